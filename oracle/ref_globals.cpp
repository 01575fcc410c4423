// ref_globals.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference driver's globals that the compiled reference sources read,
// defined here because src/main.cpp (which defines them) is not linked:
// the params key glauberVar (src/main.cpp:80, default 1: the table IC's
// column is an entropy density), read by s95p::loadSongIC (src/s95p.cpp:56).
int glauberVariable = 1;
