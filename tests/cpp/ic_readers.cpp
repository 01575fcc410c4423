// ic_readers.cpp -- test program: the C++ host layer's IC file readers
// (vhb::IcGlissando, vhb::IcTrento, vhb::IC in include/vhlle_b200.hpp; the
// reference's constructors src/icGlissando.cpp:130-160,
// src/icTrento.cpp:115-179, s95p::loadSongIC src/s95p.cpp:43-66) print what
// they parsed, one value per line (%.17g), for comparison with the Python
// readers.  No GPU is used (setIC is not called).
//
//   ic_readers glissando <file> <setup>
//   ic_readers trento <file> <setup>
//   ic_readers table <file>
//   ic_readers urqmd <file>
#include <cstdio>
#include <string>
#include <vector>

#include "vhlle_b200.hpp"

template <class T>
static void put(const char* tag, const std::vector<T>& v) {
  std::printf("%s %zu\n", tag, v.size());
  for (const T& a : v) std::printf("%.17g\n", (double)a);
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string kind = argv[1];
  try {
    if (kind == "glissando" && argc == 4) {
      vhb::IcGlissando ic(nullptr, argv[2], 0.5, argv[3]);
      put("npart", ic.npart());
      put("x", ic.x());
      put("y", ic.y());
      put("c", ic.c());
    } else if (kind == "trento" && argc == 4) {
      vhb::IcTrento ic(nullptr, argv[2], 0.5, argv[3]);
      put("npart", ic.npart());
      put("ngrid", ic.ngrid());
      put("gmax", ic.gmax());
      put("grid", ic.grid());
    } else if (kind == "urqmd") {
      vhb::IcPartUrqmd ic(nullptr, argv[2], 1.0, 1.0, 0.5);
      put("npart", ic.npart());
    } else if (kind == "table") {
      vhb::IC ic(argv[2], 1.0, 1);
      put("x", ic.x());
      put("y", ic.y());
      put("val", ic.val());
    } else {
      return 2;
    }
  } catch (const std::exception& e) {
    std::printf("error %s\n", e.what());
    return 1;
  }
  return 0;
}
