// crm_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Gives the C oracle (vh_oracle.c, vh_oracle_ic.c) the correctly rounded exp,
// log, pow and fourth root
// that the CUDA path evaluates the transport coefficients with
// (vhlle_b200/csrc/vh_crmath.cuh, compiled here as host code; every
// operation in it is an IEEE add, multiply, divide, sqrt or explicit fma, so
// the host and device builds return the same bits).  With or_trc.crmath set,
// the oracle differs from the reference only where the C library's exp or
// pow is not correctly rounded.
#include "../vhlle_b200/csrc/vh_crmath.cuh"

extern "C" double or_exp_cr(double x) { return vh::crm::exp_cr(x); }
extern "C" double or_root4_cr(double x) { return vh::crm::root4_cr(x); }
extern "C" double or_log_cr(double x) { return vh::crm::log_cr(x); }
extern "C" double or_pow_cr(double x, double y) { return vh::crm::pow_cr(x, y); }
