// host_setprimvar.cpp -- test program: the C++ host layer's IC entry,
// vhb::Fluid::setPrimVar (include/vhlle_b200.hpp; the reference's
// Cell::setPrimVar, src/cll.cpp:222-241) with the host EoS classes, on
// points read from a file.
//
//   host_setprimvar table <eos1f file> <in> <out>
//   host_setprimvar chiral <dir holding eos/> <in> <out>
//   host_setprimvar conformal <cnst> <in> <out>
//   host_setprimvar table3 <eos3f file> <in> <out>
//
// <in>: raw float64 [n][8] = tau, e, nb, nq, ns, vx, vy, vz;
// <out>: raw float64 [n][7], the Q each call stores.
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "vhlle_b200.hpp"

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s table|chiral|conformal <arg> <in> <out>\n", argv[0]);
    return 2;
  }
  const std::string kind = argv[1];
  std::unique_ptr<vhb::EoS> eos;
  if (kind == "table")
    eos.reset(new vhb::EoS1f(argv[2]));
  else if (kind == "chiral")
    eos.reset(new vhb::EoSChiral(argv[2]));
  else if (kind == "table3")
    eos.reset(new vhb::EoS3f(argv[2], 0., 0., 0., 0., 0.));
  else if (kind == "conformal")
    eos.reset(new vhb::EoSConformal(std::atof(argv[2])));
  else
    return 2;
  FILE* fi = std::fopen(argv[3], "rb");
  if (!fi) return 3;
  std::vector<double> in;
  double buf[8];
  while (std::fread(buf, sizeof(double), 8, fi) == 8) in.insert(in.end(), buf, buf + 8);
  std::fclose(fi);
  const size_t n = in.size() / 8;
  vhb::TransportCoeff tr(0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., eos.get(), 0, 0);
  vhb::Fluid f(eos.get(), eos.get(), &tr, 2, 2, 2, -1., 1., -1., 1., -1., 1., 0.1, 0.5);
  std::vector<double> out(7 * n);
  for (size_t i = 0; i < n; i++) {
    const double* a = &in[8 * i];
    f.setPrimVar(0, 0, 0, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7]);
    for (int k = 0; k < 7; k++) out[7 * i + k] = f.Q[k * 8];  // N = 8 cells, cell 0
  }
  FILE* fo = std::fopen(argv[4], "wb");
  if (!fo) return 3;
  std::fwrite(out.data(), sizeof(double), out.size(), fo);
  std::fclose(fo);
  return 0;
}
