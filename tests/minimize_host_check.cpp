// Test harness (built by tests/test_minimize_host.py with g++, run on the
// CPU): the product's minimiser (smmp-svn_b200/csrc/minimize.cpp) over the
// oracle's energy and gradient (gradient.f / opeshe.f restated) from the
// Met-enkephalin start of the README's minimisation example.
//
//   minimize_host_check <libdir/> <seqfile> <varfile> <imin>
//
// Prints "calls energy grad2 converged" and the final free dihedrals (rad).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "minimize.hpp"

extern "C" void* orc_create(const char*, int, int, int);
extern "C" int orc_init_molecule(void*, const char*, const char*, const char*, const char*);
extern "C" int orc_gradient(void*, double*, double*);
extern "C" void orc_set_vlvr(void*, const double*);
extern "C" void orc_get_vlvr(void*, double*);
extern "C" void orc_get_idvr(void*, int*);
extern "C" void orc_sizes(void*, int*);

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  void* h = orc_create(argv[1], 0, 0, 0);
  if (!h || orc_init_molecule(h, argv[2], argv[3], "nh2", "cooh")) return 2;
  int sz[7];
  orc_sizes(h, sz);
  const int ntlvr = sz[1], nvr = sz[2];
  std::vector<double> vl(ntlvr), g(ntlvr), x(nvr);
  std::vector<int> idvr(nvr);
  orc_get_vlvr(h, vl.data());
  orc_get_idvr(h, idvr.data());
  for (int k = 0; k < nvr; ++k) x[k] = vl[idvr[k] - 1];
  auto fg = [&](const double* xv, double* gv) {
    for (int k = 0; k < nvr; ++k) vl[idvr[k] - 1] = xv[k];
    orc_set_vlvr(h, vl.data());
    double e = 0.0;
    if (orc_gradient(h, &e, g.data())) std::exit(3);
    for (int k = 0; k < nvr; ++k) gv[k] = g[idvr[k] - 1];
    return e;
  };
  const smmpb200::MinimizeResult r = smmpb200::minimize(std::atoi(argv[4]), x, fg, 10000, 1e-9);
  std::printf("%d %.10f %.6g %d\n", r.calls, r.energy, r.grad2, r.converged ? 1 : 0);
  for (int k = 0; k < nvr; ++k) std::printf("%.12f\n", x[k]);
  return 0;
}
