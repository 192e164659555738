// Test harness (built by tests/test_gradient_host_port.py with nvcc, run on
// the CPU): the gradient arithmetic of smmp-svn_b200/csrc/gradient_core.cuh,
// compiled for the host, over the product's own host topology (pair chunk
// lists, 1-4 list, variable ranges, force-field tables) and the oracle's
// coordinates, bond frames and dihedral state, against the oracle's
// gradient (gradient.f / opeshe.f).
//
//   gradient_host_check <libdir/> <seqfile> [varfile|-] [ecepp2 0|1] [epsd 0|1]
//
// Prints the largest difference relative to the largest derivative for six
// conformations and exits 1 above 1e-12.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "gradient_core.cuh"
#include "molbuild.hpp"
#include "topology.hpp"

extern "C" void* orc_create(const char*, int, int, int);
extern "C" int orc_init_molecule(void*, const char*, const char*, const char*, const char*);
extern "C" int orc_gradient(void*, double*, double*);
extern "C" void orc_set_vlvr(void*, const double*);
extern "C" void orc_get_vlvr(void*, double*);
extern "C" void orc_get_coords(void*, double*);
extern "C" void orc_get_frames(void*, double*);
extern "C" void orc_get_toat(void*, double*);

using namespace smmpb200;

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string var = (argc > 3 && std::string(argv[3]) != "-") ? argv[3] : " ";
  const bool sh2 = argc > 4 && std::atoi(argv[4]) != 0;
  const bool epsd = argc > 5 && std::atoi(argv[5]) != 0;
  const ForceField ff = ecepp_forcefield(argv[1], sh2, epsd, 0);
  const ResidueLibrary lib(library_path(argv[1], sh2));
  BuildOptions opt;
  opt.sh2 = sh2;
  const MolTopo t = build_topology(lib, ff, opt, argv[2], var);
  const GradTables tab{ff.pair.a, ff.pair.a14, ff.pair.c, ff.pair.hb, ff.conv, ff.plt, ff.slp,
                       ff.epsd};
  void* h = orc_create(argv[1], sh2 ? 1 : 0, epsd ? 1 : 0, 0);
  if (!h || orc_init_molecule(h, argv[2], var.c_str(), "nh2", "cooh")) return 2;
  const int n = t.natoms, nv = t.nvar;
  std::vector<double> v0(nv);
  orc_get_vlvr(h, v0.data());
  unsigned long long lcg = 777;
  double worst = 0.0;
  for (int conf = 0; conf < 6; ++conf) {
    std::vector<double> v = v0;
    for (int i = 0; i < nv; ++i) {
      lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
      v[i] += (conf ? 0.1 : 0.0) * (double(lcg >> 11) / 9007199254740992.0 - 0.5);
    }
    orc_set_vlvr(h, v.data());
    double e_or;
    std::vector<double> g_or(nv), xyz(3 * n), frame(3 * n), toat(n);
    if (orc_gradient(h, &e_or, g_or.data())) return 2;
    orc_get_coords(h, xyz.data());
    orc_get_frames(h, frame.data());
    orc_get_toat(h, toat.data());
    // forces from every pair of the product's lists
    std::vector<double> F(3 * n, 0.0);
    double e[3] = {0.0, 0.0, 0.0};
    auto pair = [&](int i, int j, bool is14) {
      const double dx = xyz[3 * j] - xyz[3 * i], dy = xyz[3 * j + 1] - xyz[3 * i + 1],
                   dz = xyz[3 * j + 2] - xyz[3 * i + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double c = gradient_pair(tab, t.type[i], t.type[j], t.charge[i], t.charge[j], r2,
                                     is14, e);
      F[3 * i] += c * dx;
      F[3 * i + 1] += c * dy;
      F[3 * i + 2] += c * dz;
      F[3 * j] -= c * dx;
      F[3 * j + 1] -= c * dy;
      F[3 * j + 2] -= c * dz;
    };
    for (int k = 0; k < (int)t.chunks.size() * 8; ++k) {
      int i, j;
      if (gradient_chunk_pair(t.chunks.data(), k, i, j)) pair(i, j, false);
    }
    for (uint32_t w : t.pairs14) pair(int(w & 0x3fffu), int(w >> 14), true);
    // derivatives: sums over each variable's contiguous range of atoms
    double gmax = 0.0, dmax = 0.0;
    for (int vv = 0; vv < nv; ++vv) {
      double SF[3] = {0, 0, 0}, ST[3] = {0, 0, 0};
      for (int i = t.var_lo[vv]; i <= t.var_hi[vv]; ++i) {
        const double fx = F[3 * i], fy = F[3 * i + 1], fz = F[3 * i + 2];
        const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        SF[0] += fx;
        SF[1] += fy;
        SF[2] += fz;
        ST[0] += fy * z - fz * y;
        ST[1] += fz * x - fx * z;
        ST[2] += fx * y - fy * x;
      }
      const int b = t.var_base[vv];
      const double* ev = &frame[3 * b];
      const double* rb = &xyz[3 * b];
      const double fvr = gradient_torsion_force(t.var_e0[vv], t.var_sg[vv], t.var_rn[vv],
                                                toat[t.var_atom[vv]]);
      const double g = gradient_variable(ev, rb, SF, ST, fvr);
      gmax = std::max(gmax, std::fabs(g_or[vv]));
      dmax = std::max(dmax, std::fabs(g - g_or[vv]));
    }
    const double rel = dmax / std::max(1.0, gmax);
    worst = std::max(worst, rel);
    std::printf("conf %d max |dE/dv| %.6g  max difference / max |dE/dv| %.3g\n", conf, gmax, rel);
  }
  std::printf("%s worst %.3g\n", worst <= 1e-12 ? "OK" : "FAIL", worst);
  return worst <= 1e-12 ? 0 : 1;
}
