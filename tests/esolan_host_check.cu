// Test harness (built by tests/test_esolan_host_port.py with nvcc, run on the
// CPU): the per-atom area function of the analytic SASA kernel
// (smmp-svn_b200/csrc/esolan.cu, esolan_atom, compiled here for the host
// with -fmad=false as the library compiles it for the device) against the
// oracle's restatement of esolan.f on the same coordinates, atom by atom.
//
//   esolan_host_check <libdir/> <seqfile> [varfile]
//
// Six conformations: the file's start and five seeded perturbations of every
// variable.  Prints one line per conformation and exits 1 on any area that
// differs from the oracle's in any bit.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "esolan.cu"
#include "smmp_oracle.hpp"

extern "C" void* orc_create(const char*, int, int, int);
extern "C" int orc_init_molecule(void*, const char*, const char*, const char*, const char*);
extern "C" int orc_energy(void*, double*, double*);
extern "C" void orc_set_vlvr(void*, const double*);
extern "C" void orc_get_vlvr(void*, double*);

using namespace smmpb200;

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  void* h = orc_create(argv[1], 0, 0, -1);
  if (!h || orc_init_molecule(h, argv[2], argc > 3 ? argv[3] : " ", "nh2", "cooh")) return 2;
  oracle::Smmp* s = static_cast<oracle::Smmp*>(h);
  const int na = s->iatrs2[s->irsml2[s->ntlml]];
  const int nv = s->ivrml1[s->ntlml] + s->nvrml[s->ntlml] - 1;
  std::vector<double> v0(nv);
  orc_get_vlvr(h, v0.data());
  std::vector<double> scratch(kEsPerThread);
  EsWork w = es_work(scratch.data());
  unsigned long long lcg = 12345;
  int bad = 0, deferred = 0;
  for (int conf = 0; conf < 6; ++conf) {
    std::vector<double> v = v0;
    for (int i = 0; i < nv; ++i) {
      lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
      v[i] += (conf ? 0.3 : 0.0) * (double(lcg >> 11) / 9007199254740992.0 - 0.5);
    }
    orc_set_vlvr(h, v.data());
    double e, t[6];
    orc_energy(h, &e, t);   // setvar + bldmol: the coordinates both sides use
    std::vector<double> x(na + 1), y(na + 1), z(na + 1), area(na + 1), one(na + 1, 1.0);
    std::vector<double> xyz(3 * na), rv(na), sg(na);
    std::vector<int> heavy;
    for (int i = 1; i <= na; ++i) {
      x[i] = s->xat(i);
      y[i] = s->yat(i);
      z[i] = s->zat(i);
      xyz[3 * (i - 1)] = x[i];
      xyz[3 * (i - 1) + 1] = y[i];
      xyz[3 * (i - 1) + 2] = z[i];
      rv[i - 1] = s->rvdw[i];
      sg[i - 1] = s->sigma[i];
      if (rv[i - 1] > 0.0) heavy.push_back(i - 1);
    }
    oracle::esolan_areas(na, x.data(), y.data(), z.data(), s->rvdw.data(), one.data(),
                         [] { return 0.5; }, area.data());
    DMol m{};
    m.natoms = na;
    m.nheavy = (int)heavy.size();
    m.rvdw = rv.data();
    m.sigma = sg.data();
    m.heavy = heavy.data();
    double eysl = 0.0, eysl_oracle = 0.0;
    for (int i : heavy) {
      double a = -1.0;
      const int st = esolan_atom<false>(m, xyz.data(), i, w, nullptr, &a);
      if (st == kEsNeedsDraws) {
        ++deferred;
        continue;
      }
      if (st != kEsDone || a != area[i + 1]) {
        std::printf("conf %d atom %d status %d kernel %.17g oracle %.17g\n", conf, i + 1, st, a,
                    area[i + 1]);
        ++bad;
      }
      eysl = eysl + a * sg[i];
      eysl_oracle = eysl_oracle + area[i + 1] * sg[i];
    }
    std::printf("conf %d atoms %d eysl %.15g oracle %.15g\n", conf, (int)heavy.size(), eysl,
                eysl_oracle);
  }
  std::printf("%s deferred %d mismatches %d\n", bad ? "FAIL" : "OK", deferred, bad);
  return bad ? 1 : 0;
}
