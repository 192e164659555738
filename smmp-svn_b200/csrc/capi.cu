// C ABI of libsmmp_b200.so (include/smmp_b200.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/smmp_b200.h"
#include "minimize.hpp"
#include "molbuild.hpp"
#include "muca.hpp"
#include "runtime.hpp"
#include "surrogate.hpp"

using namespace smmpb200;

namespace {

thread_local std::string g_err;

template <class F>
int guard(F&& f) {
  try {
    f();
    return SMMP_OK;
  } catch (const std::invalid_argument& e) {
    g_err = e.what();
    return SMMP_ERR_ARG;
  } catch (const std::runtime_error& e) {
    g_err = e.what();
    std::string w = e.what();
    if (w.find("cuda") != std::string::npos || w.find("CUDA") != std::string::npos ||
        w.find("H2D") != std::string::npos || w.find("D2H") != std::string::npos ||
        w.find("sync") != std::string::npos)
      return SMMP_ERR_CUDA;
    if (w.find("kernel error") != std::string::npos) return SMMP_ERR_KERNEL;
    return SMMP_ERR_INPUT;
  } catch (const std::exception& e) {
    g_err = e.what();
    return SMMP_ERR_ARG;
  }
}

void need(bool ok, const char* msg) {
  if (!ok) throw std::invalid_argument(msg);
}

Config to_cfg(const smmp_config_t* c) {
  Config k;
  if (c) {
    k.sh2 = c->sh2;
    k.epsd = c->epsd;
    k.itysol = c->itysol;
    k.ientyp = c->ientyp;
    k.rndord = c->rndord;
    k.upchswitch = c->upchswitch;
  }
  need(k.ientyp == 0, "only ientyp=0 (ECEPP) is on this path");
  need(k.upchswitch == 0, "biased Gaussian steps (upchswitch!=0) are outside this path");
  need(k.itysol >= -9 && k.itysol <= 9,
       "itysol must be 0 (vacuum), a numerical SASA model 1..9 or an analytic one -1..-9");
  return k;
}

DWeight to_dweight(const smmp_weight_t* w, std::vector<void*>& tmp) {
  DWeight d{kWeightCanon, 0, 0, 1.0, nullptr, nullptr};
  if (!w || w->kind == 0) return d;
  need(w->kind == 1 || w->kind == 2, "weight kind must be 0, 1 or 2 on the GPU path");
  need(w->kmax >= w->kmin && w->b && w->alpha && w->ebin != 0.0, "bad multicanonical table");
  size_t n = (size_t)(w->kmax - w->kmin + 1);
  double *b = nullptr, *a = nullptr;
  check_cuda(cudaMalloc(&b, n * sizeof(double)), "cudaMalloc");
  tmp.push_back(b);
  check_cuda(cudaMalloc(&a, n * sizeof(double)), "cudaMalloc");
  tmp.push_back(a);
  check_cuda(cudaMemcpy(b, w->b, n * sizeof(double), cudaMemcpyHostToDevice), "H2D");
  check_cuda(cudaMemcpy(a, w->alpha, n * sizeof(double), cudaMemcpyHostToDevice), "H2D");
  d.kind = w->kind;
  d.kmin = w->kmin;
  d.kmax = w->kmax;
  d.ebin = w->ebin;
  d.b = b;
  d.alpha = a;
  return d;
}

struct TmpFree {
  std::vector<void*> p;
  ~TmpFree() {
    for (void* q : p) cudaFree(q);
  }
};

void raise_kernel_errors(Ensemble& e) {
  std::vector<int> err;
  e.get_errors(err);
  for (size_t c = 0; c < err.size(); ++c)
    if (err[c] != 0)
      throw std::runtime_error("kernel error " + std::to_string(err[c]) + " on chain " +
                               std::to_string(c));
}

// ------------------------------------------------------------------ host MT19937
// The global stream of the reference-facing layer exists before any molecule
// (main programs call sgrnd before init_molecule).  Until a molecule is on
// the GPU it is advanced here; afterwards the GPU copy is authoritative.
struct HostMT {
  uint32_t mt[kMTWords];   // device slot layout with an empty queue
  HostMT() {
    std::memset(mt, 0, sizeof mt);
    mt[kMTIdx] = 625;
  }
  void seed(uint32_t s) {
    mt[0] = s;
    for (int i = 1; i < 624; ++i) mt[i] = 69069u * mt[i - 1];
    mt[624] = 624;
  }
  double next() {
    if (mt[624] >= 624) {
      if (mt[624] == 625) seed(4357u);
      const uint32_t MATA = 0x9908B0DFu, UM = 0x80000000u, LM = 0x7fffffffu;
      int kk = 0;
      uint32_t y;
      for (; kk < 227; ++kk) {
        y = (mt[kk] & UM) | (mt[kk + 1] & LM);
        mt[kk] = mt[kk + 397] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
      }
      for (; kk < 623; ++kk) {
        y = (mt[kk] & UM) | (mt[kk + 1] & LM);
        mt[kk] = mt[kk - 227] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
      }
      y = (mt[623] & UM) | (mt[0] & LM);
      mt[623] = mt[396] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
      mt[624] = 0;
    }
    uint32_t y = mt[mt[624]++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9D2C5680u;
    y ^= (y << 15) & 0xEFC60000u;
    y ^= (y >> 18);
    return (double)y / 4294967295.0;
  }
};

constexpr double kPi = 3.141592653589793;
double h_wrap(double d) {
  d = std::fmod(d, 2.0 * kPi);
  return std::fabs(d) <= kPi ? d : d - std::copysign(2.0 * kPi, d);
}

// ------------------------------------------------------------------ global system
struct Universe {
  Config cfg;
  std::string libdir;
  bool energy_ready = false;
  std::shared_ptr<Molecule> mol;
  std::unique_ptr<Ensemble> ens;
  HostMT mt;
  double beta = 0.0;
  double terms[6] = {0, 0, 0, 0, 0, 0};
  long long ncalls = 0, nacalls = 0;
};
Universe& U() {
  static Universe u;
  return u;
}

void require_molecule() {
  need(U().ens != nullptr, "call smmp_init_molecule first");
}

void sync_beta() {
  Universe& u = U();
  u.ens->set_betas(std::vector<double>{u.beta});
}

double universe_energy() {
  Universe& u = U();
  u.ens->energy(false);
  raise_kernel_errors(*u.ens);
  std::vector<double> e, t;
  u.ens->get_eol(e);
  u.ens->get_terms(t);
  for (int k = 0; k < 6; ++k) u.terms[k] = t[k];
  return e[0];
}

double universe_grnd() {
  Universe& u = U();
  if (!u.ens) return u.mt.next();
  std::vector<double> out;
  u.ens->draw(0, 1, out);
  return out[0];
}

// Sampling weight on the host for the host-driven sweep (canon.f:135-149,
// mulcan_par_mod.f90:380-410), the arithmetic of the device's weight().
double host_weight(const smmp_weight_t* w, double beta, double x) {
  if (!w || w->kind == 0) return beta * x;
  double v = x / w->ebin + std::copysign(0.5, x);
  v = std::fmax((double)w->kmin, v);
  v = std::fmin((double)w->kmax, v);
  const int k = (int)v - w->kmin;
  if (w->kind == 1) return (beta + w->b[k]) * x + w->alpha[k];
  return w->b[k] * x + w->alpha[k];
}

// metropolis with proposals driven from the host and every energy() on the
// GPU (metropolis.f:13-184): for a host weight callback, and for the
// analytic SASA model, whose energy() may draw from the stream between a
// proposal's numbers and its acceptance number.
void metropolis_host(double* eol1, double* acz, const std::function<double(double)>& W) {
  Universe& u = U();
  const MolTopo& t = u.mol->topo;
  std::vector<double> vl;
  double eol = universe_energy();
  for (int nsw = 0; nsw < t.nfree; ++nsw) {
    int ivar = u.cfg.rndord ? (int)(t.nfree * universe_grnd()) : nsw;
    if (ivar >= t.nfree) ivar = t.nfree - 1;
    int jv = t.idvr[ivar];
    u.ens->get_vlvr(vl);
    double vold = vl[jv];
    double dv = t.axvr[jv] * (universe_grnd() - 0.5);
    vl[jv] = h_wrap(vold + dv);
    u.ens->set_vlvr(vl);
    double enw = universe_energy();
    double delta = W(enw) - W(eol);
    int up = 0;
    if (delta <= 0.0) {
      up = 1;
    } else {
      double rd = universe_grnd();
      delta = std::fmin(delta, 100.0);
      if (std::exp(-delta) >= rd) up = 1;
    }
    if (up) {
      eol = enw;
    } else {
      vl[jv] = vold;
      u.ens->set_vlvr(vl);
    }
    *acz += up;
    ++u.ncalls;
    u.nacalls += up;
  }
  double enw = universe_energy();
  if (std::fabs(eol - enw) > 1e-6 && eol < 100000)
    throw std::runtime_error("metropolis: eol and enw difference unacceptable");
  *eol1 = eol;
}

}  // namespace

// ============================================================================ layer 1
extern "C" {

const char* smmp_last_error(void) { return g_err.c_str(); }

int smmp_gpu_available(void) {
  int n = 0;
  return cudaGetDeviceCount(&n) == cudaSuccess && n > 0 ? 1 : 0;
}

int smmp_reset(void) {
  return guard([&] {
    Universe& u = U();
    u.ens.reset();
    u.mol.reset();
    u.cfg = Config();
    u.libdir.clear();
    u.energy_ready = false;
    u.mt = HostMT();
    u.beta = 0.0;
    for (double& t : u.terms) t = 0.0;
    u.ncalls = u.nacalls = 0;
  });
}

int smmp_set_config(const smmp_config_t* cfg) {
  return guard([&] {
    need(cfg != nullptr, "cfg is NULL");
    U().cfg = to_cfg(cfg);
  });
}

int smmp_get_config(smmp_config_t* cfg) {
  return guard([&] {
    need(cfg != nullptr, "cfg is NULL");
    const Config& k = U().cfg;
    cfg->sh2 = k.sh2;
    cfg->epsd = k.epsd;
    cfg->itysol = k.itysol;
    cfg->ientyp = k.ientyp;
    cfg->rndord = k.rndord;
    cfg->upchswitch = k.upchswitch;
  });
}

int smmp_init_energy(const char* libdir) {
  return guard([&] {
    need(libdir != nullptr, "libdir is NULL");
    Universe& u = U();
    std::string d = libdir;
    if (!d.empty() && d.back() != '/') d += '/';
    // validate: the library (and the sphere points of a solvation model)
    // must be readable now, as init_energy reads them
    need(u.cfg.ientyp == 0, "init_energy: only ientyp=0 (ECEPP) is on this path");
    ecepp_forcefield(d, u.cfg.sh2 != 0, u.cfg.epsd != 0, u.cfg.itysol);
    ResidueLibrary probe(library_path(d, u.cfg.sh2 != 0));
    (void)probe;
    u.libdir = d;
    u.energy_ready = true;
  });
}

int smmp_init_molecule(int iabin, const char* grpn, const char* grpc, const char* seqfile,
                       const char* varfile) {
  return guard([&] {
    Universe& u = U();
    need(u.energy_ready, "call smmp_init_energy first");
    need(iabin == 1, "only iabin=1 (sequence + variable files) is on this path");
    need(seqfile != nullptr, "seqfile is NULL");
    need(u.mol == nullptr, "one molecule per system on this path");
    need(smmp_gpu_available() == 1, "no CUDA device available");
    std::string var = varfile ? varfile : "";
    u.mol = build_molecule(u.libdir, u.cfg, seqfile, var, grpn ? grpn : "nh2",
                           grpc ? grpc : "cooh");
    u.ens.reset(new Ensemble({u.mol}, {0}, {4357}, {u.beta}, true));
    std::vector<uint32_t> mt(u.mt.mt, u.mt.mt + kMTWords);
    u.ens->set_mt(mt);
  });
}

int smmp_energy(double* e_out) {
  return guard([&] {
    require_molecule();
    double e = universe_energy();
    if (e_out) *e_out = e;
  });
}

int smmp_enysol(int nmol, double* eysl) {
  return guard([&] {
    require_molecule();
    need(nmol == 0 || nmol == 1, "molecule index out of range");
    need(U().cfg.itysol > 0, "enysol needs a numerical SASA model (itysol 1..9)");
    universe_energy();
    if (eysl) *eysl = U().terms[4];
  });
}

int smmp_energy_terms(double terms[6]) {
  return guard([&] {
    need(terms != nullptr, "terms is NULL");
    for (int k = 0; k < 6; ++k) terms[k] = U().terms[k];
  });
}

int smmp_setvar(int nml, const double* vlvrx) {
  return guard([&] {
    require_molecule();
    need(nml == 1, "molecule index out of range");
    need(vlvrx != nullptr, "vlvrx is NULL");
    Universe& u = U();
    int nv = u.mol->topo.nvar;
    std::vector<double> vl((size_t)u.ens->vstride(), 0.0);
    std::copy(vlvrx, vlvrx + nv, vl.begin());
    u.ens->set_vlvr(vl);
    universe_energy();   // setvar + bldmol (the energy terms are refreshed too)
  });
}

int smmp_metropolis(double* eol, double* acz, const smmp_weight_t* w) {
  return guard([&] {
    require_molecule();
    need(eol != nullptr && acz != nullptr, "eol/acz is NULL");
    Universe& u = U();
    if (w && w->kind == 3) {
      need(w->callback != nullptr, "weight callback is NULL");
      metropolis_host(eol, acz, [w](double x) { return w->callback(x, w->user); });
      return;
    }
    if (u.cfg.itysol < 0) {   // analytic SASA: energy() on the GPU, proposals here
      need(!w || w->kind == 0 || (w->kmax >= w->kmin && w->b && w->alpha && w->ebin != 0.0),
           "bad multicanonical table");
      const double beta = u.beta;
      metropolis_host(eol, acz, [w, beta](double x) { return host_weight(w, beta, x); });
      return;
    }
    TmpFree tmp;
    DWeight dw = to_dweight(w, tmp.p);
    sync_beta();
    std::vector<unsigned long long> a0, p0, a1, p1;
    u.ens->get_acceptance(a0, p0);
    int flags = u.cfg.rndord ? kFlagRndOrd : 0;
    u.ens->sweeps(1, flags, dw);
    raise_kernel_errors(*u.ens);
    u.ens->get_acceptance(a1, p1);
    std::vector<double> e, t;
    u.ens->get_eol(e);
    u.ens->get_terms(t);
    for (int k = 0; k < 6; ++k) u.terms[k] = t[k];
    *eol = e[0];
    *acz += (double)(a1[0] - a0[0]);
    u.ncalls += (long long)(p1[0] - p0[0]);
    u.nacalls += (long long)(a1[0] - a0[0]);
  });
}

// Text to a file, or to standard output when the name is empty or blank
// (ibegst(fileName) = 0 in outvar.f:38 / outpdb.f:62).
void write_text(const std::string& s, const char* fileName, const char* who) {
  if (fileName && std::string(fileName).find_first_not_of(' ') != std::string::npos) {
    std::FILE* f = std::fopen(fileName, "w");
    if (!f) throw std::invalid_argument(std::string(who) + ": cannot open the file");
    std::fputs(s.c_str(), f);
    std::fclose(f);
  } else {
    std::fputs(s.c_str(), stdout);
    std::fflush(stdout);
  }
}

int smmp_muca_update(int kmin, int kmax, double ebin, double beta, int* ihist, double* xhist,
                     double* g1, double* b, double* alpha, double* ent) {
  return guard([&] {
    need(kmax - kmin >= 2 && ebin > 0.0, "muca: need at least three bins and ebin > 0");
    need(ihist && xhist && g1 && b && alpha && ent, "NULL argument");
    muca_update(MucaBins{kmin, kmax, ebin, beta}, ihist, xhist, g1, b, alpha, ent);
  });
}

int smmp_muca_finish(int kmin, int kmax, double ebin, double beta, double* b, double* alpha) {
  return guard([&] {
    need(kmax - kmin >= 2 && ebin > 0.0, "muca: need at least three bins and ebin > 0");
    need(b && alpha, "NULL argument");
    muca_finish(MucaBins{kmin, kmax, ebin, beta}, b, alpha);
  });
}

int smmp_outvar(int nml, const char* fileName) {
  return guard([&] {
    require_molecule();
    need(nml == 0 || nml == 1, "outvar: no such molecule (one molecule on this path)");
    Universe& u = U();
    std::vector<double> vl;
    u.ens->get_vlvr(vl);
    write_text(outvar_text(u.mol->topo, vl.data(), 1), fileName, "outvar");
  });
}

int smmp_outpdb(int nml, const char* fileName) {
  return guard([&] {
    require_molecule();
    need(nml == 0 || nml == 1, "outpdb: no such molecule (one molecule on this path)");
    Universe& u = U();
    std::vector<double> xyz;
    u.ens->get_coords(xyz);   // the rebuild of the current variables
    write_text(outpdb_text(u.mol->topo, xyz.data()), fileName, "outpdb");
  });
}

int smmp_sgrnd(int32_t seed) {
  return guard([&] {
    Universe& u = U();
    u.mt.seed((uint32_t)seed);
    if (u.ens) u.ens->set_mt(std::vector<uint32_t>(u.mt.mt, u.mt.mt + kMTWords));
  });
}

double smmp_grnd(void) {
  double r = NAN;
  int st = guard([&] { r = universe_grnd(); });
  return st == SMMP_OK ? r : NAN;
}

// gradient() of the global system: energies and gdeyvr of chain 0.
double universe_gradient(std::vector<double>& g) {
  Universe& u = U();
  u.ens->gradient(g);
  raise_kernel_errors(*u.ens);
  std::vector<double> e, t;
  u.ens->get_eol(e);
  u.ens->get_terms(t);
  for (int k = 0; k < 6; ++k) u.terms[k] = t[k];
  return e[0];
}

int smmp_gradient(double* gdeyvr, double* eysm) {
  return guard([&] {
    require_molecule();
    need(U().cfg.itysol == 0, "the GPU gradient is for the vacuum energy (itysol 0)");
    std::vector<double> g;
    const double e = universe_gradient(g);
    if (gdeyvr) std::copy(g.begin(), g.begin() + U().mol->topo.nvar, gdeyvr);
    if (eysm) *eysm = e;
  });
}

int smmp_minim(int imin, int maxit, double eps, int* nop) {
  return guard([&] {
    require_molecule();
    need(imin == 1 || imin == 2, "imin must be 1 (quasi-Newton) or 2 (conjugate gradients)");
    need(maxit > 0 && eps >= 0.0, "bad minim arguments");
    Universe& u = U();
    need(u.cfg.itysol == 0, "the GPU gradient is for the vacuum energy (itysol 0)");
    const MolTopo& t = u.mol->topo;
    std::vector<double> vl, g;
    u.ens->get_vlvr(vl);
    std::vector<double> x(t.nfree);
    for (int k = 0; k < t.nfree; ++k) x[k] = vl[t.idvr[k]];
    auto fg = [&](const double* xv, double* gv) {
      for (int k = 0; k < t.nfree; ++k) vl[t.idvr[k]] = xv[k];
      u.ens->set_vlvr(vl);
      const double e = universe_gradient(g);
      for (int k = 0; k < t.nfree; ++k) gv[k] = g[t.idvr[k]];
      return e;
    };
    const MinimizeResult r = minimize(imin, x, fg, maxit, eps);
    for (int k = 0; k < t.nfree; ++k) vl[t.idvr[k]] = h_wrap(x[k]);   // minim.f: into (-pi, pi]
    u.ens->set_vlvr(vl);
    universe_energy();
    if (nop) *nop = r.calls;
  });
}

int smmp_canon(int nequi, int nswp, int nmes, double temp, int lrand, double* trace, double* out) {
  return guard([&] {
    require_molecule();
    need(temp > 0 && nmes > 0 && nequi >= 0 && nswp >= 0, "bad canon arguments");
    Universe& u = U();
    u.beta = 1.0 / (temp * 1.98773e-3);
    sync_beta();
    if (lrand) u.ens->random_start();
    universe_energy();
    int flags = u.cfg.rndord ? kFlagRndOrd : 0;
    DWeight w{kWeightCanon, 0, 0, 1.0, nullptr, nullptr};
    std::vector<unsigned long long> a0, p0, a1, p1;
    int k = 0;
    if (nequi > 0) u.ens->sweeps(nequi, flags, w);
    raise_kernel_errors(*u.ens);
    std::vector<double> e;
    u.ens->get_eol(e);
    double after_equi = e[0];
    u.ens->get_acceptance(a0, p0);
    // sweeps nsw = 0..nswp (canon.f:85-115), measuring when mod(nsw, nmes) == 0
    int nsw = 0;
    while (nsw <= nswp) {
      int next_meas = ((nsw + nmes - 1) / nmes) * nmes;
      int upto = std::min(next_meas, nswp);
      u.ens->sweeps(upto - nsw + 1, flags, w);
      raise_kernel_errors(*u.ens);
      nsw = upto + 1;
      if (trace && upto % nmes == 0) {
        u.ens->get_eol(e);
        trace[k++] = e[0];
      }
    }
    u.ens->get_acceptance(a1, p1);
    u.ens->get_eol(e);
    if (out) {
      out[0] = after_equi;
      out[1] = (double)(a1[0] - a0[0]) / ((double)(nswp + 1) * u.mol->topo.nfree);
      out[2] = e[0];
    }
    u.ncalls += (long long)(p1[0] - p0[0]);
    u.nacalls += (long long)(a1[0] - a0[0]);
  });
}

int smmp_anneal(int nequi, int nswp, int nmes, double tmax, double tmin, int lrand, double* out) {
  return guard([&] {
    require_molecule();
    need(tmax > 0 && tmin > 0 && nswp > 0, "bad anneal arguments");
    (void)nmes;
    Universe& u = U();
    double bmin = 1.0 / (tmax * 1.98773e-3), bmax = 1.0 / (tmin * 1.98773e-3);
    double db = std::exp(std::log(bmax / bmin) / nswp);
    if (lrand) u.ens->random_start();
    double e0 = universe_energy();
    int flags = u.cfg.rndord ? kFlagRndOrd : 0;
    DWeight w{kWeightCanon, 0, 0, 1.0, nullptr, nullptr};
    u.beta = bmin;
    sync_beta();
    if (nequi > 0) u.ens->sweeps(nequi, flags, w);
    std::vector<double> e;
    u.ens->get_eol(e);
    double after = e[0];
    std::vector<unsigned long long> a0, p0, a1, p1;
    u.ens->get_acceptance(a0, p0);
    double ymin = after;
    int nemin = 0;
    for (int nsw = 0; nsw <= nswp; ++nsw) {
      u.beta = bmin * std::pow(db, nsw);
      sync_beta();
      u.ens->sweeps(1, flags, w);
      u.ens->get_eol(e);
      if (e[0] < ymin) {
        ymin = e[0];
        nemin = nsw;
      }
    }
    raise_kernel_errors(*u.ens);
    u.ens->get_acceptance(a1, p1);
    if (out) {
      out[0] = e0;
      out[1] = after;
      out[2] = (double)(a1[0] - a0[0]) / ((double)(nswp + 1) * u.mol->topo.nfree);
      out[3] = e[0];
      out[4] = ymin;
      out[5] = nemin;
    }
  });
}

int smmp_set_beta(double beta) {
  return guard([&] {
    U().beta = beta;
    if (U().ens) sync_beta();
  });
}
double smmp_get_beta(void) { return U().beta; }

int smmp_get_sizes(int* natoms, int* ntlvr, int* nvr) {
  return guard([&] {
    require_molecule();
    const MolTopo& t = U().mol->topo;
    if (natoms) *natoms = t.natoms;
    if (ntlvr) *ntlvr = t.nvar;
    if (nvr) *nvr = t.nfree;
  });
}

int smmp_get_vlvr(double* vlvr) {
  return guard([&] {
    require_molecule();
    std::vector<double> v;
    U().ens->get_vlvr(v);
    std::copy(v.begin(), v.begin() + U().mol->topo.nvar, vlvr);
  });
}

int smmp_set_vlvr(const double* vlvr) {
  return guard([&] {
    require_molecule();
    std::vector<double> v((size_t)U().ens->vstride(), 0.0);
    std::copy(vlvr, vlvr + U().mol->topo.nvar, v.begin());
    U().ens->set_vlvr(v);
  });
}

int smmp_get_idvr(int* idvr) {
  return guard([&] {
    require_molecule();
    const MolTopo& t = U().mol->topo;
    for (int i = 0; i < t.nfree; ++i) idvr[i] = t.idvr[i] + 1;
  });
}

int smmp_get_axvr(double* axvr) {
  return guard([&] {
    require_molecule();
    const MolTopo& t = U().mol->topo;
    std::copy(t.axvr.begin(), t.axvr.end(), axvr);
  });
}

int smmp_get_coords(double* xyz) {
  return guard([&] {
    require_molecule();
    std::vector<double> c;
    U().ens->get_coords(c);
    std::copy(c.begin(), c.begin() + 3 * U().mol->topo.natoms, xyz);
  });
}

int smmp_get_acceptance(long long* ncalls, long long* nacalls) {
  return guard([&] {
    if (ncalls) *ncalls = U().ncalls;
    if (nacalls) *nacalls = U().nacalls;
  });
}

}  // extern "C"

// ============================================================================ layer 2

struct smmp_mol {
  std::shared_ptr<Molecule> m;
};
struct smmp_ens {
  std::unique_ptr<Ensemble> e;
  int flags = 0;
};

extern "C" {

smmp_mol_t* smmp_mol_build(const char* libdir, const smmp_config_t* cfg, const char* seqfile,
                           const char* varfile, const char* grpn, const char* grpc) {
  smmp_mol_t* out = nullptr;
  guard([&] {
    need(libdir && seqfile, "libdir/seqfile is NULL");
    auto m = build_molecule(libdir, to_cfg(cfg), seqfile, varfile ? varfile : "",
                            grpn ? grpn : "nh2", grpc ? grpc : "cooh");
    out = new smmp_mol{m};
  });
  return out;
}

void smmp_mol_free(smmp_mol_t* m) { delete m; }

int smmp_mol_info(const smmp_mol_t* m, long long info[6]) {
  return guard([&] {
    need(m && info, "NULL argument");
    const MolTopo& t = m->m->topo;
    info[0] = t.natoms;
    info[1] = t.nvar;
    info[2] = t.nfree;
    info[3] = t.npairs;
    info[4] = (long long)t.heavy.size();
    info[5] = t.nres;
  });
}

int smmp_mol_outvar(const smmp_mol_t* m, const double* vlvr, int iml, char* buf,
                    uint64_t* len) {
  return guard([&] {
    need(m && vlvr && len, "NULL argument");
    const std::string s = outvar_text(m->m->topo, vlvr, iml);
    if (buf) {
      need(*len >= s.size() + 1, "buffer too small");
      std::memcpy(buf, s.c_str(), s.size() + 1);
    }
    *len = s.size() + 1;
  });
}

int smmp_mol_outpdb(const smmp_mol_t* m, const double* xyz, char* buf, uint64_t* len) {
  return guard([&] {
    need(m && xyz && len, "NULL argument");
    const std::string s = outpdb_text(m->m->topo, xyz);
    if (buf) {
      need(*len >= s.size() + 1, "buffer too small");
      std::memcpy(buf, s.c_str(), s.size() + 1);
    }
    *len = s.size() + 1;
  });
}

int smmp_mol_var_ranges(const smmp_mol_t* m, int* lo, int* hi) {
  return guard([&] {
    need(m && lo && hi, "NULL argument");
    const MolTopo& t = m->m->topo;
    for (int v = 0; v < t.nvar; ++v) {
      lo[v] = t.var_lo[v];
      hi[v] = t.var_hi[v];
    }
  });
}

int smmp_mol_atoms(const smmp_mol_t* m, int* parent, int* type, double* charge, double* geom) {
  return guard([&] {
    need(m && parent && type && charge && geom, "NULL argument");
    const MolTopo& t = m->m->topo;
    for (int i = 0; i < t.natoms; ++i) {
      parent[i] = t.iow[i];
      type[i] = t.type[i] + 1;
      charge[i] = t.charge[i];
      geom[4 * i] = t.blen[i];
      geom[4 * i + 1] = std::atan2(t.sba[i], t.cba[i]);
      geom[4 * i + 2] = t.toat0[i];
      geom[4 * i + 3] = t.rvdw[i];
    }
  });
}

int smmp_mol_vars(const smmp_mol_t* m, int* info) {
  return guard([&] {
    need(m && info, "NULL argument");
    const MolTopo& t = m->m->topo;
    for (int v = 0; v < t.nvar; ++v) {
      info[4 * v] = t.var_atom[v];
      info[4 * v + 1] = t.var_class[v];
      info[4 * v + 2] = t.var_fixed[v];
      info[4 * v + 3] = t.var_residue[v];
    }
  });
}

int smmp_mol_pairs(const smmp_mol_t* m, int* pairs) {
  return guard([&] {
    need(m && pairs, "NULL argument");
    const MolTopo& t = m->m->topo;
    size_t k = 0;
    for (uint32_t w : t.chunks) {
      const int i = int(w & 0x3fffu), j0 = int((w >> 14) & 0x3fffu), len = int((w >> 28) & 7u) + 1;
      for (int j = j0; j < j0 + len; ++j) {
        pairs[k++] = i;
        pairs[k++] = j;
        pairs[k++] = 0;
      }
    }
    for (uint32_t w : t.pairs14) {
      pairs[k++] = int(w & 0x3fffu);
      pairs[k++] = int(w >> 14);
      pairs[k++] = 1;
    }
  });
}

int smmp_mol_vlvr0(const smmp_mol_t* m, double* vlvr) {
  return guard([&] {
    need(m && vlvr, "NULL argument");
    const MolTopo& t = m->m->topo;
    for (size_t k = 0; k < t.vlvr0.size(); ++k) vlvr[k] = t.vlvr0[k];
  });
}

int smmp_mol_idvr(const smmp_mol_t* m, int* idvr) {
  return guard([&] {
    need(m && idvr, "NULL argument");
    const MolTopo& t = m->m->topo;
    for (size_t k = 0; k < t.idvr.size(); ++k) idvr[k] = t.idvr[k];
  });
}

smmp_ens_t* smmp_ens_create(smmp_mol_t* const* mols, int nmols, const int* chain_mol,
                            int nchains, const int* seeds, const double* betas,
                            int shared_stream, int flags) {
  smmp_ens_t* out = nullptr;
  guard([&] {
    need(mols && nmols > 0 && chain_mol && nchains > 0 && seeds && betas, "NULL argument");
    need(smmp_gpu_available() == 1, "no CUDA device available");
    std::vector<std::shared_ptr<Molecule>> ms;
    for (int i = 0; i < nmols; ++i) {
      need(mols[i] != nullptr, "NULL molecule");
      ms.push_back(mols[i]->m);
    }
    std::vector<int> cm(chain_mol, chain_mol + nchains);
    int ns = shared_stream ? 1 : nchains;
    std::vector<int> sd(seeds, seeds + ns);
    std::vector<double> b(betas, betas + nchains);
    auto e = std::make_unique<Ensemble>(ms, cm, sd, b, shared_stream != 0);
    out = new smmp_ens{std::move(e), flags};
  });
  return out;
}

void smmp_ens_free(smmp_ens_t* e) { delete e; }

int smmp_ens_set_stream(smmp_ens_t* e, void* stream) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    e->e->set_stream(static_cast<cudaStream_t>(stream));
  });
}

int smmp_ens_random_start(smmp_ens_t* e) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    e->e->random_start();
  });
}

int smmp_ens_energy(smmp_ens_t* e, double* eol) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    e->e->energy((e->flags & SMMP_ENS_FP32) != 0);
    raise_kernel_errors(*e->e);
    if (eol) {
      std::vector<double> v;
      e->e->get_eol(v);
      std::copy(v.begin(), v.end(), eol);
    }
  });
}

int smmp_ens_equilibrate(smmp_ens_t* e, int nequi) {
  return guard([&] {
    need(e != nullptr && nequi >= 0, "bad arguments");
    e->e->equilibrate(nequi, e->flags & (kFlagFP32 | kFlagRndOrd));
    raise_kernel_errors(*e->e);
  });
}

int smmp_ens_sweeps(smmp_ens_t* e, int nsweeps, const smmp_weight_t* w) {
  return guard([&] {
    need(e != nullptr && nsweeps >= 0, "bad arguments");
    TmpFree tmp;
    DWeight dw = to_dweight(w, tmp.p);
    int flags = e->flags & (kFlagFP32 | kFlagRndOrd);
    e->e->sweeps(nsweeps, flags, dw);
    raise_kernel_errors(*e->e);
  });
}

int smmp_ens_set_pt(smmp_ens_t* e, const double* betas, int wrap, int exchange_seed) {
  return guard([&] {
    need(e != nullptr && betas != nullptr, "NULL argument");
    e->e->set_pt(std::vector<double>(betas, betas + e->e->nchains()), wrap, exchange_seed);
  });
}

int smmp_ens_pt_sweeps(smmp_ens_t* e, int nsweeps, int serial, int graph_chunk) {
  return guard([&] {
    need(e != nullptr && nsweeps >= 0, "bad arguments");
    need(e->e->has_pt(), "call smmp_ens_set_pt first");
    int flags = e->flags & (kFlagFP32 | kFlagRndOrd);
    e->e->pt_sweeps(nsweeps, flags, serial != 0, graph_chunk);
    raise_kernel_errors(*e->e);
  });
}

int smmp_ens_set_pt_fused(smmp_ens_t* e, int on, double timeout_s, int barrier_extra) {
  return guard([&] {
    need(e != nullptr, "NULL argument");
    need(timeout_s > 0.0 && barrier_extra >= 0, "bad arguments");
    e->e->set_pt_fused(on != 0, timeout_s, (unsigned)barrier_extra);
  });
}

int smmp_ens_pt_fused_last(smmp_ens_t* e, int* fused) {
  return guard([&] {
    need(e != nullptr && fused != nullptr, "NULL argument");
    *fused = e->e->pt_fused_last() ? 1 : 0;
  });
}

int smmp_ens_pt_map(smmp_ens_t* e, int* temp_chain) {
  return guard([&] {
    need(e && temp_chain && e->e->has_pt(), "bad arguments");
    std::vector<int> tc;
    e->e->pt_map(tc);
    std::copy(tc.begin(), tc.end(), temp_chain);
  });
}

int smmp_ens_pair_terms(smmp_ens_t* e, uint64_t* terms) {
  return guard([&] {
    need(e && terms, "NULL argument");
    std::vector<unsigned long long> p;
    e->e->get_pair_terms(p);
    std::copy(p.begin(), p.end(), terms);
  });
}

int smmp_ens_gradient(smmp_ens_t* e, double* grad, double* energies) {
  return guard([&] {
    need(e && grad, "NULL argument");
    std::vector<double> g;
    e->e->gradient(g);
    std::copy(g.begin(), g.end(), grad);
    if (energies) {
      std::vector<double> en;
      e->e->get_eol(en);
      std::copy(en.begin(), en.end(), energies);
    }
    raise_kernel_errors(*e->e);
  });
}

int smmp_ens_pt_stats(smmp_ens_t* e, uint64_t* stats) {
  return guard([&] {
    need(e && stats && e->e->has_pt(), "bad arguments");
    std::vector<unsigned long long> st;
    e->e->pt_stats(st);
    std::copy(st.begin(), st.end(), stats);
  });
}

int smmp_ens_sizes(smmp_ens_t* e, int* nchains, int* vstride, int* tstride) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    if (nchains) *nchains = e->e->nchains();
    if (vstride) *vstride = e->e->vstride();
    if (tstride) *tstride = e->e->tstride();
  });
}

#define ENS_GET(name, call, T)                      \
  int name(smmp_ens_t* e, T* out) {                 \
    return guard([&] {                              \
      need(e && out, "NULL argument");              \
      std::vector<T> v;                             \
      e->e->call(v);                                \
      std::copy(v.begin(), v.end(), out);           \
    });                                             \
  }
ENS_GET(smmp_ens_get_energies, get_eol, double)
ENS_GET(smmp_ens_get_terms, get_terms, double)
ENS_GET(smmp_ens_get_vlvr, get_vlvr, double)
ENS_GET(smmp_ens_get_betas, get_betas, double)
ENS_GET(smmp_ens_get_coords, get_coords, double)
ENS_GET(smmp_ens_errors, get_errors, int)
#undef ENS_GET

int smmp_ens_set_vlvr(smmp_ens_t* e, const double* vlvr) {
  return guard([&] {
    need(e && vlvr, "NULL argument");
    size_t n = (size_t)e->e->nchains() * e->e->vstride();
    e->e->set_vlvr(std::vector<double>(vlvr, vlvr + n));
  });
}

int smmp_ens_acceptance(smmp_ens_t* e, unsigned long long* acc, unsigned long long* prop) {
  return guard([&] {
    need(e && acc && prop, "NULL argument");
    std::vector<unsigned long long> a, p;
    e->e->get_acceptance(a, p);
    std::copy(a.begin(), a.end(), acc);
    std::copy(p.begin(), p.end(), prop);
  });
}

int smmp_ens_draw(smmp_ens_t* e, int slot, int n, double* out) {
  return guard([&] {
    need(e && out && n >= 0 && slot >= 0 && slot < e->e->nslots_mt(), "bad arguments");
    std::vector<double> v;
    e->e->draw(slot, n, v);
    std::copy(v.begin(), v.end(), out);
  });
}

}  // extern "C"

namespace {
struct CkptHeader {
  uint64_t magic, nchains, vstride, tstride, nmt, ntoat, npt, iswitch;
};
constexpr uint64_t kMagic = 0x534d4d5042323030ull;   // "SMMPB200"
template <class T>
void put(std::vector<char>& b, const std::vector<T>& v) {
  const char* p = reinterpret_cast<const char*>(v.data());
  b.insert(b.end(), p, p + v.size() * sizeof(T));
}
template <class T>
void get(const char*& p, const char* end, std::vector<T>& v, size_t n) {
  if ((size_t)(end - p) < n * sizeof(T)) throw std::invalid_argument("checkpoint truncated");
  v.resize(n);
  std::memcpy(v.data(), p, n * sizeof(T));
  p += n * sizeof(T);
}
std::vector<char> serialize(Ensemble& e) {
  CkptHeader h{kMagic, (uint64_t)e.nchains(), (uint64_t)e.vstride(), (uint64_t)e.tstride(),
               (uint64_t)e.nslots_mt(), (uint64_t)e.nslots_toat(), 0, 0};
  std::vector<double> vl, to, be, eo;
  std::vector<uint32_t> mt, ptmt;
  std::vector<unsigned long long> acc, prop;
  std::vector<int> tc;
  std::vector<double> ptb;
  int isw = 0;
  e.get_vlvr(vl);
  e.get_toat(to);
  e.get_betas(be);
  e.get_eol(eo);
  e.get_mt(mt);
  e.get_acceptance(acc, prop);
  if (e.has_pt()) {
    e.pt_get_state(tc, isw, ptmt, ptb);
    h.npt = tc.size();
    h.iswitch = (uint64_t)isw;
  }
  std::vector<char> b(sizeof h);
  std::memcpy(b.data(), &h, sizeof h);
  put(b, vl);
  put(b, to);
  put(b, be);
  put(b, eo);
  put(b, mt);
  put(b, acc);
  put(b, prop);
  if (h.npt) {
    put(b, tc);
    put(b, ptmt);
    put(b, ptb);
  }
  return b;
}
}  // namespace

extern "C" {

int smmp_ens_checkpoint(smmp_ens_t* e, void* buf, uint64_t* bytes) {
  return guard([&] {
    need(e && bytes, "NULL argument");
    std::vector<char> b = serialize(*e->e);
    if (!buf) {
      *bytes = b.size();
      return;
    }
    need(*bytes >= b.size(), "checkpoint buffer too small");
    std::memcpy(buf, b.data(), b.size());
    *bytes = b.size();
  });
}

int smmp_ens_restore(smmp_ens_t* e, const void* buf, uint64_t bytes) {
  return guard([&] {
    need(e && buf && bytes >= sizeof(CkptHeader), "bad arguments");
    CkptHeader h;
    std::memcpy(&h, buf, sizeof h);
    Ensemble& en = *e->e;
    need(h.magic == kMagic && h.nchains == (uint64_t)en.nchains() &&
             h.vstride == (uint64_t)en.vstride() && h.tstride == (uint64_t)en.tstride() &&
             h.nmt == (uint64_t)en.nslots_mt() && h.ntoat == (uint64_t)en.nslots_toat(),
         "checkpoint does not match this ensemble");
    const char* p = static_cast<const char*>(buf) + sizeof h;
    const char* end = static_cast<const char*>(buf) + bytes;
    std::vector<double> vl, to, be, eo, ptb;
    std::vector<uint32_t> mt, ptmt;
    std::vector<unsigned long long> acc, prop;
    std::vector<int> tc;
    get(p, end, vl, h.nchains * h.vstride);
    get(p, end, to, h.ntoat * h.tstride);
    get(p, end, be, h.nchains);
    get(p, end, eo, h.nchains);
    get(p, end, mt, h.nmt * kMTWords);
    get(p, end, acc, h.nchains);
    get(p, end, prop, h.nchains);
    en.set_vlvr(vl);
    en.set_toat(to);
    en.set_betas(be);
    en.set_mt(mt);
    en.set_acceptance(acc, prop);
    if (h.npt) {
      need(en.has_pt(), "checkpoint holds a PT state; call smmp_ens_set_pt first");
      get(p, end, tc, h.npt);
      get(p, end, ptmt, kMTWords);
      get(p, end, ptb, h.npt);
      en.pt_set_state(tc, (int)h.iswitch, ptmt, ptb);
    }
    (void)eo;
  });
}

}  // extern "C"

// ============================================================================ surrogate

struct smmp_sur {
  std::unique_ptr<Surrogate> s;
};

extern "C" {

smmp_sur_t* smmp_sur_create(int nang, uint64_t seed) {
  smmp_sur_t* out = nullptr;
  int rc = guard([&] {
    need(nang > 0, "smmp_sur_create: nang must be positive");
    auto h = std::make_unique<smmp_sur>();
    h->s.reset(new Surrogate(nang, seed));
    out = h.release();
  });
  return rc == SMMP_OK ? out : nullptr;
}

void smmp_sur_free(smmp_sur_t* s) { delete s; }

int smmp_sur_sizes(smmp_sur_t* s, int* nin, int* nin_pad, int64_t* nparams) {
  return guard([&] {
    need(s != nullptr, "null surrogate");
    if (nin) *nin = s->s->layout().nin;
    if (nin_pad) *nin_pad = s->s->layout().nin_pad;
    if (nparams) *nparams = (int64_t)s->s->layout().n;
  });
}

int smmp_sur_set_data(smmp_sur_t* s, const double* ang, const double* energy, int n, double clip) {
  return guard([&] {
    need(s && ang && energy && n > 0, "smmp_sur_set_data: bad arguments");
    s->s->set_data(ang, energy, n, clip);
  });
}

int smmp_sur_train(smmp_sur_t* s, int epochs, int batch, double lr, uint64_t shuffle_seed,
                   double* loss) {
  return guard([&] {
    need(s != nullptr, "null surrogate");
    double l = s->s->train(epochs, batch, lr, shuffle_seed);
    if (loss) *loss = l;
  });
}

int smmp_sur_predict(smmp_sur_t* s, const double* ang, int n, double* energy_out) {
  return guard([&] {
    need(s && ang && energy_out && n >= 0, "smmp_sur_predict: bad arguments");
    if (n > 0) s->s->predict(ang, n, energy_out);
  });
}

int smmp_sur_gradients(smmp_sur_t* s, const double* ang, const double* energy, int n,
                       float* grad_out, double* loss) {
  return guard([&] {
    need(s && ang && energy && grad_out && n > 0, "smmp_sur_gradients: bad arguments");
    double l = s->s->gradients(ang, energy, n, grad_out);
    if (loss) *loss = l;
  });
}

int smmp_sur_get_params(smmp_sur_t* s, float* params, float* norm) {
  return guard([&] {
    need(s != nullptr, "null surrogate");
    if (params) s->s->get_params(params);
    if (norm) {
      norm[0] = s->s->mu();
      norm[1] = s->s->sigma();
    }
  });
}

int smmp_sur_predict_noalloc(smmp_sur_t* s, const float* ang_dev, int n, double* energy_dev,
                             void* stream) {
  return guard([&] {
    need(s && ang_dev && energy_dev && n >= 0, "smmp_sur_predict_noalloc: bad arguments");
    s->s->predict_noalloc(ang_dev, n, energy_dev, static_cast<cudaStream_t>(stream));
  });
}

int smmp_ens_set_surrogate(smmp_ens_t* e, smmp_sur_t* s, double floor, int min_stage1) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    if (s) {
      DSurrogate v = s->s->device_view();
      e->e->set_surrogate(&v, (float)floor, min_stage1);
    } else {
      e->e->set_surrogate(nullptr, 0.f, 0);
    }
  });
}

int smmp_ens_autotune(smmp_ens_t* e, int* choice, double* ms) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    double t[3];
    int c = e->e->autotune(e->flags & (kFlagFP32 | kFlagRndOrd), t);
    if (choice) *choice = c;
    if (ms) {
      ms[0] = t[0];
      ms[1] = t[1];
      ms[2] = t[2];
    }
  });
}

int smmp_ens_set_window(smmp_ens_t* e, int window, int* applied) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    need(window >= 1, "window must be at least 1");
    const int k = e->e->set_window(window);
    if (applied) *applied = k;
  });
}

int smmp_ens_window(smmp_ens_t* e, int* window, double* ms) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    if (window) *window = e->e->window();
    if (ms)
      for (int k = 0; k < 3; ++k) ms[k] = e->e->window_ms()[k];
  });
}

int smmp_ens_set_pair_work(smmp_ens_t* e, int form) {
  return guard([&] {
    need(e != nullptr, "NULL ensemble");
    need(form >= 0 && form <= 2, "pair-work form must be 0, 1 or 2");
    e->e->set_pair_work(form);
  });
}

int smmp_ens_da_stats(smmp_ens_t* e, uint64_t* stage1, uint64_t* stage2) {
  return guard([&] {
    need(e && stage1 && stage2, "NULL argument");
    std::vector<unsigned long long> a, b;
    e->e->da_stats(a, b);
    for (size_t c = 0; c < a.size(); ++c) {
      stage1[c] = a[c];
      stage2[c] = b[c];
    }
  });
}

int smmp_sur_set_params(smmp_sur_t* s, const float* params, const float* norm) {
  return guard([&] {
    need(s != nullptr, "null surrogate");
    if (params) s->s->set_params(params);
    if (norm) {
      need(norm[1] > 0.f, "smmp_sur_set_params: sigma must be positive");
      s->s->set_norm(norm[0], norm[1]);
    }
  });
}

}  // extern "C"
