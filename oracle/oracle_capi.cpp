// C entry points of the CPU oracle -- TEST INFRASTRUCTURE ONLY (tests/,
// smoke() and the CPU-baseline leg of bench.py load this through ctypes).
#include <chrono>
#include <cmath>
#include <cstring>
#include <algorithm>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <vector>

#include "smmp_oracle.hpp"

using oracle::Smmp;

namespace {
thread_local std::string g_err;
template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}
Smmp* S(void* h) { return static_cast<Smmp*>(h); }
int ntlvr(Smmp* s) { return s->ivrml1[s->ntlml] + s->nvrml[s->ntlml] - 1; }
}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_create(const char* libdir, int sh2, int epsd, int itysol) {
  auto s = std::make_unique<Smmp>();
  s->sh2 = sh2 != 0;
  s->epsd = epsd != 0;
  s->itysol = itysol;
  if (guard([&] { s->init_energy(libdir); })) return nullptr;
  return s.release();
}

void* orc_clone(void* h) { return new Smmp(*S(h)); }
void orc_destroy(void* h) { delete S(h); }

int orc_init_molecule(void* h, const char* seq, const char* var, const char* grpn,
                      const char* grpc) {
  return guard([&] { S(h)->init_molecule(seq, var ? var : " ", grpn, grpc); });
}

// Sizes: [natoms, ntlvr (all variables), nvr (free variables), nres,
//         nvw (vdW domains), n14 (1-4 partners), nms (moving sets)].
void orc_sizes(void* h, int* out) {
  Smmp* s = S(h);
  int n = s->ntlml;
  out[0] = s->iatrs2[s->irsml2[n]];
  out[1] = ntlvr(s);
  out[2] = s->nvr;
  out[3] = s->irsml2[n];
  out[4] = s->ivwml1[n] + s->nvwml[n] - 1;
  out[5] = s->i14ml1[n] + s->n14ml[n] - 1;
  out[6] = s->imsml1[n] + s->nmsml[n] - 1;
}

// Energy of the current variables; terms = [eyel, eyvw, eyhb, eyvr, eysl, eysm].
int orc_energy(void* h, double* e, double* terms) {
  Smmp* s = S(h);
  return guard([&] {
    *e = s->energy();
    if (terms) {
      terms[0] = s->eyel;
      terms[1] = s->eyvw;
      terms[2] = s->eyhb;
      terms[3] = s->eyvr;
      terms[4] = s->eysl;
      terms[5] = s->eysm;
    }
  });
}

void orc_get_vlvr(void* h, double* out) {
  Smmp* s = S(h);
  for (int i = 1; i <= ntlvr(s); ++i) out[i - 1] = s->vlvr[i];
}
void orc_set_vlvr(void* h, const double* in) {
  Smmp* s = S(h);
  for (int i = 1; i <= ntlvr(s); ++i) s->vlvr[i] = in[i - 1];
}
void orc_get_idvr(void* h, int* out) {
  Smmp* s = S(h);
  for (int i = 1; i <= s->nvr; ++i) out[i - 1] = s->idvr[i];
}
void orc_get_axvr(void* h, double* out) {
  Smmp* s = S(h);
  for (int i = 1; i <= ntlvr(s); ++i) out[i - 1] = s->axvr[i];
}
void orc_get_coords(void* h, double* xyz) {
  Smmp* s = S(h);
  int na = s->iatrs2[s->irsml2[s->ntlml]];
  for (int i = 1; i <= na; ++i) {
    xyz[3 * (i - 1) + 0] = s->xat(i);
    xyz[3 * (i - 1) + 1] = s->yat(i);
    xyz[3 * (i - 1) + 2] = s->zat(i);
  }
}
// Internal state that the rebuild reads: toat (per atom).
void orc_get_toat(void* h, double* out) {
  Smmp* s = S(h);
  int na = s->iatrs2[s->irsml2[s->ntlml]];
  for (int i = 1; i <= na; ++i) out[i - 1] = s->toat[i];
}

// Topology and interaction lists, 1-based values as in the reference arrays.
//   atom_i:  per atom [ityat, iowat, nbdat, ibdat1, ibdat2, ibdat3, ixmsat,
//                      ivwat1, ivwat2, i14at1, i14at2]          (11 ints)
//   atom_d:  per atom [cgat, blat, baat, toat]                 (4 doubles)
//   var_i:   per variable [iatvr, ityvr, iclvr, iorvr, imsvr1, imsvr2,
//                          iadvr1, iadvr2, fxvr]               (9 ints)
//   ms:      per moving set [latms1, latms2]
//   vw:      per vdW domain [lvwat1, lvwat2, ixatvw]
//   l14:     per 1-4 entry  [l14at, ixat14]
void orc_get_topology(void* h, int* atom_i, double* atom_d, int* var_i, int* ms, int* vw,
                      int* l14) {
  Smmp* s = S(h);
  int sz[7];
  orc_sizes(h, sz);
  for (int i = 1; i <= sz[0]; ++i) {
    int* a = atom_i + 11 * (i - 1);
    a[0] = s->ityat[i];
    a[1] = s->iowat[i];
    a[2] = s->nbdat[i];
    a[3] = s->IBD(1, i);
    a[4] = s->IBD(2, i);
    a[5] = s->IBD(3, i);
    a[6] = s->ixmsat[i];
    a[7] = s->ivwat1[i];
    a[8] = s->ivwat2[i];
    a[9] = s->i14at1[i];
    a[10] = s->i14at2[i];
    double* d = atom_d + 4 * (i - 1);
    d[0] = s->cgat[i];
    d[1] = s->blat[i];
    d[2] = s->baat[i];
    d[3] = s->toat[i];
  }
  for (int i = 1; i <= sz[1]; ++i) {
    int* v = var_i + 9 * (i - 1);
    v[0] = s->iatvr[i];
    v[1] = s->ityvr[i];
    v[2] = s->iclvr[i];
    v[3] = s->iorvr[i];
    v[4] = s->imsvr1[i];
    v[5] = s->imsvr2[i];
    v[6] = s->iadvr1[i];
    v[7] = s->iadvr2[i];
    v[8] = s->fxvr[i];
  }
  for (int i = 1; i <= sz[6]; ++i) {
    ms[2 * (i - 1)] = s->latms1[i];
    ms[2 * (i - 1) + 1] = s->latms2[i];
  }
  for (int i = 1; i <= sz[4]; ++i) {
    vw[3 * (i - 1)] = s->lvwat1[i];
    vw[3 * (i - 1) + 1] = s->lvwat2[i];
    vw[3 * (i - 1) + 2] = s->ixatvw[i];
  }
  for (int i = 1; i <= sz[5]; ++i) {
    l14[2 * (i - 1)] = s->l14at[i];
    l14[2 * (i - 1) + 1] = s->ixat14[i];
  }
}

// Atom names (4 chars each, no terminator) and variable names (3 chars each).
void orc_get_names(void* h, char* atoms, char* vars) {
  Smmp* s = S(h);
  int sz[7];
  orc_sizes(h, sz);
  for (int i = 1; i <= sz[0]; ++i) std::memcpy(atoms + 4 * (i - 1), s->nmat[i].data(), 4);
  for (int i = 1; i <= sz[1]; ++i) std::memcpy(vars + 3 * (i - 1), s->nmvr[i].data(), 3);
}

void orc_set_beta(void* h, double beta) { S(h)->beta = beta; }
void orc_set_rndord(void* h, int r) { S(h)->rndord = r != 0; }
void orc_sgrnd(void* h, int seed) { S(h)->sgrnd(seed); }
double orc_grnd(void* h) { return S(h)->grnd(); }
void orc_get_mt(void* h, unsigned* state, int* mti) {
  std::memcpy(state, S(h)->mt, sizeof(S(h)->mt));
  *mti = S(h)->mti;
}

// Canonical random start (canon.f:60-67): vlvr(idvr(i)) = addang(pi, axvr*(grnd()-0.5)).
void orc_random_start(void* h) {
  Smmp* s = S(h);
  for (int i = 1; i <= s->nvr; ++i) {
    int iv = s->idvr[i];
    double dv = s->axvr[iv] * (s->grnd() - 0.5);
    s->vlvr[iv] = oracle::addang(3.141592653589793, dv);
  }
}

// nsweeps calls of metropolis with the canonical weight at s->beta.  If
// accept_log is given, it receives one byte per proposal (1 = accepted).
int orc_sweeps(void* h, int nsweeps, double* eol, double* acz, unsigned char* accept_log) {
  Smmp* s = S(h);
  return guard([&] {
    Smmp::Weight w;
    for (int k = 0; k < nsweeps; ++k) {
      long long before = s->nacalls;
      long long cbefore = s->ncalls;
      if (accept_log) {
        // replay the sweep proposal by proposal to record decisions
        std::vector<double> vrol(s->vlvr);
        double e = s->energy();
        for (int nsw = 1; nsw <= s->nvr; ++nsw) {
          int ivar = s->rndord ? 1 + int(s->nvr * s->grnd()) : nsw;
          int jv = s->idvr[ivar];
          vrol = s->vlvr;
          double dv = s->axvr[jv] * (s->grnd() - 0.5);
          s->vlvr[jv] = oracle::addang(vrol[jv], dv);
          double enw = s->energy();
          double delta = s->weight(w, enw) - s->weight(w, e);
          int up = 0;
          if (delta <= 0.0) {
            e = enw;
            up = 1;
          } else {
            double rd = s->grnd();
            delta = std::min(delta, 100.0);
            if (std::exp(-delta) >= rd) {
              e = enw;
              up = 1;
            } else {
              s->vlvr = vrol;
            }
          }
          *acz += up;
          ++s->ncalls;
          s->nacalls += up;
          accept_log[(size_t)k * s->nvr + (nsw - 1)] = (unsigned char)up;
        }
        double enw = s->energy();
        if (std::fabs(e - enw) > 0.000001 && e < 100000)
          throw std::runtime_error("metropolis: eol and enw difference unacceptable");
        *eol = e;
      } else {
        s->metropolis(*eol, *acz, w);
      }
      (void)before;
      (void)cbefore;
    }
  });
}

// Simulated annealing driver (anneal.f:13-152): random start, nequi sweeps at
// 1/tmax, then nswp+1 sweeps with beta = bmin*db**nsw.  out = [start energy,
// energy after equilibration, acceptance, last energy, lowest energy,
// sweep of lowest energy].
int orc_anneal(void* h, int nequi, int nswp, double tmax, double tmin, int lrand, double* out) {
  Smmp* s = S(h);
  return guard([&] {
    Smmp::Weight w;
    double bmin = 1.0 / (tmax * 1.98773e-3);
    double bmax = 1.0 / (tmin * 1.98773e-3);
    double db = std::exp(std::log(bmax / bmin) / nswp);
    if (lrand) orc_random_start(h);
    double eol = s->energy();
    out[0] = eol;
    s->beta = bmin;
    double acz = 0.0;
    for (int nsw = 1; nsw <= nequi; ++nsw) s->metropolis(eol, acz, w);
    out[1] = eol;
    acz = 0.0;
    double ymin = eol;
    int nemin = 0;
    int nsw;
    for (nsw = 0; nsw <= nswp; ++nsw) {
      s->beta = bmin * std::pow(db, nsw);
      s->metropolis(eol, acz, w);
      if (eol < ymin) {
        ymin = eol;
        nemin = nsw;
      }
    }
    out[2] = acz / double(nsw * s->nvr);
    out[3] = eol;
    out[4] = ymin;
    out[5] = nemin;
  });
}

// Serial parallel tempering (partem_s.f:13-258, newsta=.true., switch=1):
// betas[num_rep] (index k = temperature label), one shared MT stream.
// eol_out[num_rep] per replica, ipoi_out[num_rep] final temperature->replica
// map, vl_out[num_rep*nvr] final free variables of each replica.
int orc_partem(void* h, int num_rep, const double* betas, int nequi, int nswp, double* eol_out,
               int* ipoi_out, double* vl_out) {
  Smmp* s = S(h);
  return guard([&] {
    Smmp::Weight w;
    int nvr = s->nvr;
    const double pi = 3.141592653589793;
    std::vector<double> coor((size_t)nvr * num_rep), eol(num_rep + 1), acc(num_rep + 1);
    std::vector<int> ipoi(num_rep + 1);
    for (int j = 1; j <= num_rep; ++j) ipoi[j] = j;
    for (int i = 1; i <= num_rep; ++i)
      for (int j = 1; j <= nvr; ++j) {
        int iv = s->idvr[j];
        double dv = s->axvr[iv] * (s->grnd() - 0.5);
        coor[(size_t)(i - 1) * nvr + (j - 1)] = oracle::addang(pi, dv);
      }
    for (int k = 1; k <= num_rep; ++k) {
      s->beta = betas[k - 1];
      for (int i = 1; i <= nvr; ++i) s->vlvr[s->idvr[i]] = coor[(size_t)(k - 1) * nvr + i - 1];
      double energ = s->energy();
      double acz = 0.0;
      for (int nsw = 1; nsw <= nequi; ++nsw) s->metropolis(energ, acz, w);
      for (int i = 1; i <= nvr; ++i) coor[(size_t)(k - 1) * nvr + i - 1] = s->vlvr[s->idvr[i]];
      eol[k] = energ;
    }
    int iswitch = 1;
    for (int nsw = 1; nsw <= nswp; ++nsw) {
      for (int k1 = 1; k1 <= num_rep; ++k1) {
        int k = ipoi[k1];
        s->beta = betas[k1 - 1];
        double energ = eol[k];
        double acz = acc[k];
        for (int i = 1; i <= nvr; ++i) s->vlvr[s->idvr[i]] = coor[(size_t)(k - 1) * nvr + i - 1];
        s->setvar(1, s->vlvr.data());
        s->metropolis(energ, acz, w);
        for (int i = 1; i <= nvr; ++i) coor[(size_t)(k - 1) * nvr + i - 1] = s->vlvr[s->idvr[i]];
        eol[k] = energ;
        acc[k] = acz;
      }
      if (!(num_rep > 1)) continue;
      int num_rep1, nu;
      if (iswitch == 1) {
        num_rep1 = num_rep - 1;
        nu = 1;
        iswitch = 2;
      } else {
        num_rep1 = num_rep;
        nu = 2;
        iswitch = 1;
      }
      for (int i = nu; i <= num_rep1; i += 2) {
        int j = i + 1;
        if (i == num_rep) j = 1;
        int in = ipoi[i], jn = ipoi[j];
        double delta = -betas[i - 1] * eol[jn] - betas[j - 1] * eol[in] + betas[i - 1] * eol[in] +
                       betas[j - 1] * eol[jn];
        double ra = s->grnd();
        if (ra <= std::exp(delta)) {
          ipoi[i] = jn;
          ipoi[j] = in;
        }
      }
    }
    for (int k = 1; k <= num_rep; ++k) {
      eol_out[k - 1] = eol[k];
      ipoi_out[k - 1] = ipoi[k];
      for (int i = 0; i < nvr; ++i) vl_out[(size_t)(k - 1) * nvr + i] = coor[(size_t)(k - 1) * nvr + i];
    }
  });
}

}  // extern "C"

namespace {

// A reusable barrier for the chain threads of one PT ensemble.
class RoundBarrier {
 public:
  explicit RoundBarrier(int n) : n_(n) {}
  void wait() {
    std::unique_lock<std::mutex> lk(m_);
    const unsigned gen = gen_;
    if (++count_ == n_) {
      count_ = 0;
      ++gen_;
      cv_.notify_all();
    } else {
      cv_.wait(lk, [&] { return gen_ != gen; });
    }
  }

 private:
  std::mutex m_;
  std::condition_variable cv_;
  int n_, count_ = 0;
  unsigned gen_ = 0;
};

// Batched parallel tempering as the product's batched mode defines it (no
// counterpart routine in the reference; its exchange step is partem_s.f:
// 210-232): chain c is a copy of the system with its own stream
// sgrnd(seeds[c]) and a canonical random start (canon.f:60-67); a round is
// one metropolis sweep of every chain at the inverse temperature of its
// label, then one exchange step over the labels with alternating parity,
// drawing from a separate stream sgrnd(exchange_seed) once per pair in pair
// order, the periodic pair (n, 1) only when wrap.  Chains sweep on nthreads
// host threads (they share nothing); the state persists between calls.
struct BatchedPT {
  std::vector<std::unique_ptr<Smmp>> ch;
  std::unique_ptr<Smmp> ex;
  std::vector<double> betas, eol, acz;
  std::vector<int> ipoi;   // chain (0-based) at label k (1-based)
  std::vector<unsigned long long> stats;
  int n = 0, wrap = 0, iswitch = 1, nthreads = 1, exchanges = 1;

  void exchange() {
    if (n < 2 || !exchanges) return;
    int num_rep1, nu;
    if (iswitch == 1) {
      num_rep1 = n - 1;
      nu = 1;
      iswitch = 2;
    } else {
      num_rep1 = n;
      nu = 2;
      iswitch = 1;
    }
    for (int i = nu; i <= num_rep1; i += 2) {
      if (i == n && !wrap) continue;
      const int j = (i == n) ? 1 : i + 1;
      const int in = ipoi[i], jn = ipoi[j];
      const double bi = betas[i - 1], bj = betas[j - 1];
      const double delta = -bi * eol[jn] - bj * eol[in] + bi * eol[in] + bj * eol[jn];
      const double ra = ex->grnd();
      stats[2 * (i - 1)] += 1;
      if (ra <= std::exp(delta)) {
        ipoi[i] = jn;
        ipoi[j] = in;
        stats[2 * (i - 1) + 1] += 1;
      }
    }
  }

  // nrounds rounds; after each, `each(r)` on the calling thread's side.
  template <class F>
  void run(int nrounds, F each) {
    const int nt = std::max(1, std::min(nthreads, n));
    RoundBarrier bar(nt + 1);
    std::vector<std::string> errs(nt);
    std::atomic<bool> stop{false};
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
      th.emplace_back([&, t] {
        Smmp::Weight w;
        for (int r = 0; r < nrounds; ++r) {
          bar.wait();   // betas set
          if (!stop)
            try {
              for (int c = t; c < n; c += nt) ch[c]->metropolis(eol[c], acz[c], w);
            } catch (const std::exception& e) {
              errs[t] = e.what();
              stop = true;
            }
          bar.wait();   // sweeps done
        }
      });
    std::string err;
    for (int r = 0; r < nrounds; ++r) {
      for (int k = 1; k <= n; ++k) ch[ipoi[k]]->beta = betas[k - 1];
      bar.wait();
      bar.wait();
      for (auto& e : errs)
        if (!e.empty() && err.empty()) err = e;
      if (!err.empty()) continue;
      exchange();
      each(r);
    }
    for (auto& x : th) x.join();
    if (!err.empty()) throw std::runtime_error(err);
  }
};

}  // namespace

extern "C" {

// exchange = 0: independent canonical chains (rounds are sweeps only).
void* orc_pt_create(void* h, int n, const double* betas, const int* seeds, int exchange_seed,
                    int wrap, int nthreads, int exchange) {
  try {
    auto* p = new BatchedPT;
    p->exchanges = exchange;
    p->n = n;
    p->wrap = wrap;
    p->nthreads = nthreads;
    for (int c = 0; c < n; ++c) {
      p->ch.emplace_back(new Smmp(*S(h)));
      p->ch[c]->sgrnd(seeds[c]);
      orc_random_start(p->ch[c].get());
    }
    p->ex.reset(new Smmp(*S(h)));
    p->ex->sgrnd(exchange_seed);
    p->betas.assign(betas, betas + n);
    p->eol.assign(n, 0.0);
    p->acz.assign(n, 0.0);
    p->ipoi.assign(n + 1, 0);
    for (int k = 1; k <= n; ++k) p->ipoi[k] = k - 1;
    p->stats.assign(2 * n, 0);
    return p;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void orc_pt_free(void* p) { delete static_cast<BatchedPT*>(p); }

// nrounds rounds of a batched PT ensemble; returns the wall time in seconds
// (negative on error: orc_last_error).
double orc_pt_run(void* p, int nrounds) {
  auto* pt = static_cast<BatchedPT*>(p);
  try {
    auto t0 = std::chrono::steady_clock::now();
    pt->run(nrounds, [](int) {});
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1.0;
  }
}

// Per round r (0-based) of a fresh batched PT run: tc_hist[r*n+k] = chain at
// label k (0-based) after the exchange, eol_hist[r*n+c] = energy of chain c,
// vl_hist[(r*n+c)*nvr+i] = its free variables; stats[2k] / [2k+1] =
// attempts / accepts of label pair (k, k+1).
int orc_partem_batched(void* h, int n, const double* betas, const int* seeds, int exchange_seed,
                       int wrap, int nrounds, int nthreads, int* tc_hist, double* eol_hist,
                       double* vl_hist, unsigned long long* stats) {
  return guard([&] {
    std::unique_ptr<BatchedPT> pt(
        static_cast<BatchedPT*>(orc_pt_create(h, n, betas, seeds, exchange_seed, wrap, nthreads, 1)));
    if (!pt) throw std::runtime_error(g_err);
    const int nvr = S(h)->nvr;
    pt->run(nrounds, [&](int r) {
      for (int k = 1; k <= n; ++k) tc_hist[(size_t)r * n + (k - 1)] = pt->ipoi[k];
      for (int c = 0; c < n; ++c) {
        eol_hist[(size_t)r * n + c] = pt->eol[c];
        for (int i = 1; i <= nvr; ++i)
          vl_hist[((size_t)r * n + c) * nvr + (i - 1)] = pt->ch[c]->vlvr[pt->ch[c]->idvr[i]];
      }
    });
    for (int k = 0; k < 2 * n; ++k) stats[k] = pt->stats[k];
  });
}

// CPU baseline: nchains independent canonical chains (each a copy of h with
// its own MT seed seeds[c] and beta betas[c]) run for nsweeps sweeps from
// their current variables, spread over nthreads host threads.  Returns the
// wall time in seconds; energies in eol_out[nchains].
double orc_bench_chains(void* h, int nchains, const int* seeds, const double* betas, int nsweeps,
                        int nthreads, double* eol_out) {
  std::vector<std::unique_ptr<Smmp>> chains;
  for (int c = 0; c < nchains; ++c) {
    chains.emplace_back(new Smmp(*S(h)));
    chains.back()->sgrnd(seeds[c]);
    chains.back()->beta = betas[c];
  }
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> th;
  if (nthreads < 1) nthreads = 1;
  for (int t = 0; t < nthreads; ++t)
    th.emplace_back([&, t] {
      Smmp::Weight w;
      for (int c = t; c < nchains; c += nthreads) {
        Smmp* s = chains[c].get();
        double eol = s->energy(), acz = 0.0;
        try {
          for (int k = 0; k < nsweeps; ++k) s->metropolis(eol, acz, w);
        } catch (...) {
          eol = NAN;
        }
        eol_out[c] = eol;
      }
    });
  for (auto& t : th) t.join();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Test hook (not a reference routine): turn every atom's valence angle by a
// pseudo-random amount in [-amp, amp] radians, so that geometric checks on
// the rebuilt molecule meet no collinear atoms (a para ring atom on its
// ring's rotation axis keeps its distances under that rotation).
void orc_perturb_valence(void* h, unsigned seed, double amp) {
  Smmp* s = S(h);
  int na = s->iatrs2[s->irsml2[s->ntlml]];
  unsigned long long x = 0x9E3779B97F4A7C15ull ^ seed;
  for (int i = 1; i <= na; ++i) {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    const double u = (double)(x >> 11) / 9007199254740992.0;   // [0, 1)
    s->baat[i] += amp * (2.0 * u - 1.0);
    s->csbaat[i] = std::cos(s->baat[i]);
    s->snbaat[i] = std::sin(s->baat[i]);
  }
}

// gradient.f: energy (vacuum) and dE/dvlvr of every variable (grad[ntlvr]).
int orc_gradient(void* h, double* e, double* grad) {
  Smmp* s = S(h);
  return guard([&] {
    *e = s->gradient();
    for (int i = 1; i <= ntlvr(s); ++i) grad[i - 1] = s->gdeyvr[i];
  });
}

// The order-free form of the same derivatives (total atomic forces, sums
// over each variable's moved atoms), for tests of that formulation.
int orc_gradient_by_sums(void* h, double* grad) {
  Smmp* s = S(h);
  return guard([&] {
    std::vector<double> gd;
    s->gradient_by_sums(1, gd);
    for (int i = 1; i <= ntlvr(s); ++i) grad[i - 1] = gd[i];
  });
}

// mulcan_par_mod.f90 weight recursion (see muca_update / muca_finish).
// canon.f:12-132 (without its output files): beta from temp, a random
// start when lrand, nequi sweeps, then sweeps nsw = 0..nswp with the energy
// recorded when mod(nsw, nmes) == 0.  out = [energy after equilibration,
// acceptance rate, last energy].
int orc_canon(void* h, int nequi, int nswp, int nmes, double temp, int lrand, double* trace,
              double* out) {
  Smmp* s = S(h);
  return guard([&] {
    Smmp::Weight w;
    s->beta = 1.0 / (temp * 1.98773e-3);
    if (lrand) orc_random_start(h);
    double eol = s->energy(), acz = 0.0;
    for (int k = 1; k <= nequi; ++k) s->metropolis(eol, acz, w);
    out[0] = eol;
    acz = 0.0;
    int m = 0, nsw = 0;
    for (nsw = 0; nsw <= nswp; ++nsw) {
      s->metropolis(eol, acz, w);
      if (nsw % nmes == 0) trace[m++] = eol;
    }
    out[1] = acz / (double)(nsw * s->nvr);
    out[2] = eol;
  });
}

// nsweeps metropolis sweeps with a multicanonical weight (kind 1:
// muca_weight, 2: muca_weight2; mulcan_par_mod.f90:380-410) over the bins
// kmin..kmax of width ebin; eol and acz in/out as metropolis's arguments.
int orc_sweeps_muca(void* h, int nsweeps, int kind, int kmin, int kmax, double ebin,
                    const double* b, const double* alpha, double* eol, double* acz) {
  Smmp* s = S(h);
  return guard([&] {
    Smmp::Weight w;
    w.kind = kind == 1 ? Smmp::W_MUCA : Smmp::W_MUCA2;
    w.kmin = kmin;
    w.kmax = kmax;
    w.ebin = ebin;
    w.b = b;
    w.alpha = alpha;
    for (int k = 0; k < nsweeps; ++k) s->metropolis(*eol, *acz, w);
  });
}

// mulcan_par (mulcan_par_mod.f90:23-190, without its files): beta from temp,
// random start, nsweep sweeps with muca_weight, the histogram of each sweep's
// energy bin, the weights updated every nup sweeps, and at the end beta
// folded into b (muca_weight2's table).  b_out, alpha_out: [kmax-kmin+1];
// out = [acceptance, last energy].
int orc_mulcan_par(void* h, int nsweep, int nup, double temp, int kmin, int kmax, double ebin,
                   double* b_out, double* alpha_out, double* out) {
  Smmp* s = S(h);
  return guard([&] {
    const int nb = kmax - kmin + 1;
    const double beta = 1.0 / (temp * 1.98773e-3);
    s->beta = beta;
    std::vector<double> xhist(nb, 0.0), g1(nb, 0.0), b(nb, 0.0), alpha(nb, 0.0), ent(nb, 0.0);
    std::vector<int> ihist(nb, 0);
    orc_random_start(h);
    double eol = s->energy(), acz = 0.0;
    Smmp::Weight w;
    w.kind = Smmp::W_MUCA;
    w.kmin = kmin;
    w.kmax = kmax;
    w.ebin = ebin;
    w.b = b.data();
    w.alpha = alpha.data();
    for (int nsw = 1; nsw <= nsweep; ++nsw) {
      s->metropolis(eol, acz, w);
      const double x = eol / ebin + std::copysign(0.5, eol);
      const int muold = (int)std::min((double)kmax, std::max((double)kmin, x));
      ihist[muold - kmin] += 1;
      if (nsw % nup == 0)
        oracle::muca_update(kmin, kmax, ebin, beta, ihist.data(), xhist.data(), g1.data(),
                            b.data(), alpha.data(), ent.data());
    }
    out[0] = acz / (double)((nsweep + 1) * s->nvr);
    out[1] = eol;
    oracle::muca_finish(kmin, kmax, ebin, beta, b.data(), alpha.data());
    for (int k = 0; k < nb; ++k) {
      b_out[k] = b[k];
      alpha_out[k] = alpha[k];
    }
  });
}

// enysol.f:13-339: the numerical solvation energy of the current coordinates
// (after an energy() call), molecule nmol (0: all).
int orc_enysol(void* h, int nmol, double* eysl) {
  Smmp* s = S(h);
  return guard([&] { *eysl = s->enysol(nmol); });
}

// enysol.f:107-330 over n arbitrary spheres (xyz[3n], radii r[n], sigma[n]),
// with the unit-sphere points of the file tes (tessel, enysol.f:341-365):
// counts[k] = exposed points of sphere k (-1 for r <= 0), areas[k], and
// eysl = sum sigma_k areas_k in the reference's order; returns asa.
int orc_enysol_spheres(int n, const double* xyz, const double* r, const double* sigma,
                       const char* tes, int* counts, double* areas, double* eysl, double* asa) {
  return guard([&] {
    Smmp pts;
    pts.tessel(tes);
    std::vector<double> x(n + 1), y(n + 1), z(n + 1), rv(n + 1);
    for (int k = 1; k <= n; ++k) {
      x[k] = xyz[3 * (k - 1)];
      y[k] = xyz[3 * (k - 1) + 1];
      z[k] = xyz[3 * (k - 1) + 2];
      rv[k] = r[k - 1];
      counts[k - 1] = -1;
      areas[k - 1] = 0.0;
    }
    double e = 0.0, vol = 0.0;
    oracle::enysol_spheres(n, x.data(), y.data(), z.data(), rv.data(), pts.spoint.data(), pts.npnt,
                           *asa, vol, [&](int k, double area, int icount) {
                             counts[k - 1] = icount;
                             areas[k - 1] = area;
                             e = e + area * sigma[k - 1];
                           });
    *eysl = e;
  });
}

// Solvation radii (rvdw, probe included) and coefficients of every atom.
void orc_get_solvation(void* h, double* rvdw, double* sigma) {
  Smmp* s = S(h);
  int na = s->iatrs2[s->irsml2[s->ntlml]];
  for (int i = 1; i <= na; ++i) {
    rvdw[i - 1] = s->rvdw[i];
    sigma[i - 1] = s->sigma[i];
  }
}

int orc_muca_update(int kmin, int kmax, double ebin, double beta, int* ihist, double* xhist,
                    double* g1, double* b, double* alpha, double* ent) {
  return guard([&] { oracle::muca_update(kmin, kmax, ebin, beta, ihist, xhist, g1, b, alpha, ent); });
}
int orc_muca_finish(int kmin, int kmax, double ebin, double beta, double* b, double* alpha) {
  return guard([&] { oracle::muca_finish(kmin, kmax, ebin, beta, b, alpha); });
}

// Atoms moved by each variable (1-based atoms of the first molecule):
// counts[v] atoms listed from atoms[offsets[v]]; offsets has ntlvr+1 entries
// and atoms room for cap entries.
int orc_moved_atoms(void* h, int* offsets, int* atoms, int cap) {
  Smmp* s = S(h);
  return guard([&] {
    const auto moved = s->moved_atoms(1);
    int k = 0;
    for (int v = 1; v <= ntlvr(s); ++v) {
      offsets[v - 1] = k;
      for (int a : moved[v]) {
        if (k >= cap) throw std::runtime_error("orc_moved_atoms: capacity");
        atoms[k++] = a;
      }
    }
    offsets[ntlvr(s)] = k;
  });
}

// Bond-axis frame vectors xtoat/ytoat/ztoat of every atom (3 per atom).
void orc_get_frames(void* h, double* f) {
  Smmp* s = S(h);
  int na = s->iatrs2[s->irsml2[s->ntlml]];
  for (int i = 1; i <= na; ++i) {
    f[3 * (i - 1)] = s->xtoat[i];
    f[3 * (i - 1) + 1] = s->ytoat[i];
    f[3 * (i - 1) + 2] = s->ztoat[i];
  }
}

// minim.f (quasi-Newton, no regularisation): *nop function calls; log
// receives up to logcap (energy, |grad|^2) pairs, *nlog the number of pairs.
int orc_minim(void* h, int imin, int maxit, double eps, int* nop, double* log, int logcap,
              int* nlog) {
  Smmp* s = S(h);
  return guard([&] {
    std::vector<double> lg;
    *nop = s->minim(imin, maxit, eps, &lg);
    const int np = (int)lg.size() / 2;
    *nlog = np;
    for (int k = 0; k < std::min(np, logcap); ++k) {
      log[2 * k] = lg[2 * k];
      log[2 * k + 1] = lg[2 * k + 1];
    }
  });
}

// esolan.f area arithmetic on n free spheres (0-based xyz[3n], radii r[n]
// with the probe already added): areas[n] and the return value sum_i A_i.
// Re-orientation angles come from a stream seeded with `seed`.
int orc_esolan_spheres(int n, const double* xyz, const double* r, int seed, double* areas,
                       double* total) {
  return guard([&] {
    std::vector<double> x(n + 1), y(n + 1), z(n + 1), rv(n + 1), sg(n + 1, 1.0), as(n + 1);
    for (int i = 1; i <= n; ++i) {
      x[i] = xyz[3 * (i - 1)];
      y[i] = xyz[3 * (i - 1) + 1];
      z[i] = xyz[3 * (i - 1) + 2];
      rv[i] = r[i - 1];
    }
    Smmp rng;
    rng.sgrnd(seed);
    *total = oracle::esolan_areas(n, x.data(), y.data(), z.data(), rv.data(), sg.data(),
                          [&] { return rng.grnd(); }, as.data());
    for (int i = 1; i <= n; ++i) areas[i - 1] = as[i];
  });
}

// Per-atom SASA of the current conformation: the numerical areas of enysol
// (surfc counts; heavy atoms with rvdw > 0) are not kept by the reference, so
// this returns the analytic ones of esolan for all atoms (areas[natoms]).
int orc_esolan_atoms(void* h, double* areas, double* total) {
  Smmp* s = S(h);
  return guard([&] {
    int na = s->iatrs2[s->irsml2[s->ntlml]];
    std::vector<double> sg(na + 1, 1.0), as(na + 1);
    *total = oracle::esolan_areas(na, &s->xat_[2], &s->yat_[2], &s->zat_[2], s->rvdw.data(), sg.data(),
                          [s] { return s->grnd(); }, as.data());
    for (int i = 1; i <= na; ++i) areas[i - 1] = as[i];
  });
}

}  // extern "C"
