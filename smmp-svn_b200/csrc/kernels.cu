// sm_100a kernels of the SMMP energy-and-sweep path.
//
//  k_seed         per-stream MT19937 seeding (twister.f sgrnd, Knuth 69069)
//  k_draw         draw numbers from a stream (grnd)
//  k_random_start canonical random start (canon.f:60-67)
//  k_energy       setvar + full Eyring rebuild + ECEPP/3 (+ SASA) energy of a
//                 set of chains, one CTA each (energy.f)
//  k_sweep        persistent Metropolis sweeps, one CTA per chain
//                 (metropolis.f)
//  k_exchange     parallel-tempering exchange step (partem_s.f:210-232)
//
// One CTA owns one chain: coordinates, dihedral state, variables and the
// chain's MT19937 stream live in shared memory for the whole launch; the
// molecule's topology is read through the read-only cache.
//
// The proposal loop of k_sweep is built for latency, since one chain's
// proposals are strictly sequential:
//  * the dihedral state follows setvar's arithmetic exactly, but the
//    coordinates move by an in-place rotation of the variable's subtree
//    (a full Eyring rebuild runs at the start and end of every sweep);
//  * random numbers are tempered ahead into a per-chain queue together with
//    their logarithms, so the acceptance test exp(-d) >= r is decided by
//    comparing -d with log(r) (exp is evaluated only within 1e-10 of the
//    threshold, where the comparison could differ);
//  * while the pair energy of proposal k is evaluated, one warp prepares
//    proposal k+1 for both possible RNG positions (k drew one or two numbers);
//  * every warp reduces the pair sums and takes the accept/reject decision
//    itself, so there is no serial single-thread phase.
#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"
#include "gradient_core.cuh"
#include "kernels.hpp"
#include "mt.cuh"

namespace smmpb200 {
#ifdef SMMP_BLOCK_VARIANT
namespace SMMP_BLOCK_VARIANT {
#endif

namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kPi2 = 2.0 * kPi;

// ---------------------------------------------------------------- angles
// Fortran MOD(d, 2*pi) (difang.f:25, :51).  For |d| < 4*pi the result is
// d - sign(2*pi, d), exact by Sterbenz's lemma, with MOD's sign convention.
__device__ __forceinline__ double mod2pi(double d) {
  double a = fabs(d);
  if (a < kPi2) return d;
  if (a < 2.0 * kPi2) {
    double r = __dsub_rn(d, copysign(kPi2, d));
    return r == 0.0 ? copysign(0.0, d) : r;
  }
  return fmod(d, kPi2);
}
// difang.f:12-33 / :38-60: wrap into (-pi, pi].
__device__ __forceinline__ double wrap_pi(double d) {
  d = mod2pi(d);
  return fabs(d) <= kPi ? d : __dsub_rn(d, copysign(kPi2, d));
}
__device__ __forceinline__ double difang(double a1, double a2) { return wrap_pi(__dsub_rn(a2, a1)); }
__device__ __forceinline__ double addang(double a1, double a2) { return wrap_pi(__dadd_rn(a1, a2)); }

// MT19937 stream slots: mt.cuh (mt_seed, mt_twist, temper, mt_grnd, qbuf,
// stream_next).

// Append cnt (<= 32) values to the queue, and their logarithms to lq (one warp).
__device__ void rng_refill_warp(uint32_t* slot, double* lq, int cnt = 32) {
  const int lane = threadIdx.x & 31;
  if (lane == 0 && slot[kMTIdx] == 625) mt_seed(slot, 4357u);
  __syncwarp();
  uint32_t mti = slot[kMTIdx], qt = slot[kQTail];
  double* q = qbuf(slot);
  int n1 = min(cnt, 624 - (int)mti);
  if (lane < n1) {
    double v = temper(slot[mti + lane]);
    int k = (qt + lane) & (kQueue - 1);
    q[k] = v;
    lq[k] = v > 0.0 ? log(v) : -INFINITY;
  }
  __syncwarp();
  if (n1 < cnt) {
    if (lane == 0) mt_twist(slot);
    __syncwarp();
    int n2 = cnt - n1;
    if (lane < n2) {
      double v = temper(slot[lane]);
      int k = (qt + n1 + lane) & (kQueue - 1);
      q[k] = v;
      lq[k] = v > 0.0 ? log(v) : -INFINITY;
    }
    mti = n2;
  } else {
    mti += cnt;
  }
  __syncwarp();
  if (lane == 0) {
    slot[kMTIdx] = mti;
    slot[kQTail] = qt + cnt;
  }
  __syncwarp();
}

// ---------------------------------------------------------------- shared memory
struct Proposal {
  int jv, ivar, used;   // variable, its index in idvr, RNG values its setup consumed
  int b, a;             // base atom of the rotation and its parent (axis a -> b)
  int lo, hi;           // the atoms the variable moves, [lo, hi]
  int cb, ce;           // its crossing pairs, cross_idx[cb, ce)
  double vold, vnew, cth, sth;
  double enew, eold;    // torsion energy of jv at its new / current dihedral
};

struct Scalars {
  // next proposal if this one draws 1 (spec[2 * par]) or 2 (spec[2 * par + 1])
  // numbers, in two slots by the parity par of the proposal; spec[4] holds a
  // proposal made after the decision (the first of a sweep, or the same
  // variable again)
  Proposal spec[5];
  int refill;
  int hlo, hhi;          // heavy-atom indices of the proposal's subtree range
  int gsync;             // result of the last grid barrier
  // a proposal's sums over the pair warps, formed once by the last of them
  unsigned nred;         // pair warps done with the current proposal
  int dclash;            // some pair was guarded (cached terms)
  double dsum, dsl;      // pair energy (change), SASA energy
  unsigned gen;          // barrier generation seen at the last grid_arrive
  int wn;                // proposals of the current speculative window
};

struct Smem {
  double *x, *y, *z, *bx, *by, *bz;
  double* toat;
  double *fx, *fz;
  double *cq;
  uint8_t* type;
  double* vlvr;
  double* et;            // torsion energy of each variable (enyshe.f:79-80)
  uint32_t* mt;          // stream slot (kMTWords)
  double* lq;            // log of the queued values
  double* red;           // [kWarps][8] partial sums
  double *ta, *ta14, *tc, *tg;
  int* thb;
  float4* p4;            // FP32 pair path: {x_hi, y_hi, z_hi, charge}
  float4* l4;            //                 {x_lo, y_lo, z_lo, 0}, x = x_hi + x_lo
  float4* tab4;          // {A, A14, C, +-guard r^2}; negative guard: H-bond pair
  double* spt;
  float4* nbf;           // SASA neighbours per warp: (dx, dy, dz, rb2) in FP32
  int* nbj;              // and their atom index (for the exact FP64 re-test)
  int* sq;               // SASA neighbour candidates per warp (kSasaQueue)
  double* sae;           // SASA: each heavy atom's term in the current state
  double* san;           // SASA: each heavy atom's term for the proposal
  Scalars* sc;
  float* daf;            // surrogate: features (sin/cos, BF16-rounded) of the state
  __nv_bfloat16* dfe;    // surrogate: feature rows of a batch [16][kDaStride(nin_pad)]
  __nv_bfloat16* dh0;    // surrogate: hidden activations [16][264]
  __nv_bfloat16* dh1;
  float* dsv;            // surrogate energies of the batch's rows [16]
  Proposal* dprop;       // the batch's proposals [16]
  // speculative window: per proposal k, the moved atoms' rotated positions
  // ([k * n + atom]: FP64 and the FP32 hi+lo copies), the warps' partial
  // energy changes [warp * kMaxWindow + k], and the proposals of this window
  // and the next ([2][kMaxWindow], alternating)
  double *wx, *wy, *wz;
  float4 *wp4, *wl4;
  double* wred;
  Proposal* wprop;
  float* ecache;         // cached FP32 pair terms of the state, one per pair of the dense list
  float* tnew;           // the proposal's new terms of its crossing pairs
  DMol* mol;
  char* pool;            // staged topology (see stage_mol)
};

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

__host__ __device__ inline size_t smem_layout(int n, int v, int npnt, bool sasa, bool da, int win,
                                              int cpairs, int ccross, Smem* s, char* base) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off = align16(off + bytes);
    return p;
  };
  Smem t;
  t.x = (double*)take(8 * n);
  t.y = (double*)take(8 * n);
  t.z = (double*)take(8 * n);
  t.toat = (double*)take(8 * n);
  t.cq = (double*)take(8 * n);
  // The rebuild frames (fx, fz) share one region with the proposal-only
  // buffers (backup coordinates and FP32 copies): the rebuild overwrites them
  // and refreshes the FP32 copies when it finishes.  Every sub-array starts
  // on a 16-byte boundary (float4 accesses).
  const size_t a8 = align16(8 * (size_t)n);
  char* region = take(3 * a8 + 32 * (size_t)n);
  if (base) {
    t.bx = (double*)region;
    t.by = (double*)(region + a8);
    t.bz = (double*)(region + 2 * a8);
    t.p4 = (float4*)(region + 3 * a8);
    t.l4 = (float4*)(region + 3 * a8 + 16 * (size_t)n);
    t.fx = (double*)region;                  // 24n bytes <= 3 * a8
    t.fz = (double*)(region + 3 * a8);       // 24n bytes <= 32n
  }
  t.type = (uint8_t*)take(n);
  t.vlvr = (double*)take(8 * (v > 0 ? v : 1));
  t.et = (double*)take(8 * (v > 0 ? v : 1));
  t.mt = (uint32_t*)take(4 * kMTWords);
  t.lq = (double*)take(8 * kQueue);
  t.red = (double*)take(8 * kWarps * 8);
  t.ta = (double*)take(8 * kTP);
  t.ta14 = (double*)take(8 * kTP);
  t.tc = (double*)take(8 * kTP);
  t.tg = (double*)take(8 * kTP);
  t.thb = (int*)take(4 * kTP);
  t.tab4 = (float4*)take(16 * kTP);
  t.spt = (double*)take(sasa ? 8 * 3 * npnt : 8);
  t.nbf = (float4*)take(sasa ? 16 * kWarps * kMaxNeighbours : 16);
  t.nbj = (int*)take(sasa ? 4 * kWarps * kMaxNeighbours : 4);
  t.sq = (int*)take(sasa ? 4 * kWarps * kSasaQueue : 4);
  t.sae = (double*)take(sasa ? 8 * (size_t)(n > 0 ? n : 1) : 8);
  t.san = (double*)take(sasa ? 8 * (size_t)(n > 0 ? n : 1) : 8);
  const size_t fpad = ((size_t)2 * (v > 0 ? v : 1) + 15) / 16 * 16 + 8;   // row stride
  t.daf = (float*)take(da ? 4 * 2 * (size_t)(v > 0 ? v : 1) : 4);
  t.dfe = (__nv_bfloat16*)take(da ? 2 * 16 * fpad : 16);
  t.dh0 = (__nv_bfloat16*)take(da ? 2 * 16 * 264 : 16);
  t.dh1 = (__nv_bfloat16*)take(da ? 2 * 16 * 264 : 16);
  t.dsv = (float*)take(da ? 4 * 16 : 16);
  t.dprop = (Proposal*)take(da ? sizeof(Proposal) * 16 : 16);
  const size_t wn = win >= 2 ? (size_t)win * n : 1;
  t.wx = (double*)take(8 * wn);
  t.wy = (double*)take(8 * wn);
  t.wz = (double*)take(8 * wn);
  t.wp4 = (float4*)take(16 * wn);
  t.wl4 = (float4*)take(16 * wn);
  t.wred = (double*)take(win >= 2 ? 8 * kWarps * kMaxWindow : 8);
  t.wprop = (Proposal*)take(win >= 2 ? sizeof(Proposal) * 2 * kMaxWindow : 16);
  t.ecache = (float*)take(cpairs > 0 ? 4 * (size_t)cpairs : 4);
  t.tnew = (float*)take(ccross > 0 ? 4 * (size_t)ccross : 4);
  t.sc = (Scalars*)take(sizeof(Scalars));
  t.mol = (DMol*)take(sizeof(DMol));
  t.pool = take(0);
  if (s) *s = t;
  return off;
}

__device__ Smem carve(const DMolSet& set, bool sasa) {
  extern __shared__ __align__(16) char smem_raw[];
  Smem s;
  smem_layout(set.max_atoms, set.max_vars, set.f.npnt, sasa, set.da != 0, sasa ? 0 : set.window,
              sasa ? 0 : set.cache_pairs, sasa ? 0 : set.cache_cross, &s, smem_raw);
  return s;
}

// Bytes of the staged topology of one molecule: one 16-byte-aligned block per
// array, in the order stage_mol copies them (host sizing and device staging
// must agree exactly).
__host__ __device__ inline size_t stage_size(int natoms, int nvar, int nsib, int nlevels, int nfree,
                                             int nflat, int nheavy, bool rows, bool lists,
                                             int ncross) {
  size_t b = 0;
  auto a = [&](size_t elem, int n) { b += align16(elem * (size_t)(n > 0 ? n : 1)); };
  a(4, nvar);          // var_atom
  a(4, nvar);          // var_base
  a(4, nvar);          // var_lo
  a(4, nvar);          // var_hi
  a(4, nvar + 1);      // sib_off
  a(4, nsib);          // sib
  a(8, nvar);          // var_e0
  a(8, nvar);          // var_sg
  a(8, nvar);          // var_rn
  a(8, nvar);          // axvr
  a(4, nfree);         // idvr
  if (rows) {
    a(8, natoms);      // near_mask
    a(8, natoms);      // near14
  }
  a(4, nheavy);        // heavy
  a(8, natoms);        // rvdw
  a(8, natoms);        // sigma
  a(4, natoms);        // iow
  a(4, natoms);        // level_atoms
  a(4, nlevels + 1);   // level_off
  a(8, natoms);        // blen
  a(8, natoms);        // cba
  a(8, natoms);        // sba
  if (lists) {
    a(4, nflat);   // flat pair list
    if (ncross > 0) {
      a(4, nvar + 1);   // cross_off
      a(2, ncross);     // cross_idx
    }
  }
  return b;
}

// Copy the chain's molecule descriptor and its per-proposal topology into
// shared memory; the staged descriptor points at the shared copies, so the
// proposal loop never waits on a global-memory round trip.  The pair lists
// are staged when they fit (set.stage_lists), else read from global memory.
__device__ __forceinline__ unsigned dynamic_smem_bytes() {
  unsigned r;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
  return r;
}
// Copy n elements into the pool; copies nothing (and leaves the source in
// place) if the block would pass `end`, so a sizing error can never write
// outside the CTA's shared memory.
template <class T>
__device__ const T* stage_array(const T* src, int n, char*& pool, const char* end, bool& ok) {
  size_t bytes = align16(sizeof(T) * (size_t)(n > 0 ? n : 1));
  if (!ok || pool + bytes > end) {
    ok = false;
    return src;
  }
  T* dst = reinterpret_cast<T*>(pool);
  for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
  pool += bytes;
  return dst;
}
__device__ const DMol& stage_mol(const DMolSet& set, const DChains& ch, int c, Smem& s) {
  if (threadIdx.x == 0) *s.mol = set.mols[ch.mol_of_chain[c]];
  __syncthreads();
  DMol g = *s.mol;
  __syncthreads();
  extern __shared__ __align__(16) char smem_raw[];
  char* pool = s.pool;
  const char* end = smem_raw + dynamic_smem_bytes();
  bool ok = true;
  DMol m = g;
  // per-proposal arrays first: a molecule too large for the whole pool keeps
  // the rebuild arrays (used twice per sweep) in global memory
  m.var_atom = stage_array(g.var_atom, g.nvar, pool, end, ok);
  m.var_base = stage_array(g.var_base, g.nvar, pool, end, ok);
  m.var_lo = stage_array(g.var_lo, g.nvar, pool, end, ok);
  m.var_hi = stage_array(g.var_hi, g.nvar, pool, end, ok);
  m.sib_off = stage_array(g.sib_off, g.nvar + 1, pool, end, ok);
  m.sib = stage_array(g.sib, g.nsib, pool, end, ok);
  m.var_e0 = stage_array(g.var_e0, g.nvar, pool, end, ok);
  m.var_sg = stage_array(g.var_sg, g.nvar, pool, end, ok);
  m.var_rn = stage_array(g.var_rn, g.nvar, pool, end, ok);
  m.axvr = stage_array(g.axvr, g.nvar, pool, end, ok);
  m.idvr = stage_array(g.idvr, g.nfree, pool, end, ok);
  if (g.rows) {
    m.near_mask = stage_array(g.near_mask, g.natoms, pool, end, ok);
    m.near14 = stage_array(g.near14, g.natoms, pool, end, ok);
  }
  m.heavy = stage_array(g.heavy, g.nheavy, pool, end, ok);
  m.rvdw = stage_array(g.rvdw, g.natoms, pool, end, ok);
  m.sigma = stage_array(g.sigma, g.natoms, pool, end, ok);
  m.iow = stage_array(g.iow, g.natoms, pool, end, ok);
  m.level_atoms = stage_array(g.level_atoms, g.natoms, pool, end, ok);
  m.level_off = stage_array(g.level_off, g.nlevels + 1, pool, end, ok);
  m.blen = stage_array(g.blen, g.natoms, pool, end, ok);
  m.cba = stage_array(g.cba, g.natoms, pool, end, ok);
  m.sba = stage_array(g.sba, g.natoms, pool, end, ok);
  if (set.stage_lists) {
    m.flat = stage_array(g.flat, g.npairs, pool, end, ok);
    if (set.cache_pairs > 0 && g.cache) {
      m.cross_off = stage_array(g.cross_off, g.nvar + 1, pool, end, ok);
      m.cross_idx = stage_array(g.cross_idx, g.ncross, pool, end, ok);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *s.mol = m;
  __syncthreads();
  return *s.mol;
}

// Force-field tables and the molecule's per-atom constants.
__device__ void load_static(const DForceField& ff, const DMol& m, Smem& s, bool sasa) {
  for (int k = threadIdx.x; k < kTP; k += blockDim.x) {
    s.ta[k] = ff.a[k];
    s.ta14[k] = ff.a14[k];
    s.tc[k] = ff.c[k];
    s.tg[k] = ff.guard_r2[k];
    s.thb[k] = ff.hb[k];
    float g = (float)ff.guard_r2[k];
    s.tab4[k] = make_float4((float)ff.a[k], (float)ff.a14[k], (float)ff.c[k], ff.hb[k] ? -g : g);
  }
  for (int k = threadIdx.x; k < m.natoms; k += blockDim.x) {
    s.cq[k] = m.charge[k];
    s.type[k] = m.type[k];
  }
  if (sasa)
    for (int k = threadIdx.x; k < 3 * ff.npnt; k += blockDim.x) s.spt[k] = ff.spoint[k];
}

// FP32 copy of atom k's position as a hi+lo pair of floats, so that FP32
// differences of two positions keep FP64-difference accuracy; p4.w holds the
// charge and l4.w the atom type (as int bits).  hi is x with its mantissa cut
// to the 24 bits a float holds (by masking: exact as a float, and x - hi is
// exact in FP64), lo the rest rounded to a float, so hi + lo keeps 48 bits of
// x and only the two independent conversions to float remain.
__device__ __forceinline__ double float_head(double v) {
  return __longlong_as_double(__double_as_longlong(v) & (long long)0xFFFFFFFFE0000000ull);
}
__device__ __forceinline__ void split_hi_lo(double x, double y, double z, float q, float tbits,
                                            float4& p4, float4& l4) {
  const double xh = float_head(x), yh = float_head(y), zh = float_head(z);
  p4 = make_float4((float)xh, (float)yh, (float)zh, q);
  l4 = make_float4((float)(x - xh), (float)(y - yh), (float)(z - zh), tbits);
}
__device__ __forceinline__ void f32_copy(Smem& s, int k) {
  split_hi_lo(s.x[k], s.y[k], s.z[k], (float)s.cq[k], __int_as_float((int)s.type[k]), s.p4[k],
              s.l4[k]);
}
// The same for an atom that moved to (x, y, z): its charge and type words
// stay as the rebuild wrote them.
__device__ __forceinline__ void f32_move(Smem& s, int k, double x, double y, double z) {
  split_hi_lo(x, y, z, s.p4[k].w, s.l4[k].w, s.p4[k], s.l4[k]);
}

// ---------------------------------------------------------------- setvar
// setvar.f:30-56 for every variable (one lane per variable; a variable shifts
// only the children of its own base, so lanes never write the same atom).
__device__ __forceinline__ double torsion_term(const DMol& m, int v, double to) {
  double e0 = m.var_e0[v];
  return e0 != 0.0 ? e0 * (1.0 + m.var_sg[v] * cos(to * m.var_rn[v])) : 0.0;
}
__device__ __forceinline__ void setvar_one(const DMol& m, Smem& s, int v) {
  int iat = m.var_atom[v];
  double tsh = difang(s.toat[iat], s.vlvr[v]);
  if (tsh != 0.0) {
    int b = m.sib_off[v], e = m.sib_off[v + 1];
    for (int k = b; k < e; ++k) {
      int jat = m.sib[k];
      double to = __dadd_rn(s.toat[jat], tsh);
      if (fabs(to) > kPi) to = __dsub_rn(to, copysign(kPi2, to));
      s.toat[jat] = to;
    }
  }
}
__device__ void setvar_all(const DMol& m, Smem& s) {
  for (int v = threadIdx.x; v < m.nvar; v += blockDim.x) setvar_one(m, s, v);
}
__device__ void setvar_warp(const DMol& m, Smem& s) {
  for (int v = threadIdx.x & 31; v < m.nvar; v += 32) setvar_one(m, s, v);
}
// Torsion energy of every variable (enyshe.f:70-80) from the dihedral state.
__device__ void torsion_all(const DMol& m, Smem& s) {
  for (int v = threadIdx.x; v < m.nvar; v += blockDim.x)
    s.et[v] = torsion_term(m, v, s.toat[m.var_atom[v]]);
}

// ---------------------------------------------------------------- rebuild
// Frame of the first backbone atom (setgbl, bldmol.f:303-420) from the
// molecule's global axes (m.ag) and the dihedrals of i2 and i3, whose sin
// and cos wait in the x/y slots of those atoms (full_rebuild).  Single
// thread.
__device__ void first_frame(const DMol& m, Smem& s) {
  const int i1 = m.i1, i2 = m.i2, i3 = m.i3;
  double ag[3][3];
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) ag[r][q] = m.ag[r * 3 + q];
  const double st2 = s.x[i2], ct2 = s.y[i2], st3 = s.x[i3], ct3 = s.y[i3];
  double x1, x2, x3, y1, y3, z1, z2, z3;
  double sa2 = m.sba[i2];
  x1 = -m.cba[i2];
  x2 = -sa2 * ct2;
  x3 = -sa2 * st2;
  double dx = sqrt(x1 * x1 + x2 * x2 + x3 * x3);
  x1 /= dx; x2 /= dx; x3 /= dx;
  z1 = -st3 * (st2 * x3 + ct2 * x2);
  z2 = st3 * ct2 * x1 + ct3 * st2;
  z3 = st3 * st2 * x1 - ct3 * ct2;
  double dz = sqrt(z1 * z1 + z2 * z2 + z3 * z3);
  z1 /= dz; z2 /= dz; z3 /= dz;
  y1 = z2 * x3 - z3 * x2;
  y3 = z1 * x2 - z2 * x1;
  double xg[3], zg[3];
  for (int r = 0; r < 3; ++r) {
    xg[r] = ag[r][0] * x1 + ag[r][1] * y1 + ag[r][2] * z1;
    zg[r] = ag[r][0] * x3 + ag[r][1] * y3 + ag[r][2] * z3;
  }
  dx = sqrt(xg[0] * xg[0] + xg[1] * xg[1] + xg[2] * xg[2]);
  dz = sqrt(zg[0] * zg[0] + zg[1] * zg[1] + zg[2] * zg[2]);
  for (int r = 0; r < 3; ++r) {
    s.fx[3 * i1 + r] = xg[r] / dx;
    s.fz[3 * i1 + r] = zg[r] / dz;
  }
  s.x[i1] = m.gbpr[0];
  s.y[i1] = m.gbpr[1];
  s.z[i1] = m.gbpr[2];
}

// Eyring step (bldmol.f:175-242): atom i from the frame of its parent ia.
// The sin and cos of atom i's dihedral wait in its own x and y slots (see
// full_rebuild); the step reads them, then writes the coordinates there.
__device__ __forceinline__ void eyring(const double* __restrict__ cba,
                                       const double* __restrict__ sba,
                                       const double* __restrict__ blen, Smem& s, int i, int ia) {
  const double st = s.x[i], ct = s.y[i];
  double ca = cba[i], sa = sba[i], bl = blen[i];
  double x1 = s.fx[3 * ia], x2 = s.fx[3 * ia + 1], x3 = s.fx[3 * ia + 2];
  double z1 = s.fz[3 * ia], z2 = s.fz[3 * ia + 1], z3 = s.fz[3 * ia + 2];
  double y1 = z2 * x3 - z3 * x2, y2 = z3 * x1 - z1 * x3, y3 = z1 * x2 - z2 * x1;
  double h2 = -sa * ct, h3 = -sa * st;
  double nx1 = -ca * x1 + h2 * y1 + h3 * z1;
  double nx2 = -ca * x2 + h2 * y2 + h3 * z2;
  double nx3 = -ca * x3 + h2 * y3 + h3 * z3;
  double dx = rsqrt(nx1 * nx1 + nx2 * nx2 + nx3 * nx3);
  nx1 *= dx; nx2 *= dx; nx3 *= dx;
  s.fx[3 * i] = nx1;
  s.fx[3 * i + 1] = nx2;
  s.fx[3 * i + 2] = nx3;
  double nz1 = -st * y1 + ct * z1, nz2 = -st * y2 + ct * z2, nz3 = -st * y3 + ct * z3;
  double dz = rsqrt(nz1 * nz1 + nz2 * nz2 + nz3 * nz3);
  s.fz[3 * i] = nz1 * dz;
  s.fz[3 * i + 1] = nz2 * dz;
  s.fz[3 * i + 2] = nz3 * dz;
  s.x[i] = s.x[ia] + nx1 * bl;
  s.y[i] = s.y[ia] + nx2 * bl;
  s.z[i] = s.z[ia] + nx3 * bl;
}

// Full rebuild of all coordinates from the dihedral state (bldmol.f:13-93).
// The transcendental work is off the chain of dependent steps: while thread 0
// sets up the first frame, every thread takes the sin/cos of the dihedrals
// (parked in the x/y slots of the atoms, none of which is placed yet); then
// the first warp alone runs one Eyring step per depth level with warp
// syncs between levels (levels are a few atoms wide: 7 in Met-enkephalin, 12
// in a 60-residue protein), and the block refreshes the FP32 copies.
__device__ void full_rebuild(const DMol& m, Smem& s) {
  // the molecule's arrays in registers before the first shared store
  const int* __restrict__ lvl_off = m.level_off;
  const int* __restrict__ lvl_at = m.level_atoms;
  const int* __restrict__ iow = m.iow;
  const double* __restrict__ cba = m.cba;
  const double* __restrict__ sba = m.sba;
  const double* __restrict__ blen = m.blen;
  const int nlev = m.nlevels, n = m.natoms, i1 = m.i1;
  for (int k = threadIdx.x; k < n; k += blockDim.x)
    if (k != i1) sincos(s.toat[k], &s.x[k], &s.y[k]);
  __syncthreads();
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) first_frame(m, s);
    __syncwarp();
    int e = lvl_off[1];
    for (int L = 1; L < nlev; ++L) {
      const int b = e;
      e = lvl_off[L + 1];
      for (int k = b + (int)threadIdx.x; k < e; k += 32) {
        const int a = lvl_at[k];
        eyring(cba, sba, blen, s, a, iow[a]);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < m.natoms; k += blockDim.x) f32_copy(s, k);
  __syncthreads();
}

// ---------------------------------------------------------------- pair energy
// One ECEPP/3 pair (enyshe.f:112-184): Coulomb with constant or sigmoidal
// dielectric, 12-6 Lennard-Jones or 12-10 hydrogen bond.
template <bool F32>
__device__ __forceinline__ void pair_term_at(const FFScalars& ff, const Smem& s, int i, int j,
                                             bool is14, double xi, double yi, double zi,
                                             double xj, double yj, double zj, double& el,
                                             double& vw, double& hb) {
  double dx = xj - xi, dy = yj - yi, dz = zj - zi;
  double r2 = dx * dx + dy * dy + dz * dz;
  int tp = s.type[i] * kTypes + s.type[j];
  double A = is14 ? s.ta14[tp] : s.ta[tp];
  double C = s.tc[tp];
  int ishb = s.thb[tp];
  double qq = ff.conv * s.cq[i] * s.cq[j];
  if (!F32 || r2 < s.tg[tp] || ff.epsd) {
    double ri = rsqrt(r2);
    double r2i = ri * ri;
    double r6i = r2i * r2i * r2i;
    if (ff.epsd) {
      double sr = ff.slp * (r2 * ri);
      const double ep = ff.plt - (sr * sr + 2.0 * sr + 2.0) * (ff.plt - 1.0) * exp(-sr) / 2.0;
      el += qq * ri / ep;
    } else {
      el += __dmul_rn(qq, ri);   // the same bits as dividing the product by a dielectric of 1
    }
    if (!ishb)
      vw += A * r6i * r6i - C * r6i;
    else
      hb += A * r6i * r6i - C * r6i * r2i * r2i;
  } else {
    float rf = rsqrtf((float)r2);
    float r2i = rf * rf;
    float r6i = r2i * r2i * r2i;
    el += (double)((float)qq * rf);
    float Af = (float)A, Cf = (float)C;
    if (!ishb)
      vw += (double)(Af * r6i * r6i - Cf * r6i);
    else
      hb += (double)(Af * r6i * r6i - Cf * r6i * r2i * r2i);
  }
}
template <bool F32>
__device__ __forceinline__ void pair_term(const FFScalars& ff, const Smem& s, int i, int j,
                                          bool is14, double& el, double& vw, double& hb) {
  pair_term_at<F32>(ff, s, i, j, is14, s.x[i], s.y[i], s.z[i], s.x[j], s.y[j], s.z[j], el, vw, hb);
}

// Kahan-compensated FP32 accumulator.
struct KSum {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float v) {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// FP32 pair term from the hi+lo coordinates; pairs closer than the guard
// distance of their types go through the FP64 path.  Coulomb accumulates
// q_i q_j / r (the factor conv is applied to the sum).
__device__ __forceinline__ void pair32(const FFScalars& ff, const Smem& s, int i, int j, bool is14,
                                       KSum& el, KSum& vw, KSum& hb, double& el64, double& vw64,
                                       double& hb64) {
  const float4 pi = s.p4[i], pj = s.p4[j], li = s.l4[i], lj = s.l4[j];
  float dx = (pj.x - pi.x) + (lj.x - li.x);
  float dy = (pj.y - pi.y) + (lj.y - li.y);
  float dz = (pj.z - pi.z) + (lj.z - li.z);
  float r2 = dx * dx + dy * dy + dz * dz;
  const float4 pr = s.tab4[__float_as_int(li.w) * kTypes + __float_as_int(lj.w)];
  if (r2 < fabsf(pr.w)) {
    double e, v, h;
    e = v = h = 0.0;
    pair_term<false>(ff, s, i, j, is14, e, v, h);
    el64 += e;
    vw64 += v;
    hb64 += h;
    return;
  }
  float ri = rsqrtf(r2);
  float r2i = ri * ri;
  float r6i = r2i * r2i * r2i;
  el.add(pi.w * pj.w * ri);
  float A = is14 ? pr.y : pr.x;
  if (pr.w >= 0.f)
    vw.add(A * r6i * r6i - pr.z * r6i);
  else
    hb.add(A * r6i * r6i - pr.z * r6i * r2i * r2i);
}

// FP64 term of a clashing pair, out of line: it is rare, and keeping it out
// of the FP32 loop keeps that loop's registers free.
__device__ __noinline__ void pair_term_clash(const FFScalars& ff, const Smem& s, int i, int j,
                                             bool is14, double* acc) {
  pair_term<false>(ff, s, i, j, is14, acc[0], acc[1], acc[2]);
}

// Positions of the atoms as the current state holds them.
struct StatePos {
  const Smem& s;
  __device__ __forceinline__ float4 p(int a) const { return s.p4[a]; }
  __device__ __forceinline__ float4 l(int a) const { return s.l4[a]; }
  __device__ __forceinline__ void clash(const FFScalars& ff, int i, int j, bool is14,
                                        double* acc) const {
    pair_term_clash(ff, s, i, j, is14, acc);
  }
};

// FP64 term of a clashing pair at given positions (out of line, as above).
__device__ __noinline__ void pair_term_clash_at(const FFScalars& ff, const Smem& s, int i, int j,
                                                bool is14, double xi, double yi, double zi,
                                                double xj, double yj, double zj, double* acc) {
  pair_term_at<false>(ff, s, i, j, is14, xi, yi, zi, xj, yj, zj, acc[0], acc[1], acc[2]);
}

// Positions after proposal k of a speculative window: the atoms the
// proposal turns come from the window buffer k, the rest from the state.
// The proposal turns the range [lo, hi], or, when that range holds the third
// backbone atom, everything else but the axis atoms a and b.
struct WindowPos {
  const Smem& s;
  int base, lo, hi, a, b;   // base = k * atoms
  bool flip;
  __device__ __forceinline__ bool moved(int t) const {
    return flip ? ((t < lo || t > hi) && t != a && t != b) : (t >= lo && t <= hi);
  }
  __device__ __forceinline__ float4 p(int t) const { return moved(t) ? s.wp4[base + t] : s.p4[t]; }
  __device__ __forceinline__ float4 l(int t) const { return moved(t) ? s.wl4[base + t] : s.l4[t]; }
  __device__ __forceinline__ void clash(const FFScalars& ff, int i, int j, bool is14,
                                        double* acc) const {
    const bool mi = moved(i), mj = moved(j);
    pair_term_clash_at(ff, s, i, j, is14, mi ? s.wx[base + i] : s.x[i], mi ? s.wy[base + i] : s.y[i],
                       mi ? s.wz[base + i] : s.z[i], mj ? s.wx[base + j] : s.x[j],
                       mj ? s.wy[base + j] : s.y[j], mj ? s.wz[base + j] : s.z[j], acc);
  }
};

// One FP32 pair term of the row loop: t = {Coulomb, 12-6, 12-10} for pair
// (i, j), zero unless `use`; a clashing pair (closer than its guard) goes
// to the FP64 sums a64 instead.  j must be a valid atom even when !use.
template <bool TOTAL, class Pos>
__device__ __forceinline__ void row_term_at(const FFScalars& ff, const Pos& pos, int i, int j,
                                            bool use, bool is14, const float4& pi,
                                            const float4& li, float qi, const float4* trow,
                                            double* a64, float* t) {
  const float4 pj = pos.p(j), lj = pos.l(j);
  const float dx = (pj.x - pi.x) + (lj.x - li.x);
  const float dy = (pj.y - pi.y) + (lj.y - li.y);
  const float dz = (pj.z - pi.z) + (lj.z - li.z);
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float4 pr = trow[__float_as_int(lj.w)];
  const bool clash = r2 < fabsf(pr.w);
  if (use && clash) pos.clash(ff, i, j, is14, a64);
  const float ri = rsqrtf(r2);
  const float r2i = ri * ri;
  const float r6i = r2i * r2i * r2i;
  const bool ishb = pr.w < 0.f;
  const float rc = ishb ? r6i * r2i * r2i : r6i;
  const float elj = (is14 ? pr.y : pr.x) * r6i * r6i - pr.z * rc;
  const bool keep = use && !clash;
  t[0] = keep ? qi * pj.w * ri : 0.f;
  if (TOTAL) {
    t[1] = keep ? elj : 0.f;
  } else {
    t[1] = keep && !ishb ? elj : 0.f;
    t[2] = keep && ishb ? elj : 0.f;
  }
}
template <bool TOTAL>
__device__ __forceinline__ void row_term(const FFScalars& ff, const Smem& s, int i, int j,
                                         bool use, bool is14, const float4& pi, const float4& li,
                                         float qi, const float4* trow, double* a64, float* t) {
  row_term_at<TOTAL>(ff, StatePos{s}, i, j, use, is14, pi, li, qi, trow, a64, t);
}

// Pair sums by rows, for molecules whose pair set has the row form (m.rows):
// warp w of the warps [0, nw) takes rows i = w, w+nw, ...; in one pass over a
// row, lane l takes partner j = j0 + l, so the 32 partners of a pass are
// consecutive atoms (one conflict-free float4 load each) and atom i's data
// stays in registers.  The first two passes read the near-window masks of
// row i; every later partner is a normal pair.  With TOTAL the three sums
// are returned added together in `el` (the sweep's proposals need only the
// total).
template <bool F32, bool TOTAL>
__device__ void pair_rows(const FFScalars& ff, const DMol& m, const Smem& s, int nw, double& el,
                          double& vw, double& hb) {
  const int lane = threadIdx.x & 31, n = m.natoms;
  if (!F32 || ff.epsd) {
    for (int i = (threadIdx.x >> 5); i < n - 1; i += nw) {
      const unsigned long long nm = m.near_mask[i], n14 = m.near14[i];
      for (int j0 = i + 1; j0 < n; j0 += 32) {
        const int j = j0 + lane, d = j0 - i - 1;
        bool use = j < n, is14 = false;
        if (d < 64) {
          const uint32_t bn = (uint32_t)(nm >> d), b14 = (uint32_t)(n14 >> d);
          use = use && (((bn | b14) >> lane) & 1u);
          is14 = ((b14 >> lane) & 1u) != 0;
        }
        if (use) pair_term<false>(ff, s, i, j, is14, el, vw, hb);
      }
    }
    if (TOTAL) {
      el = (el + vw) + hb;
      vw = hb = 0.0;
    }
    return;
  }
  KSum ke, kv, kh;
  double a64[3] = {0.0, 0.0, 0.0};
  const float convf = (float)ff.conv;
  auto add = [&](const float (&t)[3]) {
    if (TOTAL) {
      ke.add(t[0] + t[1]);
    } else {
      ke.add(t[0]);
      kv.add(t[1]);
      kh.add(t[2]);
    }
  };
  for (int i = (threadIdx.x >> 5); i < n - 1; i += nw) {
    const float4 pi = s.p4[i], li = s.l4[i];
    const float qi = convf * pi.w;
    const float4* trow = s.tab4 + __float_as_int(li.w) * kTypes;
    float t[3];
    {   // partners i+1 .. i+64: the near-window masks
      const unsigned long long nm = m.near_mask[i], n14 = m.near14[i];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = i + 1 + 32 * h + lane;
        const uint32_t bn = (uint32_t)(nm >> (32 * h)), b14 = (uint32_t)(n14 >> (32 * h));
        const bool use = j < n && (((bn | b14) >> lane) & 1u);
        const bool is14 = ((b14 >> lane) & 1u) != 0;
        row_term<TOTAL>(ff, s, i, use ? j : i + 1, use, is14, pi, li, qi, trow, a64, t);
        add(t);
      }
    }
    // every later partner is a normal pair
    for (int j = i + 65 + lane; j < n + lane; j += 32) {
      const bool use = j < n;
      row_term<TOTAL>(ff, s, i, use ? j : i + 1, use, false, pi, li, qi, trow, a64, t);
      add(t);
    }
  }
  if (TOTAL) {
    el += ((ke.value() + a64[0]) + a64[1]) + a64[2];
  } else {
    el += ke.value() + a64[0];
    vw += kv.value() + a64[1];
    hb += kh.value() + a64[2];
  }
}

// Energy of the pairs that cross the partition {lo..hi} | rest (the pairs
// whose distance a rotation of either side changes), this thread's share, for
// warps [0, nw): rows i < lo take partners lo..hi, rows i in lo..hi take
// partners beyond hi (row form: the first 64 partners of a row are masked).
// A proposal's energy change is this sum after the rotation minus the same
// sum before it, computed by the same threads over the same pairs.
template <bool F32, class Pos>
__device__ double cross_rows_at(const FFScalars& ff, const DMol& m, const Smem& s, const Pos& pos,
                                int nw, int lo, int hi) {
  const int lane = threadIdx.x & 31, n = m.natoms;
  double e64[3] = {0.0, 0.0, 0.0};
  KSum ke;
  const float convf = (float)ff.conv;
  for (int i = (threadIdx.x >> 5); i <= hi && i < n - 1; i += nw) {
    const int jb = i < lo ? lo : hi + 1;
    const int je = i < lo ? hi : n - 1;
    if (jb > je) continue;
    const unsigned long long nm = m.near_mask[i], n14 = m.near14[i];
    if (!F32 || ff.epsd) {   // FP64 terms read the state (the one-at-a-time sweep only)
      for (int j = jb + lane; j <= je; j += 32) {
        const int d = j - i - 1;
        bool use = true, is14 = false;
        if (d < 64) {
          use = (((nm | n14) >> d) & 1ull) != 0;
          is14 = ((n14 >> d) & 1ull) != 0;
        }
        if (use) pair_term<false>(ff, s, i, j, is14, e64[0], e64[1], e64[2]);
      }
      continue;
    }
    const float4 pi = pos.p(i), li = pos.l(i);
    const float qi = convf * pi.w;
    const float4* trow = s.tab4 + __float_as_int(li.w) * kTypes;
    for (int j0 = jb; j0 <= je; j0 += 32) {
      const int j = j0 + lane, d = j - i - 1;
      bool use = j <= je, is14 = false;
      if (use && d < 64) {
        use = (((nm | n14) >> d) & 1ull) != 0;
        is14 = ((n14 >> d) & 1ull) != 0;
      }
      float t[3];
      row_term_at<true>(ff, pos, i, use ? j : jb, use, is14, pi, li, qi, trow, e64, t);
      ke.add(t[0] + t[1]);
    }
  }
  return ((ke.value() + e64[0]) + e64[1]) + e64[2];
}
template <bool F32>
__device__ double cross_rows(const FFScalars& ff, const DMol& m, const Smem& s, int nw, int lo,
                             int hi) {
  return cross_rows_at<F32>(ff, m, s, StatePos{s}, nw, lo, hi);
}

// Pair sums of the threads [0, nthr): by rows when the molecule has the row
// form (kernels built with ROWS), else the dense pair list (the mklist pairs,
// 1-4 pairs flagged).
template <bool F32, bool ROWS>
__device__ void pair_energy(const FFScalars& ff, const DMol& m, const Smem& s, int tid, int nthr,
                            double& el, double& vw, double& hb) {
  if (ROWS && m.rows) {
    pair_rows<F32, false>(ff, m, s, nthr >> 5, el, vw, hb);
    return;
  }
  // the dense pair list: thread tid takes pairs tid, tid + nthr, ...
  const int np = m.npairs;
  if (!F32) {
    for (int t = tid; t < np; t += nthr) {
      const uint32_t w = m.flat[t];
      pair_term<false>(ff, s, int(w & 0x3fffu), int((w >> 14) & 0x3fffu), (w >> 28) != 0u, el, vw,
                       hb);
    }
    return;
  }
  if (ff.epsd) {   // sigmoidal dielectric: FP64 terms
    pair_energy<false, ROWS>(ff, m, s, tid, nthr, el, vw, hb);
    return;
  }
  KSum ke, kv, kh;
  double e64 = 0.0, v64 = 0.0, h64 = 0.0;
  int t = tid;
  for (; t + nthr < np; t += 2 * nthr) {   // two pairs in flight per thread
    const uint32_t w0 = m.flat[t], w1 = m.flat[t + nthr];
    pair32(ff, s, int(w0 & 0x3fffu), int((w0 >> 14) & 0x3fffu), (w0 >> 28) != 0u, ke, kv, kh, e64,
           v64, h64);
    pair32(ff, s, int(w1 & 0x3fffu), int((w1 >> 14) & 0x3fffu), (w1 >> 28) != 0u, ke, kv, kh, e64,
           v64, h64);
  }
  for (; t < np; t += nthr) {
    const uint32_t w = m.flat[t];
    pair32(ff, s, int(w & 0x3fffu), int((w >> 14) & 0x3fffu), (w >> 28) != 0u, ke, kv, kh, e64,
           v64, h64);
  }
  el += ff.conv * ke.value() + e64;
  vw += kv.value() + v64;
  hb += kh.value() + h64;
}

// ---------------------------------------------------------------- cached pair terms
// For molecules with per-variable crossing lists (m.cache), a sweep keeps
// the FP32 total term of every pair of the state in s.ecache, filled after
// each opening energy().  A proposal then evaluates only the pairs its turn
// changes and sums (new - cached) for the change of the pair energy; an
// accepted proposal writes its new terms into the cache.  A pair closer than
// its types' guard distance is summed in FP64 (as everywhere in the FP32
// mode) and makes the cache unusable once such a pair enters the state (the
// rest of the sweep then sums every pair in full, as without the cache).

// Total term of pair word w from the FP32 copies: Coulomb (conv folded into
// the charge product) plus the 12-6 or 12-10 term.  Returns true for a pair
// inside its guard distance, whose FP64 total is then in t64.
__device__ __forceinline__ bool cache_term(const FFScalars& ff, const Smem& s, uint32_t w,
                                           float convf, float& term, double& t64) {
  const int i = int(w & 0x3fffu), j = int((w >> 14) & 0x3fffu);
  const bool is14 = (w >> 28) != 0u;
  const float4 pi = s.p4[i], pj = s.p4[j], li = s.l4[i], lj = s.l4[j];
  const float dx = (pj.x - pi.x) + (lj.x - li.x);
  const float dy = (pj.y - pi.y) + (lj.y - li.y);
  const float dz = (pj.z - pi.z) + (lj.z - li.z);
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float4 pr = s.tab4[__float_as_int(li.w) * kTypes + __float_as_int(lj.w)];
  if (r2 < fabsf(pr.w)) {
    double e = 0.0, v = 0.0, h = 0.0;
    pair_term<false>(ff, s, i, j, is14, e, v, h);
    t64 = (e + v) + h;
    term = 0.f;
    return true;
  }
  const float ri = rsqrtf(r2);
  const float r2i = ri * ri;
  const float r6i = r2i * r2i * r2i;
  const float rc = pr.w < 0.f ? r6i * r2i * r2i : r6i;
  term = convf * pi.w * pj.w * ri + ((is14 ? pr.y : pr.x) * r6i * r6i - pr.z * rc);
  return false;
}

// Fill the cache from the current coordinates (whole block); returns, in
// every thread, whether some pair of the state is inside its guard distance.
__device__ bool fill_pair_cache(const FFScalars& ff, const DMol& m, Smem& s) {
  const float convf = (float)ff.conv;
  int clash = 0;
  for (int t = threadIdx.x; t < m.npairs; t += blockDim.x) {
    float term;
    double t64;
    if (cache_term(ff, s, m.flat[t], convf, term, t64)) clash = 1;
    s.ecache[t] = term;
  }
  return __syncthreads_or(clash) != 0;
}

// The proposal's change of the pair energy over the crossing pairs of
// variable v, this thread's share (threads [0, nthr)); its new terms go to
// s.tnew, and nclash counts its pairs inside their guard distance.
__device__ double cached_delta(const FFScalars& ff, const DMol& m, Smem& s, int b, int e, int tid,
                               int nthr, int& nclash) {
  const float convf = (float)ff.conv;
  KSum k;
  double d64 = 0.0;
  for (int q = b + tid; q < e; q += nthr) {
    const int t = m.cross_idx[q];
    float term;
    double t64;
    if (cache_term(ff, s, m.flat[t], convf, term, t64)) {
      d64 += t64 - (double)s.ecache[t];
      ++nclash;
    } else {
      k.add(term - s.ecache[t]);
    }
    s.tnew[q - b] = term;
  }
  return k.value() + d64;
}

// ---------------------------------------------------------------- SASA
// enysol.f:192-306: an atom's sphere point is exposed when it lies outside
// every neighbour sphere (neighbours: d <= r_i + r_j).  FP64 with the
// reference's division and summation order and no fused multiply-add, so the
// exposed-point counts are those of the reference arithmetic.  Warps
// [w0, w0+nw) take one heavy atom at a time; returns this thread's share of
// eysl.
// Cheap pre-test with a margin for "heavy atom j may be a neighbour of i";
// sasa_exact decides.
__device__ __forceinline__ bool sasa_near(const DMol& m, const Smem& s, int j, double trad,
                                          double xi, double yi, double zi) {
  double ex = xi - s.x[j], ey = yi - s.y[j], ez = zi - s.z[j];
  double lim = trad + m.rvdw[j];
  return ex * ex + ey * ey + ez * ez <= lim * lim * 1.0000001 + 1e-12;
}

// Is heavy atom j a neighbour of atom i (enysol.f:232-250: the spheres of
// radius rvdw overlap), and its offset / squared radius in units of trad.
__device__ __forceinline__ bool sasa_exact(const DMol& m, const Smem& s, int j, double trad,
                                           double xi, double yi, double zi, double& dx,
                                           double& dy, double& dz, double& rb2) {
  double rj = m.rvdw[j];
  dx = __ddiv_rn(xi - s.x[j], trad);
  dy = __ddiv_rn(yi - s.y[j], trad);
  dz = __ddiv_rn(zi - s.z[j], trad);
  double dd = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  double akrad = __ddiv_rn(rj, trad);
  double dr = __dadd_rn(1.0, akrad);
  dr = __dmul_rn(dr, dr);
  rb2 = __dmul_rn(akrad, akrad);
  return dd <= dr;
}

__device__ __forceinline__ bool sasa_neighbour(const DMol& m, const Smem& s, int i, int j,
                                               double trad, double xi, double yi, double zi,
                                               double& dx, double& dy, double& dz, double& rb2) {
  return j != i && sasa_near(m, s, j, trad, xi, yi, zi) &&
         sasa_exact(m, s, j, trad, xi, yi, zi, dx, dy, dz, rb2);
}

// Is the surface point (s0, s1, s2) inside the neighbour sphere (enysol.f:267-275).
__device__ __forceinline__ bool sasa_buried(double s0, double s1, double s2, double dx, double dy,
                                            double dz, double rb2) {
  double t0 = __dadd_rn(dx, s0), t1 = __dadd_rn(dy, s1), t2 = __dadd_rn(dz, s2);
  double sdd = __dadd_rn(__dadd_rn(__dmul_rn(t0, t0), __dmul_rn(t1, t1)), __dmul_rn(t2, t2));
  return sdd <= rb2;
}

constexpr float kSasaMargin = 1e-4f;

// Incremental SASA of a proposal.  Only the proposal's moved atoms change
// position; a heavy atom that did not move and has no moved heavy atom among
// its neighbour candidates before or after the move (pre-test on the new and
// the backed-up positions) keeps its neighbours and their positions, hence
// its exposed-point count: its term is taken from `cache` instead of being
// recounted.  Terms are written to `out` (per heavy atom) when it is set.
struct SasaInc {
  const double* cache;   // nullptr: count every atom
  double* out;
  int lo, span, a, b;
  bool flip;
  int hlo, hhi;          // heavy-atom indices with atom index in [lo, lo + span)
  __device__ __forceinline__ bool moved(int j) const {
    return flip ? ((j < lo || j >= lo + span) && j != a && j != b) : (j >= lo && j < lo + span);
  }
};

__device__ double sasa_energy(const FFScalars& ff, const DMol& m, Smem& s, int w0, int nw,
                              int* err, const SasaInc& inc = SasaInc{nullptr, nullptr, 0, 0, 0, 0, false, 0, 0}) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float4* nbf = s.nbf + (size_t)warp * kMaxNeighbours;
  int* nbj = s.nbj + (size_t)warp * kMaxNeighbours;
  int* q = s.sq + warp * kSasaQueue;
  double eysl = 0.0;
  const int npnt = ff.npnt;
  for (int h = warp - w0; h < m.nheavy; h += nw) {
    int i = m.heavy[h];
    double trad = m.rvdw[i];
    double xi = s.x[i], yi = s.y[i], zi = s.z[i];
    // Candidates that pass the cheap pre-test are queued, and the exact
    // test (four FP64 divisions) runs on full warps of queued candidates.
    int nn = 0, nq = 0;
    auto exact32 = [&](int cnt) {
      const int j = lane < cnt ? q[lane] : 0;
      double dx = 0, dy = 0, dz = 0, rb2 = 0;
      const bool take = lane < cnt && sasa_exact(m, s, j, trad, xi, yi, zi, dx, dy, dz, rb2);
      const unsigned mask = __ballot_sync(0xffffffffu, take);
      const int pos = nn + __popc(mask & ((1u << lane) - 1u));
      if (take && pos < kMaxNeighbours) {
        nbf[pos] = make_float4((float)dx, (float)dy, (float)dz, (float)rb2);
        nbj[pos] = j;
      }
      nn += __popc(mask);
    };
    if (inc.cache != nullptr && !inc.moved(i)) {
      // is a moved heavy atom a neighbour candidate, before or after the move?
      bool touched = false;
      const int inner = inc.hhi - inc.hlo;
      const int nmv = inc.flip ? m.nheavy - inner : inner;
      for (int t = lane; t < nmv; t += 32) {
        const int hj = inc.flip ? (t < inc.hlo ? t : t + inner) : inc.hlo + t;
        const int j = m.heavy[hj];
        if (inc.flip && (j == inc.a || j == inc.b)) continue;
        const double lim = trad + m.rvdw[j];
        const double l2 = lim * lim * 1.0000001 + 1e-12;
        const double ex = xi - s.x[j], ey = yi - s.y[j], ez = zi - s.z[j];
        const double ox = xi - s.bx[j], oy = yi - s.by[j], oz = zi - s.bz[j];
        touched = touched || ex * ex + ey * ey + ez * ez <= l2 || ox * ox + oy * oy + oz * oz <= l2;
      }
      if (!__any_sync(0xffffffffu, touched)) {   // unchanged: the cached term
        if (lane == 0) {
          const double tv = inc.cache[h];
          eysl += tv;
          if (inc.out) inc.out[h] = tv;
        }
        __syncwarp();
        continue;
      }
    }
    for (int base = 0; base < m.nheavy; base += 32) {
      const int hj = base + lane;
      const int j = hj < m.nheavy ? m.heavy[hj] : i;
      const bool cand = j != i && sasa_near(m, s, j, trad, xi, yi, zi);
      const unsigned mask = __ballot_sync(0xffffffffu, cand);
      if (cand) q[nq + __popc(mask & ((1u << lane) - 1u))] = j;   // nq < 32: fits
      nq += __popc(mask);
      __syncwarp();
      if (nq >= 32) {
        exact32(32);
        const int rest = nq - 32;
        const int v = lane < rest ? q[32 + lane] : 0;
        __syncwarp();
        if (lane < rest) q[lane] = v;
        __syncwarp();
        nq = rest;
      }
    }
    if (nq > 0) exact32(nq);
    __syncwarp();
    int cnt = 0;
    if (nn <= kMaxNeighbours) {
      // FP32 test with a margin; a point within the margin of a sphere is
      // re-tested in FP64 with the reference's arithmetic.  With neighbour
      // offsets below 3 radii (radii within a factor 2, checked on the
      // host) and unit points, the FP32 error of sdd is below 2e-5.  Each
      // lane takes its (up to) four points through the neighbour list
      // together, so the four tests are independent work.
      constexpr int R = 4;   // points per lane: npnt <= 128
      float f[R][3];
      unsigned buried = 0, valid = 0;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int p = lane + 32 * r;
        const bool ok = p < npnt;
        valid |= ok ? (1u << r) : 0u;
        f[r][0] = ok ? (float)s.spt[3 * p] : 0.f;
        f[r][1] = ok ? (float)s.spt[3 * p + 1] : 0.f;
        f[r][2] = ok ? (float)s.spt[3 * p + 2] : 0.f;
      }
      unsigned done = ~valid & 0xfu;
      for (int k = 0; k < nn && done != 0xfu; ++k) {
        const float4 c = nbf[k];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (done & (1u << r)) continue;
          const float t0 = c.x + f[r][0], t1 = c.y + f[r][1], t2 = c.z + f[r][2];
          const float sdd = t0 * t0 + t1 * t1 + t2 * t2;
          bool b = sdd < c.w - kSasaMargin;
          if (!b && sdd <= c.w + kSasaMargin) {
            const int p = lane + 32 * r;
            double dx, dy, dz, rb2;
            sasa_exact(m, s, nbj[k], trad, xi, yi, zi, dx, dy, dz, rb2);
            b = sasa_buried(s.spt[3 * p], s.spt[3 * p + 1], s.spt[3 * p + 2], dx, dy, dz, rb2);
          }
          if (b) {
            buried |= 1u << r;
            done |= 1u << r;
          }
        }
      }
      cnt = __popc(valid & ~buried);
    } else {
      // More neighbours than the buffer holds (crowded, clashing
      // conformations): test each point against every heavy atom directly,
      // with the same arithmetic, so the count is the same.
      for (int p = lane; p < npnt; p += 32) {
        double s0 = s.spt[3 * p], s1 = s.spt[3 * p + 1], s2 = s.spt[3 * p + 2];
        bool exposed = true;
        for (int hj = 0; hj < m.nheavy && exposed; ++hj) {
          double dx, dy, dz, rb2;
          if (sasa_neighbour(m, s, i, m.heavy[hj], trad, xi, yi, zi, dx, dy, dz, rb2) &&
              sasa_buried(s0, s1, s2, dx, dy, dz, rb2))
            exposed = false;
        }
        cnt += exposed;
      }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) {
      double sdr = __ddiv_rn(__dmul_rn(__dmul_rn(4.0 * kPi, trad), trad), (double)npnt);
      double area = __dmul_rn(sdr, (double)cnt);
      const double t = __dmul_rn(area, m.sigma[i]);
      eysl += t;
      if (inc.out) inc.out[h] = t;
    }
    __syncwarp();
  }
  return eysl;
}

// ---------------------------------------------------------------- reduction
// Warp partials of (eyel, eyvw, eyhb, eyvr, eysl) into s.red[warp].
__device__ __forceinline__ void warp_partials(Smem& s, double v0, double v1, double v2, double v3,
                                              double v4) {
  double v[5] = {v0, v1, v2, v3, v4};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0) {
    int w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) s.red[w * 8 + k] = v[k];
  }
}
// Every warp sums the warp partials the same way (call after a barrier).
__device__ __forceinline__ void all_sums(const Smem& s, double* out) {
  const int lane = threadIdx.x & 31;
  double v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) v[k] = lane < kWarps ? s.red[lane * 8 + k] : 0.0;
  // full butterfly: every lane of every warp ends with the same bits, since
  // each round adds two partial sums in either order (a + b == b + a)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
#pragma unroll
  for (int k = 0; k < 5; ++k) out[k] = v[k];
}
// Sum of nw <= 16 warp partials in the order of a 32-lane xor butterfly
// (v += shfl_xor(v, o) for o = 16 .. 1) whose lanes nw..31 hold zero: the
// decision phase's butterfly over a warp and tree_sum16 in one thread give
// the same bits (lane 0's tree; every lane ends with its bits).
__device__ __forceinline__ double tree_sum16(const double* p, int stride, int nw) {
  double t[16];
#pragma unroll
  for (int l = 0; l < 16; ++l) t[l] = (l < nw ? p[l * stride] : 0.0) + 0.0;
#pragma unroll
  for (int o = 8; o > 0; o >>= 1)
#pragma unroll
    for (int l = 0; l < o; ++l) t[l] = t[l] + t[l + o];
  return t[0];
}
__device__ __forceinline__ double total_of(const double* sum) {
  // energy.f: eysm = eyel + eyvw + eyhb + eyvr, then + eysl
  return ((sum[0] + sum[1]) + sum[2]) + sum[3] + sum[4];
}

// Full evaluation of the current coordinates by the whole block; partials in
// s.red (read them with all_sums after a barrier).
template <bool F32, bool ROWS, bool SASA>
__device__ void evaluate_block(const FFScalars& ff, const DMol& m, Smem& s, int* err) {
  double el = 0.0, vw = 0.0, hb = 0.0, sl = 0.0, vr = 0.0;
  pair_energy<F32, ROWS>(ff, m, s, threadIdx.x, blockDim.x, el, vw, hb);
  for (int v = threadIdx.x; v < m.nvar; v += blockDim.x) vr += s.et[v];
  if (SASA) sl = sasa_energy(ff, m, s, 0, kWarps, err, SasaInc{nullptr, s.sae, 0, 0, 0, 0, false, 0, 0});
  warp_partials(s, el, vw, hb, vr, sl);
}

// Sampling weight (canon.f:135-149, mulcan_par_mod.f90:380-410), FP64 with
// separately rounded products as in the reference.
__device__ double weight(const DWeight& w, double beta, double x) {
  if (w.kind == kWeightCanon) return __dmul_rn(beta, x);
  double v = __dadd_rn(__ddiv_rn(x, w.ebin), copysign(0.5, x));
  v = fmax((double)w.kmin, v);
  v = fmin((double)w.kmax, v);
  int k = (int)v - w.kmin;
  if (w.kind == kWeightMuca) return __dadd_rn(__dmul_rn(__dadd_rn(beta, w.b[k]), x), w.alpha[k]);
  return __dadd_rn(__dmul_rn(w.b[k], x), w.alpha[k]);
}

__device__ __forceinline__ void set_err(int* err, int code) {
  if (*err == 0) *err = code;
}

// Prepare a proposal (metropolis.f:42-66) from queue position `pos`:
// variable, new value and the cos/sin of the rotation it implies.
// part 0 fills every field but enew, part 1 only enew; the two parts run
// on two lanes through one sincos call (of the step and of the torsion
// argument), so that neither waits for the other.  part < 0: both, one
// after the other.
__device__ void make_proposal(const DMol& m, const Smem& s, int p, uint32_t pos, bool rndord,
                              Proposal& out, int part = -1) {
  const double* q = qbuf(s.mt);
  uint32_t k = pos;
  int ivar = p;
  if (rndord) {
    ivar = (int)__dmul_rn((double)m.nfree, q[k & (kQueue - 1)]);
    if (ivar >= m.nfree) ivar = m.nfree - 1;
    ++k;
  }
  int jv = m.idvr[ivar];
  double vold = s.vlvr[jv];
  double dv = __dmul_rn(m.axvr[jv], __dsub_rn(q[k & (kQueue - 1)], 0.5));
  ++k;
  double vnew = addang(vold, dv);
  if (part >= 0) {
    double x;
    if (part == 0) {
      x = difang(vold, vnew);
    } else {   // dihedral of the primary atom after this proposal's setvar (setvar.f:40-53)
      const double t0 = s.toat[m.var_atom[jv]];
      double to = __dadd_rn(t0, difang(t0, vnew));
      if (fabs(to) > kPi) to = __dsub_rn(to, copysign(kPi2, to));
      x = to * m.var_rn[jv];
    }
    double sv, cv;
    sincos(x, &sv, &cv);
    if (part == 0) {
      out.jv = jv;
      out.ivar = ivar;
      out.used = (int)(k - pos);
      out.b = m.var_base[jv];
      out.a = m.iow[out.b];
      out.lo = m.var_lo[jv];
      out.hi = m.var_hi[jv];
      out.cb = m.cross_off[jv];
      out.ce = m.cross_off[jv + 1];
      out.vold = vold;
      out.vnew = vnew;
      out.cth = cv;
      out.sth = sv;
      out.eold = s.et[jv];
    } else {
      const double e0 = m.var_e0[jv];
      out.enew = e0 != 0.0 ? e0 * (1.0 + m.var_sg[jv] * cv) : 0.0;
    }
    return;
  }
  {
    double sv, cv;
    sincos(difang(vold, vnew), &sv, &cv);
    out.jv = jv;
    out.ivar = ivar;
    out.used = (int)(k - pos);
    out.b = m.var_base[jv];
    out.a = m.iow[out.b];
    out.lo = m.var_lo[jv];
    out.hi = m.var_hi[jv];
    out.cb = m.cross_off[jv];
    out.ce = m.cross_off[jv + 1];
    out.vold = vold;
    out.vnew = vnew;
    out.cth = cv;
    out.sth = sv;
    out.eold = s.et[jv];
  }
  {
    // dihedral of the primary atom after this proposal's setvar (setvar.f:40-53)
    int iat = m.var_atom[jv];
    double t0 = s.toat[iat];
    double to = __dadd_rn(t0, difang(t0, vnew));
    if (fabs(to) > kPi) to = __dsub_rn(to, copysign(kPi2, to));
    out.enew = torsion_term(m, jv, to);
  }
}

// Load the chain's state into shared memory.
__device__ void load_chain(const DChains& ch, const DMol& m, int c, Smem& s) {
  const double* tg = ch.toat + (size_t)ch.toat_slot[c] * ch.tstride;
  for (int k = threadIdx.x; k < m.natoms; k += blockDim.x) s.toat[k] = tg[k];
  const double* vg = ch.vlvr + (size_t)c * ch.vstride;
  for (int k = threadIdx.x; k < m.nvar; k += blockDim.x) s.vlvr[k] = vg[k];
  const uint32_t* mg = ch.mt + (size_t)ch.mt_slot[c] * kMTWords;
  for (int k = threadIdx.x; k < kMTWords; k += blockDim.x) s.mt[k] = mg[k];
}

__device__ void store_chain(const DChains& ch, const DMol& m, int c, Smem& s) {
  double* tg = ch.toat + (size_t)ch.toat_slot[c] * ch.tstride;
  for (int k = threadIdx.x; k < m.natoms; k += blockDim.x) tg[k] = s.toat[k];
  double* vg = ch.vlvr + (size_t)c * ch.vstride;
  for (int k = threadIdx.x; k < m.nvar; k += blockDim.x) vg[k] = s.vlvr[k];
  uint32_t* mg = ch.mt + (size_t)ch.mt_slot[c] * kMTWords;
  for (int k = threadIdx.x; k < kMTWords; k += blockDim.x) mg[k] = s.mt[k];
  if (ch.coords) {
    double* cg = ch.coords + (size_t)c * 3 * ch.tstride;
    for (int k = threadIdx.x; k < m.natoms; k += blockDim.x) {
      cg[3 * k] = s.x[k];
      cg[3 * k + 1] = s.y[k];
      cg[3 * k + 2] = s.z[k];
    }
  }
}

__device__ void write_terms(const DChains& ch, int c, const double* sum) {
  double* t = ch.terms + (size_t)c * 6;
  for (int k = 0; k < 5; ++k) t[k] = sum[k];
  t[5] = ((sum[0] + sum[1]) + sum[2]) + sum[3];
}

}  // namespace

// ============================================================================ kernels

__global__ void k_seed(uint32_t* mt, const int* seeds, int nslots) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nslots) {
    uint32_t* slot = mt + (size_t)i * kMTWords;
    mt_seed(slot, (uint32_t)seeds[i]);
    slot[kQHead] = 0;
    slot[kQTail] = 0;
  }
}

__global__ void k_draw(uint32_t* mt, int slot, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0)
    for (int i = 0; i < n; ++i) out[i] = stream_next(mt + (size_t)slot * kMTWords);
}

// canon.f:60-67 random start, chains visited in the given order so that a
// shared stream is consumed exactly as the reference does.
__global__ void k_random_start(DMolSet set, DChains ch, const int* order, int n) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int q = 0; q < n; ++q) {
    int c = order[q];
    const DMol& m = set.mols[ch.mol_of_chain[c]];
    uint32_t* slot = ch.mt + (size_t)ch.mt_slot[c] * kMTWords;
    double* vl = ch.vlvr + (size_t)c * ch.vstride;
    for (int i = 0; i < m.nfree; ++i) {
      int iv = m.idvr[i];
      double dv = __dmul_rn(m.axvr[iv], __dsub_rn(stream_next(slot), 0.5));
      vl[iv] = addang(kPi, dv);
    }
  }
}

// Metropolis sweeps of the analytic SASA model, driven from the host one
// proposal at a time across all chains (metropolis.f:13-184 with energy()
// called per proposal, as the reference does, because esolan's random
// re-orientation draws from the stream between a proposal's numbers and its
// acceptance number).  One thread per chain in [first, first+n).
// k_propose: the proposal's numbers (metropolis.f:41-60) and the new value.
__global__ void k_propose(DMolSet set, DChains ch, int first, int n, int p, int rndord,
                          double* vold, int* jvar) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int c = first + t;
  const DMol& m = set.mols[ch.mol_of_chain[c]];
  uint32_t* slot = ch.mt + (size_t)ch.mt_slot[c] * kMTWords;
  int ivar = p;
  if (rndord) {
    ivar = (int)__dmul_rn((double)m.nfree, stream_next(slot));
    if (ivar >= m.nfree) ivar = m.nfree - 1;
  }
  const int jv = m.idvr[ivar];
  double* vl = ch.vlvr + (size_t)c * ch.vstride;
  const double vo = vl[jv];
  const double dv = __dmul_rn(m.axvr[jv], __dsub_rn(stream_next(slot), 0.5));
  vl[jv] = addang(vo, dv);
  vold[c] = vo;
  jvar[c] = jv;
}

// k_decide: acceptance of the proposal whose energy() is now in ch.eol
// (metropolis.f:72-87; -d against log r, exp only within 1e-10 of the
// threshold, as in k_sweep); eolc holds each chain's current energy.
__global__ void k_decide(DChains ch, DWeight w, int first, int n, const double* vold,
                         const int* jvar, double* eolc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int c = first + t;
  const double enw = ch.eol[c], eol = eolc[c], beta = ch.beta[c];
  const double delta = __dsub_rn(weight(w, beta, enw), weight(w, beta, eol));
  int up;
  if (delta <= 0.0) {
    up = 1;
  } else {
    uint32_t* slot = ch.mt + (size_t)ch.mt_slot[c] * kMTWords;
    const double rd = stream_next(slot);
    const double d = fmin(delta, 100.0);
    const double margin = -d - (rd > 0.0 ? log(rd) : -INFINITY);
    if (margin > 1e-10) up = 1;
    else if (margin < -1e-10) up = 0;
    else up = exp(-d) >= rd ? 1 : 0;
  }
  if (up) {
    eolc[c] = enw;
    ch.nacc[c] += 1;
  } else {
    ch.vlvr[(size_t)c * ch.vstride + jvar[c]] = vold[c];
  }
  ch.nprop[c] += 1;
  if (!isfinite(enw) && ch.err[c] == 0) ch.err[c] = kErrNonFinite;
}

// k_close: the closing energy() is in ch.eol; consistency check
// (metropolis.f:172-179), then eol is the tracked energy again.
__global__ void k_close(DChains ch, int first, int n, const double* eolc, int check,
                        double check_tol) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int c = first + t;
  const double eol = eolc[c], enew = ch.eol[c];
  if (check && fabs(eol - enew) > check_tol && eol < 100000.0 && ch.err[c] == 0)
    ch.err[c] = kErrConsistency;
  ch.eol[c] = eol;
}

__global__ void k_copy_eol(DChains ch, int first, int n, double* eolc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) eolc[first + t] = ch.eol[first + t];
}

// energy(): setvar + rebuild + energy for chains [first, first+gridDim.x).
// The dihedral state is updated in place exactly as the reference's energy()
// does; terms and eol of each chain receive the result.
template <bool F32, bool ROWS, bool SASA>
__global__ void __launch_bounds__(kThreads, 1) k_energy(DMolSet set, DChains ch, int first) {
  int c = first + blockIdx.x;
  const bool sasa = SASA;
  Smem s = carve(set, sasa);
  const DMol& m = stage_mol(set, ch, c, s);
  load_static(*set.ff, m, s, sasa);
  load_chain(ch, m, c, s);
  __syncthreads();
  setvar_all(m, s);
  __syncthreads();
  torsion_all(m, s);
  full_rebuild(m, s);
  evaluate_block<F32, ROWS, SASA>(set.f, m, s, &ch.err[c]);
  __syncthreads();
  double sum[5];
  all_sums(s, sum);
  if (threadIdx.x == 0) {
    double e = total_of(sum);
    ch.eol[c] = e;
    write_terms(ch, c, sum);
    if (!isfinite(e)) set_err(&ch.err[c], kErrNonFinite);
  }
  store_chain(ch, m, c, s);
}

// dE/dvlvr of every variable and the energy (gradient.f:13 with opeshe.f:12-317,
// vacuum) for chains [first, first + gridDim.x), in the order-free form of
// gradient_core.cuh: setvar and a full FP64 rebuild of the chain's variables,
// the force on every atom from all of its pairs of the mklist lists
// (shared-memory atomics), then one warp per variable sums the forces and
// torques over the atoms it moves, its contiguous range [var_lo, var_hi].
// grad[c * vstride + v]; the energy to ch.eol and its terms to ch.terms.
__global__ void __launch_bounds__(kThreads, 1) k_gradient(DMolSet set, DChains ch, int first,
                                                          double* grad) {
  const int c = first + blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Smem s = carve(set, false);
  const DMol& m = stage_mol(set, ch, c, s);
  load_static(*set.ff, m, s, false);
  load_chain(ch, m, c, s);
  __syncthreads();
  setvar_all(m, s);
  __syncthreads();
  torsion_all(m, s);
  full_rebuild(m, s);
  // forces in the rebuild frames' region, free after the rebuild
  double *Fx = s.bx, *Fy = s.by, *Fz = s.bz;
  for (int k = threadIdx.x; k < m.natoms; k += blockDim.x) Fx[k] = Fy[k] = Fz[k] = 0.0;
  __syncthreads();
  const GradTables tab{s.ta, s.ta14, s.tc, s.thb, set.f.conv, set.f.plt, set.f.slp, set.f.epsd};
  double e[3] = {0.0, 0.0, 0.0};
  auto pair = [&](int i, int j, bool is14) {
    const double dx = s.x[j] - s.x[i], dy = s.y[j] - s.y[i], dz = s.z[j] - s.z[i];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double f = gradient_pair(tab, s.type[i], s.type[j], s.cq[i], s.cq[j], r2, is14, e);
    atomicAdd(&Fx[i], f * dx);
    atomicAdd(&Fy[i], f * dy);
    atomicAdd(&Fz[i], f * dz);
    atomicAdd(&Fx[j], -f * dx);
    atomicAdd(&Fy[j], -f * dy);
    atomicAdd(&Fz[j], -f * dz);
  };
  for (int t = threadIdx.x; t < m.nchunks * 8; t += blockDim.x) {
    int i, j;
    if (gradient_chunk_pair(m.chunks, t, i, j)) pair(i, j, false);
  }
  for (int t = threadIdx.x; t < m.n14; t += blockDim.x) {
    const uint32_t w = m.pairs14[t];
    pair(int(w & 0x3fffu), int(w >> 14), true);
  }
  double vr = 0.0;
  for (int v = threadIdx.x; v < m.nvar; v += blockDim.x) vr += s.et[v];
  warp_partials(s, e[0], e[1], e[2], vr, 0.0);
  __syncthreads();
  for (int v = warp; v < m.nvar; v += kWarps) {
    double S[6] = {0, 0, 0, 0, 0, 0};
    for (int a = m.var_lo[v] + lane; a <= m.var_hi[v]; a += 32) {
      const double fx = Fx[a], fy = Fy[a], fz = Fz[a], x = s.x[a], y = s.y[a], z = s.z[a];
      S[0] += fx;
      S[1] += fy;
      S[2] += fz;
      S[3] += fy * z - fz * y;
      S[4] += fz * x - fx * z;
      S[5] += fx * y - fy * x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int k = 0; k < 6; ++k) S[k] += __shfl_xor_sync(0xffffffffu, S[k], o);
    if (lane == 0) {
      const int b = m.var_base[v], o = m.iow[b];
      double ev[3] = {s.x[b] - s.x[o], s.y[b] - s.y[o], s.z[b] - s.z[o]};
      const double inv = 1.0 / sqrt(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]);
      ev[0] *= inv;
      ev[1] *= inv;
      ev[2] *= inv;
      const double rb[3] = {s.x[b], s.y[b], s.z[b]};
      const double fvr = gradient_torsion_force(m.var_e0[v], m.var_sg[v], m.var_rn[v],
                                                s.toat[m.var_atom[v]]);
      grad[(size_t)c * ch.vstride + v] = gradient_variable(ev, rb, S, S + 3, fvr);
    }
  }
  double sum[5];
  all_sums(s, sum);
  if (threadIdx.x == 0) {
    const double en = total_of(sum);
    ch.eol[c] = en;
    write_terms(ch, c, sum);
    if (!isfinite(en)) set_err(&ch.err[c], kErrNonFinite);
  }
  store_chain(ch, m, c, s);
}

// Replica exchange (partem_s.f:210-232): alternate even/odd neighbour pairs,
// replica num_rep pairs with 1 when `wrap` is set.  temp_chain[k] is the chain
// at temperature label k (ipoi); betas[k] the inverse temperature of label k.
// One warp: the pairs of one parity step are disjoint, so lane k decides the
// k-th pair with the k-th uniform of the exchange stream (the order in which
// the reference's loop draws them).  `slot` is the exchange stream's slot
// (shared or global memory, used by this warp only); `lq` receives the logs
// the refill computes.  Energies are read past L1: in the fused sweep other
// blocks wrote them.
// Pairs of an exchange step of parity sw: i = nu, nu+2, ..., num_rep1
// (1-based); i == n is the wrap pair.
__device__ __forceinline__ int exchange_pairs(int n, int sw, int wrap) {
  const int num_rep1 = sw == 1 ? n - 1 : n, nu = sw == 1 ? 1 : 2;
  int npairs = 0;
  for (int i = nu; i <= num_rep1; i += 2)
    if (i != n || wrap) ++npairs;
  return npairs;
}

__device__ void exchange_core(const DChains& ch, int* temp_chain, const double* betas, int n,
                              uint32_t* slot, double* lq, int* iswitch, int wrap,
                              unsigned long long* stats) {
  const int lane = threadIdx.x & 31;
  if (n > 1) {
    const int sw = *iswitch;
    const int nu = sw == 1 ? 1 : 2;
    const int npairs = exchange_pairs(n, sw, wrap);
    uint32_t head = slot[kQHead];
    for (int base = 0; base < npairs; base += 32) {
      const int cnt = min(32, npairs - base);
      while ((int)(slot[kQTail] - head) < cnt) rng_refill_warp(slot, lq);   // < 32 before: fits
      __syncwarp();
      if (lane < cnt) {
        const int i = nu + 2 * (base + lane);   // the wrap pair, if any, is the last
        int j = i + 1;
        if (i == n) j = 1;
        const int in = temp_chain[i - 1], jn = temp_chain[j - 1];
        const double bi = betas[i - 1], bj = betas[j - 1];
        const double ein = __ldcg(&ch.eol[in]), ejn = __ldcg(&ch.eol[jn]);
        double delta = __dsub_rn(-__dmul_rn(bi, ejn), __dmul_rn(bj, ein));
        delta = __dadd_rn(delta, __dmul_rn(bi, ein));
        delta = __dadd_rn(delta, __dmul_rn(bj, ejn));
        const double ra = qbuf(slot)[(head + lane) & (kQueue - 1)];
        stats[2 * (i - 1)] += 1;
        if (ra <= exp(delta)) {
          temp_chain[i - 1] = jn;
          temp_chain[j - 1] = in;
          stats[2 * (i - 1) + 1] += 1;
        }
      }
      head += cnt;
      __syncwarp();
    }
    if (lane == 0) {
      slot[kQHead] = head;
      *iswitch = sw == 1 ? 2 : 1;
    }
  }
  __threadfence_block();
  __syncwarp();
  for (int k = lane; k < n; k += 32) ch.beta[temp_chain[k]] = betas[k];
  __threadfence();
  __syncwarp();
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier of all blocks of a cooperative launch (every block resident), with
// a bounded wait: after timeout_ns a block gives up, records kErrTimeout and
// returns false, and the caller ends its sweeps.  bar[0] counts arrivals
// (the barrier opens at `expected`, the launch's block count), bar[1] is the
// generation.  Returns the same value in every thread.
__device__ bool grid_barrier(unsigned* bar, unsigned expected, unsigned long long timeout_ns,
                             int* err, int* flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    if (arrived == expected) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      while (*gen == g) {
        if (global_ns() - t0 > timeout_ns) {
          ok = 0;
          if (*err == 0) *err = kErrTimeout;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    *flag = ok;
  }
  __syncthreads();
  return *flag != 0;
}

// Barrier of the pair warps 0 .. kWarps-2 of k_sweep (named barrier 1; the
// last warp does not take part).
__device__ __forceinline__ void pair_warps_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"((kWarps - 1) * 32) : "memory");
}

// The same barrier in two halves: grid_arrive counts this block in and
// returns the generation it saw (the barrier opens when the count reaches
// `expected`); grid_wait waits, bounded as above, for the generation to move
// on.  The block may work in between.  (The fused exchange's master block
// uses grid_count_in / grid_wait_round instead.)
__device__ unsigned grid_arrive(unsigned* bar, unsigned expected, unsigned* gen_seen) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    if (arrived == expected) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    }
    *gen_seen = g;
  }
  __syncthreads();
  return *gen_seen;
}
__device__ bool grid_wait(unsigned* bar, unsigned g, unsigned long long timeout_ns, int* err,
                          int* flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned* gen = bar + 1;
    const unsigned long long t0 = global_ns();
    while (*gen == g) {
      if (global_ns() - t0 > timeout_ns) {
        ok = 0;
        if (*err == 0) *err = kErrTimeout;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    *flag = ok;
  }
  __syncthreads();
  return *flag != 0;
}

// The master block of a fused parallel-tempering launch (the launch's extra
// last block, on an SM no chain uses): for each of the nsweeps rounds it
// waits, bounded, until all `expected` chains have arrived, runs the
// exchange with its first warp and opens the barrier; then
// it tops up the exchange stream's queue for the next round while the
// chains sweep.  It alone touches the exchange stream during the launch.  A
// wait that runs out ends it (the chains' own waits then run out too and
// record the timeout).
__device__ void pt_master(const DChains& ch, const DPTFused& pt, int nsweeps, unsigned expected) {
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  volatile unsigned* cnt = pt.bar;
  for (int r = 0; r < nsweeps; ++r) {
    int ok = 1;
    if (lane == 0) {
      // the count is never reset within the launch: round r is complete
      // when (r + 1) * expected chains have arrived
      const unsigned target = expected * (unsigned)(r + 1);
      const unsigned long long t0 = global_ns();
      while (*cnt < target) {   // (spinning: the master's SM has nothing else to do)
        if (global_ns() - t0 > pt.timeout_ns) {
          ok = 0;
          break;
        }
      }
      __threadfence();
    }
    if (!__shfl_sync(0xffffffffu, ok, 0)) return;
    exchange_core(ch, pt.temp_chain, pt.betas, pt.n, pt.mt, pt.lq, pt.iswitch, pt.wrap, pt.stats);
    if (lane == 0) atomicAdd(pt.bar + 1, 1u);   // the exchange's writes are fenced
    __syncwarp();
    // the refill the next exchange would start with, done now (the same
    // values at the same points of the stream)
    if (r + 1 < nsweeps && pt.n > 1) {
      const int need = min(32, exchange_pairs(pt.n, *pt.iswitch, pt.wrap));
      while ((int)(pt.mt[kQTail] - pt.mt[kQHead]) < need) rng_refill_warp(pt.mt, pt.lq);
    }
    __syncwarp();
  }
}

// A chain's arrival at the exchange master's barrier (no generation read).
__device__ void grid_count_in(unsigned* bar) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
  }
}
// Wait, bounded, until the master has opened `round` rounds (spinning: the
// wait is short and on the chains' critical path).
__device__ bool grid_wait_round(unsigned* bar, unsigned round, unsigned long long timeout_ns,
                                int* err, int* flag) {
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned* gen = bar + 1;
    const unsigned long long t0 = global_ns();
    while ((int)(*gen - round) < 0) {
      if (global_ns() - t0 > timeout_ns) {
        ok = 0;
        if (*err == 0) *err = kErrTimeout;
        break;
      }
    }
    __threadfence();
    *flag = ok;
  }
  __syncthreads();
  return *flag != 0;
}

// Atom t of the set a proposal moves: the subtree [lo, lo+span) or, when
// `flip`, every other atom.
__device__ __forceinline__ int moved_atom(int t, int lo, int span, bool flip) {
  return flip ? (t < lo ? t : t + span) : lo + t;
}

// The rotation a proposal applies: about the unit axis a -> b through b, by
// (cth, sth); by -theta when the complement of the subtree turns.
struct Axis {
  double px, py, pz, kx, ky, kz, cth, sth;
};
__device__ __forceinline__ Axis proposal_axis(const Smem& s, const Proposal& cur, bool flip) {
  Axis ax;
  ax.cth = cur.cth;
  ax.sth = flip ? -cur.sth : cur.sth;
  ax.px = s.x[cur.b];
  ax.py = s.y[cur.b];
  ax.pz = s.z[cur.b];
  double kx = ax.px - s.x[cur.a], ky = ax.py - s.y[cur.a], kz = ax.pz - s.z[cur.a];
  double inv = rsqrt(kx * kx + ky * ky + kz * kz);
  ax.kx = kx * inv;
  ax.ky = ky * inv;
  ax.kz = kz * inv;
  return ax;
}
// Rodrigues' rotation of one point (the in-place move of the one-at-a-time
// sweep and the copies of the speculative window use this one expression).
__device__ __forceinline__ void rotate_point(const Axis& ax, double x, double y, double z,
                                             double& ox, double& oy, double& oz) {
  double vx = x - ax.px, vy = y - ax.py, vz = z - ax.pz;
  double kd = ax.kx * vx + ax.ky * vy + ax.kz * vz;
  double cx = ax.ky * vz - ax.kz * vy, cy = ax.kz * vx - ax.kx * vz, cz = ax.kx * vy - ax.ky * vx;
  double f = kd * (1.0 - ax.cth);
  ox = ax.px + vx * ax.cth + cx * ax.sth + ax.kx * f;
  oy = ax.py + vy * ax.cth + cy * ax.sth + ax.ky * f;
  oz = ax.pz + vz * ax.cth + cz * ax.sth + ax.kz * f;
}

// Proposal k of a speculative window (metropolis.f:42-66) from the window's
// state, as the one-at-a-time sweep would make it after k rejected
// proposals: those leave the coordinates, the other variables and the
// energies as they were, the stream k * (used + 1) numbers further on, and
// the dihedral state after k more setvar replays, which on this variable's
// own atom (its base carries no other variable) move it towards its value
// until it stops changing.
__device__ void make_proposal_w(const DMol& m, const Smem& s, int p, uint32_t pos, bool rndord,
                                int replays, Proposal& out) {
  const double* q = qbuf(s.mt);
  uint32_t k = pos;
  int ivar = p;
  if (rndord) {
    ivar = (int)__dmul_rn((double)m.nfree, q[k & (kQueue - 1)]);
    if (ivar >= m.nfree) ivar = m.nfree - 1;
    ++k;
  }
  int jv = m.idvr[ivar];
  double vold = s.vlvr[jv];
  double dv = __dmul_rn(m.axvr[jv], __dsub_rn(q[k & (kQueue - 1)], 0.5));
  ++k;
  double vnew = addang(vold, dv);
  double sv, cv;
  sincos(difang(vold, vnew), &sv, &cv);
  int iat = m.var_atom[jv];
  double t0 = s.toat[iat];
  for (int r = 0; r < replays; ++r) {   // setvar_one on iat with vlvr = vold
    const double tsh = difang(t0, vold);
    if (tsh == 0.0) break;
    t0 = __dadd_rn(t0, tsh);
    if (fabs(t0) > kPi) t0 = __dsub_rn(t0, copysign(kPi2, t0));
  }
  double to = __dadd_rn(t0, difang(t0, vnew));
  if (fabs(to) > kPi) to = __dsub_rn(to, copysign(kPi2, to));
  out.jv = jv;
  out.ivar = ivar;
  out.used = (int)(k - pos);
  out.b = m.var_base[jv];
  out.a = m.iow[out.b];
  out.lo = m.var_lo[jv];
  out.hi = m.var_hi[jv];
  out.cb = m.cross_off[jv];
  out.ce = m.cross_off[jv + 1];
  out.vold = vold;
  out.vnew = vnew;
  out.cth = cv;
  out.sth = sv;
  out.enew = torsion_term(m, jv, to);
  out.eold = s.et[jv];
}

// The speculative window of the next proposals from p0 (one warp): up to
// set.window of them, ending before the 16th-proposal re-sum point and
// before a variable the window already holds; written to wp[0..wn).
__device__ void build_window(const DMolSet& set, const DMol& m, Smem& s, int p0, uint32_t hd,
                             bool rndord, Proposal* wp, int* err) {
  const int lane = threadIdx.x & 31;
  const int u = rndord ? 2 : 1;
  int wn = min(min(set.window, kMaxWindow), m.nfree - p0);
  wn = min(wn, 16 - (p0 & 15));
  // The window's numbers are in the queue: the sweep's first window tops it
  // up before any decision reads it, and every window's pair-sum phase tops
  // it up to 48 past its head, so a window of up to 8 (rndord: 3 numbers
  // each) finds its numbers without a refill here, where other warps may
  // still read the queue.  Anything else is a bug: the window shrinks to
  // what is queued and the chain reports a consistency error.
  const uint32_t avail = s.mt[kQTail] - hd;
  if ((uint32_t)(wn * (u + 1)) > avail) {
    wn = max(1, (int)(avail / (u + 1)));
    if (lane == 0) set_err(err, kErrConsistency);
  }
  Proposal P;
  int jv = -1;
  if (lane < wn) {
    make_proposal_w(m, s, p0 + lane, hd + (uint32_t)(lane * (u + 1)), rndord, lane, P);
    jv = P.jv;
  }
  bool again = false;
  for (int j = 0; j < kMaxWindow - 1; ++j) {
    const int jj = __shfl_sync(0xffffffffu, jv, j);
    if (j < lane && lane < wn && jj == jv) again = true;
  }
  const unsigned rm = __ballot_sync(0xffffffffu, again);
  if (rm) wn = min(wn, __ffs(rm) - 1);
  if (lane < wn) wp[lane] = P;
  if (lane == 0) s.sc->wn = wn;
  __syncwarp();
}

// The proposals of the rest of a sweep in speculative windows (FP32 pair
// terms, row-form molecules, relaxed states: the sweep's incremental mode).
// The proposals of a window are made from the same state, each as if the
// earlier ones had been rejected, which is exactly the state a rejection
// leaves.  Their energy changes are summed in one pass; the first accepted
// proposal ends the window and the later ones are dropped.  Each proposal
// draws the same numbers, is summed over the same pairs by the same threads
// in the same order and decided with the same arithmetic as in the
// one-at-a-time loop of k_sweep, so the trajectory is the same bit for bit:
// a window of w proposals costs three block barriers instead of 3w.
template <bool F32>
__device__ __noinline__ void sweep_windows(const DMolSet& set, const DMol& m, Smem& s,
                                           const DWeight& w, double beta, int* err, bool rndord,
                                           double& eol, double& etor, double& ep, uint32_t& head,
                                           unsigned long long& nacc, unsigned long long& nprop,
                                           unsigned long long& pterms) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int spec_warp = kWarps - 1;
  const int n = m.natoms;
  const int u = rndord ? 2 : 1;
  if (warp == spec_warp) {
    while (s.mt[kQTail] - head < 24) rng_refill_warp(s.mt, s.lq);   // nobody reads the queue yet
    build_window(set, m, s, 0, head, rndord, s.wprop, err);
  }
  __syncthreads();
  int p = 0, half = 0;
  while (p < m.nfree) {
    const Proposal* wp = s.wprop + half * kMaxWindow;
    const int wn = s.sc->wn;
    const bool resum = p > 0 && (p & 15) == 0;
    // ---- phase R: each proposal's moved atoms, turned, into its buffer;
    // the state's pair energy summed afresh every 16 proposals
    for (int idx = threadIdx.x; idx < wn * n; idx += blockDim.x) {
      const int k = idx / n, t = idx - k * n;
      const Proposal& P = wp[k];
      const int lo = m.var_lo[P.jv], hi = m.var_hi[P.jv];
      const bool flip = lo <= m.i3 && m.i3 <= hi;
      const int span = hi - lo + 1;
      if (t >= (flip ? n - span : span)) continue;
      const int a = moved_atom(t, lo, span, flip);
      if (flip && (a == P.a || a == P.b)) continue;   // on the axis
      const Axis ax = proposal_axis(s, P, flip);
      double ox, oy, oz;
      rotate_point(ax, s.x[a], s.y[a], s.z[a], ox, oy, oz);
      const int o = k * n + a;
      s.wx[o] = ox;
      s.wy[o] = oy;
      s.wz[o] = oz;
      split_hi_lo(ox, oy, oz, s.p4[a].w, s.l4[a].w, s.wp4[o], s.wl4[o]);
    }
    if (resum) {
      pterms += (unsigned long long)m.npairs;
      double el = 0.0, vw = 0.0, hb = 0.0;
      pair_rows<F32, true>(set.f, m, s, kWarps, el, vw, hb);
      double v = el;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) s.red[warp * 8 + 2] = v;
    }
    __syncthreads();
    if (resum) {
      double fresh_ep = 0.0;
      for (int k = 0; k < kWarps; ++k) fresh_ep += s.red[k * 8 + 2];
      eol = (eol - ep) + fresh_ep;
      ep = fresh_ep;
    }
    // ---- phase S: every proposal's energy change over the pairs across its
    // bond (after minus before, per thread, as the one-at-a-time sweep forms
    // it); meanwhile the last warp tops the stream's queue up to 48 numbers
    // past the head (16 at a time: at most 63 of its 64 places are taken)
    if (warp == spec_warp) {
      while (s.mt[kQTail] - head < 48) rng_refill_warp(s.mt, s.lq, 16);
    } else {
      for (int k = 0; k < wn; ++k) {
        const Proposal& P = wp[k];
        const int lo = m.var_lo[P.jv], hi = m.var_hi[P.jv];
        const bool flip = lo <= m.i3 && m.i3 <= hi;
        const double before = cross_rows_at<F32>(set.f, m, s, StatePos{s}, kWarps - 1, lo, hi);
        const double after = cross_rows_at<F32>(
            set.f, m, s, WindowPos{s, k * n, lo, hi, P.a, P.b, flip}, kWarps - 1, lo, hi);
        double v = ((after - before) + 0.0) + 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s.wred[warp * kMaxWindow + k] = v;
      }
    }
    __syncthreads();
    // ---- phase D: every warp decides the window the same way; lane k
    // takes proposal k (metropolis.f:72-87)
    double dpair = 0.0, enw = 0.0, etn = 0.0;
    int up = 0, drew = 1;
    if (lane < wn) {
      const Proposal& P = wp[lane];
      dpair = tree_sum16(s.wred + lane, kMaxWindow, kWarps - 1);
      const double epair = (ep + dpair) + 0.0;
      etn = (etor - P.eold) + P.enew;
      enw = epair + etn;
      const double delta = __dsub_rn(weight(w, beta, enw), weight(w, beta, eol));
      if (delta <= 0.0) {
        up = 1;
        drew = 0;
      } else {
        const uint32_t kq = (head + (uint32_t)(lane * (u + 1) + P.used)) & (kQueue - 1);
        const double rd = qbuf(s.mt)[kq], lrd = s.lq[kq];
        const double d = fmin(delta, 100.0);
        const double margin = -d - lrd;
        if (margin > 1e-10)
          up = 1;
        else if (margin < -1e-10)
          up = 0;
        else
          up = exp(-d) >= rd ? 1 : 0;
      }
    }
    const unsigned am = __ballot_sync(0xffffffffu, lane < wn && up);
    const int ks = am ? __ffs(am) - 1 : -1;
    const int last = ks >= 0 ? ks : wn - 1;
    const unsigned bad = __ballot_sync(0xffffffffu, lane <= last && !isfinite(enw));
    if (threadIdx.x == 0 && bad) set_err(err, kErrNonFinite);
    const int src = ks >= 0 ? ks : 0;
    const double enw_k = __shfl_sync(0xffffffffu, enw, src);
    const double etn_k = __shfl_sync(0xffffffffu, etn, src);
    const double dpair_k = __shfl_sync(0xffffffffu, dpair, src);
    const int drew_last = ks >= 0 ? __shfl_sync(0xffffffffu, drew, src) : 1;
    // ---- phase C: the accepted proposal's atoms take their turned copies;
    // the last warp replays the window's setvar calls on the dihedral state
    // and makes the next window
    if (ks >= 0) {
      const Proposal& P = wp[ks];
      const int lo = m.var_lo[P.jv], hi = m.var_hi[P.jv];
      const bool flip = lo <= m.i3 && m.i3 <= hi;
      const int span = hi - lo + 1;
      const int nmoved = flip ? n - span : span;
      for (int t = threadIdx.x; t < nmoved; t += blockDim.x) {
        const int a = moved_atom(t, lo, span, flip);
        if (flip && (a == P.a || a == P.b)) continue;
        const int o = ks * n + a;
        s.x[a] = s.wx[o];
        s.y[a] = s.wy[o];
        s.z[a] = s.wz[o];
        s.p4[a] = s.wp4[o];
        s.l4[a] = s.wl4[o];
      }
    }
    head += (uint32_t)(last * (u + 1) + u + drew_last);
    nprop += (unsigned long long)(last + 1);
    for (int k = 0; k < wn; ++k) pterms += 2ull * (unsigned long long)m.var_cross[wp[k].jv];
    if (ks >= 0) {
      ++nacc;
      eol = enw_k;
      etor = etn_k;
      ep += dpair_k;
    }
    p += last + 1;
    if (warp == spec_warp) {
      for (int j = 0; j <= last; ++j) {   // metropolis.f:53-87 through energy()'s setvar
        if (lane == 0) s.vlvr[wp[j].jv] = wp[j].vnew;
        __syncwarp();
        setvar_warp(m, s);
        __syncwarp();
        if (lane == 0 && j != ks) s.vlvr[wp[j].jv] = wp[j].vold;
        __syncwarp();
      }
      if (lane == 0 && ks >= 0) s.et[wp[ks].jv] = wp[ks].enew;
      __syncwarp();
      if (p < m.nfree)
        build_window(set, m, s, p, head, rndord, s.wprop + (half ^ 1) * kMaxWindow, err);
    }
    half ^= 1;
    __syncthreads();
  }
}

// nsweeps Metropolis sweeps (metropolis.f:13-184) of chains
// [first, first+gridDim.x).  Per sweep the reference calls energy() nvr+2
// times; here the start of every sweep does a full setvar and evaluation
// (with a rebuild: every sweep with FP64 pair terms, the first of the launch
// with FP32 ones), each proposal updates the dihedral state with the same
// setvar arithmetic, rotates the moving subtree in place and evaluates the
// pairs it changes (all of the lists, the crossing rows, or the crossing
// pairs against cached terms),
// and the closing consistency check of the launch's last sweep does a full
// evaluation (earlier sweeps are checked against the next opening one).
// With pt.on every sweep is followed by a replica exchange of all chains of
// the (cooperative) launch.
// Kernels are built per (F32, ROWS, SASA): a launch whose molecules have no
// row form, or that runs without solvation, carries none of that code (and
// none of its registers).
template <bool F32, bool ROWS, bool SASA>
__global__ void __launch_bounds__(kThreads, 1) k_sweep(DMolSet set, DChains ch, DWeight w, int first,
                                                       int nsweeps, int flags, double check_tol,
                                                       DPTFused pt) {
  if (pt.on && pt.master && blockIdx.x == gridDim.x - 1) {
    pt_master(ch, pt, nsweeps, gridDim.x - 1 + pt.extra);
    return;
  }
  const int c = first + blockIdx.x;
  const bool sasa = SASA;
  const bool rndord = (flags & kFlagRndOrd) != 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int spec_warp = kWarps - 1;            // setvar replay + next proposal
  const int nthr_pairs = (kWarps - 1) * 32;    // the other warps evaluate pairs
  Smem s = carve(set, sasa);
  Scalars& sc = *s.sc;
  const DMol& m = stage_mol(set, ch, c, s);
  load_static(*set.ff, m, s, sasa);
  load_chain(ch, m, c, s);
  double beta = ch.beta[c];
  int* err = &ch.err[c];
  unsigned long long nacc = 0, nprop = 0, pterms = 0;
  if (threadIdx.x == 0) sc.nred = 0;
  __syncthreads();
  // logs of the values already queued, then fill the queue
  if (warp == spec_warp) {
    uint32_t h = s.mt[kQHead], t = s.mt[kQTail];
    const double* q = qbuf(s.mt);
    for (uint32_t k = h + lane; k < t; k += 32) {
      double v = q[k & (kQueue - 1)];
      s.lq[k & (kQueue - 1)] = v > 0.0 ? log(v) : -INFINITY;
    }
    __syncwarp();
    while (s.mt[kQTail] - s.mt[kQHead] < 24) rng_refill_warp(s.mt, s.lq);
  }
  __syncthreads();
  uint32_t head = s.mt[kQHead];   // identical in every thread from here on
  double eol = ch.eol[c], enew = 0.0, etor = 0.0;
  double ep = 0.0;   // pair energy of the state (row-form molecules: updated by differences)
  // The closing energy() of a sweep that another sweep of this launch
  // follows is not evaluated on its own: that sweep's opening energy() (one
  // more setvar on the same variables, then the rebuild) stands in for it in
  // the consistency check.  energy() calls setvar every time (energy.f:47)
  // and setvar is not idempotent to the last bit, so it is the opening
  // evaluation that the trajectory must start from.
  bool check_pending = false;
  // The opening energy() of a sweep reads nothing of the temperature, so with
  // the fused exchange it is evaluated while the chain waits for the other
  // chains to arrive at the exchange (opened: done ahead).
  bool opened = false;
  // proposals sum only the pairs their turn changes against the cached terms
  // (cok: the cache holds the state, which has no pair inside its guard)
  const bool cmode = F32 && !SASA && set.cache_pairs > 0 && m.cache && !m.rows && !set.f.epsd;
  bool cok = false;
  // With FP32 pair terms only the launch's first sweep rebuilds the
  // coordinates from the dihedrals: later sweeps start from the coordinates
  // their predecessor's accepted rotations left, which differ from a rebuild
  // by FP64 rounding alone, far below what FP32 terms resolve.  FP64 pair
  // terms rebuild every sweep, as energy() does (metropolis.f:35).
  auto opening = [&](bool rebuild) {
    if (flags & kFlagExtraSetvar) {   // partem_s.f:194-198: setvar(i, vlvr) first
      setvar_all(m, s);
      __syncthreads();
    }
    // ---- eol = energy() (metropolis.f:35)
    setvar_all(m, s);
    __syncthreads();
    pterms += (unsigned long long)m.npairs;
    torsion_all(m, s);
    if (rebuild)
      full_rebuild(m, s);
    else
      __syncthreads();
    evaluate_block<F32, ROWS, SASA>(set.f, m, s, err);
    __syncthreads();
    double sum[5];
    all_sums(s, sum);
    enew = total_of(sum);
    etor = sum[3];
    ep = (sum[0] + sum[1]) + sum[2];
    if (cmode) {
      pterms += (unsigned long long)m.npairs;
      cok = !fill_pair_cache(set.f, m, s);
    }
  };

  // The sweep's first proposal (by the last warp; with the fused exchange it
  // is made while the chain waits for the exchange: it reads nothing of the
  // temperature).
  bool prepared = false;
  auto first_proposal = [&]() {
    if (warp == spec_warp) {
      if (lane < 2) make_proposal(m, s, 0, head, rndord, sc.spec[4], lane);
      __syncwarp();
      if (lane == 0) {
        s.vlvr[sc.spec[4].jv] = sc.spec[4].vnew;
        sc.refill = 0;
      }
    }
  };

  for (int sw = 0; sw < nsweeps; ++sw) {
    if (!opened) opening(!F32 || sw == 0);
    opened = false;
    if (check_pending && threadIdx.x == 0 && !(flags & kFlagNoCheck) &&
        fabs(eol - enew) > check_tol && eol < 100000.0)
      set_err(err, kErrConsistency);
    check_pending = false;
    eol = enew;
    const bool relaxed = fabs(eol) < 1e4;
    bool windowed = false;
    if constexpr (ROWS && F32 && !SASA) {
      // the incremental mode in speculative windows (same trajectory, fewer barriers)
      windowed = m.rows && !set.f.epsd && relaxed && set.window >= 2 && m.nfree > 0;
      if (windowed)
        sweep_windows<F32>(set, m, s, w, beta, err, rndord, eol, etor, ep, head, nacc, nprop,
                           pterms);
    }
    if (!windowed && m.nfree > 0 && !prepared) first_proposal();
    prepared = false;
    __syncthreads();

    int cur_slot = 4;   // sc.spec slot of the current proposal
    for (int p = 0, par = 0; p < (windowed ? 0 : m.nfree); ++p, par ^= 1) {
      const Proposal cur = sc.spec[cur_slot];
      const int lo = cur.lo, hi = cur.hi;
      // The rebuild holds the first three backbone atoms in place (setgbl):
      // when the subtree holds i3 (the dihedral about i1-i2), the rest of the
      // molecule turns by -theta instead, so the coordinates keep the
      // rebuild's orientation (the SASA test points are fixed in space).
      const bool flip = lo <= m.i3 && m.i3 <= hi;
      const int span = hi - lo + 1;
      const int nmoved = flip ? m.natoms - span : span;
      if (SASA && threadIdx.x == 0) {   // heavy-atom index range of [lo, hi]
        int l = 0, r = m.nheavy;
        while (l < r) {
          const int mid = (l + r) >> 1;
          if (m.heavy[mid] < lo) l = mid + 1; else r = mid;
        }
        sc.hlo = l;
        r = m.nheavy;
        while (l < r) {
          const int mid = (l + r) >> 1;
          if (m.heavy[mid] <= hi) l = mid + 1; else r = mid;
        }
        sc.hhi = l;
      }
      // ---- phase A0 (row-form molecules): energy of the pairs across the
      // rotating bond before the move; after it, phase B computes the same
      // sum again and the pair energy changes by the difference
      // (FP32 pair terms only: in FP64 mode every proposal is summed in full,
      // so that eol carries no accumulated rounding into the reference's
      // 1e-6 consistency check)
      // The FP32 differences carry the rounding of the terms they touch, so
      // they are used only for relaxed states (|E| < 1e4 kcal/mol at the
      // sweep's start: no clash terms) and the state's pair energy is summed
      // afresh every 16 proposals (same coordinates; eol follows).
      const bool incr = ROWS && F32 && m.rows && !set.f.epsd && relaxed;
      const bool cached = cmode && cok;
      double xold = 0.0;
      pterms += incr     ? 2ull * (unsigned long long)m.var_cross[cur.jv]
                : cached ? (unsigned long long)(cur.ce - cur.cb)
                         : (unsigned long long)m.npairs;
      if (incr && p > 0 && (p & 15) == 0) {
        pterms += (unsigned long long)m.npairs;
        double el = 0.0, vw = 0.0, hb = 0.0;
        pair_rows<F32, true>(set.f, m, s, kWarps, el, vw, hb);
        double v = el;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s.red[warp * 8 + 2] = v;
        __syncthreads();
        double fresh_ep = 0.0;
        for (int k = 0; k < kWarps; ++k) fresh_ep += s.red[k * 8 + 2];
        eol = (eol - ep) + fresh_ep;
        ep = fresh_ep;
        __syncthreads();
      }
      // ---- phase A: rotate the subtree of cur.jv about its bond (+theta),
      // by the pair warps alone (they sync among themselves); the last warp,
      // which reads no coordinates, goes straight on to its phase B work
      if (warp != spec_warp) {
        if (incr) {
          xold = cross_rows<F32>(set.f, m, s, kWarps - 1, lo, hi);
          pair_warps_sync();
        }
        const Axis ax = proposal_axis(s, cur, flip);
        for (int t = threadIdx.x; t < nmoved; t += nthr_pairs) {
          const int k = moved_atom(t, lo, span, flip);
          if (flip && (k == cur.a || k == cur.b)) continue;   // on the axis
          const double x0 = s.x[k], y0 = s.y[k], z0 = s.z[k];
          s.bx[k] = x0;
          s.by[k] = y0;
          s.bz[k] = z0;
          double ox, oy, oz;
          rotate_point(ax, x0, y0, z0, ox, oy, oz);
          s.x[k] = ox;
          s.y[k] = oy;
          s.z[k] = oz;
          if (F32) f32_move(s, k, ox, oy, oz);
        }
        pair_warps_sync();
      }
      // ---- phase B: pair energy; the last warp replays this proposal's
      // setvar call on the dihedral state and prepares proposal p+1
      if (warp != spec_warp) {
        double el = 0.0, vw = 0.0, hb = 0.0, sl = 0.0;
        if (incr) {
          el = cross_rows<F32>(set.f, m, s, kWarps - 1, lo, hi) - xold;   // the change
        } else if (cached) {   // the change, and in sl the count of guarded pairs
          int nc = 0;
          el = cached_delta(set.f, m, s, cur.cb, cur.ce, threadIdx.x, nthr_pairs, nc);
          sl = (double)nc;
        } else if (ROWS && m.rows) {
          pair_rows<F32, true>(set.f, m, s, kWarps - 1, el, vw, hb);
        } else {
          pair_energy<F32, false>(set.f, m, s, threadIdx.x, nthr_pairs, el, vw, hb);
        }
        if (sasa)
          sl = sasa_energy(set.f, m, s, 0, kWarps - 1, err,
                           SasaInc{s.sae, s.san, lo, span, cur.a, cur.b, flip, sc.hlo, sc.hhi});
        double v = (el + vw) + hb;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (sasa) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) sl += __shfl_xor_sync(0xffffffffu, sl, o);
        } else {   // the cached terms need only whether some pair was guarded
          sl = __any_sync(0xffffffffu, sl > 0.0) ? 1.0 : 0.0;
        }
        if (lane == 0) {
          s.red[warp * 8] = v;
          s.red[warp * 8 + 1] = sl;
        }
        // the last pair warp to get here sums the warps' partials once, in
        // a fixed order (the butterfly of tree_sum16), for every warp to read
        unsigned last = 0;
        if (lane == 0) {
          __threadfence_block();
          last = atomicAdd(&sc.nred, 1u) == (unsigned)(kWarps - 2) ? 1u : 0u;
        }
        if (__shfl_sync(0xffffffffu, last, 0)) {
          __threadfence_block();
          // at most 16 partials: lanes 16-31 hold zeros, and the butterfly's
          // first step (offset 16) would only add them
          static_assert(kWarps - 1 <= 16, "pair-warp partials fit in 16 lanes");
          double t = lane < kWarps - 1 ? s.red[lane * 8] : 0.0;
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
          double e1 = 0.0;
          if (sasa) {
            e1 = lane < kWarps - 1 ? s.red[lane * 8 + 1] : 0.0;
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) e1 += __shfl_xor_sync(0xffffffffu, e1, o);
          }
          const bool anyc = __any_sync(0xffffffffu, lane < kWarps - 1 && s.red[lane * 8 + 1] > 0.0);
          if (lane == 0) {
            sc.dsum = t;
            sc.dsl = e1;
            sc.dclash = anyc ? 1 : 0;
            sc.nred = 0;
          }
        }
      } else {
        setvar_warp(m, s);
        __syncwarp();
        if (sc.refill) rng_refill_warp(s.mt, s.lq);
        if (lane < 4 && p + 1 < m.nfree)   // two proposals, each on two lanes
          make_proposal(m, s, p + 1, head + cur.used + (lane & 1), rndord,
                        sc.spec[2 * par + (lane & 1)], lane >> 1);
      }
      __syncthreads();
      // ---- phase C: every warp sums and decides (metropolis.f:72-87)
      const double dpair = sc.dsum;
      const double esl = sasa ? sc.dsl : 0.0;
      const bool pclash = cached && sc.dclash != 0;   // some warp met a guarded pair
      // pair energy of the proposal: the state's plus the change (row form,
      // cached terms), or the full sum
      const double epair = ((incr || cached) ? ep + dpair : dpair) + esl;
      // every value read here was written before the last barrier
      const double etor_new = (etor - cur.eold) + cur.enew;
      const double enw = epair + etor_new;
      double delta = __dsub_rn(weight(w, beta, enw), weight(w, beta, eol));
      int up, drew;
      if (delta <= 0.0) {
        up = 1;
        drew = 0;
      } else {
        drew = 1;
        uint32_t k = (head + cur.used) & (kQueue - 1);
        double rd = qbuf(s.mt)[k], lrd = s.lq[k];
        double d = fmin(delta, 100.0);
        double margin = -d - lrd;
        if (margin > 1e-10)
          up = 1;
        else if (margin < -1e-10)
          up = 0;
        else
          up = exp(-d) >= rd ? 1 : 0;
      }
      if (up) {
        eol = enw;
        etor = etor_new;
        if (incr || cached) ep += dpair;
        if (sasa)   // the proposal's SASA terms become the state's
          for (int h = threadIdx.x; h < m.nheavy; h += blockDim.x) s.sae[h] = s.san[h];
        if (cached) {   // the new terms become the state's (a guarded pair: full sums from here)
          if (pclash) {
            cok = false;
          } else {
            const int cb = cur.cb, ce = cur.ce;
            for (int q = cb + (int)threadIdx.x; q < ce; q += blockDim.x)
              s.ecache[m.cross_idx[q]] = s.tnew[q - cb];
          }
        }
      } else {
        for (int t = threadIdx.x; t < nmoved; t += blockDim.x) {
          const int k = moved_atom(t, lo, span, flip);
          if (flip && (k == cur.a || k == cur.b)) continue;
          const double x0 = s.bx[k], y0 = s.by[k], z0 = s.bz[k];
          s.x[k] = x0;
          s.y[k] = y0;
          s.z[k] = z0;
          if (F32) f32_move(s, k, x0, y0, z0);
        }
      }
      head += cur.used + drew;
      ++nprop;
      nacc += up;
      // the state's bookkeeping on the last warp, which restores no atoms
      // (it moves none) and so reaches this point first
      if (threadIdx.x == spec_warp * 32) {
        if (up)
          s.et[cur.jv] = cur.enew;
        else
          s.vlvr[cur.jv] = cur.vold;
        if (!isfinite(enw)) set_err(err, kErrNonFinite);
        if (p + 1 < m.nfree) {
          Proposal& nx = sc.spec[2 * par + drew];
          if (nx.jv == cur.jv) {   // same variable again: from the state after this decision
            make_proposal(m, s, p + 1, head, rndord, sc.spec[4]);
            s.vlvr[cur.jv] = sc.spec[4].vnew;
          } else {
            s.vlvr[nx.jv] = nx.vnew;
          }
        }
        sc.refill = (s.mt[kQTail] - head) < 24 ? 1 : 0;
      }
      __syncthreads();
      // the next proposal's slot (every thread reads the same words)
      if (p + 1 < m.nfree) cur_slot = sc.spec[2 * par + drew].jv == cur.jv ? 4 : 2 * par + drew;
    }
    // with the exchange master, the sweep's energy is published and the chain
    // counted in at once: the closing setvar and checks need no temperature
    if (pt.on && pt.master) {
      if (threadIdx.x == 0) ch.eol[c] = eol;
      grid_count_in(pt.bar);
    }
    // ---- closing energy() and consistency check (metropolis.f:172-179)
    if (warp == spec_warp) {
      const bool low = __shfl_sync(0xffffffffu, (s.mt[kQTail] - head) < 24u ? 1 : 0, 0) != 0;
      if (low) rng_refill_warp(s.mt, s.lq);
    }
    setvar_all(m, s);
    __syncthreads();
    if (sw + 1 == nsweeps) {
      pterms += (unsigned long long)m.npairs;
      torsion_all(m, s);
      full_rebuild(m, s);
      evaluate_block<F32, ROWS, SASA>(set.f, m, s, err);
      __syncthreads();
      double sum[5];
      all_sums(s, sum);
      enew = total_of(sum);
      if (threadIdx.x == 0) {
        if (!(flags & kFlagNoCheck) && fabs(eol - enew) > check_tol && eol < 100000.0)
          set_err(err, kErrConsistency);
        write_terms(ch, c, sum);
      }
      __syncthreads();
    } else {
      check_pending = true;
    }
    if (pt.on) {
      // fused parallel tempering: every chain's energy is in place, the
      // exchange runs (in the master block, or else in block 0's first warp
      // between two barriers), then every chain takes up its new
      // temperature; between its arrival and its wait, a chain evaluates the
      // opening energy of its next sweep
      // (with the master the chain arrived above, and the generation is the
      // number of rounds exchanged, so it need not be read before arriving)
      const unsigned nchain = gridDim.x - (pt.master ? 1u : 0u) + pt.extra;
      unsigned gen = 0u;
      if (!pt.master) {
        if (threadIdx.x == 0) ch.eol[c] = eol;
        gen = grid_arrive(pt.bar, nchain, &sc.gen);
      }
      if (sw + 1 < nsweeps) {
        opening(!F32);
        opened = true;
        bool win_next = false;   // the next sweep runs in speculative windows
        if constexpr (ROWS && F32 && !SASA)
          win_next = m.rows && !set.f.epsd && fabs(enew) < 1e4 && set.window >= 2 && m.nfree > 0;
        if (!win_next && m.nfree > 0) {
          first_proposal();
          prepared = true;
        }
      }
      if (pt.master) {
        if (!grid_wait_round(pt.bar, (unsigned)(sw + 1), pt.timeout_ns, err, &sc.gsync)) break;
      } else if (!grid_wait(pt.bar, gen, pt.timeout_ns, err, &sc.gsync)) {
        break;
      }
      if (!pt.master) {
        if (blockIdx.x == 0 && warp == 0)
          exchange_core(ch, pt.temp_chain, pt.betas, pt.n, pt.mt, pt.lq, pt.iswitch, pt.wrap,
                        pt.stats);
        if (!grid_barrier(pt.bar, nchain, pt.timeout_ns, err, &sc.gsync)) break;
      }
      beta = __ldcg(&ch.beta[c]);
    }
  }
  if (threadIdx.x == 0) {
    ch.eol[c] = eol;
    ch.nacc[c] += nacc;
    ch.nprop[c] += nprop;
    ch.pterms[c] += pterms;
    s.mt[kQHead] = head;
  }
  __syncthreads();
  store_chain(ch, m, c, s);
}

// ============================================================================ delayed acceptance
// Two-stage Metropolis step (delayed acceptance) with the energy surrogate as
// the first stage.  For a proposal y from state x (same proposal as the plain
// sweep, metropolis.f:42-66):
//   stage 1: d1 = W(s(y)) - W(s(x)), pass with min(1, exp(-d1));
//   stage 2 (only when stage 1 passes): the exact energy E(y);
//            d2 = [W(E(y)) - W(E(x))] - d1, accept with min(1, exp(-d2)).
// W is the sampling weight (beta*E canonically) and s the surrogate, a fixed
// function of the state, so the chain keeps the exact stationary
// distribution.  A chain whose stage-2 acceptance falls below the floor (after
// da_min stage-1 passes) takes plain steps (stage 1 skipped) from its next
// sweep on.  Uniforms come from the chain's own MT19937 stream as in the plain
// sweep; the extra stage-1 draws make the stream's use differ from it.

__device__ __forceinline__ float bf16_round(float v) {
  return __bfloat162float(__float2bfloat16(v));
}
__device__ __forceinline__ float silu_f(float z) { return z / (1.f + expf(-z)); }

// Features of the current state: sin/cos of every free dihedral, rounded to
// BF16 as the training kernels round them.
__device__ void sur_features(const DMol& m, Smem& s) {
  for (int k = threadIdx.x; k < m.nfree; k += blockDim.x) {
    float sn, cs;
    sincosf((float)s.vlvr[m.idvr[k]], &sn, &cs);
    s.daf[2 * k] = bf16_round(sn);
    s.daf[2 * k + 1] = bf16_round(cs);
  }
}

__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}
__device__ __forceinline__ uint32_t ldg32(const __nv_bfloat16* p) {
  return __ldg(reinterpret_cast<const unsigned int*>(p));
}
__device__ __forceinline__ void mma_bf16_16816(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One dense layer for the 16 rows of a batch on the tensor cores:
// out[r][n] = bf16(silu(b[n] + sum_k A[r][k] Wt[n][k])), A [16][K] BF16 in
// shared memory (row stride lda), Wt [256][K] BF16 (the transposed weights,
// K contiguous, read from L2).  Warp w computes columns 16w..16w+15 (two
// m16n8k16 tiles).  Every row is computed by the same instructions, so a
// row's result does not depend on the other rows.
__device__ void mlp_layer16(const __nv_bfloat16* __restrict__ Wt, const float* __restrict__ b,
                            const __nv_bfloat16* A, int lda, int K, __nv_bfloat16* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int n0 = warp * 16;
  const __nv_bfloat16* w0 = Wt + (size_t)(n0 + g) * K + 2 * t;
  const __nv_bfloat16* w1 = Wt + (size_t)(n0 + 8 + g) * K + 2 * t;
  float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
  for (int kk = 0; kk < K; kk += 16) {
    const uint32_t b0[2] = {ldg32(w0 + kk), ldg32(w0 + kk + 8)};
    const uint32_t b1[2] = {ldg32(w1 + kk), ldg32(w1 + kk + 8)};
    const uint32_t a[4] = {lds32(A + g * lda + kk + 2 * t), lds32(A + (g + 8) * lda + kk + 2 * t),
                           lds32(A + g * lda + kk + 2 * t + 8),
                           lds32(A + (g + 8) * lda + kk + 2 * t + 8)};
    mma_bf16_16816(c0, a, b0);
    mma_bf16_16816(c1, a, b1);
  }
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int r = g + 8 * h;
      const int n = n0 + 2 * t + q;
      out[r * 264 + n] = __float2bfloat16(silu_f(c0[2 * h + q] + b[n]));
      out[r * 264 + n + 8] = __float2bfloat16(silu_f(c1[2 * h + q] + b[n + 8]));
    }
  __syncthreads();
}

// Surrogate energies (kcal/mol) of the 16 feature rows in s.dfe, into
// s.dsv.  Needs 16 warps.
__device__ void sur_batch(const DSurrogate& S, Smem& s) {
  const int lda1 = S.nin_pad + 8;
  mlp_layer16(S.w1t, S.b1, s.dfe, lda1, S.nin_pad, s.dh0);
  mlp_layer16(S.w2t, S.b2, s.dh0, 264, 256, s.dh1);
  mlp_layer16(S.w3t, S.b3, s.dh1, 264, 256, s.dh0);
  const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
  float v = 0.f;
  for (int n = lane; n < 256; n += 32)
    v += __bfloat162float(s.dh0[r * 264 + n]) * __bfloat162float(S.w4[n]);
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) s.dsv[r] = S.mu + S.sigma * (v + S.b4[0]);
  __syncthreads();
}

// Feature row r of the batch: the state's features with free dihedral kx
// set to angle a (kx < 0: the state itself); padding columns zero.
__device__ void sur_row(const DSurrogate& S, Smem& s, int r, int kx, double a) {
  const int lda1 = S.nin_pad + 8;
  float sn = 0.f, cs = 0.f;
  if (kx >= 0) sincosf((float)a, &sn, &cs);
  for (int c = threadIdx.x & 31; c < S.nin_pad; c += 32) {
    float v = c < S.nin ? s.daf[c] : 0.f;
    if ((c >> 1) == kx) v = (c & 1) ? bf16_round(cs) : bf16_round(sn);
    s.dfe[r * lda1 + c] = __float2bfloat16(v);
  }
}

// Metropolis test of exp(-d) against queue position k (as the plain sweep).
__device__ __forceinline__ int mh_accept(const Smem& s, uint32_t k, double d) {
  const double rd = qbuf(s.mt)[k & (kQueue - 1)], lrd = s.lq[k & (kQueue - 1)];
  d = fmin(d, 100.0);
  const double margin = -d - lrd;
  if (margin > 1e-10) return 1;
  if (margin < -1e-10) return 0;
  return exp(-d) >= rd ? 1 : 0;
}

template <bool F32, bool ROWS, bool SASA>
__global__ void __launch_bounds__(kThreads, 1) k_sweep_da(DMolSet set, DChains ch, DWeight w,
                                                          int first, int nsweeps, int flags,
                                                          double check_tol) {
  const int c = first + blockIdx.x;
  const bool rndord = (flags & kFlagRndOrd) != 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Smem s = carve(set, SASA);
  const DMol& m = stage_mol(set, ch, c, s);
  load_static(*set.ff, m, s, SASA);
  load_chain(ch, m, c, s);
  const double beta = ch.beta[c];
  int* err = &ch.err[c];
  const DSurrogate& S = ch.sur;
  unsigned long long nacc = 0, nprop = 0, n1 = ch.da_n1[c], n2 = ch.da_n2[c];
  const unsigned long long n1_0 = n1, n2_0 = n2;
  __syncthreads();
  if (warp == 0) {
    uint32_t h = s.mt[kQHead], t = s.mt[kQTail];
    const double* q = qbuf(s.mt);
    for (uint32_t k = h + lane; k < t; k += 32) {
      double v = q[k & (kQueue - 1)];
      s.lq[k & (kQueue - 1)] = v > 0.0 ? log(v) : -INFINITY;
    }
    __syncwarp();
    while (s.mt[kQTail] - s.mt[kQHead] < 24) rng_refill_warp(s.mt, s.lq);
  }
  __syncthreads();
  uint32_t head = s.mt[kQHead];
  double eol = 0.0, etor = 0.0;
  bool check_pending = false;   // as in k_sweep: the next opening energy() checks

  for (int sw = 0; sw < nsweeps; ++sw) {
    // stage-2 acceptance n2 / max(n1, 1) below the floor, once n1 >= da_min
    const bool plain = n1 >= (unsigned long long)ch.da_min &&
                       (double)n2 < (double)ch.da_floor * (double)(n1 > 0 ? n1 : 1);
    // ---- energy() and surrogate of the sweep's starting state
    setvar_all(m, s);
    __syncthreads();
    torsion_all(m, s);
    full_rebuild(m, s);
    evaluate_block<F32, ROWS, SASA>(set.f, m, s, err);
    __syncthreads();
    {
      double sum[5];
      all_sums(s, sum);
      const double enew = total_of(sum);
      if (check_pending && threadIdx.x == 0 && !(flags & kFlagNoCheck) &&
          fabs(eol - enew) > check_tol && eol < 100000.0)
        set_err(err, kErrConsistency);
      check_pending = false;
      eol = enew;
      etor = sum[3];
    }
    sur_features(m, s);
    __syncthreads();
    float s_cur = 0.f;
    if (!plain) {   // the state's own surrogate energy: row 0 of a batch
      if (warp == 0) sur_row(S, s, 0, -1, 0.0);
      __syncthreads();
      sur_batch(S, s);
      s_cur = s.dsv[0];
    }
    // Proposals are drawn in batches of up to 16 (variables p, p+1, ... in
    // turn; each one from the current state) and screened together on the
    // tensor cores.  They are then decided in order; an accepted move changes
    // the state, so the batch ends there and the next one starts after it.
    // Drawn proposals that a batch's end leaves unused are dropped (their
    // uniforms are independent of everything else).
    int p = 0;
    while (p < m.nfree) {
      const int per = rndord ? 2 : 1;              // uniforms per proposal
      // the 64-entry queue is refilled 32 at a time below 32 entries: a
      // batch takes at most 30 of them and leaves two for its first decisions
      const int nb = plain ? 1 : min(min(16, 30 / per), m.nfree - p);
      if (warp == 0) {
        while (true) {   // room for the batch's proposals and two decisions
          const bool low =
              __shfl_sync(0xffffffffu, (s.mt[kQTail] - head) < (uint32_t)(nb * per + 2) ? 1 : 0, 0) != 0;
          if (!low) break;
          rng_refill_warp(s.mt, s.lq);
        }
        if (lane < nb) make_proposal(m, s, p + lane, head + lane * per, rndord, s.dprop[lane]);
      }
      __syncthreads();
      head += nb * per;
      if (!plain) {
        for (int r = warp; r < 16; r += kWarps) {
          if (r < nb)
            sur_row(S, s, r, s.dprop[r].ivar, s.dprop[r].vnew);
          else
            sur_row(S, s, r, -1, 0.0);
        }
        __syncthreads();
        sur_batch(S, s);
      }
      int next = p + nb;
      for (int j = 0; j < nb; ++j) {
        if (warp == 0) {   // at most two decisions per proposal
          const bool low = __shfl_sync(0xffffffffu, (s.mt[kQTail] - head) < 2u ? 1 : 0, 0) != 0;
          if (low) rng_refill_warp(s.mt, s.lq);
        }
        __syncthreads();
        const Proposal cur = s.dprop[j];
        ++nprop;
        // ---- stage 1: surrogate
        double d1 = 0.0;
        float s_new = s_cur;
        if (!plain) {
          s_new = s.dsv[j];
          d1 = __dsub_rn(weight(w, beta, (double)s_new), weight(w, beta, (double)s_cur));
          int pass = 1;
          if (d1 > 0.0) {
            pass = mh_accept(s, head, d1);
            head += 1;
          }
          if (!pass) continue;   // rejected without the exact energy
          ++n1;
        }
        // ---- stage 2: exact energy of the proposal
        __syncthreads();
        if (threadIdx.x == 0) s.vlvr[cur.jv] = cur.vnew;
        const int lo = m.var_lo[cur.jv], hi = m.var_hi[cur.jv];
        const bool flip = lo <= m.i3 && m.i3 <= hi;
        const int span = hi - lo + 1;
        const int nmoved = flip ? m.natoms - span : span;
        {
          const double sth = flip ? -cur.sth : cur.sth;
          double px = s.x[cur.b], py = s.y[cur.b], pz = s.z[cur.b];
          double kx = px - s.x[cur.a], ky = py - s.y[cur.a], kz = pz - s.z[cur.a];
          double inv = rsqrt(kx * kx + ky * ky + kz * kz);
          kx *= inv;
          ky *= inv;
          kz *= inv;
          __syncthreads();   // every thread has read the axis
          for (int t = threadIdx.x; t < nmoved; t += blockDim.x) {
            const int k = moved_atom(t, lo, span, flip);
            if (flip && (k == cur.a || k == cur.b)) continue;
            double vx = s.x[k] - px, vy = s.y[k] - py, vz = s.z[k] - pz;
            s.bx[k] = s.x[k];
            s.by[k] = s.y[k];
            s.bz[k] = s.z[k];
            double kd = kx * vx + ky * vy + kz * vz;
            double cx = ky * vz - kz * vy, cy = kz * vx - kx * vz, cz = kx * vy - ky * vx;
            double f = kd * (1.0 - cur.cth);
            s.x[k] = px + vx * cur.cth + cx * sth + kx * f;
            s.y[k] = py + vy * cur.cth + cy * sth + ky * f;
            s.z[k] = pz + vz * cur.cth + cz * sth + kz * f;
            if (F32) f32_copy(s, k);
          }
        }
        __syncthreads();
        {
          double el = 0.0, vw = 0.0, hb = 0.0, sl = 0.0;
          if (ROWS && m.rows)
            pair_rows<F32, true>(set.f, m, s, kWarps, el, vw, hb);
          else
            pair_energy<F32, false>(set.f, m, s, threadIdx.x, blockDim.x, el, vw, hb);
          if (SASA) sl = sasa_energy(set.f, m, s, 0, kWarps, err);
          double v = ((el + vw) + hb) + sl;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) s.red[warp * 8] = v;
        }
        __syncthreads();
        double epair = 0.0;
        for (int k = 0; k < kWarps; ++k) epair += s.red[k * 8];
        const double etor_new = (etor - cur.eold) + cur.enew;
        const double enw = epair + etor_new;
        const double d2 =
            __dsub_rn(__dsub_rn(weight(w, beta, enw), weight(w, beta, eol)), d1);
        int up = 1;
        if (d2 > 0.0) {
          up = mh_accept(s, head, d2);
          head += 1;
        }
        __syncthreads();   // every thread has read s.red and the queue
        if (up) {
          eol = enw;
          etor = etor_new;
          s_cur = s_new;
          ++nacc;
          if (!plain) ++n2;
          if (threadIdx.x == 0) {
            s.et[cur.jv] = cur.enew;
            float sn, cs;
            sincosf((float)cur.vnew, &sn, &cs);
            s.daf[2 * cur.ivar] = bf16_round(sn);
            s.daf[2 * cur.ivar + 1] = bf16_round(cs);
          }
        } else {
          for (int t = threadIdx.x; t < nmoved; t += blockDim.x) {
            const int k = moved_atom(t, lo, span, flip);
            if (flip && (k == cur.a || k == cur.b)) continue;
            s.x[k] = s.bx[k];
            s.y[k] = s.by[k];
            s.z[k] = s.bz[k];
            if (F32) f32_copy(s, k);
          }
          if (threadIdx.x == 0) s.vlvr[cur.jv] = cur.vold;
        }
        if (!isfinite(enw) && threadIdx.x == 0) set_err(err, kErrNonFinite);
        __syncthreads();
        // the dihedral state follows the variables (the setvar of energy())
        setvar_all(m, s);
        __syncthreads();
        if (up) {   // the state changed: the batch's later proposals are stale
          next = p + j + 1;
          break;
        }
      }
      p = next;
    }
    // ---- closing energy() and consistency check (metropolis.f:172-179)
    setvar_all(m, s);
    __syncthreads();
    if (sw + 1 < nsweeps) {
      check_pending = true;
      continue;
    }
    torsion_all(m, s);
    full_rebuild(m, s);
    evaluate_block<F32, ROWS, SASA>(set.f, m, s, err);
    __syncthreads();
    {
      double sum[5];
      all_sums(s, sum);
      const double enew = total_of(sum);
      if (threadIdx.x == 0) {
        if (!(flags & kFlagNoCheck) && fabs(eol - enew) > check_tol && eol < 100000.0)
          set_err(err, kErrConsistency);
        write_terms(ch, c, sum);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ch.eol[c] = eol;
    ch.nacc[c] += nacc;
    ch.nprop[c] += nprop;
    ch.da_n1[c] = n1;
    ch.da_n2[c] = n2;
    s.mt[kQHead] = head;
  }
  (void)n1_0;
  (void)n2_0;
  __syncthreads();
  store_chain(ch, m, c, s);
}

// Replica exchange step as a kernel: the stream slot is copied into shared
// memory, worked on by exchange_core and written back.
__global__ void __launch_bounds__(32) k_exchange(DChains ch, int* temp_chain, const double* betas,
                                                 int n, uint32_t* mt, int* iswitch, int wrap,
                                                 unsigned long long* stats) {
  __shared__ uint32_t slot[kMTWords];
  __shared__ double lq[kQueue];
  const int lane = threadIdx.x;
  if (blockIdx.x != 0) return;
  for (int k = lane; k < kMTWords; k += 32) slot[k] = mt[k];
  __syncwarp();
  exchange_core(ch, temp_chain, betas, n, slot, lq, iswitch, wrap, stats);
  __syncwarp();
  for (int k = lane; k < kMTWords; k += 32) mt[k] = slot[k];
}

// ============================================================================ host wrappers

// (under another name for the calls below: in the 384-thread build the
// 512-thread build's sweep_smem_bytes is also visible through the argument)
static size_t launch_smem_bytes(const DMolSet& set) {
  const bool sasa = set.f.itysol > 0;
  return smem_layout(set.max_atoms, set.max_vars, set.f.npnt, sasa, set.da != 0,
                     sasa ? 0 : set.window, sasa ? 0 : set.cache_pairs,
                     sasa ? 0 : set.cache_cross, nullptr, nullptr) +
         (size_t)set.stage_bytes;
}
size_t sweep_smem_bytes(const DMolSet& set) { return launch_smem_bytes(set); }

size_t stage_bytes_of(const DMol& d, bool lists) {
  return stage_size(d.natoms, d.nvar, d.nsib, d.nlevels, d.nfree, d.npairs, d.nheavy,
                    d.rows != 0, lists, d.cache ? d.ncross : 0);
}

cudaError_t launch_seed(uint32_t* mt, const int* seeds, int nslots, cudaStream_t st) {
  k_seed<<<(nslots + 127) / 128, 128, 0, st>>>(mt, seeds, nslots);
  return cudaGetLastError();
}

cudaError_t launch_draw(uint32_t* mt, int slot, int n, double* out, cudaStream_t st) {
  k_draw<<<1, 1, 0, st>>>(mt, slot, n, out);
  return cudaGetLastError();
}

cudaError_t launch_random_start(const DMolSet& set, const DChains& ch, const int* order, int n,
                                cudaStream_t st) {
  k_random_start<<<1, 1, 0, st>>>(set, ch, order, n);
  return cudaGetLastError();
}

cudaError_t launch_propose(const DMolSet& set, const DChains& ch, int first, int n, int p,
                           int rndord, double* vold, int* jvar, cudaStream_t st) {
  k_propose<<<(n + 127) / 128, 128, 0, st>>>(set, ch, first, n, p, rndord, vold, jvar);
  return cudaGetLastError();
}
cudaError_t launch_decide(const DChains& ch, const DWeight& w, int first, int n,
                          const double* vold, const int* jvar, double* eolc, cudaStream_t st) {
  k_decide<<<(n + 127) / 128, 128, 0, st>>>(ch, w, first, n, vold, jvar, eolc);
  return cudaGetLastError();
}
cudaError_t launch_close(const DChains& ch, int first, int n, const double* eolc, int check,
                         double check_tol, cudaStream_t st) {
  k_close<<<(n + 127) / 128, 128, 0, st>>>(ch, first, n, eolc, check, check_tol);
  return cudaGetLastError();
}
cudaError_t launch_copy_eol(const DChains& ch, int first, int n, double* eolc, cudaStream_t st) {
  k_copy_eol<<<(n + 127) / 128, 128, 0, st>>>(ch, first, n, eolc);
  return cudaGetLastError();
}

// Raise a kernel's dynamic shared-memory limit once per size, so that the
// launches captured into CUDA graphs make no attribute calls.
static cudaError_t prep_smem(const void* fn, size_t bytes) {
  constexpr int kSlots = 32;
  static const void* fns[kSlots] = {nullptr};
  static size_t done[kSlots] = {0};
  int k = 0;
  while (k < kSlots && fns[k] && fns[k] != fn) ++k;
  if (k < kSlots && fns[k] == fn && done[k] >= bytes) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && k < kSlots) {
    fns[k] = fn;
    done[k] = bytes;
  }
  return e;
}

template <bool F32, bool ROWS, bool SASA>
static cudaError_t launch_energy_t(const DMolSet& set, const DChains& ch, int first, int count,
                                   size_t sm, cudaStream_t st) {
  cudaError_t e = prep_smem((const void*)k_energy<F32, ROWS, SASA>, sm);
  if (e != cudaSuccess || count <= 0) return e;
  k_energy<F32, ROWS, SASA><<<count, kThreads, sm, st>>>(set, ch, first);
  return cudaGetLastError();
}

template <bool F32, bool ROWS, bool SASA>
static cudaError_t launch_sweep_t(const DMolSet& set, const DChains& ch, const DWeight& w,
                                  int first, int count, int nsweeps, int flags, double check_tol,
                                  size_t sm, cudaStream_t st) {
  if (ch.sur.w1 != nullptr) {   // delayed acceptance with the surrogate
    cudaError_t e = prep_smem((const void*)k_sweep_da<F32, ROWS, SASA>, sm);
    if (e != cudaSuccess || count <= 0) return e;
    k_sweep_da<F32, ROWS, SASA><<<count, kThreads, sm, st>>>(set, ch, w, first, nsweeps, flags,
                                                             check_tol);
    return cudaGetLastError();
  }
  cudaError_t e = prep_smem((const void*)k_sweep<F32, ROWS, SASA>, sm);
  if (e != cudaSuccess || count <= 0) return e;
  k_sweep<F32, ROWS, SASA><<<count, kThreads, sm, st>>>(set, ch, w, first, nsweeps, flags,
                                                        check_tol, DPTFused{});
  return cudaGetLastError();
}

// One cooperative launch of nsweeps (sweep, exchange) rounds over chains
// [0, count).  Returns cudaErrorCooperativeLaunchTooLarge when the chains
// cannot all be resident at once, cudaErrorNotSupported when the device has
// no cooperative launch; nothing is launched then.
template <bool F32, bool ROWS, bool SASA>
static cudaError_t launch_sweep_pt_t(DMolSet set, DChains ch, DWeight w, int count, int nsweeps,
                                     int flags, double check_tol, DPTFused pt, size_t sm,
                                     cudaStream_t st) {
  const void* fn = (const void*)k_sweep<F32, ROWS, SASA>;
  cudaError_t e = prep_smem(fn, sm);
  if (e != cudaSuccess) return e;
  int dev = 0, coop = 0, nsm = 0, per = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kThreads, sm)) != cudaSuccess)
    return e;
  if (!coop) return cudaErrorNotSupported;
  if ((long long)per * nsm < count) return cudaErrorCooperativeLaunchTooLarge;
  // one more block, when it fits, to run the exchanges (pt_master)
  pt.master = (long long)per * nsm >= (long long)count + 1 ? 1 : 0;
  int first = 0;
  void* args[] = {&set, &ch, &w, &first, &nsweeps, &flags, &check_tol, &pt};
  return cudaLaunchCooperativeKernel(fn, dim3(count + pt.master), dim3(kThreads), args, sm, st);
}

static int variant(const DMolSet& set, bool fp32) {
  return (fp32 ? 4 : 0) | (set.any_rows ? 2 : 0) | (set.f.itysol > 0 ? 1 : 0);
}

cudaError_t launch_energy(const DMolSet& set, const DChains& ch, int first, int count, bool fp32,
                          cudaStream_t st) {
  const size_t sm = launch_smem_bytes(set);
  switch (variant(set, fp32)) {
    case 0: return launch_energy_t<false, false, false>(set, ch, first, count, sm, st);
    case 1: return launch_energy_t<false, false, true>(set, ch, first, count, sm, st);
    case 2: return launch_energy_t<false, true, false>(set, ch, first, count, sm, st);
    case 3: return launch_energy_t<false, true, true>(set, ch, first, count, sm, st);
    case 4: return launch_energy_t<true, false, false>(set, ch, first, count, sm, st);
    case 5: return launch_energy_t<true, false, true>(set, ch, first, count, sm, st);
    case 6: return launch_energy_t<true, true, false>(set, ch, first, count, sm, st);
    default: return launch_energy_t<true, true, true>(set, ch, first, count, sm, st);
  }
}

cudaError_t launch_sweep(const DMolSet& set, const DChains& ch, const DWeight& w, int first,
                         int count, int nsweeps, int flags, double check_tol, cudaStream_t st) {
  const size_t sm = launch_smem_bytes(set);
#define SMMP_SWEEP(a, b, c) \
  launch_sweep_t<a, b, c>(set, ch, w, first, count, nsweeps, flags, check_tol, sm, st)
  switch (variant(set, (flags & kFlagFP32) != 0)) {
    case 0: return SMMP_SWEEP(false, false, false);
    case 1: return SMMP_SWEEP(false, false, true);
    case 2: return SMMP_SWEEP(false, true, false);
    case 3: return SMMP_SWEEP(false, true, true);
    case 4: return SMMP_SWEEP(true, false, false);
    case 5: return SMMP_SWEEP(true, false, true);
    case 6: return SMMP_SWEEP(true, true, false);
    default: return SMMP_SWEEP(true, true, true);
  }
#undef SMMP_SWEEP
}

cudaError_t launch_sweep_pt(const DMolSet& set, const DChains& ch, const DWeight& w, int count,
                            int nsweeps, int flags, double check_tol, const DPTFused& pt,
                            cudaStream_t st) {
  if (ch.sur.w1 != nullptr || pt.n != count) return cudaErrorNotSupported;
  const size_t sm = launch_smem_bytes(set);
#define SMMP_SWEEP(a, b, c) \
  launch_sweep_pt_t<a, b, c>(set, ch, w, count, nsweeps, flags, check_tol, pt, sm, st)
  switch (variant(set, (flags & kFlagFP32) != 0)) {
    case 0: return SMMP_SWEEP(false, false, false);
    case 1: return SMMP_SWEEP(false, false, true);
    case 2: return SMMP_SWEEP(false, true, false);
    case 3: return SMMP_SWEEP(false, true, true);
    case 4: return SMMP_SWEEP(true, false, false);
    case 5: return SMMP_SWEEP(true, false, true);
    case 6: return SMMP_SWEEP(true, true, false);
    default: return SMMP_SWEEP(true, true, true);
  }
#undef SMMP_SWEEP
}

cudaError_t launch_gradient(const DMolSet& set, const DChains& ch, int first, int count,
                            double* grad, cudaStream_t st) {
  const size_t sm = launch_smem_bytes(set);
  cudaError_t e = prep_smem((const void*)k_gradient, sm);
  if (e != cudaSuccess || count <= 0) return e;
  k_gradient<<<count, kThreads, sm, st>>>(set, ch, first, grad);
  return cudaGetLastError();
}

cudaError_t launch_exchange(const DChains& ch, int* temp_chain, const double* betas, int n,
                            uint32_t* mt, int* iswitch, int wrap, unsigned long long* stats,
                            cudaStream_t st) {
  k_exchange<<<1, 32, 0, st>>>(ch, temp_chain, betas, n, mt, iswitch, wrap, stats);
  return cudaGetLastError();
}

#ifdef SMMP_BLOCK_VARIANT
}  // namespace SMMP_BLOCK_VARIANT
#endif
}  // namespace smmpb200
