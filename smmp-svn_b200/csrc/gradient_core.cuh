// Derivatives of the ECEPP/3 energy with respect to the dihedrals, in the
// order-free form of opeshe.f:12-317: the force on every atom from all of
// its pairs, then for each variable the force and torque sums over the atoms
// it moves -- the contiguous range [var_lo, var_hi] of the atom order, so the
// sums are differences of prefix sums over atoms.  The reference's ordered
// recursion over moving sets gives the same sums (to rounding); which atoms
// a variable moves is the same set in both (checked on the host topology).
//
// Host and device share this arithmetic.  k_gradient (kernels.cu) runs the
// pair loop over the block's threads (forces accumulated with FP64 atomics)
// and the force and torque sums of each variable over one warp; a host build
// of the same functions over the product's topology is checked against the
// oracle's gradient to 1e-12 of the largest derivative (ECEPP/3, ECEPP/2 and
// the sigmoidal dielectric).
#pragma once
#include <cmath>
#include <cstdint>

#include "device.cuh"

namespace smmpb200 {

struct GradTables {
  const double* a;     // [kTypes * kTypes] repulsion (ahb for H-bond type pairs)
  const double* a14;   // 1-4 repulsion
  const double* c;     // attraction (chb for H-bond type pairs)
  const int* hb;       // 1: 12-10 H-bond pair
  double conv, plt, slp;
  int epsd;
};

// Pair (i, j) at squared distance r2: the factor c with F_i += c (r_j - r_i)
// and F_j -= c (r_j - r_i) (opeshe.f:165-225), and its energy terms added to
// e = {Coulomb, van der Waals, H-bond}.
__host__ __device__ inline double gradient_pair(const GradTables& t, int ti, int tj, double qi,
                                                double qj, double r2, bool is14, double* e) {
  const double rij4 = r2 * r2, rij6 = rij4 * r2, rij = sqrt(r2);
  const double cqi = t.conv * qi;
  double eel, deel;
  if (t.epsd) {
    const double sr = t.slp * rij, sr2 = sr * sr;
    const double xsr = (t.plt - 1.0) * exp(-sr) / 2.0;
    const double ep = t.plt - (sr2 + 2.0 * sr + 2.0) * xsr;
    eel = cqi * qj / (rij * ep);
    deel = eel + cqi * qj * (t.slp * sr2 * xsr) / (ep * ep);
  } else {
    eel = cqi * qj / rij;
    deel = eel;
  }
  e[0] += eel;
  const int k = ti * kTypes + tj;
  const double a = is14 ? t.a14[k] : t.a[k];
  const double eyrp = a / (rij6 * rij6);
  if (t.hb[k]) {
    const double eyds = t.c[k] / (rij6 * rij4);
    e[2] += eyrp - eyds;
    return (-12.0 * eyrp + 10.0 * eyds - deel) / r2;
  }
  const double eyds = t.c[k] / rij6;
  e[1] += eyrp - eyds;
  return (-12.0 * eyrp + 6.0 * eyds - deel) / r2;
}

// The pair of chunk-list item t (chunk t/8, partner t%8; the word packs
// i | j0 << 14 | (len-1) << 28): false for an empty slot.
__host__ __device__ inline bool gradient_chunk_pair(const uint32_t* chunks, int t, int& i,
                                                    int& j) {
  const uint32_t w = chunks[t >> 3];
  const int l = t & 7;
  i = int(w & 0x3fffu);
  j = int((w >> 14) & 0x3fffu) + l;
  return l <= int((w >> 28) & 7u);
}

// Derivative of variable v (opeshe.f:302-310): e the unit axis of its bond
// (frame axis of the base atom b), SF and ST the sums of the atomic forces
// and of r x F over the atoms it moves, fvr its torsion force
// e0 sg rn sin(rn toat).
__host__ __device__ inline double gradient_variable(const double* e, const double* b,
                                                    const double* SF, const double* ST,
                                                    double fvr) {
  return (e[1] * b[2] - e[2] * b[1]) * SF[0] + (e[2] * b[0] - e[0] * b[2]) * SF[1] +
         (e[0] * b[1] - e[1] * b[0]) * SF[2] + e[0] * ST[0] + e[1] * ST[1] + e[2] * ST[2] - fvr;
}

__host__ __device__ inline double gradient_torsion_force(double e0, double sg, double rn,
                                                         double toat) {
  return e0 != 0.0 ? e0 * sg * rn * sin(toat * rn) : 0.0;
}

}  // namespace smmpb200
