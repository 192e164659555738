// Multicanonical weight recursion (mulcan_par_mod.f90:93-145, 163-168): the
// histogram of the last nup sweeps updates the weight parameters b and alpha
// of muca_weight (mulcan_par_mod.f90:380-395), which the GPU sweep kernels
// evaluate; host arithmetic, compiled with -ffp-contract=off.  The
// reference's float() conversions and REAL*4 logarithms stay in single
// precision.  Bins kmin..kmax, arrays indexed k - kmin.
#include "muca.hpp"

#include <algorithm>
#include <cmath>

namespace smmpb200 {

void muca_update(const MucaBins& q, int* ihist, double* xhist, double* g1, double* b,
                 double* alpha, double* ent) {
  const int lo = q.kmin, hi = q.kmax;
  const int n = hi - lo;   // index of kmax
  xhist[n] += ihist[n];
  xhist[n - 1] += ihist[n - 1];
  for (int k = n - 2; k >= 0; --k) {
    xhist[k] += ihist[k];
    const int h0 = ihist[k], h1 = ihist[k + 1];
    if (h0 > 1 && h1 > 1) {
      const float prod = (float)h1 * (float)h0;
      double g0 = (double)prod / (double)(float)(h0 + h1);
      g1[k] += g0;
      g0 /= g1[k];
      const double l1 = (double)std::log((float)h1), l0 = (double)std::log((float)h0);
      b[k] += g0 * (l1 - l0) / q.ebin;
    } else if (xhist[k] < 2.0) {
      b[k] = std::max(0.0, b[k + 1]);
    }
  }
  b[n] = b[n - 2];
  b[n - 1] = b[n - 2];
  alpha[n] = 0.0;
  ent[n] = (q.beta + b[n]) * (double)(float)hi * q.ebin + alpha[n];
  ihist[n] = 0;
  for (int k = n - 1; k >= 0; --k) {
    const int bin = lo + k;
    ihist[k] = 0;
    alpha[k] = alpha[k + 1] + (b[k + 1] - b[k]) * (bin + 0.5) * q.ebin;
    ent[k] = (q.beta + b[k]) * (double)(float)bin * q.ebin + alpha[k];
  }
}

void muca_finish(const MucaBins& q, double* b, double* alpha) {
  const int n = q.kmax - q.kmin;
  alpha[n] = 0.0;
  b[n] += q.beta;
  for (int k = n - 1; k >= 0; --k) {
    b[k] += q.beta;
    alpha[k] = alpha[k + 1] + (b[k + 1] - b[k]) * (q.kmin + k + 0.5) * q.ebin;
  }
}

}  // namespace smmpb200
