// CPU oracle -- TEST INFRASTRUCTURE ONLY (see smmp_oracle.hpp).
//
// The multicanonical weight recursion of mulcan_par_mod.f90 (mulcan_par,
// :93-145 every nup sweeps, :163-168 at the end).  Arrays are indexed
// k - kmin for the bins kmin..kmax.  The Fortran's float()/Float() and
// log() of REAL*4 arguments are single-precision operations, kept so.
#include <algorithm>
#include <cmath>

#include "smmp_oracle.hpp"

namespace oracle {

void muca_update(int kmin, int kmax, double ebin, double beta, int* ihist, double* xhist,
                 double* g1, double* b, double* alpha, double* ent) {
  auto H = [&](int k) -> int& { return ihist[k - kmin]; };
  auto X = [&](int k) -> double& { return xhist[k - kmin]; };
  auto G = [&](int k) -> double& { return g1[k - kmin]; };
  auto B = [&](int k) -> double& { return b[k - kmin]; };
  auto A = [&](int k) -> double& { return alpha[k - kmin]; };
  auto E = [&](int k) -> double& { return ent[k - kmin]; };
  X(kmax) = X(kmax) + H(kmax);
  X(kmax - 1) = X(kmax - 1) + H(kmax - 1);
  for (int i = kmax - 2; i >= kmin; --i) {
    X(i) = X(i) + H(i);
    if (H(i) > 1 && H(i + 1) > 1) {
      double g0 = (double)((float)H(i + 1) * (float)H(i));   // REAL*4 product
      g0 = g0 / (double)(float)(H(i) + H(i + 1));
      G(i) = G(i) + g0;
      g0 = g0 / G(i);
      const double bi_1 = (double)std::log((float)H(i + 1));   // REAL*4 log
      const double bi = (double)std::log((float)H(i));
      B(i) = B(i) + g0 * (bi_1 - bi) / ebin;
    } else if (X(i) < 2.0) {
      B(i) = std::max(0.0, B(i + 1));
    }
  }
  B(kmax) = B(kmax - 2);
  B(kmax - 1) = B(kmax - 2);
  A(kmax) = 0.0;
  E(kmax) = (beta + B(kmax)) * (double)(float)kmax * ebin + A(kmax);
  H(kmax) = 0;
  for (int i = kmax - 1; i >= kmin; --i) {
    H(i) = 0;
    A(i) = A(i + 1) + (B(i + 1) - B(i)) * (i + 0.5) * ebin;
    E(i) = (beta + B(i)) * (double)(float)i * ebin + A(i);
  }
}

void muca_finish(int kmin, int kmax, double ebin, double beta, double* b, double* alpha) {
  alpha[kmax - kmin] = 0.0;
  b[kmax - kmin] = b[kmax - kmin] + beta;
  for (int i = kmax - 1; i >= kmin; --i) {
    b[i - kmin] = b[i - kmin] + beta;
    alpha[i - kmin] = alpha[i + 1 - kmin] + (b[i + 1 - kmin] - b[i - kmin]) * (i + 0.5) * ebin;
  }
}

}  // namespace oracle
