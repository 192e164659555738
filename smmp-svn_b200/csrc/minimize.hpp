// Minimisation of the energy over the free dihedrals with its analytic
// gradient (the role of minim.f:13 with imin = 1 quasi-Newton, imin = 2
// conjugate gradients).  The energy and gradient come from a callback (the
// GPU gradient kernel behind the C ABI); this file is host code only.
//
// imin = 1: BFGS on the inverse Hessian; imin = 2: nonlinear conjugate
// gradients (Polak-Ribiere+ with restarts).  Both take steps by a line search
// satisfying the strong Wolfe conditions (bracketing, then cubic zooming).
// Iteration stops when the squared gradient falls below eps, when maxit
// function calls are used, or when a line search makes no progress.
#pragma once
#include <functional>
#include <vector>

namespace smmpb200 {

// f(x, g) returns E(x) and writes dE/dx to g (both of size n).
using EnergyGradient = std::function<double(const double* x, double* g)>;

struct MinimizeResult {
  int calls = 0;        // energy + gradient evaluations
  double energy = 0.0;
  double grad2 = 0.0;   // squared gradient at the end
  bool converged = false;
};

MinimizeResult minimize(int imin, std::vector<double>& x, const EnergyGradient& fg, int maxit,
                        double eps);

}  // namespace smmpb200
