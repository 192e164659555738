// Minimisation over the free dihedrals (see minimize.hpp).
#include "minimize.hpp"

#include <algorithm>
#include <cmath>

namespace smmpb200 {

namespace {

double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t k = 0; k < a.size(); ++k) s += a[k] * b[k];
  return s;
}

// Minimiser of the cubic through (a, fa, da) and (b, fb, db), kept inside
// the middle of [a, b] (bisection when the cubic does not help).
double cubic_step(double a, double fa, double da, double b, double fb, double db) {
  const double lo = std::min(a, b), hi = std::max(a, b);
  const double d1 = da + db - 3.0 * (fa - fb) / (a - b);
  const double disc = d1 * d1 - da * db;
  double t = 0.5 * (a + b);
  if (disc >= 0.0) {
    const double d2 = std::copysign(std::sqrt(disc), b - a);
    const double den = db - da + 2.0 * d2;
    if (den != 0.0) t = b - (b - a) * (db + d2 - d1) / den;
  }
  const double w = hi - lo;
  if (!(t > lo + 0.1 * w && t < hi - 0.1 * w)) t = 0.5 * (a + b);
  return t;
}

struct LineSearch {
  const EnergyGradient& fg;
  const std::vector<double>& x;
  const std::vector<double>& p;
  std::vector<double> xt, gt;
  int& calls;
  int maxcalls;
  double phi(double a, double& dphi) {
    for (size_t k = 0; k < x.size(); ++k) xt[k] = x[k] + a * p[k];
    const double f = fg(xt.data(), gt.data());
    ++calls;
    dphi = dot(gt, p);
    return f;
  }
};

// Strong Wolfe line search (bracketing, then zooming with cubic steps):
// returns the accepted step (0: none) with its point, energy and gradient in
// ls.xt, f_out and ls.gt.
double wolfe(LineSearch& ls, double f0, double d0, double a1, double amax, double c2,
             double& f_out) {
  const double c1 = 1e-4;
  double a_prev = 0.0, f_prev = f0, d_prev = d0, a = std::min(a1, amax);
  for (int it = 0; it < 30 && ls.calls < ls.maxcalls; ++it) {
    double d;
    const double f = ls.phi(a, d);
    auto zoom = [&](double lo, double flo, double dlo, double hi, double fhi, double dhi) {
      for (int z = 0; z < 40 && ls.calls < ls.maxcalls; ++z) {
        const double t = cubic_step(lo, flo, dlo, hi, fhi, dhi);
        double dt;
        const double ft = ls.phi(t, dt);
        if (!std::isfinite(ft) || ft > f0 + c1 * t * d0 || ft >= flo) {
          hi = t;
          fhi = ft;
          dhi = dt;
        } else {
          if (std::fabs(dt) <= -c2 * d0) {
            f_out = ft;
            return t;
          }
          if (dt * (hi - lo) >= 0.0) {
            hi = lo;
            fhi = flo;
            dhi = dlo;
          }
          lo = t;
          flo = ft;
          dlo = dt;
        }
        if (std::fabs(hi - lo) < 1e-14 * std::max(1.0, std::fabs(lo))) break;
      }
      // best point found: the low end (it satisfies the sufficient decrease)
      if (lo > 0.0) {
        double dl;
        f_out = ls.phi(lo, dl);
        return lo;
      }
      return 0.0;
    };
    if (!std::isfinite(f) || f > f0 + c1 * a * d0 || (it > 0 && f >= f_prev))
      return zoom(a_prev, f_prev, d_prev, a, std::isfinite(f) ? f : 1e300, d);
    if (std::fabs(d) <= -c2 * d0) {
      f_out = f;
      return a;
    }
    if (d >= 0.0) return zoom(a, f, d, a_prev, f_prev, d_prev);
    a_prev = a;
    f_prev = f;
    d_prev = d;
    if (a >= amax) {
      f_out = f;
      return a;
    }
    a = std::min(2.0 * a, amax);
  }
  return 0.0;
}

}  // namespace

MinimizeResult minimize(int imin, std::vector<double>& x, const EnergyGradient& fg, int maxit,
                        double eps) {
  const size_t n = x.size();
  MinimizeResult r;
  std::vector<double> g(n), p(n), s(n), y(n), gnew(n), H;
  double f = fg(x.data(), g.data());
  r.calls = 1;
  const bool bfgs = imin != 2;
  if (bfgs) {
    H.assign(n * n, 0.0);
    for (size_t k = 0; k < n; ++k) H[k * n + k] = 1.0;
  }
  LineSearch ls{fg, x, p, std::vector<double>(n), std::vector<double>(n), r.calls, maxit};
  double g2 = dot(g, g);
  std::vector<double> gprev;
  double fprev = f;
  int since_restart = 0;
  bool first = true;
  while (g2 > eps && r.calls < maxit && n > 0) {
    // direction
    if (bfgs) {
      for (size_t i = 0; i < n; ++i) {
        double v = 0.0;
        for (size_t j = 0; j < n; ++j) v -= H[i * n + j] * g[j];
        p[i] = v;
      }
    } else {
      double beta = 0.0;
      if (!first && since_restart < (int)n) {
        double num = 0.0;
        for (size_t k = 0; k < n; ++k) num += g[k] * (g[k] - gprev[k]);
        beta = std::max(0.0, num / dot(gprev, gprev));
      } else {
        since_restart = 0;
      }
      for (size_t k = 0; k < n; ++k) p[k] = -g[k] + beta * p[k];
    }
    double d0 = dot(g, p);
    if (!(d0 < 0.0)) {   // not a descent direction: steepest descent
      for (size_t k = 0; k < n; ++k) p[k] = -g[k];
      d0 = -g2;
      if (bfgs) {
        std::fill(H.begin(), H.end(), 0.0);
        for (size_t k = 0; k < n; ++k) H[k * n + k] = 1.0;
      }
      since_restart = 0;
    }
    // no dihedral moves by more than half a radian in one trial step
    double pmax = 0.0;
    for (size_t k = 0; k < n; ++k) pmax = std::max(pmax, std::fabs(p[k]));
    const double amax = pmax > 0.0 ? 0.5 / pmax : 1.0;
    // first trial step.  Quasi-Newton: at most a unit gradient step on the
    // first iteration, then 1.  Conjugate gradients: the step that would
    // lower the energy by 10 kcal/mol (mincjg.f's expected first decrease,
    // AMF), then the one that repeats the last decrease; a steep start then
    // moves by a short step instead of to the line minimum far downhill.
    double a1 = 1.0;
    if (bfgs) {
      if (first) a1 = std::min(1.0, 1.0 / std::sqrt(g2));
    } else {
      a1 = first ? 10.0 / -d0 : std::min(1.0, 2.02 * (f - fprev) / -d0);
    }
    if (!(a1 > 0.0)) a1 = 1.0;
    double fnew = f;
    const double a = wolfe(ls, f, d0, a1, amax, bfgs ? 0.9 : 0.3, fnew);
    if (a <= 0.0 || !(fnew <= f)) break;   // no progress
    for (size_t k = 0; k < n; ++k) {
      s[k] = a * p[k];
      gnew[k] = ls.gt[k];
      y[k] = gnew[k] - g[k];
    }
    if (bfgs) {
      const double sy = dot(s, y);
      if (sy > 1e-12 * std::sqrt(dot(s, s) * dot(y, y))) {
        if (first) {   // scale the initial inverse Hessian
          const double sc = sy / dot(y, y);
          for (size_t k = 0; k < n * n; ++k) H[k] *= sc;
        }
        // H <- (I - rho s y^T) H (I - rho y s^T) + rho s s^T
        const double rho = 1.0 / sy;
        std::vector<double> Hy(n, 0.0);
        for (size_t i = 0; i < n; ++i)
          for (size_t j = 0; j < n; ++j) Hy[i] += H[i * n + j] * y[j];
        const double yHy = dot(y, Hy);
        for (size_t i = 0; i < n; ++i)
          for (size_t j = 0; j < n; ++j)
            H[i * n + j] += -rho * (Hy[i] * s[j] + s[i] * Hy[j]) +
                            (rho * rho * yHy + rho) * s[i] * s[j];
      }
    }
    x = ls.xt;
    fprev = f;
    gprev = g;
    g = gnew;
    f = fnew;
    g2 = dot(g, g);
    first = false;
    ++since_restart;
  }
  r.energy = f;
  r.grad2 = g2;
  r.converged = g2 <= eps;
  return r;
}

}  // namespace smmpb200
