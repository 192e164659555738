// CPU oracle -- TEST INFRASTRUCTURE ONLY (see smmp_oracle.hpp).
//
// minim.f:12-258 (no regularisation) with move (minim.f:262-360), minqsn.f
// (imin = 1: quasi-Newton, BFGS updates of a Cholesky-factored Hessian,
// mc11a/mc11e, cubic line searches) and mincjg.f (imin = 2: conjugate
// gradients with restarts).  Arrays are 1-based;
// the reference's single-precision literals (.01, .1) are kept as floats
// promoted to double, as the Fortran evaluates them.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <vector>

#include "smmp_oracle.hpp"

namespace oracle {

namespace {

// mc11a (minqsn.f:250-370): rank-one update a + sig z z^T of a factorised
// symmetric matrix in packed storage.  z and w may be the same array.
void mc11a(double* a, int n, double* z, double sig, double* w, int& ir, int mk, double eps) {
  if (n > 1) {
    if (sig == 0.0 || ir == 0) return;
    const int np = n + 1;
    int ij = 1, mm = 0;
    double ti = 0.0, tim = 0.0;
    bool label1 = false;
    if (sig < 0.0) {
      ti = 1.0 / sig;
      ij = 1;
      if (mk == 0) {
        for (int i = 1; i <= n; ++i) w[i] = z[i];
        for (int i = 1; i <= n; ++i) {
          if (a[ij] > 0.0) {
            const double v = w[i];
            ti = ti + (v * v) / a[ij];
            if (i < n)
              for (int j = i + 1; j <= n; ++j) {
                ij = ij + 1;
                w[j] = w[j] - v * a[ij];
              }
            ij = ij + 1;
          } else {
            w[i] = 0.0;
            ij = ij + np - i;
          }
        }
      } else {
        for (int i = 1; i <= n; ++i) {
          if (a[ij] != 0.0) ti = ti + (w[i] * w[i]) / a[ij];
          ij = ij + np - i;
        }
      }
      if (ir <= 0) {
        ti = 0.0;
        ir = -ir - 1;
      } else if (ti > 0.0) {
        if (eps != 0.0) {
          ti = eps / sig;
        } else {
          ir = ir - 1;
          ti = 0.0;
        }
      } else if (mk <= 1) {
        label1 = true;
      }
      if (!label1) {
        mm = 1;
        tim = ti;
        for (int i = 1; i <= n; ++i) {
          const int j = np - i;
          ij = ij - i;
          if (a[ij] != 0.0) tim = ti - (w[j] * w[j]) / a[ij];
          w[j] = ti;
          ti = tim;
        }
      }
    } else {
      label1 = true;
    }
    if (label1) {   // label 1
      mm = 0;
      tim = 1.0 / sig;
    }
    ij = 1;   // label 2
    for (int i = 1; i <= n; ++i) {
      const double v = z[i];
      if (a[ij] > 0.0) {
        const double al = v / a[ij];
        if (mm <= 0)
          ti = tim + v * al;
        else
          ti = w[i];
        const double r = ti / tim;
        a[ij] = a[ij] * r;
        if (r == 0.0 || i == n) break;   // goto 3
        const double b = al / ti;
        if (r > 4.0) {
          const double gm = tim / ti;
          for (int j = i + 1; j <= n; ++j) {
            ij = ij + 1;
            const double y = a[ij];
            a[ij] = b * z[j] + y * gm;
            z[j] = z[j] - v * y;
          }
        } else {
          for (int j = i + 1; j <= n; ++j) {
            ij = ij + 1;
            z[j] = z[j] - v * a[ij];
            a[ij] = a[ij] + b * z[j];
          }
        }
        tim = ti;
        ij = ij + 1;
      } else if (ir > 0 || sig < 0.0 || v == 0.0) {
        ti = tim;
        ij = ij + np - i;
      } else {
        ir = 1 - ir;
        a[ij] = (v * v) / tim;
        if (i == n) return;
        for (int j = i + 1; j <= n; ++j) {
          ij = ij + 1;
          a[ij] = z[j] / v;
        }
        return;
      }
    }
    if (ir < 0) ir = -ir;   // label 3
  } else {
    a[1] = a[1] + sig * (z[1] * z[1]);
    ir = 1;
    if (a[1] > 0.0) return;
    a[1] = 0.0;
    ir = 0;
  }
}

// mc11e (minqsn.f:372-420): solve a z = z with the factorised matrix.
void mc11e(const double* a, int n, double* z, double* w, int ir) {
  if (ir < n) return;
  w[1] = z[1];
  if (n > 1) {
    int ij = 0;
    for (int i = 2; i <= n; ++i) {
      ij = i;
      const int i1 = i - 1;
      double v = z[i];
      for (int j = 1; j <= i1; ++j) {
        v = v - a[ij] * z[j];
        ij = ij + n - j;
      }
      z[i] = v;
      w[i] = v;
    }
    z[n] = z[n] / a[ij];
    const int np = n + 1;
    for (int nip = 2; nip <= n; ++nip) {
      const int i = np - nip;
      int ii = ij - nip;
      double v = z[i] / a[ii];
      const int ip = i + 1;
      ij = ii;
      for (int j = ip; j <= n; ++j) {
        ii = ii + 1;
        v = v - a[ii] * z[j];
      }
      z[i] = v;
    }
  } else {
    z[1] = z[1] / a[1];
  }
}

}  // namespace

// move (minim.f:262-360, ireg = 0): variables from x, energy and gradient,
// the free variables' derivatives in g; one log entry (energy, |grad|^2).
void Smmp::minim_move(int n, double& f, const double* x, double* g,
                      std::vector<double>* log) {
  const int ntlvr = ivrml1[ntlml] + nvrml[ntlml] - 1;
  int k = 0;
  for (int i = 1; i <= ntlvr; ++i)
    if (!fxvr[i]) vlvr[i] = x[++k];
  gradient();
  double gdsmey = 0.0;
  k = 0;
  for (int i = 1; i <= ntlvr; ++i)
    if (!fxvr[i]) {
      g[++k] = gdeyvr[i];
      gdsmey = gdsmey + gdeyvr[i] * gdeyvr[i];
    }
  (void)n;
  f = eysm;
  if (log) {
    log->push_back(f);
    log->push_back(gdsmey);
  }
}

// minqsn.f:13-247.  Returns the number of function calls (nfun).
int Smmp::minqsn(int n, double* x, double& f, double* g, const double* scal, double acur,
                 int maxfun, std::vector<double>* log) {
  const double eps1 = 0.1, eps2 = 0.7, tiny = 1.e-32;
  const double f01 = (double)0.01f, f1 = (double)0.1f;   // REAL*4 literals .01 and .1
  std::vector<double> H(n * (n + 1) / 2 + 1), D(n + 1), W(n + 1), XA(n + 1), GA(n + 1),
      XB(n + 1), GB(n + 1);
  double *h = H.data(), *d = D.data(), *w = W.data(), *xa = XA.data(), *ga = GA.data(),
         *xb = XB.data(), *gb = GB.data();
  int nfun = 0, itr = 0, isfv = 0, ir = 0;
  double dff = 0.0, c = 0.0, fa = 0.0, dga = 0.0, fmin = 0.0, gmin = 0.0, stmin = 0.0,
         stepub = 0.0, steplb = 0.0, step = 0.0, fb = 0.0, dgb = 0.0;
  (void)itr;
  c = 0.0;
  for (int i = 1; i <= n; ++i) c = std::max(c, std::fabs(g[i] * scal[i]));
  if (c <= 0.0) c = 1.0;
  const int n1 = n + 1, i1 = (n * n1) / 2;
  for (int i = 1; i <= i1; ++i) h[i] = 0.0;
  int j = 1;
  for (int i = 1; i <= n; ++i) {
    h[j] = f01 * c / (scal[i] * scal[i]);
    j = j + n1 - i;
  }
  enum { L1, L2, L3, L4, L5 } at = L1;
  for (;;) {
    switch (at) {
      case L1:   // re-start the search from the best point so far
        isfv = 1;
        fa = f;
        for (int i = 1; i <= n; ++i) {
          xa[i] = x[i];
          ga[i] = g[i];
        }
        at = L2;
        break;
      case L2: {   // a new line search from A
        ++itr;
        for (int i = 1; i <= n; ++i) d[i] = -ga[i];
        mc11e(h, n, d, w, n);
        c = 0.0;
        dga = 0.0;
        for (int i = 1; i <= n; ++i) {
          const double di = d[i];
          c = std::max(c, std::fabs(di / scal[i]));
          dga = dga + ga[i] * di;
        }
        c = 1.0 / c;
        if (dga >= 0.0) {   // uphill
          at = L5;
          break;
        }
        fmin = fa;
        gmin = dga;
        stmin = 0.0;
        stepub = 0.0;
        steplb = acur * c;
        if (dff > 0.0)
          step = std::min(1.0, (dff + dff) / (-dga));
        else
          step = std::min(1.0, c);
        at = L3;
        break;
      }
      case L3: {
        if (nfun >= maxfun) return nfun;
        c = stmin + step;
        for (int i = 1; i <= n; ++i) xb[i] = xa[i] + c * d[i];
        nfun = nfun + 1;
        minim_move(n, fb, xb, gb, log);
        isfv = std::min(2, isfv);
        at = L4;
        if (fb <= f) {
          if (fb == f) {
            double gl1 = 0.0, gl2 = 0.0;
            for (int i = 1; i <= n; ++i) {
              const double si = scal[i] * scal[i];
              gl1 = gl1 + si * (g[i] * g[i]);
              gl2 = gl2 + si * (gb[i] * gb[i]);
            }
            if (gl2 >= gl1) break;   // goto 4
          }
          f = fb;
          for (int i = 1; i <= n; ++i) {
            x[i] = xb[i];
            g[i] = gb[i];
          }
          isfv = 3;
        }
        break;
      }
      case L4: {
        dgb = 0.0;
        for (int i = 1; i <= n; ++i) dgb = dgb + gb[i] * d[i];
        if (fb - fa <= eps1 * c * dga) {   // sufficient reduction
          stmin = c;
          fmin = fb;
          gmin = dgb;
          stepub = stepub - step;
          if (stepub > 0.0)
            step = 0.5 * stepub;
          else
            step = 9.0 * stmin;
          c = dga + 3.0 * dgb - 4.0 * (fb - fa) / stmin;
          if (c > 0.0) step = std::min(step, stmin * std::max(1.0, -dgb / c));
          if (dgb < eps2 * dga) {
            at = L3;
            break;
          }
          isfv = 4 - isfv;
          if (stmin + step > steplb) {   // line search complete: update the Hessian
            for (int i = 1; i <= n; ++i) {
              xa[i] = xb[i];
              xb[i] = ga[i];
              d[i] = gb[i] - ga[i];
              ga[i] = gb[i];
            }
            ir = -n;
            double sig = 1.0 / dga;
            mc11a(h, n, xb, sig, w, ir, 1, 0.0);
            ir = -ir;
            sig = 1.0 / (stmin * (dgb - dga));
            mc11a(h, n, d, sig, d, ir, 0, 0.0);
            if (ir == n) {
              dff = fa - fb;
              fa = fb;
              at = L2;
            } else {
              return nfun;   // rank of the Hessian < n
            }
            break;
          }
          at = L5;
          break;
        } else if (step > steplb) {   // insufficient reduction: cubic interpolation
          stepub = step;
          c = gmin + dgb - 3.0 * (fb - fmin) / step;
          c = c + gmin - std::sqrt(c * c - gmin * dgb);
          if (std::fabs(c) < tiny)
            step = f1 * step;
          else
            step = step * std::max(0.1, gmin / c);
          at = L3;
          break;
        }
        at = L5;
        break;
      }
      case L5:
        if (isfv >= 2) {
          at = L1;
          break;
        }
        nfun = nfun + 1;
        minim_move(n, f, x, g, log);
        return nfun;
    }
  }
}

// mincjg.f: conjugate gradients with restarts (no scaling).  Returns nfun.
int Smmp::mincjg(int n, double* x, double& f, double* g, double acur, int maxfun,
                 std::vector<double>* log) {
  const double AMF = 10.0, TOL = 1.e-7, EPS = .7;
  const int MXFCON = 2, MAXLIN = 5;
  std::vector<double> D(n + 1), XA(n + 1), GA(n + 1), DT(n + 1), YT(n + 1), GT(n + 1);
  double *d = D.data(), *xa = XA.data(), *ga = GA.data(), *dt = DT.data(), *yt = YT.data(),
         *gt = GT.data();
  int ier = 0, iter = 0, iterfm = 0, iterrs = 0, nfun = 0, nfopt = nfun, nfbeg = 0, iretry = 0;
  double gsqrd = 0.0, fmin = f, gsq2, gnew, dfpr, stmin, fuit = 0.0, gdit = 0.0, gdmi = 0.0,
         sbound = 0.0, stepch = 0.0, step = 0.0, wo = 0.0, sum = 0.0, fch = 0.0, ddspln = 0.0,
         gspln = 0.0, beta = 0.0, gama = 0.0, gamden = 0.0;
  for (int i = 1; i <= n; ++i) {
    const double t = g[i];
    ga[i] = t;
    d[i] = -t;
    gsqrd = gsqrd + t * t;
    xa[i] = x[i];
  }
  gsq2 = .2 * gsqrd;
  gnew = -gsqrd;
  dfpr = AMF;
  stmin = AMF / gsqrd;
  (void)gnew;
  enum { L1, L2, L3, L4, L5, L6 } at = L1;
  for (;;) {
    switch (at) {
      case L1:
        iter = iter + 1;
        fuit = f;
        gdit = 0.0;
        for (int i = 1; i <= n; ++i) {
          gt[i] = g[i];
          gdit = gdit + d[i] * g[i];
        }
        if (gdit >= 0.0) {   // uphill
          ier = 3;
          at = L6;
          break;
        }
        gdmi = gdit;
        sbound = -1.0;
        nfbeg = nfun;
        iretry = -1;
        stepch = std::min(stmin, std::fabs(dfpr / gdit));
        stmin = 0.0;
        at = L2;
        break;
      case L2: {
        step = stmin + stepch;
        wo = 0.0;
        for (int i = 1; i <= n; ++i) {
          const double t = stepch * d[i];
          wo = std::max(wo, std::fabs(t));
          x[i] = xa[i] + t;
        }
        if (wo > TOL) {
          nfun = nfun + 1;
          minim_move(n, f, x, g, log);
          gnew = 0.0;
          sum = 0.0;
          for (int i = 1; i <= n; ++i) {
            const double t = g[i];
            gnew = gnew + d[i] * t;
            sum = sum + t * t;
          }
          fch = f - fmin;
          if (fch <= 0.0) {
            if (fch < 0.0 || (gnew / gdmi) >= -1.0) {
              fmin = f;
              gsqrd = sum;
              gsq2 = .2 * gsqrd;
              nfopt = nfun;
              for (int i = 1; i <= n; ++i) {
                xa[i] = x[i];
                ga[i] = g[i];
              }
            }
            if (sum <= acur) return nfun;   // normal end
          }
          if (nfun == maxfun) return nfun;   // ier = 1
        } else {   // stepch is effectively zero
          if (nfun > nfbeg + 1 || std::fabs(gdmi / gdit) > EPS) ier = 2;
          at = L6;
          break;
        }
        wo = (fch + fch) / stepch - gnew - gdmi;
        ddspln = (gnew - gdmi) / stepch;
        if (nfun <= nfopt) {
          if (gdmi * gnew <= 0.0) sbound = stmin;
          stmin = step;
          gdmi = gnew;
          stepch = -stepch;
        } else {
          sbound = step;
        }
        if (fch != 0.0) ddspln = ddspln + (wo + wo) / stepch;
        if (gdmi == 0.0) {
          at = L6;
          break;
        }
        if (nfun <= nfbeg + 1) {
          at = L4;
          break;
        }
        if (std::fabs(gdmi / gdit) <= EPS) {
          at = L6;
          break;
        }
        at = L3;
        break;
      }
      case L3:
        if (nfun >= nfopt + MAXLIN) {
          ier = 2;
          at = L6;
          break;
        }
        at = L4;
        break;
      case L4:
        if (sbound < -.5)
          stepch = 9.0 * stmin;
        else
          stepch = .5 * (sbound - stmin);
        gspln = gdmi + stepch * ddspln;
        if ((gdmi * gspln) < 0.0) stepch = stepch * gdmi / (gdmi - gspln);
        at = L2;
        break;
      case L5: {
        sum = 0.0;
        for (int i = 1; i <= n; ++i) sum = sum + g[i] * gt[i];
        beta = (gsqrd - sum) / (gdmi - gdit);
        if (std::fabs(beta * gdmi) > gsq2) {
          iretry = iretry + 1;
          if (iretry <= 0) {
            at = L3;
            break;
          }
        }
        if (f < fuit) iterfm = iter;
        if (iter >= iterfm + MXFCON) return nfun;   // ier = 4
        dfpr = stmin * gdit;
        if (iretry > 0) {
          for (int i = 1; i <= n; ++i) d[i] = -g[i];
          iterrs = 0;
        } else {
          if (iterrs != 0 && (iter - iterrs) < (n - 1) && std::fabs(sum) < gsq2) {
            gama = 0.0;
            sum = 0.0;
            for (int i = 1; i <= n; ++i) {
              const double t = g[i];
              gama = gama + t * yt[i];
              sum = sum + t * dt[i];
            }
            gama = gama / gamden;
            if (std::fabs(beta * gdmi + gama * sum) < gsq2) {
              for (int i = 1; i <= n; ++i) d[i] = -g[i] + beta * d[i] + gama * dt[i];
              at = L1;
              break;
            }
          }
          gamden = gdmi - gdit;
          for (int i = 1; i <= n; ++i) {
            const double t = g[i], di = d[i];
            dt[i] = di;
            yt[i] = t - gt[i];
            d[i] = -t + beta * di;
          }
          iterrs = iter;
        }
        at = L1;
        break;
      }
      case L6:
        if (nfun != nfopt) {   // back to the best point
          f = fmin;
          for (int i = 1; i <= n; ++i) {
            x[i] = xa[i];
            g[i] = ga[i];
          }
        }
        if (ier == 0) {
          at = L5;
          break;
        }
        nfun = nfun + 1;
        minim_move(n, f, x, g, log);
        return nfun;
    }
  }
}

// minim.f:12-258 without regularisation, imin = 1 (quasi-Newton) or 2
// (conjugate gradients): returns the number of function calls; log receives
// (energy, |gradient|^2) of each.
int Smmp::minim(int imin, int maxit, double eps, std::vector<double>* log) {
  if (imin != 1 && imin != 2) throw std::runtime_error("minim: imin must be 1 or 2");
  gradient();
  const int ntlvr = ivrml1[ntlml] + nvrml[ntlml] - 1;
  std::vector<double> vlvrn(ntlvr + 1), gdvr(ntlvr + 1), scl(ntlvr + 1);
  int nv = 0;
  for (int i = 1; i <= ntlvr; ++i)
    if (!fxvr[i]) {
      ++nv;
      vlvrn[nv] = vlvr[i];
      scl[nv] = 1.0;
      gdvr[nv] = gdeyvr[i];
    }
  double esm = eysm;
  const int nop = imin == 1
                      ? minqsn(nv, vlvrn.data(), esm, gdvr.data(), scl.data(), eps, maxit, log)
                      : mincjg(nv, vlvrn.data(), esm, gdvr.data(), eps, maxit, log);
  energy();
  nv = 0;
  for (int i = 1; i <= ntlvr; ++i)   // minim.f:213-225
    if (!fxvr[i]) {
      double vr = vlvrn[++nv];
      if (std::fabs(vr) > 3.141592653589793) vr = vr - std::copysign(2.0 * 3.141592653589793, vr);
      vlvr[i] = vr;
    }
  return nop;
}

}  // namespace oracle
