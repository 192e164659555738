// CPU oracle -- TEST INFRASTRUCTURE ONLY (see smmp_oracle.hpp).
//
// esolan.f:12-1050: solvation energy sum_i sigma_i A_i from the analytic
// solvent-accessible surface (projection method, J Comp Phys 26, 334-343,
// 2005).  Only the area arithmetic is restated: the gradient arrays (grad,
// gradan; esolan.f:553-575, 718-902, 1000-1030) never feed back into A_i.
// Evaluation order, branch structure, the in-place deletions from the
// neighbour list and the random re-orientation that draws from the global
// MT19937 stream follow the Fortran statement by statement.  Arrays are
// 1-based as in the reference.
#include <algorithm>
#include <cmath>
#include <functional>
#include <stdexcept>
#include <vector>

#include "smmp_oracle.hpp"

namespace oracle {

namespace {
constexpr double pi = 3.141592653589793;
constexpr double pi2 = 2.0 * pi;
constexpr double pi4 = 4.0 * pi;
inline double sq(double x) { return x * x; }   // Fortran x**2
}  // namespace

// The area arithmetic over atoms 1..numat (1-based arrays; radii already
// include the water probe, as init_molecule.f:194-209 leaves them); returns
// sum_i sigma_i A_i and, when As_out is given, A_i in As_out[1..numat].
double esolan_areas(int numat, const double* xa, const double* ya, const double* za,
                    const double* rvdw, const double* sigma, const std::function<double()>& grnd,
                    double* As_out, double* gradan) {
  auto xat = [&](int i) { return xa[i]; };
  auto yat = [&](int i) { return ya[i]; };
  auto zat = [&](int i) { return za[i]; };
  double sss = 0.0;
  std::vector<double> pol(numat + 1), As(numat + 1);
  for (int i = 1; i <= numat; ++i) {   // esolan.f:105-111
    pol[i] = rvdw[i] * rvdw[i];
    As[i] = pi4 * pol[i];
  }
  // per-atom work arrays, indexed by atom number (ddat, neibor) or position
  std::vector<int> neib(numat + 2), neibp(numat + 2), fullarc(numat + 2), al(2 * numat + 2),
      ta2(numat + 2), ta3(numat + 2);
  std::vector<double> ddat(5 * (numat + 1)), neibor(5 * (numat + 1));
  auto DD = [&](int k, int c) -> double& { return ddat[5 * k + c]; };
  auto NB = [&](int k, int c) -> double& { return neibor[5 * k + c]; };
  struct Vertex {
    double t, s, c3, c4;   // vertex(iv, 1..4): (t, s) and the two circles
  };
  std::vector<Vertex> vertex(1);   // 1-based
  std::vector<double> ayx1, ax1, ax2, ay1, ay2, probe;
  std::vector<int> ivrx;
  // gradient row of atom i: grad(i, j, 1..3) (esolan.f:553-575, 718-902)
  std::vector<double> gr(gradan ? 3 * (numat + 1) : 0);
  if (gradan)
    for (int j = 0; j < 3 * (numat + 1); ++j) gradan[j] = 0.0;

  const double rdpcut = (double)1e-10f;   // esolan.f:133, a single-precision literal

  for (int i = 1; i <= numat; ++i) {   // do 1 i = 1, numat
    if (gradan) std::fill(gr.begin(), gr.end(), 0.0);
    bool assemble = false;   // label 11 reached with the circles known
    int ifu_g = 0, ine_g = 0;
    double cf = 0, sf = 0, cg = 0, sg = 0;
    int jjj = 0;
    do {   // one pass; `break` is the Fortran `goto 1` / `goto 11`
      const double R = rvdw[i];
      int jj = 0;
      bool enclosed = false;
      for (int j = 1; j <= numat; ++j) {   // esolan.f:127-152
        if (i == j) continue;
        double ddp = sq(xat(j) - xat(i)) + sq(yat(j) - yat(i)) + sq(zat(j) - zat(i));
        if (ddp < rdpcut) throw std::runtime_error("esolan: centres of two atoms coincide");
        ddp = std::sqrt(ddp);
        if (ddp + R <= rvdw[j]) {   // atom i inside atom j
          As[i] = 0.0;
          enclosed = true;
          break;
        }
        if (!(ddp <= R - rvdw[j] || ddp >= R + rvdw[j])) neib[++jj] = j;
      }
      if (enclosed) break;
      neib[0] = jj;
      if (neib[0] == 0) break;

      const double R2 = R * R, R22 = R2 + R2, R42 = R22 + R22, R22p = R22 * pi;
      for (int j = 1; j <= neib[0]; ++j) {   // esolan.f:166-172
        int k = neib[j];
        DD(k, 2) = xat(k) - xat(i);
        DD(k, 3) = yat(k) - yat(i);
        DD(k, 4) = zat(k) - zat(i);
        DD(k, 1) = rvdw[k];
      }
      DD(i, 2) = DD(i, 3) = DD(i, 4) = 0.0;
      DD(i, 1) = R;

      // north point too close to an intersection line: random re-orientation
      // (esolan.f:180-238)
      int k = neib[1];
      double ddp = std::fabs(sq(DD(k, 2)) + sq(DD(k, 3)) + sq(R - DD(k, 4)) - pol[k]);
      for (int j = 2; j <= neib[0]; ++j) {
        k = neib[j];
        double ddp2 = std::fabs(sq(DD(k, 2)) + sq(DD(k, 3)) + sq(R - DD(k, 4)) - pol[k]);
        if (ddp2 < ddp) ddp = ddp2;
      }
      while (ddp < 1.0e-6) {
        ++jjj;
        double uga = grnd();
        double ufi = grnd();
        uga = pi * uga / 2;
        ufi = pi * ufi / 2;
        cf = std::cos(ufi);
        sf = std::sin(ufi);
        cg = std::cos(uga);
        sg = std::sin(uga);
        const double cfsg = cf * sg, cfcg = cf * cg;
        const double xx = R * cfsg, yy = R * sf, zz = R * cfcg;
        k = neib[1];
        ddp = std::fabs(sq(xx - DD(k, 2)) + sq(yy - DD(k, 3)) + sq(zz - DD(k, 4)) - pol[k]);
        for (int j = 2; j <= neib[0]; ++j) {
          k = neib[j];
          double ddp2 =
              std::fabs(sq(xx - DD(k, 2)) + sq(yy - DD(k, 3)) + sq(zz - DD(k, 4)) - pol[k]);
          if (ddp2 < ddp) ddp = ddp2;
        }
      }
      if (jjj != 0) {   // esolan.f:240-253
        const double sfsg = sf * sg, sfcg = sf * cg, cfsg = cf * sg, cfcg = cf * cg;
        for (int j = 1; j <= neib[0]; ++j) {
          k = neib[j];
          const double xx = DD(k, 2), yy = DD(k, 3), zz = DD(k, 4);
          DD(k, 2) = xx * cg - zz * sg;
          DD(k, 3) = -(xx * sfsg) + yy * cf - zz * sfcg;
          DD(k, 4) = xx * cfsg + yy * sf + zz * cfcg;
        }
      }

      // a (t^2 + s^2) + b t + c s + d = 0 of every neighbour circle
      // (esolan.f:257-268)
      const double pom8 = 8.0 * pol[i];
      for (int q = 1; q <= neib[0]; ++q) {
        const int j = neib[q];
        NB(j, 1) = sq(DD(j, 2)) + sq(DD(j, 3)) + sq(DD(j, 4) - R) - pol[j];
        NB(j, 2) = -(pom8 * DD(j, 2));
        NB(j, 3) = -(pom8 * DD(j, 3));
        NB(j, 4) = 4.0 * pol[i] * (sq(DD(j, 2)) + sq(DD(j, 3)) + sq(R + DD(j, 4)) - pol[j]);
      }

      // mutual disposition of every pair of circles (esolan.f:272-466)
      int iv = 0;
      vertex.resize(1);
      const int nb = neib[0];
      auto remove_at = [&](int pos) {
        neib[0] = neib[0] - 1;
        for (int j = pos; j <= neib[0]; ++j) neib[j] = neib[j + 1];
      };
      bool covered = false;   // `goto 11`: the whole surface is buried
      k = neib[0];
      while (k > 1 && !covered) {
        k = k - 1;
        const int lfirst = neib[0];   // the DO bounds are fixed on entry
        for (int L = lfirst; L >= k + 1; --L) {
          const double ak1 = NB(neib[k], 1), al1 = NB(neib[L], 1);
          if (!((ak1 > 0.0 || ak1 < 0.0) && (al1 > 0.0 || al1 < 0.0))) continue;
          const double b1 = NB(neib[k], 2) / ak1, c1 = NB(neib[k], 3) / ak1,
                       d1 = NB(neib[k], 4) / ak1;
          const double b2 = NB(neib[L], 2) / al1, c2 = NB(neib[L], 3) / al1,
                       d2 = NB(neib[L], 4) / al1;
          const double D = 4.0 * ((b1 - b2) * (b2 * d1 - b1 * d2) +
                                  (c1 - c2) * (c2 * d1 - c1 * d2) - sq(d1 - d2)) +
                           sq(b1 * c2 - b2 * c1);
          const double dist = std::sqrt(sq(b1 - b2) + sq(c1 - c2));
          const double s2 = std::sqrt(b2 * b2 + c2 * c2 - 4.0 * d2);
          const double s1 = std::sqrt(b1 * b1 + c1 * c1 - 4.0 * d1);
          auto add_vertices = [&]() {
            const double am = 2.0 * (sq(b1 - b2) + sq(c1 - c2));
            const double t = -(2.0 * (b1 - b2) * (d1 - d2)) - (b2 * c1 - b1 * c2) * (c1 - c2);
            const double s = -(2.0 * (c1 - c2) * (d1 - d2)) + (b2 * c1 - b1 * c2) * (b1 - b2);
            const double pom = std::sqrt(D);
            const double p1 = (c1 - c2) * pom, p2 = (b1 - b2) * pom;
            vertex.push_back({(t + p1) / am, (s - p2) / am, double(neib[k]), double(neib[L])});
            vertex.push_back({(t - p1) / am, (s + p2) / am, double(neib[k]), double(neib[L])});
            iv += 2;
          };
          bool next_k = false;   // `goto 12`
          if (ak1 > 0.0 && al1 > 0.0) {   // a01
            if (D <= 0.0 && dist <= s2 - s1) {
              remove_at(k);   // circle L encloses circle k
              next_k = true;
            } else if (D <= 0.0 && dist <= -s2 + s1) {
              remove_at(L);   // circle k encloses circle L
            } else if (D > 0.0) {
              add_vertices();
            }
          } else if (ak1 > 0.0 && al1 < 0.0) {   // a03
            if (D <= 0.0 && dist <= -s2 + s1) {
              As[i] = 0.0;
              covered = true;
              break;
            } else if (D <= 0.0 && dist >= s2 + s1) {
              remove_at(k);
              next_k = true;
            } else if (D > 0.0) {
              add_vertices();
            }
          } else if (ak1 < 0.0 && al1 > 0.0) {   // a07
            if (D <= 0.0 && dist <= s2 - s1) {
              As[i] = 0.0;   // the reference goes on with the next k (goto 12)
              next_k = true;
            } else if (D <= 0.0 && dist >= s2 + s1) {
              remove_at(L);
            } else if (D > 0.0) {
              add_vertices();
            }
          } else {   // a09: both negative
            if (D <= 0.0 && dist <= s2 - s1) {
              remove_at(L);
            } else if (D <= 0.0 && dist <= -s2 + s1) {
              remove_at(k);
              next_k = true;
            } else if (D <= 0.0) {
              As[i] = 0.0;
              covered = true;
              break;
            } else {
              add_vertices();
            }
          }
          if (next_k) break;
        }
      }
      if (covered) break;   // goto 11 (only gradients follow)

      // circles that are lines, circles whose inside is the buried side
      // (esolan.f:468-517)
      int ita2 = 0, ita3 = 0;
      for (int j = 1; j <= neib[0]; ++j) {
        if (NB(neib[j], 1) == 0.0) ta2[++ita2] = j;
        if (NB(neib[j], 1) < 0.0) ta3[++ita3] = j;
      }
      if (ita2 > 0 && ita3 < 1) {
        As[i] = R22p;
        if (ita2 > 1) {
          double amial = pi, amaal = -pi, amibe = pi, amabe = -pi;
          for (int j = 1; j <= ita2; ++j) {
            const int q = ta2[j];
            const double p1 = NB(neib[q], 3), p2 = NB(neib[q], 2);
            const double alp = std::atan2(p1, p2);
            double bet = alp;
            if (alp <= 0.0) bet = bet + pi2;
            if (amial > alp) amial = alp;
            if (amaal < alp) amaal = alp;
            if (amibe > bet) amibe = bet;
            if (amabe < bet) amabe = bet;
          }
          const double dal = amaal - amial, dbe = amabe - amibe;
          if (dal < pi)
            As[i] = R22 * (pi - dal);
          else if (dbe < pi)
            As[i] = R22 * (pi - dbe);
          else
            As[i] = 0.0;
        }
      } else if ((nb > 0 && neib[0] < 1) || ita3 > 0) {
        As[i] = 0.0;
      }

      // full arcs (no intersection point) and circles with intersection
      // points (esolan.f:519-531)
      neibp[0] = neib[0];
      for (int j = 1; j <= neib[0]; ++j) neibp[j] = neib[j];
      int ifu = 0, ine = 0;
      for (int j = 1; j <= neibp[0]; ++j) {
        bool has_ip = false;
        for (int q = 1; q <= iv; ++q)
          if (double(neibp[j]) == vertex[q].c3 || double(neibp[j]) == vertex[q].c4) {
            has_ip = true;
            break;
          }
        if (has_ip) {
          neib[++ine] = neibp[j];
        } else {
          ++ifu;
          fullarc[ifu] = neibp[j];
          al[ifu] = neibp[j];
        }
      }
      neib[0] = ine;
      fullarc[0] = ifu;
      al[0] = ifu;

      assemble = gradan != nullptr;
      ifu_g = ifu;
      ine_g = ine;
      for (int q = 1; q <= ifu; ++q) {   // esolan.f:533-578
        const double a = NB(fullarc[q], 1), aia = a < 0.0 ? -1.0 : 1.0;
        const double b = NB(fullarc[q], 2), c = NB(fullarc[q], 3), d = NB(fullarc[q], 4);
        if (a != 0.0) {
          As[i] = As[i] - aia * R22p *
                              (1.0 + (-(d / a) - R42) * std::fabs(a) /
                                         std::sqrt(sq(R42 * a - d) + R42 * (b * b + c * c)));
          if (gradan) {   // esolan.f:547-569
            const int fk = fullarc[q];
            double dadx[5][4];
            dadx[1][1] = 2.0 * DD(fk, 2);
            dadx[1][2] = 2.0 * DD(fk, 3);
            dadx[1][3] = 2.0 * (DD(fk, 4) - R);
            dadx[2][1] = -8.0 * pol[i];
            dadx[2][2] = 0.0;
            dadx[2][3] = 0.0;
            dadx[3][1] = 0.0;
            dadx[3][2] = dadx[2][1];
            dadx[3][3] = 0.0;
            dadx[4][1] = 8.0 * pol[i] * DD(fk, 2);
            dadx[4][2] = 8.0 * pol[i] * DD(fk, 3);
            dadx[4][3] = 8.0 * pol[i] * (DD(fk, 4) + R);
            const double R42p = R22p + R22p;
            const double div =
                R22 * R42p / std::pow(sq(R42 * a - d) + R42 * (b * b + c * c), 1.5);
            double gp[5];
            gp[1] = (R42 * (b * b + c * c - 2.0 * a * d) + 2.0 * d * d) * div;
            gp[2] = -b * (d + R42 * a) * div;
            gp[3] = -c * (d + R42 * a) * div;
            gp[4] = (b * b + c * c - 2.0 * a * d + (R42 + R42) * a * a) * div;
            for (int x = 1; x <= 3; ++x)
              gr[3 * fk + x - 1] = gp[1] * dadx[1][x] + gp[2] * dadx[2][x] +
                                   gp[3] * dadx[3][x] + gp[4] * dadx[4][x];
          }
        } else
          As[i] = As[i] + R22p * d / std::sqrt(R42 * (b * b + c * c) + d * d);
      }

      for (int q = 1; q <= ine; ++q) {   // esolan.f:580-996
        const int jk = neib[q];
        const double a = NB(jk, 1), ak = a * a, daba = std::fabs(a);
        const double aia = a < 0.0 ? -1.0 : 1.0;
        const double b = NB(jk, 2), c = NB(jk, 3), d = NB(jk, 4);
        const double b2c2 = b * b + c * c;
        const double vv = std::sqrt(sq(R42 * a - d) + R42 * b2c2);
        const double vv1 = 1.0 / vv;
        const double wv = std::sqrt(b2c2 - 4.0 * a * d);
        // the intersection points on this circle; each vertex keeps this
        // circle as its third component from here on (esolan.f:602-622)
        int nyx = 0;
        ay1.assign(1, 0.0);
        ay2.assign(1, 0.0);
        ivrx.assign(1, 0);
        for (int j = 1; j <= iv; ++j) {
          if (vertex[j].c3 == double(jk)) {
            ++nyx;
            ay1.push_back(vertex[j].t);
            ay2.push_back(vertex[j].s);
            ivrx.push_back(j);
          }
          if (vertex[j].c4 == double(jk)) {
            ++nyx;
            ay1.push_back(vertex[j].t);
            ay2.push_back(vertex[j].s);
            std::swap(vertex[j].c3, vertex[j].c4);
            ivrx.push_back(j);
          }
        }
        int ial = ifu;   // the other active circles (esolan.f:624-631)
        for (int j = 1; j <= ine; ++j)
          if (neib[j] != jk) al[++ial] = neib[j];
        al[0] = ial;
        auto buried = [&](double p1, double p2) {
          for (int ij = 1; ij <= ial; ++ij)
            if (NB(al[ij], 1) * (p1 * p1 + p2 * p2) + NB(al[ij], 2) * p1 + NB(al[ij], 3) * p2 +
                    NB(al[ij], 4) <
                0.0)
              return true;
          return false;
        };

        if (a != 0.0) {   // esolan.f:633-717
          const double aa = 0.5 / a, ba = b * aa, ca = c * aa;
          const double bcd = b2c2 - 2.0 * a * d;
          for (int j = 1; j <= nyx; ++j) {
            ay1[j] = ay1[j] + ba;
            ay2[j] = ay2[j] + ca;
          }
          const double ct = -ba, cs = -ca, rr = 0.5 * wv / daba;
          ayx1.assign(nyx + 2, 0.0);
          for (int j = 1; j <= nyx; ++j) ayx1[j] = std::atan2(ay2[j], ay1[j]);
          for (int j = 1; j <= nyx - 1; ++j) {   // selection sort, ascending
            double a1 = ayx1[j];
            int jm = j;
            for (int ij = j + 1; ij <= nyx; ++ij)
              if (a1 > ayx1[ij]) {
                a1 = ayx1[ij];
                jm = ij;
              }
            if (jm != j) {
              a1 = ayx1[jm];
              ayx1[jm] = ayx1[j];
              ayx1[j] = a1;
              std::swap(ivrx[jm], ivrx[j]);
            }
          }
          ayx1[nyx + 1] = ayx1[1] + pi2;
          ivrx.push_back(ivrx[1]);   // vrx(nyx+1, .) = vrx(1, .)
          const double vv2 = vv1 * vv1;
          const double xv = (d + R42 * a) * vv1;
          const double yv = (bcd + 2.0 * R42 * ak) / daba * vv1;
          const double zv = wv / a * vv1;
          for (int j = 1; j <= nyx; ++j) {
            if (std::fabs(ayx1[j + 1] - ayx1[j]) < 1e-8) continue;   // a 'bad' intersection
            const double prob = (ayx1[j] + ayx1[j + 1]) / 2.0;
            const double ap1 = ct + rr * std::cos(prob), ap2 = cs + rr * std::sin(prob);
            if (buried(ap1, ap2)) continue;   // the arc's middle point is covered
            const double alp = ayx1[j], bet = ayx1[j + 1];
            const double dcbetmalp = std::cos(5e-1 * (bet - alp));
            const double dcbetpalp = std::cos(5e-1 * (bet + alp));
            const double dsbetmalp = std::sin(5e-1 * (bet - alp));
            const double dsbetpalp = std::sin(5e-1 * (bet + alp));
            const double uv = daba * (bcd + 2.0 * R42 * ak) * dcbetmalp -
                              a * std::sqrt(b2c2 - 4.0 * a * d) * (b * dcbetpalp + c * dsbetpalp);
            As[i] = As[i] + R2 * (aia * (alp - bet) +
                                  (d + R42 * a) * vv1 *
                                      (pi - 2.0 * std::atan(uv / (2.0 * ak * vv * dsbetmalp))));
            if (gradan) {   // esolan.f:718-899
              const double dsalp = std::sin(alp), dcalp = std::cos(alp);
              const double dsbet = std::sin(bet), dcbet = std::cos(bet);
              const double dcotbma = 1.0 / std::tan(5e-1 * (bet - alp));
              const int kk = (int)vertex[ivrx[j]].c4, LL = (int)vertex[ivrx[j + 1]].c4;
              const double P = b * dcbetpalp + c * dsbetpalp;
              const double Q = -b * dsbetpalp + c * dcbetpalp;
              const double s2 = dsbetmalp * dsbetmalp;
              const double tt = yv * dcotbma - zv * P / dsbetmalp;
              const double a1 = NB(kk, 1), b1 = NB(kk, 2), c1 = NB(kk, 3), d1 = NB(kk, 4);
              const double a2 = NB(LL, 1), b2 = NB(LL, 2), c2 = NB(LL, 3), d2 = NB(LL, 4);
              const double ab1 = a * b1 - b * a1, ac1 = a * c1 - c * a1;
              const double ab2 = a * b2 - b * a2, ac2 = a * c2 - c * a2;
              const double am1 = wv * aia * a1 * (ab1 * dsalp - ac1 * dcalp);
              const double am2 = wv * aia * a2 * (ab2 * dsbet - ac2 * dcbet);
              double dalp[5], dbet[5], daalp[5], dabet[5], dv[5], ddx[5], ddy[5], ddz[5],
                  dt[5], di[5];
              auto ang = [&](double* out, double A1, double B1, double C1, double D1, double AB,
                             double AC, double cs_, double sn_, double am) {
                out[1] = (B1 * AB + C1 * AC - 2.0 * d * A1 * A1 -
                          a * (B1 * B1 + C1 * C1 - 4.0 * A1 * D1) -
                          2.0 * d * aia * A1 * (AB * cs_ + AC * sn_) / wv +
                          wv * aia * A1 * (B1 * cs_ + C1 * sn_)) /
                         am;
                out[2] = (-A1 * AB + b * A1 * A1 + b * aia * A1 * (AB * cs_ + AC * sn_) / wv -
                          wv * aia * A1 * A1 * cs_) /
                         am;
                out[3] = (-A1 * AC + c * A1 * A1 + c * aia * A1 * (AB * cs_ + AC * sn_) / wv -
                          wv * aia * A1 * A1 * sn_) /
                         am;
                out[4] = (-2.0 * a * A1 * A1 - 2.0 * daba * A1 * (AB * cs_ + AC * sn_) / wv) / am;
              };
              ang(dalp, a1, b1, c1, d1, ab1, ac1, dcalp, dsalp, am1);
              ang(dbet, a2, b2, c2, d2, ab2, ac2, dcbet, dsbet, am2);
              auto dang = [&](double* out, double A1, double B1, double C1, double D1, double AB,
                              double AC, double cs_, double sn_, double am) {
                out[1] = (-b * AB - c * AC + wv * wv * A1 + 2.0 * ak * D1 +
                          wv * aia * ((AB - b * A1) * cs_ + (AC - c * A1) * sn_)) /
                         am;
                out[2] = (a * AB - ak * B1 + wv * daba * A1 * cs_) / am;
                out[3] = (a * AC - ak * C1 + wv * daba * A1 * sn_) / am;
                out[4] = (2.0 * ak * A1) / am;
              };
              dang(daalp, a1, b1, c1, d1, ab1, ac1, dcalp, dsalp, am1);
              dang(dabet, a2, b2, c2, d2, ab2, ac2, dcbet, dsbet, am2);
              dv[2] = R42 * b * vv1;
              dv[3] = R42 * c * vv1;
              dv[4] = (d - R42 * a) * vv1;
              dv[1] = -dv[4] * R42;
              ddx[1] = R42 * vv1 - (d + R42 * a) * dv[1] * vv2;
              ddx[2] = -(d + R42 * a) * dv[2] * vv2;
              ddx[3] = -(d + R42 * a) * dv[3] * vv2;
              ddx[4] = 1.0 * vv1 - (d + R42 * a) * dv[4] * vv2;
              const double Y = b * b + c * c - 2.0 * a * d + 2.0 * R42 * ak;
              ddy[1] = (-2.0 * d + 4.0 * R42 * a) / daba * vv1 -
                       Y * (aia * vv + daba * dv[1]) / ak * vv2;
              ddy[2] = 2.0 * b / daba * vv1 - Y * aia * dv[2] / a * vv2;
              ddy[3] = 2.0 * c / daba * vv1 - Y * aia * dv[3] / a * vv2;
              ddy[4] = -2.0 * a / daba * vv1 - Y * aia * dv[4] / a * vv2;
              ddz[1] = -2.0 * d / wv / a * vv1 - wv * (vv + a * dv[1]) / ak * vv2;
              ddz[2] = b / wv / a * vv1 - wv * dv[2] / a * vv2;
              ddz[3] = c / wv / a * vv1 - wv * dv[3] / a * vv2;
              ddz[4] = -2.0 / wv * vv1 - wv * dv[4] / a * vv2;
              for (int x = 1; x <= 4; ++x) {
                const double extra =
                    x == 2 ? dcbetpalp * 2.0 * dsbetmalp : (x == 3 ? dsbetpalp * 2.0 * dsbetmalp : 0.0);
                dt[x] = dcotbma * ddy[x] - 5e-1 * yv * (dbet[x] - dalp[x]) / s2 -
                        (P / dsbetmalp) * ddz[x] -
                        5e-1 * zv *
                            (Q * dsbetmalp * (dalp[x] + dbet[x]) -
                             P * dcbetmalp * (dbet[x] - dalp[x]) + extra) /
                            s2;
                di[x] = R2 * (aia * (dalp[x] - dbet[x]) + (pi - 2.0 * std::atan(5e-1 * tt)) * ddx[x] -
                              4.0 * xv * dt[x] / (4.0 + tt * tt));
              }
              double dii[5][4];
              dii[1][1] = 2.0 * DD(jk, 2);
              dii[1][2] = 2.0 * DD(jk, 3);
              dii[1][3] = 2.0 * (DD(jk, 4) - R);
              dii[2][1] = -R42 - R42;
              dii[2][2] = 0.0;
              dii[2][3] = 0.0;
              dii[3][1] = 0.0;
              dii[3][2] = dii[2][1];
              dii[3][3] = 0.0;
              dii[4][1] = dii[1][1] * R42;
              dii[4][2] = dii[1][2] * R42;
              dii[4][3] = 2.0 * (DD(jk, 4) + R) * R42;
              for (int x = 1; x <= 3; ++x)
                gr[3 * jk + x - 1] += di[1] * dii[1][x] + di[2] * dii[2][x] + di[3] * dii[3][x] +
                                      di[4] * dii[4][x];
              double dta[5], dtb[5], di1[5], di2[5];
              for (int x = 1; x <= 4; ++x) {
                dta[x] = 5e-1 * daalp[x] * ((yv - zv * (Q * dsbetmalp + P * dcbetmalp)) / s2);
                dtb[x] = 5e-1 * dabet[x] * ((-yv - zv * (Q * dsbetmalp - P * dcbetmalp)) / s2);
                di1[x] = R2 * (aia * daalp[x] - 4.0 * xv * dta[x] / (4.0 + tt * tt));
                di2[x] = R2 * (-aia * dabet[x] - 4.0 * xv * dtb[x] / (4.0 + tt * tt));
              }
              auto rows = [&](int m) {
                dii[1][1] = 2.0 * DD(m, 2);
                dii[1][2] = 2.0 * DD(m, 3);
                dii[1][3] = 2.0 * (DD(m, 4) - R);
                dii[4][1] = dii[1][1] * R42;
                dii[4][2] = dii[1][2] * R42;
                dii[4][3] = 2.0 * (DD(m, 4) + R) * R42;
              };
              rows(kk);
              for (int x = 1; x <= 3; ++x)
                gr[3 * kk + x - 1] += di1[1] * dii[1][x] + di1[2] * dii[2][x] +
                                      di1[3] * dii[3][x] + di1[4] * dii[4][x];
              rows(LL);
              for (int x = 1; x <= 3; ++x)
                gr[3 * LL + x - 1] += di2[1] * dii[1][x] + di2[2] * dii[2][x] +
                                      di2[3] * dii[3][x] + di2[4] * dii[4][x];
            }
          }
        } else {   // the circle is a line (esolan.f:904-994)
          const double ang = std::atan2(b, c);
          double a1 = std::sin(ang), a2 = std::cos(ang);
          ax1.assign(nyx + 1, 0.0);
          ax2.assign(nyx + 1, 0.0);
          for (int j = 1; j <= nyx; ++j) {
            ax1[j] = ay1[j] * a2 - ay2[j] * a1;
            ax2[j] = ay1[j] * a1 + ay2[j] * a2;
          }
          for (int j = 1; j <= nyx - 1; ++j) {   // selection sort by ax(.,1)
            double m = ax1[j];
            int jm = j;
            for (int L = j + 1; L <= nyx; ++L)
              if (m > ax1[L]) {
                m = ax1[L];
                jm = L;
              }
            if (jm != j) {
              std::swap(ax1[jm], ax1[j]);
              std::swap(ax2[jm], ax2[j]);
              std::swap(ay1[jm], ay1[j]);
              std::swap(ay2[jm], ay2[j]);
            }
          }
          ayx1.assign(nyx + 2, 0.0);
          if (c != 0.0)
            for (int j = 1; j <= nyx; ++j) ayx1[j] = (ay1[j] - ay1[1]) / c;
          else
            for (int j = 1; j <= nyx; ++j) ayx1[j] = -(ay2[j] - ay2[1]) / b;
          probe.assign(nyx + 2, 0.0);
          probe[1] = -1.0;
          for (int j = 1; j <= nyx - 1; ++j) probe[j + 1] = (ayx1[j] + ayx1[j + 1]) / 2.0;
          probe[nyx + 1] = ayx1[nyx] + 1.0;
          const double bc = b * b + c * c;
          const double cc = std::sqrt(R42 * bc + d * d);
          const double caba = c * ay1[1] - b * ay2[1];
          double p1 = ay1[1] + c * probe[1], p2 = ay2[1] - b * probe[1];
          if (!buried(p1, p2)) {
            const double arg2 = bc * ayx1[1] + caba;
            As[i] = As[i] + R22 * d * (std::atan(arg2 / cc) + pi / 2.0) / cc;
          }
          for (int j = 2; j <= nyx; ++j) {
            p1 = ay1[1] + c * probe[j];
            p2 = ay2[1] - b * probe[j];
            if (buried(p1, p2)) continue;
            const double arg1 = bc * ayx1[j - 1] + caba, arg2 = bc * ayx1[j] + caba;
            As[i] = As[i] + R22 * d * (std::atan(arg2 / cc) - std::atan(arg1 / cc)) / cc;
          }
          p1 = ay1[1] + c * probe[nyx + 1];
          p2 = ay2[1] - b * probe[nyx + 1];
          if (!buried(p1, p2)) {
            const double arg1 = bc * ayx1[nyx] + caba;
            As[i] = As[i] + R22 * d * (pi / 2.0 - std::atan(arg1 / cc)) / cc;
          }
        }
      }
    } while (false);
    if (assemble) {   // label 11 (esolan.f:998-1030): grad(i, i) and the frame turned back
      for (int j = 1; j <= ine_g; ++j) al[ifu_g + j] = neib[j];
      al[0] = ifu_g + ine_g;
      for (int x = 0; x < 3; ++x) {
        double ss = 0.0;
        for (int j2 = 1; j2 <= al[0]; ++j2) ss = ss + gr[3 * al[j2] + x];
        gr[3 * i + x] = -ss;
      }
      if (jjj != 0) {
        const double sfsg = sf * sg, sfcg = sf * cg, cfsg = cf * sg, cfcg = cf * cg;
        auto turn = [&](int j) {
          const double xx = gr[3 * j], yy = gr[3 * j + 1], zz = gr[3 * j + 2];
          gr[3 * j] = xx * cg - yy * sfsg + zz * cfsg;
          gr[3 * j + 1] = yy * cf + zz * sf;
          gr[3 * j + 2] = -xx * sg - yy * sfcg + zz * cfcg;
        };
        turn(i);
        for (int j2 = 1; j2 <= al[0]; ++j2) turn(al[j2]);
      }
    }
    if (gradan)   // esolan.f:1034-1042, in atom order i
      for (int j = 1; j <= numat; ++j)
        for (int x = 0; x < 3; ++x) gradan[3 * j + x] = gradan[3 * j + x] + sigma[i] * gr[3 * j + x];
    sss = sss + As[i] * sigma[i];   // label 1
  }
  if (As_out)
    for (int i = 1; i <= numat; ++i) As_out[i] = As[i];
  return sss;
}

double Smmp::esolan(int nmol) {
  int numat;
  if (nmol == 0)
    numat = iatrs2[irsml2[ntlml]] - iatrs1[irsml1[1]] + 1;   // esolan.f:93-97
  else
    numat = iatrs2[irsml2[nmol]] - iatrs1[irsml1[nmol]] + 1;
  return esolan_areas(numat, &xat_[2], &yat_[2], &zat_[2], rvdw.data(), sigma.data(),
                      [this] { return grnd(); }, nullptr, nullptr);
}

}  // namespace oracle
