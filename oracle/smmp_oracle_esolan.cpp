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
                    double* As_out) {
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

  const double rdpcut = (double)1e-10f;   // esolan.f:133, a single-precision literal

  for (int i = 1; i <= numat; ++i) {   // do 1 i = 1, numat
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
      int jjj = 0;
      int k = neib[1];
      double ddp = std::fabs(sq(DD(k, 2)) + sq(DD(k, 3)) + sq(R - DD(k, 4)) - pol[k]);
      for (int j = 2; j <= neib[0]; ++j) {
        k = neib[j];
        double ddp2 = std::fabs(sq(DD(k, 2)) + sq(DD(k, 3)) + sq(R - DD(k, 4)) - pol[k]);
        if (ddp2 < ddp) ddp = ddp2;
      }
      double cf = 0, sf = 0, cg = 0, sg = 0;
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

      for (int q = 1; q <= ifu; ++q) {   // esolan.f:533-578
        const double a = NB(fullarc[q], 1), aia = a < 0.0 ? -1.0 : 1.0;
        const double b = NB(fullarc[q], 2), c = NB(fullarc[q], 3), d = NB(fullarc[q], 4);
        if (a != 0.0)
          As[i] = As[i] - aia * R22p *
                              (1.0 + (-(d / a) - R42) * std::fabs(a) /
                                         std::sqrt(sq(R42 * a - d) + R42 * (b * b + c * c)));
        else
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
        for (int j = 1; j <= iv; ++j) {
          if (vertex[j].c3 == double(jk)) {
            ++nyx;
            ay1.push_back(vertex[j].t);
            ay2.push_back(vertex[j].s);
          }
          if (vertex[j].c4 == double(jk)) {
            ++nyx;
            ay1.push_back(vertex[j].t);
            ay2.push_back(vertex[j].s);
            std::swap(vertex[j].c3, vertex[j].c4);
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
            }
          }
          ayx1[nyx + 1] = ayx1[1] + pi2;
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
                      [this] { return grnd(); }, nullptr);
}

}  // namespace oracle
