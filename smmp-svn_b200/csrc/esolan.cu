// Analytic solvent-accessible surface and its solvation energy on the GPU
// (esolan.f:12-1050, the itysol < 0 model of energy.f:79-82): for every
// atom, the neighbour spheres cut circles on its surface; in the stereographic
// projection from the north point each circle is a*(t^2+s^2) + b*t + c*s + d
// = 0, circles inside others are dropped, intersection points are found, and
// the exposed area is summed arc by arc in closed form.  The gradients the
// reference also computes never feed back into the areas and are not built.
//
// One CTA per chain, one thread per atom (the per-atom work is sequential
// and data dependent: in-place deletions from the circle list, sorting of
// the intersection angles), scratch for each thread in global memory.  When
// the north point of an atom lies within 1e-6 of a neighbour sphere the
// reference turns the neighbours by two random angles drawn from the global
// stream (esolan.f:180-253): such atoms are left for a second pass in which
// one thread takes them in atom order and draws from the chain's stream, so
// the numbers drawn, and their order, are the reference's.
//
// This file is compiled with -fmad=false: every multiply and add is rounded
// separately, in the reference's order, as in the oracle's restatement.
#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"
#include "kernels.hpp"
#include "mt.cuh"

namespace smmpb200 {

namespace {

constexpr double kPiE = 3.141592653589793;
constexpr double kPi2E = 2.0 * kPiE;
constexpr double kPi4E = 4.0 * kPiE;
constexpr int kEsNb = 256;       // neighbour spheres of one atom
constexpr int kEsVert = 4096;    // intersection points of one atom
constexpr int kEsCircle = 2 * kEsNb + 2;
constexpr int kEsThreads = 128;
// per-thread scratch, in doubles: dd, nbr (4 per neighbour), vertices (4
// each), six arrays of one circle's points, then the integer arrays
constexpr size_t kEsDoubles = 8 * kEsNb + 4 * kEsVert + 6 * kEsCircle;
constexpr size_t kEsInts = 5 * (kEsNb + 2) + 2 * kEsNb + 2;
constexpr size_t kEsPerThread = kEsDoubles + (kEsInts + 1) / 2;

__host__ __device__ __forceinline__ double sq(double x) { return x * x; }   // Fortran x**2

struct EsWork {
  double* dd;     // [4p + 0..3]: radius, x, y, z of neighbour p relative to atom i
  double* nbr;    // [4p + 0..3]: a, b, c, d of circle p
  double* vert;   // [4v + 0..3]: t, s, circle, circle
  double *ay1, *ay2, *ayx1, *ax1, *ax2, *probe;
  int *neib, *neibp, *fullarc, *al, *ta2, *atom;
};

__host__ __device__ EsWork es_work(double* base) {
  EsWork w;
  double* p = base;
  w.dd = p;
  p += 4 * kEsNb;
  w.nbr = p;
  p += 4 * kEsNb;
  w.vert = p;
  p += 4 * kEsVert;
  w.ay1 = p;
  p += kEsCircle;
  w.ay2 = p;
  p += kEsCircle;
  w.ayx1 = p;
  p += kEsCircle;
  w.ax1 = p;
  p += kEsCircle;
  w.ax2 = p;
  p += kEsCircle;
  w.probe = p;
  p += kEsCircle;
  int* q = reinterpret_cast<int*>(p);
  w.neib = q;
  q += kEsNb + 2;
  w.neibp = q;
  q += kEsNb + 2;
  w.fullarc = q;
  q += kEsNb + 2;
  w.ta2 = q;
  q += kEsNb + 2;
  w.atom = q;
  q += kEsNb + 2;
  w.al = q;
  return w;
}

enum EsStatus : int { kEsDone = 0, kEsNeedsDraws = 1, kEsOverflow = 2, kEsCoincident = 3 };

// Exposed area of atom i (esolan.f:113-996).  Circles are numbered by their
// position p in the neighbour list (neighbours in atom order, as the
// reference's atom numbers order them); list entries neib[1..] hold p.
// Without DRAW an atom that needs the random re-orientation returns
// kEsNeedsDraws and draws nothing.  Host-callable so that a CPU test can
// check this arithmetic against the oracle bit for bit (the library itself
// calls it only from k_esolan).
template <bool DRAW>
__host__ __device__ int esolan_atom(const DMol& m, const double* xyz, int i, EsWork& w, uint32_t* slot,
                           double* area) {
  const double R = m.rvdw[i];
  double As = kPi4E * (R * R);
  const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
  int nbn = 0;
  for (int q = 0; q < m.nheavy; ++q) {   // esolan.f:127-152 (atoms of radius 0 never count)
    const int j = m.heavy[q];
    if (j == i) continue;
    const double xj = xyz[3 * j], yj = xyz[3 * j + 1], zj = xyz[3 * j + 2];
    double ddp = sq(xj - xi) + sq(yj - yi) + sq(zj - zi);
    if (ddp < (double)1e-10f) return kEsCoincident;
    ddp = sqrt(ddp);
    const double rj = m.rvdw[j];
    if (ddp + R <= rj) {   // atom i inside atom j
      *area = 0.0;
      return kEsDone;
    }
    if (!(ddp <= R - rj || ddp >= R + rj)) {
      if (nbn == kEsNb) return kEsOverflow;
      const int p = nbn;   // position in the neighbour list (0-based)
      w.neib[p + 1] = p;
      ++nbn;
      w.atom[p] = j;
      w.dd[4 * p] = rj;
      w.dd[4 * p + 1] = xj - xi;
      w.dd[4 * p + 2] = yj - yi;
      w.dd[4 * p + 3] = zj - zi;
    }
  }
  w.neib[0] = nbn;
  if (nbn == 0) {
    *area = As;
    return kEsDone;
  }
  const double pol_i = R * R;
  const double R2 = R * R, R22 = R2 + R2, R42 = R22 + R22, R22p = R22 * kPiE;
  auto pol = [&](int p) { return w.dd[4 * p] * w.dd[4 * p]; };

  // north point against every neighbour sphere (esolan.f:180-238)
  int p = w.neib[1];
  double ddp = fabs(sq(w.dd[4 * p + 1]) + sq(w.dd[4 * p + 2]) + sq(R - w.dd[4 * p + 3]) - pol(p));
  for (int j = 2; j <= w.neib[0]; ++j) {
    p = w.neib[j];
    const double d2 =
        fabs(sq(w.dd[4 * p + 1]) + sq(w.dd[4 * p + 2]) + sq(R - w.dd[4 * p + 3]) - pol(p));
    if (d2 < ddp) ddp = d2;
  }
  if (ddp < 1.0e-6) {
    if constexpr (!DRAW) {
      return kEsNeedsDraws;
    } else {
      double cf = 0, sf = 0, cg = 0, sg = 0;
      int tries = 0;
      while (ddp < 1.0e-6) {
        // the reference retries without bound; a thousand draws that all land
        // within 1e-6 of a neighbour sphere mean coinciding atoms
        if (++tries > 1000) return kEsCoincident;
        double uga = stream_next(slot);
        double ufi = stream_next(slot);
        uga = kPiE * uga / 2;
        ufi = kPiE * ufi / 2;
        cf = cos(ufi);
        sf = sin(ufi);
        cg = cos(uga);
        sg = sin(uga);
        const double cfsg = cf * sg, cfcg = cf * cg;
        const double xx = R * cfsg, yy = R * sf, zz = R * cfcg;
        p = w.neib[1];
        ddp = fabs(sq(xx - w.dd[4 * p + 1]) + sq(yy - w.dd[4 * p + 2]) + sq(zz - w.dd[4 * p + 3]) -
                   pol(p));
        for (int j = 2; j <= w.neib[0]; ++j) {
          p = w.neib[j];
          const double d2 = fabs(sq(xx - w.dd[4 * p + 1]) + sq(yy - w.dd[4 * p + 2]) +
                                 sq(zz - w.dd[4 * p + 3]) - pol(p));
          if (d2 < ddp) ddp = d2;
        }
      }
      const double sfsg = sf * sg, sfcg = sf * cg, cfsg = cf * sg, cfcg = cf * cg;
      for (int j = 1; j <= w.neib[0]; ++j) {   // esolan.f:240-253
        p = w.neib[j];
        const double xx = w.dd[4 * p + 1], yy = w.dd[4 * p + 2], zz = w.dd[4 * p + 3];
        w.dd[4 * p + 1] = xx * cg - zz * sg;
        w.dd[4 * p + 2] = -(xx * sfsg) + yy * cf - zz * sfcg;
        w.dd[4 * p + 3] = xx * cfsg + yy * sf + zz * cfcg;
      }
    }
  }

  // circle coefficients (esolan.f:257-268)
  const double pom8 = 8.0 * pol_i;
  for (int q = 1; q <= w.neib[0]; ++q) {
    p = w.neib[q];
    const double dx = w.dd[4 * p + 1], dy = w.dd[4 * p + 2], dz = w.dd[4 * p + 3];
    w.nbr[4 * p] = sq(dx) + sq(dy) + sq(dz - R) - pol(p);
    w.nbr[4 * p + 1] = -(pom8 * dx);
    w.nbr[4 * p + 2] = -(pom8 * dy);
    w.nbr[4 * p + 3] = 4.0 * pol_i * (sq(dx) + sq(dy) + sq(R + dz) - pol(p));
  }
  auto A = [&](int q) { return w.nbr[4 * q]; };
  auto B = [&](int q) { return w.nbr[4 * q + 1]; };
  auto C = [&](int q) { return w.nbr[4 * q + 2]; };
  auto Dd = [&](int q) { return w.nbr[4 * q + 3]; };

  // every pair of circles (esolan.f:272-466)
  int iv = 0;
  const int nb = w.neib[0];
  bool covered = false;
  int k = w.neib[0];
  while (k > 1 && !covered) {
    k = k - 1;
    const int lfirst = w.neib[0];   // the DO bounds are fixed on entry
    for (int L = lfirst; L >= k + 1; --L) {
      const int pk = w.neib[k], pl = w.neib[L];
      const double ak1 = A(pk), al1 = A(pl);
      if (!((ak1 > 0.0 || ak1 < 0.0) && (al1 > 0.0 || al1 < 0.0))) continue;
      const double b1 = B(pk) / ak1, c1 = C(pk) / ak1, d1 = Dd(pk) / ak1;
      const double b2 = B(pl) / al1, c2 = C(pl) / al1, d2 = Dd(pl) / al1;
      const double D = 4.0 * ((b1 - b2) * (b2 * d1 - b1 * d2) + (c1 - c2) * (c2 * d1 - c1 * d2) -
                              sq(d1 - d2)) +
                       sq(b1 * c2 - b2 * c1);
      const double dist = sqrt(sq(b1 - b2) + sq(c1 - c2));
      const double s2 = sqrt(b2 * b2 + c2 * c2 - 4.0 * d2);
      const double s1 = sqrt(b1 * b1 + c1 * c1 - 4.0 * d1);
      int action = 0;   // 1 vertices, 2 drop k (next k), 3 drop L, 4 covered, 5 As=0 next k
      if (ak1 > 0.0 && al1 > 0.0) {   // a01
        if (D <= 0.0 && dist <= s2 - s1) action = 2;
        else if (D <= 0.0 && dist <= -s2 + s1) action = 3;
        else if (D > 0.0) action = 1;
      } else if (ak1 > 0.0 && al1 < 0.0) {   // a03
        if (D <= 0.0 && dist <= -s2 + s1) action = 4;
        else if (D <= 0.0 && dist >= s2 + s1) action = 2;
        else if (D > 0.0) action = 1;
      } else if (ak1 < 0.0 && al1 > 0.0) {   // a07
        if (D <= 0.0 && dist <= s2 - s1) action = 5;
        else if (D <= 0.0 && dist >= s2 + s1) action = 3;
        else if (D > 0.0) action = 1;
      } else {   // a09
        if (D <= 0.0 && dist <= s2 - s1) action = 3;
        else if (D <= 0.0 && dist <= -s2 + s1) action = 2;
        else if (D <= 0.0) action = 4;
        else action = 1;
      }
      if (action == 1) {
        if (iv + 2 > kEsVert) return kEsOverflow;
        const double am = 2.0 * (sq(b1 - b2) + sq(c1 - c2));
        const double t = -(2.0 * (b1 - b2) * (d1 - d2)) - (b2 * c1 - b1 * c2) * (c1 - c2);
        const double s = -(2.0 * (c1 - c2) * (d1 - d2)) + (b2 * c1 - b1 * c2) * (b1 - b2);
        const double pom = sqrt(D);
        const double p1 = (c1 - c2) * pom, p2 = (b1 - b2) * pom;
        double* v = w.vert + 4 * iv;
        v[0] = (t + p1) / am;
        v[1] = (s - p2) / am;
        v[2] = pk;
        v[3] = pl;
        v[4] = (t - p1) / am;
        v[5] = (s + p2) / am;
        v[6] = pk;
        v[7] = pl;
        iv += 2;
      } else if (action == 2 || action == 3) {
        const int pos = action == 2 ? k : L;
        w.neib[0] = w.neib[0] - 1;
        for (int j = pos; j <= w.neib[0]; ++j) w.neib[j] = w.neib[j + 1];
        if (action == 2) break;
      } else if (action == 4) {
        As = 0.0;
        covered = true;
        break;
      } else if (action == 5) {
        As = 0.0;   // the reference goes on with the next k
        break;
      }
    }
  }
  if (covered) {
    *area = As;
    return kEsDone;
  }

  // lines and inside-buried circles (esolan.f:468-517)
  int ita2 = 0, ita3 = 0;
  for (int j = 1; j <= w.neib[0]; ++j) {
    if (A(w.neib[j]) == 0.0) w.ta2[++ita2] = j;
    if (A(w.neib[j]) < 0.0) ++ita3;
  }
  if (ita2 > 0 && ita3 < 1) {
    As = R22p;
    if (ita2 > 1) {
      double amial = kPiE, amaal = -kPiE, amibe = kPiE, amabe = -kPiE;
      for (int j = 1; j <= ita2; ++j) {
        const int q = w.neib[w.ta2[j]];
        const double alp = atan2(C(q), B(q));
        double bet = alp;
        if (alp <= 0.0) bet = bet + kPi2E;
        if (amial > alp) amial = alp;
        if (amaal < alp) amaal = alp;
        if (amibe > bet) amibe = bet;
        if (amabe < bet) amabe = bet;
      }
      const double dal = amaal - amial, dbe = amabe - amibe;
      if (dal < kPiE) As = R22 * (kPiE - dal);
      else if (dbe < kPiE) As = R22 * (kPiE - dbe);
      else As = 0.0;
    }
  } else if ((nb > 0 && w.neib[0] < 1) || ita3 > 0) {
    As = 0.0;
  }

  // full arcs and circles with intersection points (esolan.f:519-531)
  w.neibp[0] = w.neib[0];
  for (int j = 1; j <= w.neib[0]; ++j) w.neibp[j] = w.neib[j];
  int ifu = 0, ine = 0;
  for (int j = 1; j <= w.neibp[0]; ++j) {
    const double pj = w.neibp[j];
    bool has_ip = false;
    for (int q = 0; q < iv; ++q)
      if (pj == w.vert[4 * q + 2] || pj == w.vert[4 * q + 3]) {
        has_ip = true;
        break;
      }
    if (has_ip) {
      w.neib[++ine] = w.neibp[j];
    } else {
      ++ifu;
      w.fullarc[ifu] = w.neibp[j];
      w.al[ifu] = w.neibp[j];
    }
  }
  w.neib[0] = ine;

  for (int q = 1; q <= ifu; ++q) {   // esolan.f:533-578
    const int f = w.fullarc[q];
    const double a = A(f), aia = a < 0.0 ? -1.0 : 1.0;
    const double b = B(f), c = C(f), d = Dd(f);
    if (a != 0.0)
      As = As - aia * R22p *
                    (1.0 + (-(d / a) - R42) * fabs(a) / sqrt(sq(R42 * a - d) + R42 * (b * b + c * c)));
    else
      As = As + R22p * d / sqrt(R42 * (b * b + c * c) + d * d);
  }

  for (int q = 1; q <= ine; ++q) {   // esolan.f:580-996
    const int jk = w.neib[q];
    const double a = A(jk), ak = a * a, daba = fabs(a);
    const double aia = a < 0.0 ? -1.0 : 1.0;
    const double b = B(jk), c = C(jk), d = Dd(jk);
    const double b2c2 = b * b + c * c;
    const double vv = sqrt(sq(R42 * a - d) + R42 * b2c2);
    const double vv1 = 1.0 / vv;
    const double wv = sqrt(b2c2 - 4.0 * a * d);
    int nyx = 0;
    const double djk = jk;
    for (int j = 0; j < iv; ++j) {   // esolan.f:602-622
      double* v = w.vert + 4 * j;
      if (v[2] == djk) {
        ++nyx;
        w.ay1[nyx] = v[0];
        w.ay2[nyx] = v[1];
      }
      if (v[3] == djk) {
        ++nyx;
        w.ay1[nyx] = v[0];
        w.ay2[nyx] = v[1];
        const double t = v[2];
        v[2] = v[3];
        v[3] = t;
      }
    }
    int ial = ifu;
    for (int j = 1; j <= ine; ++j)
      if (w.neib[j] != jk) w.al[++ial] = w.neib[j];
    auto buried = [&](double p1, double p2) {
      for (int ij = 1; ij <= ial; ++ij) {
        const int g = w.al[ij];
        if (A(g) * (p1 * p1 + p2 * p2) + B(g) * p1 + C(g) * p2 + Dd(g) < 0.0) return true;
      }
      return false;
    };
    if (a != 0.0) {   // esolan.f:633-717
      const double aa = 0.5 / a, ba = b * aa, ca = c * aa;
      const double bcd = b2c2 - 2.0 * a * d;
      for (int j = 1; j <= nyx; ++j) {
        w.ay1[j] = w.ay1[j] + ba;
        w.ay2[j] = w.ay2[j] + ca;
      }
      const double ct = -ba, cs = -ca, rr = 0.5 * wv / daba;
      for (int j = 1; j <= nyx; ++j) w.ayx1[j] = atan2(w.ay2[j], w.ay1[j]);
      for (int j = 1; j <= nyx - 1; ++j) {   // selection sort, ascending
        double a1 = w.ayx1[j];
        int jm = j;
        for (int ij = j + 1; ij <= nyx; ++ij)
          if (a1 > w.ayx1[ij]) {
            a1 = w.ayx1[ij];
            jm = ij;
          }
        if (jm != j) {
          a1 = w.ayx1[jm];
          w.ayx1[jm] = w.ayx1[j];
          w.ayx1[j] = a1;
        }
      }
      w.ayx1[nyx + 1] = w.ayx1[1] + kPi2E;
      for (int j = 1; j <= nyx; ++j) {
        if (fabs(w.ayx1[j + 1] - w.ayx1[j]) < 1e-8) continue;
        const double prob = (w.ayx1[j] + w.ayx1[j + 1]) / 2.0;
        const double ap1 = ct + rr * cos(prob), ap2 = cs + rr * sin(prob);
        if (buried(ap1, ap2)) continue;
        const double alp = w.ayx1[j], bet = w.ayx1[j + 1];
        const double dcbetmalp = cos(5e-1 * (bet - alp));
        const double dcbetpalp = cos(5e-1 * (bet + alp));
        const double dsbetmalp = sin(5e-1 * (bet - alp));
        const double dsbetpalp = sin(5e-1 * (bet + alp));
        const double uv = daba * (bcd + 2.0 * R42 * ak) * dcbetmalp -
                          a * sqrt(b2c2 - 4.0 * a * d) * (b * dcbetpalp + c * dsbetpalp);
        As = As + R2 * (aia * (alp - bet) +
                        (d + R42 * a) * vv1 * (kPiE - 2.0 * atan(uv / (2.0 * ak * vv * dsbetmalp))));
      }
    } else {   // the circle is a line (esolan.f:904-994)
      const double ang = atan2(b, c);
      const double a1 = sin(ang), a2 = cos(ang);
      for (int j = 1; j <= nyx; ++j) {
        w.ax1[j] = w.ay1[j] * a2 - w.ay2[j] * a1;
        w.ax2[j] = w.ay1[j] * a1 + w.ay2[j] * a2;
      }
      for (int j = 1; j <= nyx - 1; ++j) {
        double mn = w.ax1[j];
        int jm = j;
        for (int L = j + 1; L <= nyx; ++L)
          if (mn > w.ax1[L]) {
            mn = w.ax1[L];
            jm = L;
          }
        if (jm != j) {
          double t = w.ax1[jm]; w.ax1[jm] = w.ax1[j]; w.ax1[j] = t;
          t = w.ax2[jm]; w.ax2[jm] = w.ax2[j]; w.ax2[j] = t;
          t = w.ay1[jm]; w.ay1[jm] = w.ay1[j]; w.ay1[j] = t;
          t = w.ay2[jm]; w.ay2[jm] = w.ay2[j]; w.ay2[j] = t;
        }
      }
      if (c != 0.0)
        for (int j = 1; j <= nyx; ++j) w.ayx1[j] = (w.ay1[j] - w.ay1[1]) / c;
      else
        for (int j = 1; j <= nyx; ++j) w.ayx1[j] = -(w.ay2[j] - w.ay2[1]) / b;
      w.probe[1] = -1.0;
      for (int j = 1; j <= nyx - 1; ++j) w.probe[j + 1] = (w.ayx1[j] + w.ayx1[j + 1]) / 2.0;
      w.probe[nyx + 1] = w.ayx1[nyx] + 1.0;
      const double bc = b * b + c * c;
      const double cc = sqrt(R42 * bc + d * d);
      const double caba = c * w.ay1[1] - b * w.ay2[1];
      double p1 = w.ay1[1] + c * w.probe[1], p2 = w.ay2[1] - b * w.probe[1];
      if (!buried(p1, p2)) {
        const double arg2 = bc * w.ayx1[1] + caba;
        As = As + R22 * d * (atan(arg2 / cc) + kPiE / 2.0) / cc;
      }
      for (int j = 2; j <= nyx; ++j) {
        p1 = w.ay1[1] + c * w.probe[j];
        p2 = w.ay2[1] - b * w.probe[j];
        if (buried(p1, p2)) continue;
        const double arg1 = bc * w.ayx1[j - 1] + caba, arg2 = bc * w.ayx1[j] + caba;
        As = As + R22 * d * (atan(arg2 / cc) - atan(arg1 / cc)) / cc;
      }
      p1 = w.ay1[1] + c * w.probe[nyx + 1];
      p2 = w.ay2[1] - b * w.probe[nyx + 1];
      if (!buried(p1, p2)) {
        const double arg1 = bc * w.ayx1[nyx] + caba;
        As = As + R22 * d * (kPiE / 2.0 - atan(arg1 / cc)) / cc;
      }
    }
  }
  *area = As;
  return kEsDone;
}

// Chains [first, first + gridDim.x): area[c * tstride + h] of heavy atom h,
// then eysl = sum_i sigma_i A_i in atom order (esolan.f:997-1040); the
// chain's eol (the vacuum energy from k_energy) gains eysl, terms[4] = eysl.
__global__ void __launch_bounds__(kEsThreads) k_esolan(DMolSet set, DChains ch, int first,
                                                       double* scratch, double* area) {
  const int c = first + blockIdx.x;
  const DMol& m = set.mols[ch.mol_of_chain[c]];
  const double* xyz = ch.coords + (size_t)c * 3 * ch.tstride;
  double* ar = area + (size_t)c * ch.tstride;
  int* err = &ch.err[c];
  EsWork w = es_work(scratch + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * kEsPerThread);
  __shared__ int deferred;
  if (threadIdx.x == 0) deferred = 0;
  __syncthreads();
  for (int h = threadIdx.x; h < m.nheavy; h += blockDim.x) {
    double a = 0.0;
    const int st = esolan_atom<false>(m, xyz, m.heavy[h], w, nullptr, &a);
    if (st == kEsNeedsDraws) {
      a = __longlong_as_double(0x7ff8dead00000000ll);   // marked for the second pass
      atomicExch(&deferred, 1);
    } else if (st == kEsOverflow) {
      atomicCAS(err, 0, (int)kErrNeighbours);
      a = 0.0;
    } else if (st == kEsCoincident) {
      atomicCAS(err, 0, (int)kErrNonFinite);
      a = 0.0;
    }
    ar[h] = a;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  if (deferred) {   // atoms that draw, in atom order, from the chain's stream
    uint32_t* slot = ch.mt + (size_t)ch.mt_slot[c] * kMTWords;
    for (int h = 0; h < m.nheavy; ++h) {
      if (__double_as_longlong(ar[h]) != 0x7ff8dead00000000ll) continue;
      double a = 0.0;
      const int st = esolan_atom<true>(m, xyz, m.heavy[h], w, slot, &a);
      if (st != kEsDone) {
        if (*err == 0) *err = st == kEsOverflow ? kErrNeighbours : kErrNonFinite;
        a = 0.0;
      }
      ar[h] = a;
    }
  }
  double sss = 0.0;
  for (int h = 0; h < m.nheavy; ++h) sss = sss + ar[h] * m.sigma[m.heavy[h]];
  ch.terms[(size_t)c * 6 + 4] = sss;
  ch.eol[c] = ch.eol[c] + sss;
  if (!isfinite(sss)) {
    if (*err == 0) *err = kErrNonFinite;
  }
}

}  // namespace

size_t esolan_scratch_bytes(int count) {
  return (size_t)count * kEsThreads * kEsPerThread * sizeof(double);
}

cudaError_t launch_esolan(const DMolSet& set, const DChains& ch, int first, int count,
                          double* scratch, double* area, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  k_esolan<<<count, kEsThreads, 0, st>>>(set, ch, first, scratch, area);
  return cudaGetLastError();
}

}  // namespace smmpb200
