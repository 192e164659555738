// Host-side internal->Cartesian rebuild used while a molecule is assembled
// (bldmol after getmol, eyring inside rplgrp, setvar inside redvar).  The
// per-proposal rebuild of the sampling path runs on the GPU.  Restates
// setvar.f, bldmol.f, dihedr.f and difang.f of SMMP trunk.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "assembly.hpp"

namespace smmpb200 {

namespace {
constexpr double pi = 3.141592653589793;
constexpr double pi2 = 2.0 * pi;
double fsign(double a, double b) { return b >= 0 ? std::fabs(a) : -std::fabs(a); }
}  // namespace

// difang.f:12-33
double difang(double a1, double a2) {
  double d = std::fmod(a2 - a1, pi2);
  return std::fabs(d) <= pi ? d : d - fsign(pi2, d);
}
// difang.f:38-60
double addang(double a1, double a2) {
  double d = std::fmod(a1 + a2, pi2);
  return std::fabs(d) <= pi ? d : d - fsign(pi2, d);
}

// setvar.f:13-72: set variables of molecule nml (phase angles of sibling
// branches shift together) and rebuild.
void Assembly::setvar(int nml, const double* vlvrx) {
  int i1vr = ivrml1[nml];
  for (int i = i1vr; i <= i1vr + nvrml[nml] - 1; ++i) {
    int iat = iatvr[i], ity = ityvr[i];
    if (ity == 3) {
      double tsh = difang(toat[iat], vlvrx[i]);
      int iow = iowat[iat];
      for (int j = 1; j <= nbdat[iow]; ++j) {
        int jat = IBD(j, iow);
        if (iowat[jat] == iow) {
          double to = toat[jat] + tsh;
          if (std::fabs(to) > pi) to = to - fsign(pi2, to);
          toat[jat] = to;
          sntoat[jat] = std::sin(to);
          cstoat[jat] = std::cos(to);
        }
      }
    } else if (ity == 2) {
      double ba = vlvrx[i];
      baat[iat] = ba;
      snbaat[iat] = std::sin(ba);
      csbaat[iat] = std::cos(ba);
    } else if (ity == 1) {
      blat[iat] = vlvrx[i];
    }
  }
  bldmol(nml);
}

// bldmol.f:13-93
void Assembly::bldmol(int nml) {
  int i1, i2, i3;
  fnd3ba(nml, i1, i2, i3);
  ixrfpt[1][nml] = i1;
  ixrfpt[2][nml] = i2;
  ixrfpt[3][nml] = i3;
  xat(i1) = gbpr[1][nml];
  yat(i1) = gbpr[2][nml];
  zat(i1) = gbpr[3][nml];
  rfpt[1][nml] = xat(i1);
  rfpt[2][nml] = yat(i1);
  rfpt[3][nml] = zat(i1);
  double xg[3], zg[3];
  setgbl(nml, i1, i2, i3, xg, zg);
  xbaat[i1] = zg[0];
  ybaat[i1] = zg[1];
  zbaat[i1] = zg[2];
  xtoat[i1] = xg[0];
  ytoat[i1] = xg[1];
  ztoat[i1] = xg[2];
  int ifirs = irsml1[nml];
  for (int i = ifirs; i <= irsml2[nml]; ++i) {
    int jj = (i == ifirs) ? iatrs1[i] + 1 : iatrs1[i];
    for (int j = jj; j <= iatrs2[i]; ++j) eyring(j, iowat[j]);
  }
  double x1, x2, x3, y1, y2, y3, z1, z2, z3;
  setsys(i1, i2, i3, x1, x2, x3, y1, y2, y3, z1, z2, z3);
  xrfax[1][nml] = x1; xrfax[2][nml] = x2; xrfax[3][nml] = x3;
  yrfax[1][nml] = -y1; yrfax[2][nml] = -y2; yrfax[3][nml] = -y3;
  zrfax[1][nml] = -z1; zrfax[2][nml] = -z2; zrfax[3][nml] = -z3;
}

// fnd3ba (bldmol.f:95-173): first three backbone atoms of molecule nml.
void Assembly::fnd3ba(int nml, int& i1, int& i2, int& i3) {
  int irs = irsml1[nml];
  i1 = iatrs1[irs];
  int i, ix, irg2;
  bool bb;
  fndbrn(nml, irs, i1, i, ix, irg2, bb);
  i2 = i + 1;
  int ibd[5] = {0, iowat[i1], IBD(1, i1), IBD(2, i1), IBD(3, i1)};
  ix = 0;
  for (int k = 1; k <= nbdat[i1] + 1; ++k)
    if (iowat[ibd[k]] != i1) {
      if (ix != 0) throw std::runtime_error("fnd3ba> Can handle only simple ring at 1st atom");
      ix = ibd[k];
    }
  ix = ixatrs[irs];
  if (i2 == ix) {
    if (irs < irsml2[nml]) {
      i3 = iatrs1[irs + 1];
      return;
    }
  } else {
    for (int k = ix; k >= i2 + 1; --k)
      if (iowat[k] == i2) {
        i3 = k;
        return;
      }
  }
  throw std::runtime_error("fnd3ba> Cannot find backbone atom");
}

// eyring (bldmol.f:175-242): place atom i from the local frame of atom ia.
void Assembly::eyring(int i, int ia) {
  double ct = cstoat[i], st = sntoat[i], ca = csbaat[i], sa = snbaat[i], bl = blat[i];
  double x1 = xtoat[ia], x2 = ytoat[ia], x3 = ztoat[ia];
  double z1 = xbaat[ia], z2 = ybaat[ia], z3 = zbaat[ia];
  double y1 = z2 * x3 - z3 * x2;
  double y2 = z3 * x1 - z1 * x3;
  double y3 = z1 * x2 - z2 * x1;
  double h2 = -sa * ct, h3 = -sa * st;
  x1 = -ca * x1 + h2 * y1 + h3 * z1;
  x2 = -ca * x2 + h2 * y2 + h3 * z2;
  x3 = -ca * x3 + h2 * y3 + h3 * z3;
  double dx = 1.0 / std::sqrt(x1 * x1 + x2 * x2 + x3 * x3);
  x1 = x1 * dx;
  x2 = x2 * dx;
  x3 = x3 * dx;
  xtoat[i] = x1;
  ytoat[i] = x2;
  ztoat[i] = x3;
  z1 = -st * y1 + ct * z1;
  z2 = -st * y2 + ct * z2;
  z3 = -st * y3 + ct * z3;
  double dz = 1.0 / std::sqrt(z1 * z1 + z2 * z2 + z3 * z3);
  xbaat[i] = z1 * dz;
  ybaat[i] = z2 * dz;
  zbaat[i] = z3 * dz;
  xat(i) = xat(ia) + x1 * bl;
  yat(i) = yat(ia) + x2 * bl;
  zat(i) = zat(ia) + x3 * bl;
}

// setsys (bldmol.f:244-300)
void Assembly::setsys(int i1, int i2, int i3, double& x1, double& x2, double& x3, double& y1,
                  double& y2, double& y3, double& z1, double& z2, double& z3) {
  double h1 = xat(i2), h2 = yat(i2), h3 = zat(i2);
  x1 = h1 - xat(i1);
  x2 = h2 - yat(i1);
  x3 = h3 - zat(i1);
  y1 = h1 - xat(i3);
  y2 = h2 - yat(i3);
  y3 = h3 - zat(i3);
  z1 = x2 * y3 - x3 * y2;
  z2 = x3 * y1 - x1 * y3;
  z3 = x1 * y2 - x2 * y1;
  double dx = 1.0 / std::sqrt(x1 * x1 + x2 * x2 + x3 * x3);
  x1 = x1 * dx;
  x2 = x2 * dx;
  x3 = x3 * dx;
  double dz = 1.0 / std::sqrt(z1 * z1 + z2 * z2 + z3 * z3);
  z1 = z1 * dz;
  z2 = z2 * dz;
  z3 = z3 * dz;
  y1 = z2 * x3 - z3 * x2;
  y2 = z3 * x1 - z1 * x3;
  y3 = z1 * x2 - z2 * x1;
}

// setgbl (bldmol.f:303-420): frame of the first atom from the global angles.
void Assembly::setgbl(int nml, int, int i2, int i3, double* xg, double* zg) {
  double ag[3][3];
  double ca = std::cos(gbpr[4][nml]), sa = std::sin(gbpr[4][nml]);
  double cb = std::cos(gbpr[5][nml]), sb = std::sin(gbpr[5][nml]);
  double cg = std::cos(gbpr[6][nml]), sg = std::sin(gbpr[6][nml]);
  double x1 = ca * cg - sa * sb * sg, x2 = sa * cg + ca * sb * sg, x3 = -cb * sg;
  double d = std::sqrt(x1 * x1 + x2 * x2 + x3 * x3);
  ag[0][0] = x1 / d; ag[1][0] = x2 / d; ag[2][0] = x3 / d;
  double y1 = -sa * cb, y2 = ca * cb, y3 = sb;
  d = std::sqrt(y1 * y1 + y2 * y2 + y3 * y3);
  ag[0][1] = y1 / d; ag[1][1] = y2 / d; ag[2][1] = y3 / d;
  double z1 = ca * sg + sa * sb * cg, z2 = sa * sg - ca * sb * cg, z3 = cb * cg;
  d = std::sqrt(z1 * z1 + z2 * z2 + z3 * z3);
  ag[0][2] = z1 / d; ag[1][2] = z2 / d; ag[2][2] = z3 / d;
  double ct2 = cstoat[i2], st2 = sntoat[i2], sa2 = snbaat[i2];
  x1 = -csbaat[i2];
  x2 = -sa2 * ct2;
  x3 = -sa2 * st2;
  double dx = std::sqrt(x1 * x1 + x2 * x2 + x3 * x3);
  x1 = x1 / dx; x2 = x2 / dx; x3 = x3 / dx;
  double st3 = sntoat[i3], ct3 = cstoat[i3];
  z1 = -st3 * (st2 * x3 + ct2 * x2);
  z2 = st3 * ct2 * x1 + ct3 * st2;
  z3 = st3 * st2 * x1 - ct3 * ct2;
  double dz = std::sqrt(z1 * z1 + z2 * z2 + z3 * z3);
  z1 = z1 / dz; z2 = z2 / dz; z3 = z3 / dz;
  y1 = z2 * x3 - z3 * x2;
  y3 = z1 * x2 - z2 * x1;
  xg[0] = ag[0][0] * x1 + ag[0][1] * y1 + ag[0][2] * z1;
  xg[1] = ag[1][0] * x1 + ag[1][1] * y1 + ag[1][2] * z1;
  xg[2] = ag[2][0] * x1 + ag[2][1] * y1 + ag[2][2] * z1;
  dx = std::sqrt(xg[0] * xg[0] + xg[1] * xg[1] + xg[2] * xg[2]);
  zg[0] = ag[0][0] * x3 + ag[0][1] * y3 + ag[0][2] * z3;
  zg[1] = ag[1][0] * x3 + ag[1][1] * y3 + ag[1][2] * z3;
  zg[2] = ag[2][0] * x3 + ag[2][1] * y3 + ag[2][2] * z3;
  dz = std::sqrt(zg[0] * zg[0] + zg[1] * zg[1] + zg[2] * zg[2]);
  for (int i = 0; i < 3; ++i) {
    xg[i] = xg[i] / dx;
    zg[i] = zg[i] / dz;
  }
}

// valang (dihedr.f:73-110)
double Assembly::valang(int i1, int i2, int i3) {
  double h1 = xat(i2), h2 = yat(i2), h3 = zat(i2);
  double x1 = xat(i1) - h1, x2 = yat(i1) - h2, x3 = zat(i1) - h3;
  double y1 = xat(i3) - h1, y2 = yat(i3) - h2, y3 = zat(i3) - h3;
  double x = x1 * x1 + x2 * x2 + x3 * x3;
  double y = y1 * y1 + y2 * y2 + y3 * y3;
  double u = x * y;
  if (u == 0.0) throw std::runtime_error("valang> Error in coordinates");
  double a = (x1 * y1 + x2 * y2 + x3 * y3) / std::sqrt(u);
  a = std::max(a, -1.0);
  a = std::min(a, 1.0);
  return std::acos(a);
}

// dihedr (dihedr.f:12-70)
double Assembly::dihedr(int i1, int i2, int i3, int i4) {
  double x1 = xat(i2) - xat(i1), y1 = yat(i2) - yat(i1), z1 = zat(i2) - zat(i1);
  double x2 = xat(i3) - xat(i2), y2 = yat(i3) - yat(i2), z2 = zat(i3) - zat(i2);
  double ux1 = y1 * z2 - z1 * y2, uy1 = z1 * x2 - x1 * z2, uz1 = x1 * y2 - y1 * x2;
  x1 = xat(i4) - xat(i3);
  y1 = yat(i4) - yat(i3);
  z1 = zat(i4) - zat(i3);
  double ux2 = z1 * y2 - y1 * z2, uy2 = x1 * z2 - z1 * x2, uz2 = y1 * x2 - x1 * y2;
  double u1 = ux1 * ux1 + uy1 * uy1 + uz1 * uz1;
  double u2 = ux2 * ux2 + uy2 * uy2 + uz2 * uz2;
  double u = u1 * u2;
  if (u == 0.0) throw std::runtime_error("dihedr> Error in coordinates");
  double a = (ux1 * ux2 + uy1 * uy2 + uz1 * uz2) / std::sqrt(u);
  a = std::max(a, -1.0);
  a = std::min(a, 1.0);
  double d = std::acos(a);
  if (ux1 * (uy2 * z2 - uz2 * y2) + uy1 * (uz2 * x2 - ux2 * z2) + uz1 * (ux2 * y2 - uy2 * x2) <
      0.0)
    d = -d;
  return d;
}

}  // namespace smmpb200
