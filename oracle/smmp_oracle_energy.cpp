// CPU oracle (test infrastructure only): rebuild, ECEPP/3 energy, SASA
// solvation, MT19937 and Metropolis sweep.  Restates setvar.f, bldmol.f,
// dihedr.f, energy.f, enyshe.f, enysol.f, twister.f, difang.f, metropolis.f,
// canon.f (can_weight) and mulcan_par_mod.f90 (muca_weight*) of SMMP trunk.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "smmp_oracle.hpp"

namespace oracle {

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
void Smmp::setvar(int nml, const double* vlvrx) {
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
void Smmp::bldmol(int nml) {
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
void Smmp::fnd3ba(int nml, int& i1, int& i2, int& i3) {
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
void Smmp::eyring(int i, int ia) {
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
void Smmp::setsys(int i1, int i2, int i3, double& x1, double& x2, double& x3, double& y1,
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
void Smmp::setgbl(int nml, int, int i2, int i3, double* xg, double* zg) {
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
double Smmp::valang(int i1, int i2, int i3) {
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
double Smmp::dihedr(int i1, int i2, int i3, int i4) {
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

// energy.f:12-119 (ientyp=0; one or more molecules; eninteract is zero for a
// single chain and is included for several).
double Smmp::energy() {
  double esm = 0.0, teysm = 0.0, teyel = 0.0, teyvw = 0.0, teyhb = 0.0, teyvr = 0.0,
         teysl = 0.0;
  for (int i = 1; i <= ntlml; ++i) {
    eysm = eyel = eyvr = eyhb = eyvw = eysl = 0.0;
    setvar(i, vlvr.data());
    esm = esm + enyshe(i);
    teysm += eysm;
    teyel += eyel;
    teyhb += eyhb;
    teyvr += eyvr;
    teyvw += eyvw;
  }
  if (itysol > 0) {
    esm = esm + enysol(0);
    teysl = teysl + eysl;
  } else if (itysol < 0) {   // energy.f:79-82
    eysl = esolan(0);
    teysl = teysl + eysl;
    esm = esm + eysl;
  } else {
    eysl = 0.0;
  }
  eysm = teysm;
  eyel = teyel;
  eyvw = teyvw;
  eyhb = teyhb;
  eyvr = teyvr;
  eysl = teysl;
  double einter = 0.0;
  if (ntlml > 1) throw std::runtime_error("energy: several molecules are outside this path");
  return esm + einter;
}

// enyshe.f:13-197: ECEPP/3 energy of molecule nml over the moving-set lists.
double Smmp::enyshe(int nml) {
  int ntlvr = nvrml[nml];
  if (ntlvr == 0) return 0.0;
  eyel = eyvw = eyhb = eyvr = 0.0;
  int ifivr = ivrml1[nml];
  int i1s = imsml1[nml] + nmsml[nml];
  for (int io = ifivr + ntlvr - 1; io >= ifivr; --io) {
    int iv = iorvr[io], ia = iatvr[iv], it = ityvr[iv], ic = iclvr[iv];
    if (it == 3) {
      double e0 = e0to[ic];
      if (e0 != 0.0) eyvr = eyvr + e0 * (1.0 + sgto[ic] * std::cos(toat[ia] * rnto[ic]));
    }
    int i2s = i1s - 1;
    i1s = imsvr1[iv];
    for (int ims = i1s; ims <= i2s; ++ims) {
      for (int i = latms1[ims]; i <= latms2[ims]; ++i) {
        int ity = ityat[i];
        double cqi = conv * cgat[i];
        double xi = xat(i), yi = yat(i), zi = zat(i);
        for (int ivw = ivwat1[i]; ivw <= ivwat2[i]; ++ivw) {
          for (int j = lvwat1[ivw]; j <= lvwat2[ivw]; ++j) {
            int jty = ityat[j];
            double xij = xat(j) - xi, yij = yat(j) - yi, zij = zat(j) - zi;
            double rij2 = xij * xij + yij * yij + zij * zij;
            double rij4 = rij2 * rij2, rij6 = rij4 * rij2;
            double rij = std::sqrt(rij2);
            double ep = 1.0;
            if (epsd) {
              double sr = slp * rij;
              ep = plt - (sr * sr + 2.0 * sr + 2.0) * (plt - 1.0) * std::exp(-sr) / 2.0;
            }
            eyel = eyel + cqi * cgat[j] / (rij * ep);
            if (ihbty[ity][jty] == 0)
              eyvw = eyvw + aij[ity][jty] / (rij6 * rij6) - cij[ity][jty] / rij6;
            else
              eyhb = eyhb + ahb[ity][jty] / (rij6 * rij6) - chb[ity][jty] / (rij6 * rij4);
          }
        }
        for (int i14 = i14at1[i]; i14 <= i14at2[i]; ++i14) {
          int j = l14at[i14];
          int jty = ityat[j];
          double xij = xat(j) - xi, yij = yat(j) - yi, zij = zat(j) - zi;
          double rij2 = xij * xij + yij * yij + zij * zij;
          double rij4 = rij2 * rij2, rij6 = rij4 * rij2;
          double rij = std::sqrt(rij2);
          double ep = 1.0;
          if (epsd) {
            double sr = slp * rij;
            ep = plt - (sr * sr + 2.0 * sr + 2.0) * (plt - 1.0) * std::exp(-sr) / 2.0;
          }
          eyel = eyel + cqi * cgat[j] / (rij * ep);
          if (ihbty[ity][jty] == 0)
            eyvw = eyvw + a14[ity][jty] / (rij6 * rij6) - cij[ity][jty] / rij6;
          else
            eyhb = eyhb + ahb[ity][jty] / (rij6 * rij6) - chb[ity][jty] / (rij6 * rij4);
        }
      }
    }
  }
  eysm = eyel + eyvw + eyhb + eyvr;
  return eysm;
}

// enysol.f:107-330 over the spheres 1..numat (1-based arrays; x[1] is the
// first sphere): cubic boxes of the largest diameter, each sphere tested
// against the spheres of its own and the 26 adjacent boxes, then the npnt
// unit-sphere points scaled to its radius counted as exposed when outside
// every neighbour.  Spheres with radius <= 0 take no part.  per_atom(k, area,
// icount) is called for each sphere in the reference's box order; asa and
// vdvol are summed in that order.
void enysol_spheres(int numat, const double* x, const double* y, const double* z,
                    const double* rv, const double* spoint, int npnt, double& asa, double& vdvol,
                    const std::function<void(int, double, int)>& per_atom) {
  asa = vdvol = 0.0;
  if (numat <= 0) return;
  double avr_x = x[1], avr_y = y[1], avr_z = z[1];
  double xmin = x[1], ymin = y[1], zmin = z[1];
  double xmax = xmin, ymax = ymin, zmax = zmin;
  double rmax = rv[1];
  for (int j = 2; j <= numat; ++j) {
    if (x[j] <= xmin) xmin = x[j];
    else if (x[j] >= xmax) xmax = x[j];
    avr_x = avr_x + x[j];
    if (y[j] <= ymin) ymin = y[j];
    else if (y[j] >= ymax) ymax = y[j];
    avr_y = avr_y + y[j];
    if (z[j] <= zmin) zmin = z[j];
    else if (z[j] >= zmax) zmax = z[j];
    avr_z = avr_z + z[j];
    if (rv[j] >= rmax) rmax = rv[j];
  }
  avr_x = avr_x / double(numat);
  avr_y = avr_y / double(numat);
  avr_z = avr_z / double(numat);
  double diamax = 2.0 * rmax;
  double sizex = xmax - xmin, sizey = ymax - ymin, sizez = zmax - zmin;
  int ndx = int(sizex / diamax + 1), ndy = int(sizey / diamax + 1), ndz = int(sizez / diamax + 1);
  int nqxy = ndx * ndy, ncbox = nqxy * ndz;
  double shiftx = (double(ndx) * diamax - sizex) / 2.0;
  double shifty = (double(ndy) * diamax - sizey) / 2.0;
  double shiftz = (double(ndz) * diamax - sizez) / 2.0;
  xmin = xmin - shiftx;
  ymin = ymin - shifty;
  zmin = zmin - shiftz;
  std::vector<int> inbox(ncbox + 2, 0), numbox(numat + 1, 0), indsort(numat + 2, 0);
  for (int j = 1; j <= numat; ++j) {
    int mx = std::min(int(std::max((x[j] - xmin) / diamax, 0.0)), ndx - 1);
    int my = std::min(int(std::max((y[j] - ymin) / diamax, 0.0)), ndy - 1);
    int mz = std::min(int(std::max((z[j] - zmin) / diamax, 0.0)), ndz - 1);
    int nboxj = mx + my * ndx + mz * nqxy + 1;
    numbox[j] = nboxj;
    inbox[nboxj] = inbox[nboxj] + 1;
  }
  for (int i = 1; i <= ncbox; ++i) inbox[i + 1] = inbox[i + 1] + inbox[i];
  for (int i = 1; i <= numat; ++i) {
    int j = numbox[i], jj = inbox[j];
    indsort[jj] = i;
    inbox[j] = jj - 1;
  }
  std::vector<int> look(numat + 2);
  std::vector<double> xyz(3 * (numat + 2)), radb2(numat + 2);
  for (int iz = 0; iz <= ndz - 1; ++iz)
    for (int iy = 0; iy <= ndy - 1; ++iy)
      for (int ix = 0; ix <= ndx - 1; ++ix) {
        int ibox = ix + iy * ndx + iz * nqxy + 1;
        int lbn = inbox[ibox + 1] - inbox[ibox];
        if (lbn <= 0) continue;
        int nsx = std::max(ix - 1, 0), nsy = std::max(iy - 1, 0), nsz = std::max(iz - 1, 0);
        int nex = std::min(ix + 1, ndx - 1), ney = std::min(iy + 1, ndy - 1),
            nez = std::min(iz + 1, ndz - 1);
        int jcnt = 1;
        for (int jz = nsz; jz <= nez; ++jz)
          for (int jy = nsy; jy <= ney; ++jy)
            for (int jx = nsx; jx <= nex; ++jx) {
              int jbox = jx + jy * ndx + jz * nqxy + 1;
              for (int ii = inbox[jbox] + 1; ii <= inbox[jbox + 1]; ++ii)
                if (rv[indsort[ii]] > 0.0) look[jcnt++] = indsort[ii];
            }
        for (int ia = inbox[ibox] + 1; ia <= inbox[ibox + 1]; ++ia) {
          int jbi = indsort[ia];
          double trad = rv[jbi];
          if (!(trad > 0.0)) continue;
          int nnei = 0;
          for (int ib = 1; ib <= jcnt - 1; ++ib) {
            int jtk = look[ib];
            if (jtk == jbi) continue;
            double dx = (x[jbi] - x[jtk]) / trad;
            double dy = (y[jbi] - y[jtk]) / trad;
            double dz = (z[jbi] - z[jtk]) / trad;
            double dd = dx * dx + dy * dy + dz * dz;
            double akrad = rv[jtk] / trad;
            double dr = 1.0 + akrad;
            dr = dr * dr;
            if (dd <= dr) {
              ++nnei;
              xyz[3 * nnei + 0] = dx;
              xyz[3 * nnei + 1] = dy;
              xyz[3 * nnei + 2] = dz;
              radb2[nnei] = akrad * akrad;
            }
          }
          // A point is exposed when it lies outside every neighbour sphere.  The
          // reference first re-tests the neighbour that buried the previous point
          // (enysol.f:260-283); that only reorders the search.
          int icount = 0;
          double sx = 0.0, sy = 0.0, sz = 0.0;
          for (int il = 1; il <= npnt; ++il) {
            const double* sp = &spoint[(il - 1) * 3];
            bool exposed = true;
            for (int ik = 1; ik <= nnei; ++ik) {
              double sdd = 0.0;
              for (int k = 0; k < 3; ++k) {
                double t = xyz[3 * ik + k] + sp[k];
                sdd = sdd + t * t;
              }
              if (sdd <= radb2[ik]) {
                exposed = false;
                break;
              }
            }
            if (exposed) {
              ++icount;
              sx = sx + sp[0];
              sy = sy + sp[1];
              sz = sz + sp[2];
            }
          }
          double sdr = 4.0 * pi * trad * trad / double(npnt);
          double area = sdr * double(icount);
          double volume = sdr / 3.0 *
                          (trad * double(icount) + (x[jbi] - avr_x) * sx +
                           (y[jbi] - avr_y) * sy + (z[jbi] - avr_z) * sz);
          asa = asa + area;
          vdvol = vdvol + volume;
          per_atom(jbi, area, icount);
        }
      }
}

// enysol.f:13-339: solvation energy from the numerical SASA (point test) of
// the atoms of molecule nmol (0: all molecules).
double Smmp::enysol(int nmol) {
  eyslh = eyslp = 0.0;
  int nrslow, nrshi;
  if (nmol == 0) {
    nrslow = irsml1[1];
    nrshi = irsml2[ntlml];
  } else {
    nrslow = irsml1[nmol];
    nrshi = irsml2[nmol];
  }
  int nlow = iatrs1[nrslow], nup = iatrs2[nrshi];
  for (int i = nrslow; i <= nrshi; ++i) surfres[i] = 0.0;
  eysl = 0.0;
  const int off = nlow - 1;   // sphere k is atom off + k
  enysol_spheres(nup - nlow + 1, &xat(off), &yat(off), &zat(off), rvdw.data() + off,
                 spoint.data(), npnt, asa, vdvol, [&](int k, double area, int) {
                   const int jbi = off + k;
                   eysl = eysl + area * sigma[jbi];
                   if (sigma[jbi] < 0) {
                     eyslp = eyslp + area * sigma[jbi];
                     asap = asap + area;
                   }
                   if (sigma[jbi] > 0) {
                     eyslh = eyslh + area * sigma[jbi];
                     asah = asah + area;
                   }
                   int jres = nursat(jbi);
                   surfres[jres] = surfres[jres] + area;
                 });
  return eysl;
}

// sgrnd (twister.f:64-91): Knuth-69069 seeding of the 624-word state.
void Smmp::sgrnd(int32_t seed) {
  mt[0] = (uint32_t)seed;
  for (int i = 1; i < 624; ++i) mt[i] = 69069u * mt[i - 1];
  mti = 624;
}

// grnd (twister.f:104-177): MT19937 double in [0,1], y/(2^32-1).
double Smmp::grnd() {
  const int N = 624, M = 397;
  const uint32_t MATA = 0x9908B0DFu, UM = 0x80000000u, LM = 0x7fffffffu;
  if (mti >= N) {
    if (mti == N + 1) sgrnd(4357);
    int kk;
    uint32_t y;
    for (kk = 0; kk < N - M; ++kk) {
      y = (mt[kk] & UM) | (mt[kk + 1] & LM);
      mt[kk] = mt[kk + M] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    }
    for (; kk < N - 1; ++kk) {
      y = (mt[kk] & UM) | (mt[kk + 1] & LM);
      mt[kk] = mt[kk + (M - N)] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    }
    y = (mt[N - 1] & UM) | (mt[0] & LM);
    mt[N - 1] = mt[M - 1] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    mti = 0;
  }
  uint32_t y = mt[mti++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9D2C5680u;
  y ^= (y << 15) & 0xEFC60000u;
  y ^= (y >> 18);
  return double(y) / (4294967296.0 - 1.0);
}

// can_weight (canon.f:135-149), muca_weight / muca_weight2
// (mulcan_par_mod.f90:380-410).
double Smmp::weight(const Weight& w, double x) const {
  if (w.kind == W_CANON) return beta * x;
  double xmin = w.kmin, xmax = w.kmax;
  int k = int(std::min(xmax, std::max(xmin, x / w.ebin + fsign(0.5, x))));
  if (w.kind == W_MUCA) return (beta + w.b[k - w.kmin]) * x + w.alpha[k - w.kmin];
  return w.b[k - w.kmin] * x + w.alpha[k - w.kmin];
}

// metropolis.f:13-184 (upchswitch=0: single-dihedral pivot moves only).
void Smmp::metropolis(double& eol1, double& acz, const Weight& w) {
  if (upchswitch != 0) throw std::runtime_error("metropolis: BGS moves are outside this path");
  std::vector<double> vrol(vlvr);
  double eol = energy();
  for (int nsw = 1; nsw <= nvr; ++nsw) {
    int ivar = rndord ? 1 + int(nvr * grnd()) : nsw;
    int jv = idvr[ivar];
    vrol = vlvr;
    double dv = axvr[jv] * (grnd() - 0.5);
    vlvr[jv] = addang(vrol[jv], dv);
    double enw = energy();
    double delta = weight(w, enw) - weight(w, eol);
    int up = 0;
    if (delta <= 0.0) {
      eol = enw;
      up = 1;
    } else {
      double rd = grnd();
      delta = std::min(delta, 100.0);
      double ex = std::exp(-delta);
      if (ex >= rd) {
        eol = enw;
        up = 1;
      } else {
        vlvr = vrol;
      }
    }
    acz = acz + up * 1.0;
    ++ncalls;
    nacalls += up;
  }
  double enw = energy();
  if (std::fabs(eol - enw) > 0.000001 && eol < 100000)
    throw std::runtime_error("metropolis: eol and enw difference unacceptable");
  eol1 = eol;
}

}  // namespace oracle
