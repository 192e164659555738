// CPU oracle -- TEST INFRASTRUCTURE ONLY (see smmp_oracle.hpp).
//
// gradient.f:12-70 and opeshe.f:12-317: the ECEPP/3 energy of a molecule and
// its derivatives with respect to the variables, by the recursive force and
// torque sums over the moving sets (Noguti and Go 1984; Abe, Braun, Noguti
// and Go 1984), in the reference's loop order: variables in descending
// order, the atoms of each variable's moving sets, their van der Waals and
// 1-4 partners, then the sums carried over from the variables added to it.
#include <cmath>
#include <stdexcept>
#include <vector>

#include "smmp_oracle.hpp"

namespace oracle {

// opeshe.f:12-317: energy terms of molecule nml (eyel, eyvw, eyhb, eyvr,
// eysm) and gdeyvr[iv] = dE/d(variable iv) for its variables.
double Smmp::opeshe(int nml) {
  eyel = eyvw = eyhb = eyvr = eysm = 0.0;
  const int ntlvr = nvrml[nml];
  if (ntlvr == 0) return 0.0;
  const int ifivr = ivrml1[nml], ilavr = ifivr + ntlvr - 1;
  if ((int)gdeyvr.size() < ilavr + 1) gdeyvr.assign(ilavr + 1, 0.0);
  std::vector<double> xfvr(ilavr + 1, 0.0), yfvr(ilavr + 1, 0.0), zfvr(ilavr + 1, 0.0),
      xfrvr(ilavr + 1, 0.0), yfrvr(ilavr + 1, 0.0), zfrvr(ilavr + 1, 0.0);
  const int ifiat = iatrs1[irsml1[nml]], ilaat = iatrs2[irsml2[nml]];
  std::vector<double> xfat(ilaat + 1, 0.0), yfat(ilaat + 1, 0.0), zfat(ilaat + 1, 0.0);
  for (int i = ifivr; i <= ilavr; ++i) gdeyvr[i] = 0.0;
  (void)ifiat;

  int i1s = imsml1[nml] + nmsml[nml];
  int i1a = iadml1[nml] + nadml[nml];

  // one pair (i, j): energies and the force on j from i (opeshe.f:165-225)
  auto pair = [&](int i, int j, bool is14, double cqi, int ity, double xi, double yi, double zi,
                  double& xfi, double& yfi, double& zfi) {
    const int jty = ityat[j];
    const double xij = xat(j) - xi, yij = yat(j) - yi, zij = zat(j) - zi;
    const double rij2 = xij * xij + yij * yij + zij * zij;
    const double rij4 = rij2 * rij2;
    const double rij6 = rij4 * rij2;
    const double rij = std::sqrt(rij2);
    double eel, deel;
    if (epsd) {
      const double sr = slp * rij;
      const double sr2 = sr * sr;
      const double xsr = (plt - 1.0) * std::exp(-sr) / 2.0;
      const double ep = plt - (sr2 + 2.0 * sr + 2.0) * xsr;
      eel = cqi * cgat[j] / (rij * ep);
      deel = eel + cqi * cgat[j] * (slp * sr2 * xsr) / (ep * ep);
    } else {
      eel = cqi * cgat[j] / rij;
      deel = eel;
    }
    eyel = eyel + eel;
    double c;
    if (ihbty[ity][jty] != 0) {
      const double eyrp = ahb[ity][jty] / (rij6 * rij6);
      const double eyds = chb[ity][jty] / (rij6 * rij4);
      eyhb = eyhb + eyrp - eyds;
      c = (-12.0 * eyrp + 10.0 * eyds - deel) / rij2;
    } else {
      const double eyrp = (is14 ? a14[ity][jty] : aij[ity][jty]) / (rij6 * rij6);
      const double eyds = cij[ity][jty] / rij6;
      eyvw = eyvw + eyrp - eyds;
      c = (-12.0 * eyrp + 6.0 * eyds - deel) / rij2;
    }
    const double xfji = c * xij, yfji = c * yij, zfji = c * zij;
    xfi = xfi + xfji;
    yfi = yfi + yfji;
    zfi = zfi + zfji;
    xfat[j] = xfat[j] - xfji;
    yfat[j] = yfat[j] - yfji;
    zfat[j] = zfat[j] - zfji;
  };

  for (int io = ilavr; io >= ifivr; --io) {   // variables in descending order
    const int iv = iorvr[io];
    const int ia = iatvr[iv];
    const int ib = iowat[ia];
    const double xb = xat(ib), yb = yat(ib), zb = zat(ib);
    const int it = ityvr[iv], ic = iclvr[iv];
    double fvr = 0.0, ex = 0.0, ey = 0.0, ez = 0.0;
    if (it == 3) {   // torsion
      ex = xtoat[ib];
      ey = ytoat[ib];
      ez = ztoat[ib];
      const double vr = toat[ia];
      const double e0 = e0to[ic];
      if (e0 != 0.0) {
        const double vrn = vr * rnto[ic];
        eyvr = eyvr + e0 * (1.0 + sgto[ic] * std::cos(vrn));
        fvr = esnto[ic] * std::sin(vrn);   // force from the variable
      }
    } else if (it == 2) {   // bond angle
      ex = xbaat[ia];
      ey = ybaat[ia];
      ez = zbaat[ia];
    } else if (it == 1) {   // bond length
      ex = xtoat[ia];
      ey = ytoat[ia];
      ez = ztoat[ia];
    }

    double xfiv = 0.0, yfiv = 0.0, zfiv = 0.0, xfriv = 0.0, yfriv = 0.0, zfriv = 0.0;
    const int i2s = i1s - 1;   // last moving set of iv
    i1s = imsvr1[iv];          // first
    for (int ims = i1s; ims <= i2s; ++ims) {
      for (int i = latms1[ims]; i <= latms2[ims]; ++i) {
        const int ity = ityat[i];
        const double cqi = conv * cgat[i];
        const double xi = xat(i), yi = yat(i), zi = zat(i);
        double xfi = xfat[i], yfi = yfat[i], zfi = zfat[i];
        for (int ivw = ivwat1[i]; ivw <= ivwat2[i]; ++ivw)
          for (int j = lvwat1[ivw]; j <= lvwat2[ivw]; ++j)
            pair(i, j, false, cqi, ity, xi, yi, zi, xfi, yfi, zfi);
        for (int i14 = i14at1[i]; i14 <= i14at2[i]; ++i14)
          pair(i, l14at[i14], true, cqi, ity, xi, yi, zi, xfi, yfi, zfi);
        xfat[i] = xfi;
        yfat[i] = yfi;
        zfat[i] = zfi;
        xfiv = xfiv + xfi;
        yfiv = yfiv + yfi;
        zfiv = zfiv + zfi;
        xfriv = xfriv + yfi * zi - zfi * yi;
        yfriv = yfriv + zfi * xi - xfi * zi;
        zfriv = zfriv + xfi * yi - yfi * xi;
      }
    }
    const int i2a = i1a - 1;   // last variable added to iv
    i1a = iadvr1[iv];          // first
    for (int iad = i1a; iad <= i2a; ++iad) {
      const int lad = ladvr[iad];
      xfiv = xfiv + xfvr[lad];
      yfiv = yfiv + yfvr[lad];
      zfiv = zfiv + zfvr[lad];
      xfriv = xfriv + xfrvr[lad];
      yfriv = yfriv + yfrvr[lad];
      zfriv = zfriv + zfrvr[lad];
    }
    xfvr[iv] = xfiv;
    yfvr[iv] = yfiv;
    zfvr[iv] = zfiv;
    xfrvr[iv] = xfriv;
    yfrvr[iv] = yfriv;
    zfrvr[iv] = zfriv;
    if (it == 3 || it == 2)
      gdeyvr[iv] = (ey * zb - ez * yb) * xfiv + (ez * xb - ex * zb) * yfiv +
                   (ex * yb - ey * xb) * zfiv + ex * xfriv + ey * yfriv + ez * zfriv - fvr;
    else if (it == 1)
      gdeyvr[iv] = -(ex * xfiv + ey * yfiv + ez * zfiv) - fvr;
  }
  eysm = eyel + eyvw + eyhb + eyvr;
  return eysm;
}

// opesol.f:12-240: the analytic solvation energy (esolan) and its
// derivatives with respect to the variables, by the same recursion over the
// moving sets as opeshe with the atomic forces -gradan; a variable whose axis
// is the molecule's reference axis (ixrfpt(2)) takes the forces of its
// primary atom's interaction partners with the opposite sign.
void Smmp::opesol(int nml, std::vector<double>& gdeysl) {
  const int ntlvr = nvrml[nml];
  if (ntlvr == 0) return;
  const int ix2 = ixrfpt[2][nml];
  const int ifivr = ivrml1[nml], ilavr = ifivr + ntlvr - 1;
  gdeysl.assign(ilavr + 1, 0.0);
  std::vector<double> xfvr(ilavr + 1, 0.0), yfvr(ilavr + 1, 0.0), zfvr(ilavr + 1, 0.0),
      xfrvr(ilavr + 1, 0.0), yfrvr(ilavr + 1, 0.0), zfrvr(ilavr + 1, 0.0);
  // esolan(nml): energy and gradan
  int numat = iatrs2[irsml2[nml]] - iatrs1[irsml1[nml]] + 1;
  std::vector<double> gradan(3 * (numat + 1));
  eysl = esolan_areas(numat, &xat_[2], &yat_[2], &zat_[2], rvdw.data(), sigma.data(),
                      [this] { return grnd(); }, nullptr, gradan.data());
  const int ifiat = iatrs1[irsml1[nml]], ilaat = iatrs2[irsml2[nml]];
  std::vector<double> xfat(ilaat + 1), yfat(ilaat + 1), zfat(ilaat + 1), xfrat(ilaat + 1),
      yfrat(ilaat + 1), zfrat(ilaat + 1);
  for (int i = ifiat; i <= ilaat; ++i) {   // f = -sigma dA/dr, g = f x r
    const double dx = -gradan[3 * i], dy = -gradan[3 * i + 1], dz = -gradan[3 * i + 2];
    xfat[i] = dx;
    yfat[i] = dy;
    zfat[i] = dz;
    const double xi = xat(i), yi = yat(i), zi = zat(i);
    xfrat[i] = dy * zi - dz * yi;
    yfrat[i] = dz * xi - dx * zi;
    zfrat[i] = dx * yi - dy * xi;
  }
  int i1s = imsml1[nml] + nmsml[nml], i1a = iadml1[nml] + nadml[nml];
  for (int io = ilavr; io >= ifivr; --io) {
    bool lnb = false;
    const int iv = iorvr[io], it = ityvr[iv], ia = iatvr[iv], ib = iowat[ia];
    const double xb = xat(ib), yb = yat(ib), zb = zat(ib);
    double ex = 0, ey = 0, ez = 0;
    if (it == 3) {
      ex = xtoat[ib];
      ey = ytoat[ib];
      ez = ztoat[ib];
      if (ib == ix2) lnb = true;
    } else if (it == 2) {
      ex = xbaat[ia];
      ey = ybaat[ia];
      ez = zbaat[ia];
      if (ib == ix2) lnb = true;
    } else if (it == 1) {
      ex = xtoat[ia];
      ey = ytoat[ia];
      ez = ztoat[ia];
      if (ia == ix2) lnb = true;
    }
    double xfiv = 0, yfiv = 0, zfiv = 0, xfriv = 0, yfriv = 0, zfriv = 0;
    if (!lnb) {
      const int i2s = i1s - 1;
      i1s = imsvr1[iv];
      for (int ims = i1s; ims <= i2s; ++ims)
        for (int i = latms1[ims]; i <= latms2[ims]; ++i) {
          xfiv = xfiv + xfat[i];
          yfiv = yfiv + yfat[i];
          zfiv = zfiv + zfat[i];
          xfriv = xfriv + xfrat[i];
          yfriv = yfriv + yfrat[i];
          zfriv = zfriv + zfrat[i];
        }
      const int i2a = i1a - 1;
      i1a = iadvr1[iv];
      for (int iad = i1a; iad <= i2a; ++iad) {
        const int lad = ladvr[iad];
        xfiv = xfiv + xfvr[lad];
        yfiv = yfiv + yfvr[lad];
        zfiv = zfiv + zfvr[lad];
        xfriv = xfriv + xfrvr[lad];
        yfriv = yfriv + yfrvr[lad];
        zfriv = zfriv + zfrvr[lad];
      }
    } else {
      auto sub = [&](int j) {
        xfiv = xfiv - xfat[j];
        yfiv = yfiv - yfat[j];
        zfiv = zfiv - zfat[j];
        xfriv = xfriv - xfrat[j];
        yfriv = yfriv - yfrat[j];
        zfriv = zfriv - zfrat[j];
      };
      for (int ivw = ivwat1[ia]; ivw <= ivwat2[ia]; ++ivw)
        for (int j = lvwat1[ivw]; j <= lvwat2[ivw]; ++j) sub(j);
      for (int i14 = i14at1[ia]; i14 <= i14at2[ia]; ++i14) sub(l14at[i14]);
    }
    xfvr[iv] = xfiv;
    yfvr[iv] = yfiv;
    zfvr[iv] = zfiv;
    xfrvr[iv] = xfriv;
    yfrvr[iv] = yfriv;
    zfrvr[iv] = zfriv;
    if (it == 3 || it == 2)
      gdeysl[iv] = (ey * zb - ez * yb) * xfiv + (ez * xb - ex * zb) * yfiv +
                   (ex * yb - ey * xb) * zfiv + ex * xfriv + ey * yfriv + ez * zfriv;
    else if (it == 1)
      gdeysl[iv] = -(ex * xfiv + ey * yfiv + ez * zfiv);
  }
}

// gradient.f:12-70: vacuum (itysol = 0) or analytic solvation (itysol < 0,
// opesol); the reference stops for the numerical model (itysol > 0).
double Smmp::gradient() {
  if (itysol > 0) throw std::runtime_error("gradient> Set itysol < 0");
  double esm = 0.0;
  for (int i = 1; i <= ntlml; ++i) {
    setvar(i, vlvr.data());
    opeshe(i);
    esm = esm + eysm;
    if (itysol < 0) {
      std::vector<double> gs;
      opesol(i, gs);
      esm = esm + eysl;
      const int ivr1 = ivrml1[i], ivr2 = ivr1 + nvrml[i] - 1;
      for (int j = ivr1; j <= ivr2; ++j) gdeyvr[j] = gdeyvr[j] + gs[j];
    } else {
      eysl = 0.0;
    }
  }
  eysm = esm;
  return esm;
}

std::vector<std::vector<int>> Smmp::moved_atoms(int nml) {
  const int ifivr = ivrml1[nml], ilavr = ifivr + nvrml[nml] - 1;
  std::vector<std::vector<int>> moved(ilavr + 1);
  int i1s = imsml1[nml] + nmsml[nml], i1a = iadml1[nml] + nadml[nml];
  for (int io = ilavr; io >= ifivr; --io) {   // descending: added variables come first
    const int iv = iorvr[io];
    const int i2s = i1s - 1;
    i1s = imsvr1[iv];
    for (int ims = i1s; ims <= i2s; ++ims)
      for (int i = latms1[ims]; i <= latms2[ims]; ++i) moved[iv].push_back(i);
    const int i2a = i1a - 1;
    i1a = iadvr1[iv];
    for (int iad = i1a; iad <= i2a; ++iad) {
      const std::vector<int>& m = moved[ladvr[iad]];
      moved[iv].insert(moved[iv].end(), m.begin(), m.end());
    }
  }
  return moved;
}

// The same derivatives without the ordered recursion: total force on every
// atom from all of its pairs, then for each variable the force and torque
// sums over the atoms it moves (its moving sets and, recursively, those of
// the variables added to it).  This is the order-free form a parallel
// implementation computes; test infrastructure checks it against opeshe.
void Smmp::gradient_by_sums(int nml, std::vector<double>& gd) {
  setvar(nml, vlvr.data());
  const int ifivr = ivrml1[nml], ilavr = ifivr + nvrml[nml] - 1;
  const int ifiat = iatrs1[irsml1[nml]], ilaat = iatrs2[irsml2[nml]];
  std::vector<double> fx(ilaat + 1, 0.0), fy(ilaat + 1, 0.0), fz(ilaat + 1, 0.0);
  auto force = [&](int i, int j, bool is14) {
    const int ity = ityat[i], jty = ityat[j];
    const double cqi = conv * cgat[i];
    const double xij = xat(j) - xat(i), yij = yat(j) - yat(i), zij = zat(j) - zat(i);
    const double rij2 = xij * xij + yij * yij + zij * zij;
    const double rij4 = rij2 * rij2, rij6 = rij4 * rij2, rij = std::sqrt(rij2);
    double deel;
    if (epsd) {
      const double sr = slp * rij, sr2 = sr * sr;
      const double xsr = (plt - 1.0) * std::exp(-sr) / 2.0;
      const double ep = plt - (sr2 + 2.0 * sr + 2.0) * xsr;
      const double eel = cqi * cgat[j] / (rij * ep);
      deel = eel + cqi * cgat[j] * (slp * sr2 * xsr) / (ep * ep);
    } else {
      deel = cqi * cgat[j] / rij;
    }
    double c;
    if (ihbty[ity][jty] != 0)
      c = (-12.0 * ahb[ity][jty] / (rij6 * rij6) + 10.0 * chb[ity][jty] / (rij6 * rij4) - deel) /
          rij2;
    else
      c = (-12.0 * (is14 ? a14[ity][jty] : aij[ity][jty]) / (rij6 * rij6) +
           6.0 * cij[ity][jty] / rij6 - deel) /
          rij2;
    fx[i] += c * xij;
    fy[i] += c * yij;
    fz[i] += c * zij;
    fx[j] -= c * xij;
    fy[j] -= c * yij;
    fz[j] -= c * zij;
  };
  for (int i = ifiat; i <= ilaat; ++i) {
    for (int ivw = ivwat1[i]; ivw <= ivwat2[i]; ++ivw)
      for (int j = lvwat1[ivw]; j <= lvwat2[ivw]; ++j) force(i, j, false);
    for (int i14 = i14at1[i]; i14 <= i14at2[i]; ++i14) force(i, l14at[i14], true);
  }
  const std::vector<std::vector<int>> moved = moved_atoms(nml);
  gd.assign(ilavr + 1, 0.0);
  for (int io = ilavr; io >= ifivr; --io) {
    const int iv = iorvr[io];
    double sx = 0, sy = 0, sz = 0, tx = 0, ty = 0, tz = 0;
    for (int i : moved[iv]) {
      sx += fx[i];
      sy += fy[i];
      sz += fz[i];
      tx += fy[i] * zat(i) - fz[i] * yat(i);
      ty += fz[i] * xat(i) - fx[i] * zat(i);
      tz += fx[i] * yat(i) - fy[i] * xat(i);
    }
    const int ia = iatvr[iv], ib = iowat[ia], ic = iclvr[iv];
    const double ex = xtoat[ib], ey = ytoat[ib], ez = ztoat[ib];
    const double xb = xat(ib), yb = yat(ib), zb = zat(ib);
    double fvr = 0.0;
    if (e0to[ic] != 0.0) fvr = esnto[ic] * std::sin(toat[ia] * rnto[ic]);
    gd[iv] = (ey * zb - ez * yb) * sx + (ez * xb - ex * zb) * sy + (ex * yb - ey * xb) * sz +
             ex * tx + ey * ty + ez * tz - fvr;
  }
}

}  // namespace oracle
