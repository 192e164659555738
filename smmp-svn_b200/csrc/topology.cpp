// Flattening of an assembled molecule into the GPU topology (see topology.hpp).
#include "topology.hpp"

#include <algorithm>
#include <cstdio>
#include <string>
#include <cmath>
#include <stdexcept>

namespace smmpb200 {

namespace {
[[noreturn]] void fail(const std::string& m) { throw std::runtime_error(m); }
// Squared distance below which a term of the pair can exceed `g` kcal/mol.
double guard_r2(double a, double c, int hb, double g) {
  double r2a = a > 0 ? std::pow(a / g, 1.0 / 6.0) : 0.0;   // A/r^12 > g
  double r2c = 0.0;
  if (c > 0) r2c = hb ? std::pow(c / g, 1.0 / 5.0)          // C/r^10 > g
                      : std::pow(c / g, 1.0 / 3.0);         // C/r^6  > g
  return std::max(r2a, r2c);
}
}  // namespace

ForceField make_forcefield(const Assembly& a) {
  ForceField ff;
  // Pairs whose van der Waals / H-bond terms can exceed g kcal/mol (clashes)
  // are evaluated in FP64; below it the FP32 rounding of a term (~1e-7
  // relative) stays under 1e-5 kcal/mol.
  const double g = 100.0;
  for (int i = 0; i < kNumTypes; ++i)
    for (int j = 0; j < kNumTypes; ++j) {
      int k = i * kNumTypes + j;
      int hb = a.ihbty[i + 1][j + 1] != 0;
      ff.pair.hb[k] = hb;
      ff.pair.a[k] = hb ? a.ahb[i + 1][j + 1] : a.aij[i + 1][j + 1];
      ff.pair.a14[k] = hb ? a.ahb[i + 1][j + 1] : a.a14[i + 1][j + 1];
      ff.pair.c[k] = hb ? a.chb[i + 1][j + 1] : a.cij[i + 1][j + 1];
      double amax = std::max(ff.pair.a[k], ff.pair.a14[k]);
      ff.pair.guard_r2[k] = guard_r2(amax, ff.pair.c[k], hb, g);
    }
  ff.conv = a.conv;
  ff.plt = a.plt;
  ff.slp = a.slp;
  ff.epsd = a.epsd ? 1 : 0;
  ff.itysol = a.itysol;
  ff.npnt = a.npnt;
  ff.spoint = a.spoint;
  return ff;
}

MolTopo flatten(Assembly& a, int nml) {
  MolTopo t;
  int ifiat = a.iatrs1[a.irsml1[nml]], ilaat = a.iatrs2[a.irsml2[nml]];
  int n = ilaat - ifiat + 1;
  if (n > kMaxAtoms) fail("flatten: molecule has more atoms than the packed pair words hold");
  t.natoms = n;
  auto A = [&](int i1based) { return i1based - ifiat; };   // 0-based atom index
  int i1, i2, i3;
  a.fnd3ba(nml, i1, i2, i3);
  t.i1 = A(i1);
  t.i2 = A(i2);
  t.i3 = A(i3);
  for (int k = 0; k < 6; ++k) t.gbpr[k] = a.gbpr[k + 1][nml];
  t.iow.resize(n);
  t.type.resize(n);
  t.charge.resize(n);
  t.blen.resize(n);
  t.cba.resize(n);
  t.sba.resize(n);
  t.toat0.resize(n);
  t.rvdw.resize(n);
  t.sigma.resize(n);
  t.atom_name.resize(n);
  t.residue_of_atom.resize(n);
  for (int i = ifiat; i <= ilaat; ++i) {
    int k = A(i);
    t.iow[k] = (i == i1) ? -1 : A(a.iowat[i]);
    t.type[k] = uint8_t(a.ityat[i] - 1);
    t.charge[k] = a.cgat[i];
    t.blen[k] = a.blat[i];
    t.cba[k] = a.csbaat[i];
    t.sba[k] = a.snbaat[i];
    t.toat0[k] = a.toat[i];
    t.rvdw[k] = a.rvdw[i];
    t.sigma[k] = a.sigma[i];
    t.atom_name[k] = a.nmat[i];
    t.residue_of_atom[k] = a.nursat(i) - a.irsml1[nml];
    if (a.rvdw[i] > 0.0) t.heavy.push_back(k);
  }
  t.nres = a.irsml2[nml] - a.irsml1[nml] + 1;
  // outpdb.f:137-176: bonded partners j > i (the first atom of the molecule
  // also lists its parent), only for atoms with bonds
  t.conect_off.assign(1, 0);
  for (int r = a.irsml1[nml]; r <= a.irsml2[nml]; ++r) {
    t.res_name.push_back(a.seq[r]);
    t.res_atom0.push_back(A(a.iatrs1[r]));
    for (int i = a.iatrs1[r]; i <= a.iatrs2[r]; ++i) {
      if (a.nbdat[i] > 0) {
        int ibd[4], jj;
        if (r == a.irsml1[nml] && i == a.iatrs1[r]) {
          ibd[0] = a.iowat[i];
          ibd[1] = a.IBD(1, i);
          ibd[2] = a.IBD(2, i);
          ibd[3] = a.IBD(3, i);
          jj = 4;
        } else {
          ibd[0] = a.IBD(1, i);
          ibd[1] = a.IBD(2, i);
          ibd[2] = a.IBD(3, i);
          jj = 3;
        }
        for (int j = 0; j < jj; ++j)
          if (ibd[j] > i) t.conect.push_back(A(ibd[j]));
      }
      t.conect_off.push_back((int)t.conect.size());
    }
  }
  // depth levels in bldmol order (every atom but i1 is built from its parent)
  std::vector<int> depth(n, -1);
  depth[t.i1] = 0;
  int maxd = 0;
  for (int res = a.irsml1[nml]; res <= a.irsml2[nml]; ++res) {
    int jj = (res == a.irsml1[nml]) ? a.iatrs1[res] + 1 : a.iatrs1[res];
    for (int j = jj; j <= a.iatrs2[res]; ++j) {
      int k = A(j), p = t.iow[k];
      if (p < 0 || p >= n || depth[p] < 0) fail("flatten: atom built before its parent");
      depth[k] = depth[p] + 1;
      maxd = std::max(maxd, depth[k]);
    }
  }
  t.level_off.assign(maxd + 2, 0);
  for (int k = 0; k < n; ++k) {
    if (depth[k] < 0) fail("flatten: atom not reached by the rebuild");
    t.level_off[depth[k] + 1]++;
  }
  for (int d = 0; d <= maxd; ++d) t.level_off[d + 1] += t.level_off[d];
  t.level_atoms.assign(n, 0);
  {
    std::vector<int> fill(t.level_off.begin(), t.level_off.end() - 1);
    for (int k = 0; k < n; ++k) t.level_atoms[fill[depth[k]]++] = k;
  }
  // variables
  int ifivr = a.ivrml1[nml], nv = a.nvrml[nml];
  t.nvar = nv;
  t.sib_off.push_back(0);
  for (int v = ifivr; v < ifivr + nv; ++v) {
    if (a.ityvr[v] != 3) fail("flatten: only torsion variables exist in the ECEPP libraries");
    int iat = a.iatvr[v], iow = a.iowat[iat];
    if (A(iow) == t.i1)
      fail("flatten: a variable turns about the first backbone atom, which has no parent bond");
    t.var_atom.push_back(A(iat));
    t.var_base.push_back(A(iow));
    for (int j = 1; j <= a.nbdat[iow]; ++j) {
      int jat = a.IBD(j, iow);
      if (a.iowat[jat] == iow) t.sib.push_back(A(jat));
    }
    t.sib_off.push_back((int)t.sib.size());
    // rotating range: union of the branches hanging from the base
    int ir = a.nursvr(v), lo = 0, hi = -1;
    for (int j = 1; j <= a.nbdat[iow]; ++j) {
      int jat = a.IBD(j, iow);
      if (a.iowat[jat] != iow) continue;
      int k, irg1, irg2;
      bool bb;
      a.fndbrn(nml, ir, jat, k, irg1, irg2, bb);
      if (bb) k = ilaat;
      if (hi < lo) {
        lo = jat;
        hi = k;
      } else {
        if (jat > hi + 1 || k < lo - 1) fail("flatten: disjoint rotating ranges");
        lo = std::min(lo, jat);
        hi = std::max(hi, k);
      }
    }
    t.var_lo.push_back(A(lo));
    t.var_hi.push_back(A(hi));
    int ic = a.iclvr[v];
    t.var_class.push_back(ic);
    t.var_e0.push_back(a.e0to[ic]);
    t.var_sg.push_back(a.sgto[ic]);
    t.var_rn.push_back(a.rnto[ic]);
    t.var_fixed.push_back(a.fxvr[v] ? 1 : 0);
    t.axvr.push_back(a.axvr[v]);
    t.vlvr0.push_back(a.vlvr[v]);
    t.var_name.push_back(a.nmvr[v]);
    t.var_residue.push_back(ir - a.irsml1[nml]);
  }
  for (int i = 1; i <= a.nvr; ++i) {
    int v = a.idvr[i];
    if (v >= ifivr && v < ifivr + nv) t.idvr.push_back(v - ifivr);
  }
  t.nfree = (int)t.idvr.size();
  // pair work from the vdW-domain and 1-4 lists
  for (int i = ifiat; i <= ilaat; ++i) {
    for (int ivw = a.ivwat1[i]; ivw <= a.ivwat2[i]; ++ivw) {
      int j1 = a.lvwat1[ivw], j2 = a.lvwat2[ivw];
      for (int j0 = j1; j0 <= j2; j0 += kChunk) {
        int len = std::min(kChunk, j2 - j0 + 1);
        t.chunks.push_back(uint32_t(A(i)) | (uint32_t(A(j0)) << 14) | (uint32_t(len - 1) << 28));
        t.npairs += len;
      }
    }
    for (int k = a.i14at1[i]; k <= a.i14at2[i]; ++k) {
      t.pairs14.push_back(uint32_t(A(i)) | (uint32_t(A(a.l14at[k])) << 14));
      t.npairs += 1;
    }
  }
  // row form of the same pair set
  t.near_mask.assign(n, 0);
  t.near14.assign(n, 0);
  bool ok = true;
  long long far = 0;
  for (uint32_t w : t.chunks) {
    int i = int(w & 0x3fffu), j0 = int((w >> 14) & 0x3fffu), len = int((w >> 28) & 7u) + 1;
    for (int j = j0; j < j0 + len; ++j) {
      int lo = std::min(i, j), d = std::abs(i - j);
      if (d == 0) fail("flatten: self pair in the lists");
      if (d <= kNearWindow) {
        uint64_t bit = 1ull << (d - 1);
        if (t.near_mask[lo] & bit) ok = false;   // listed twice
        t.near_mask[lo] |= bit;
      } else {
        ++far;
      }
    }
  }
  for (uint32_t w : t.pairs14) {
    int i = int(w & 0x3fffu), j = int(w >> 14);
    int lo = std::min(i, j), d = std::abs(i - j);
    if (d == 0) fail("flatten: self pair in the lists");
    if (d > kNearWindow) {
      ok = false;
      continue;
    }
    uint64_t bit = 1ull << (d - 1);
    if ((t.near14[lo] | t.near_mask[lo]) & bit) ok = false;
    t.near14[lo] |= bit;
  }
  // Distant pairs: the count equals that of the full triangle beyond the
  // window, and no pair is listed twice (bitmap check; larger molecules keep
  // the list form).
  long long far_all = 0;
  for (int i = 0; i < n; ++i) far_all += std::max(0, n - 1 - i - kNearWindow);
  if (ok && far == far_all && n <= 4096) {
    std::vector<bool> seen((size_t)n * n, false);
    for (uint32_t w : t.chunks) {
      int i = int(w & 0x3fffu), j0 = int((w >> 14) & 0x3fffu), len = int((w >> 28) & 7u) + 1;
      for (int j = j0; j < j0 + len; ++j) {
        if (std::abs(i - j) <= kNearWindow) continue;
        size_t key = (size_t)std::min(i, j) * n + std::max(i, j);
        if (seen[key]) ok = false;
        seen[key] = true;
      }
    }
  } else {
    ok = false;
  }
  t.rows_ok = ok;
  return t;
}

// outvar.f:50-121.  crd is the reference's literal (INCL.H:41), not 180/pi.
std::string outvar_text(const MolTopo& t, const double* vlvr, int iml) {
  const double crd = 57.2957795130823;
  char mlfd[32], line[256];
  std::snprintf(mlfd, sizeof mlfd, "%4d : ", iml);   // (i4,a3)
  std::string out;
  bool any = false;
  for (int k = 0; k < 6; ++k) any = any || t.gbpr[k] != 0.0;
  if (any) {   // '@' line of the global parameters: (1x,2a,1x,12a), f17.6 trimmed
    out += " @ ";
    out += mlfd;
    out += " ";
    for (int k = 0; k < 6; ++k) {
      std::snprintf(line, sizeof line, "%.6f", k < 3 ? t.gbpr[k] : t.gbpr[k] * crd);
      out += line;
      if (k < 5) out += ",";
    }
    out += "\n";
  }
  for (int v = 0; v < t.nvar; ++v) {   // (3x,a,i3,1x,a,1x,a,1x,a,1x,f10.3[,1x,a])
    std::string name = t.var_name[v];
    name.resize(3, ' ');   // character nmvr*3
    std::snprintf(line, sizeof line, "   %s%3d : %s : %10.3f%s\n", mlfd, t.var_residue[v] + 1,
                  name.c_str(), vlvr[v] * crd, t.var_fixed[v] ? "  &" : "");
    out += line;   // every variable of these libraries is a torsion (ityvr = 3)
  }
  return out;
}

// outpdb.f:12-185 for a system of one molecule (chain id blank, atom
// numbers from 1).  Lines are 80 characters, blank-filled, as (a80) writes
// them; the formats are outpdb.f:181-183.
std::string outpdb_text(const MolTopo& t, const double* xyz) {
  auto pad80 = [](std::string s) {
    s.resize(80, ' ');
    return s + "\n";
  };
  auto upper = [](std::string s) {
    for (char& ch : s)
      if (ch >= 'a' && ch <= 'z') ch = char(ch - 'a' + 'A');
    return s;
  };
  std::string out, res;
  char line[128];
  int iat = 0;
  for (int r = 0; r < t.nres; ++r) {
    const std::string raw = t.res_name[r].substr(0, 3);
    const char* linty = (raw != "ace" && raw != "nme") ? "ATOM  " : "HETATM";
    res = upper(raw);
    res.resize(3, ' ');
    const int a1 = t.res_atom0[r], a2 = r + 1 < t.nres ? t.res_atom0[r + 1] : t.natoms;
    for (int i = a1; i < a2; ++i) {
      ++iat;
      std::string nm = t.atom_name[i];
      nm.resize(4, ' ');
      std::string atnm = " " + nm;   // atnm(2:5) = nmat(i)
      if (atnm[1] == 'h') {           // hydrogens: a trailing digit moves to column 1
        const size_t j = atnm.find_last_not_of(' ');
        if (j != std::string::npos && atnm[j] >= '0' && atnm[j] <= '9') {
          atnm[0] = atnm[j];
          atnm[j] = ' ';
        }
      }
      atnm = upper(atnm);
      // (a6,i5,1x,a5,a3,1x,a1,i4,a1,3x,3f8.3,2(1x,f5.2))
      std::snprintf(line, sizeof line, "%s%5d %s%s  %4d    %8.3f%8.3f%8.3f %5.2f %5.2f", linty,
                    iat, atnm.c_str(), res.c_str(), r + 1, xyz[3 * i], xyz[3 * i + 1],
                    xyz[3 * i + 2], 1.0, 0.0);
      out += pad80(line);
    }
  }
  ++iat;
  std::snprintf(line, sizeof line, "TER   %5d      %s  ", iat, res.c_str());   // (a6,i5,6x,a3,1x,a1)
  out += pad80(line);
  for (int i = 0; i < t.natoms; ++i) {   // (a6,5i5)
    const int b = t.conect_off[i], e = t.conect_off[i + 1];
    if (e == b) continue;
    std::string l = "CONECT";
    std::snprintf(line, sizeof line, "%5d", i + 1);
    l += line;
    for (int k = b; k < e; ++k) {
      std::snprintf(line, sizeof line, "%5d", t.conect[k] + 1);
      l += line;
    }
    out += pad80(l);
  }
  out += pad80("END");
  return out;
}

}  // namespace smmpb200
