// Host-side molecule assembly (product): builds the static topology the GPU
// kernels read (atoms, internal coordinates, variables, moving sets and
// interaction lists) from a residue library, a sequence file and a .var file.
// Restates init_energy.f, redseq.f, getmol.f, addend.f, setmvs.f, mklist.f,
// redvar.f, init_molecule.f and nursvr.f of SMMP trunk.
#include "assembly.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>

namespace smmpb200 {

namespace {
constexpr double pi = 3.141592653589793;
constexpr double pi2 = 2.0 * pi;
constexpr double cdr = 1.745329251994330e-2;   // INCL.H:45

[[noreturn]] void fail(const std::string& m) { throw std::runtime_error(m); }

std::string lower(std::string s) {   // redstr.f tolost
  for (auto& c : s)
    if (c >= 'A' && c <= 'Z') c = char(c - 'A' + 'a');
  return s;
}
std::string pad(const std::string& s, size_t n) {
  std::string r = s.substr(0, std::min(n, s.size()));
  r.resize(n, ' ');
  return r;
}
// Fortran 1-based substring s(a:b) of a blank-padded line.
std::string sub(const std::string& s, int a, int b) {
  if (b < a) return std::string();
  std::string r;
  for (int i = a; i <= b; ++i) r += (i - 1 < (int)s.size()) ? s[i - 1] : ' ';
  return r;
}
int ibegst(const std::string& s) {
  for (size_t i = 0; i < s.size(); ++i)
    if (s[i] != ' ') return int(i) + 1;
  return 0;
}
int iendst(const std::string& s) {
  for (int i = int(s.size()); i >= 1; --i)
    if (s[i - 1] != ' ') return i;
  return 0;
}
int index1(const std::string& s, char c) {   // Fortran INDEX, 1-based, 0 if absent
  auto p = s.find(c);
  return p == std::string::npos ? 0 : int(p) + 1;
}
// Formatted numeric field reader (Fortran Iw / Dw.d input with BLANK='NULL').
long read_int_field(const std::string& f) {
  std::string t;
  for (char c : f)
    if (c != ' ') t += c;
  if (t.empty()) return 0;
  char* e = nullptr;
  long v = std::strtol(t.c_str(), &e, 10);
  if (*e) fail("bad integer field >" + f + "<");
  return v;
}
double read_real_field(const std::string& f, int d) {
  std::string t;
  for (char c : f)
    if (c != ' ') t += c;
  if (t.empty()) return 0.0;
  char* e = nullptr;
  double v = std::strtod(t.c_str(), &e);
  if (*e) fail("bad real field >" + f + "<");
  if (t.find('.') == std::string::npos) v /= std::pow(10.0, d);
  return v;
}
double fsign(double a, double b) { return b >= 0 ? std::fabs(a) : -std::fabs(a); }

// extstr (redstr.f): extract next substring of str(ib:ie) up to separator spr.
void extstr(char spr, int& ib, int ie, const std::string& str, std::string& strn, int& l,
            int ln = 132) {
  l = 0;
  strn.assign(ln, ' ');
  std::string seg = sub(str, ib, ie);
  int is = index1(seg, spr);
  if (is < 1) {
    l = ie - ib + 1;
    if (l > 0) strn.replace(0, l, seg);
    ib = ie + 1;
  } else if (is == 1) {
    ib = ib + 1;
    return;
  } else {
    l = is - 1;
    strn.replace(0, l, seg.substr(0, l));
    ib = ib + is;
  }
  int i = ibegst(strn);
  if (i < 1) {
    l = 0;
    strn.assign(ln, ' ');
  } else if (i > 1) {
    int j = iendst(strn);
    l = j - i + 1;
    std::string t = strn.substr(i - 1, l);
    strn.assign(ln, ' ');
    strn.replace(0, l, t);
  } else {
    l = iendst(strn);
  }
}
// iredin (redstr.f): read a non-negative integer made of digits only.
int iredin(const std::string& line, int& in) {
  int ib = ibegst(line);
  if (ib <= 0) return 0;
  int ie = iendst(line);
  if (ie - ib >= 9) return 0;
  for (int i = ib; i <= ie; ++i)
    if (line[i - 1] < '0' || line[i - 1] > '9') return 0;
  in = std::atoi(line.substr(ib - 1, ie - ib + 1).c_str());
  return 1;
}
// iredrl (redstr.f): read a real of at most 17 characters / 6 decimals.
int iredrl(const std::string& line, double& r) {
  int ib = ibegst(line);
  if (ib <= 0) return 0;
  int ie = iendst(line);
  std::string f = line.substr(ib - 1, ie - ib + 1);
  if (f.find(',') != std::string::npos) return 0;
  int il = ie - ib + 1;
  int ip = index1(line, '.');
  if (ip > 0) {
    int ibp = ip - ib;
    if (!(il <= 17 && ibp < 11 && ie - ip <= 6)) return 0;
  } else {
    if (!(il < 11)) return 0;
  }
  char* e = nullptr;
  r = std::strtod(f.c_str(), &e);
  if (*e) return 0;
  return 1;
}

// ----------------------------------------------------------------------------
// ECEPP/3 parameter tables (init_energy.f BLOCK DATA :315-610).  Values given
// in the reference as default-REAL literals are widened from float, as the
// Fortran DATA statements do.
const float atpl_s[18] = {42., 42., 42., 42., 42., 42., 93., 151., 115., 59., 84., 59.,
                          93., 93., 93., 220., 42., 93.};
const float efel_s[18] = {85., 85., 85., 85., 85., 85., 520., 520., 520., 700., 700., 700.,
                          610., 610., 610., 1480., 85., 520.};
const float rmin_s[18] = {292., 293., 268., 268., 283., 293., 412., 374., 370., 324., 312.,
                          324., 351., 351., 351., 415., 248., 412.};
const bool do_s[18] = {0, 0, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
const bool ac_s[18] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 0, 0, 0};
// chb_s / ahb_s (mxhbdo=4, mxhbac=6), column-major as in the DATA statement.
const float chb_s[24] = {2624., 2624., 4610., 0., 4014., 4014., 5783., 0.,
                         2624., 2624., 4610., 0., 8244., 8244., 8244., 0.,
                         8244., 8244., 8244., 0., 8244., 8244., 8244., 0.};
const float ahb_s[24] = {5890., 5890., 11220., 0., 12040., 12040., 16583., 0.,
                         5890., 5890., 11220., 0., 32897., 32897., 32897., 0.,
                         32897., 32897., 32897., 0., 32897., 32897., 32897., 0.};
const float e0to_s[19] = {20., 0., 0., 2.7f, .6f, 1.8f, 1.8f, 0., 0., 0., 0., 0., 2., 1.5f,
                          3.5f, 8., 18., 20., 15.};
const float sgto_s[19] = {-1., 0., 0., 1., 1., 1., 1., 0., 0., 0., 0., 0., 1., 1., -1.,
                          -1., -1., -1., -1.};
const float rnto_s[19] = {2., 0., 0., 3., 3., 3., 3., 0., 0., 0., 0., 0., 3., 3., 2.,
                          2., 2., 2., 2.};
// Diagonal overrides of setpar (init_energy.f:204-239).
const double cdiag[18] = {45.5, 45.5, 45.5, 45.5, 45.5, 45.5, 370.5, 766.6, 509.5, 217.2,
                          369.0, 217.2, 401.3, 401.3, 401.3, 2274.4, 45.5, 370.5};
const double adiag[18] = {14090.0, 14380.0, 8420.0, 8420.0, 11680.0, 14380.0, 906100.0,
                          1049000.0, 653600.0, 125600.0, 170200.0, 125600.0, 375200.0,
                          375200.0, 375200.0, 5809000.0, 5340.0, 909000.0};
// Solvation coefficients / radii per (solvent model 1..9, atom type 1..18)
// (init_energy.f:582-608), stored [type][model].
const float coef_tab[18][9] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0.008f, 0.216f, 0.012f, 0.018f, 0.013f, 0.004f, 0.0325f, 0.016f, 1.000f},
    {0.427f, -0.732f, 0.012f, 0.018f, 0.013f, 0.004f, 0.0325f, 0.016f, 1.000f},
    {-.008f, -0.678f, 0.012f, 0.018f, 0.013f, 0.004f, 0.0325f, 0.016f, 1.000f},
    {-.172f, -0.910f, -0.116f, -0.009f, -0.007f, -0.113f, -0.0175f, -0.006f, 0.000f},
    {-.038f, -0.262f, -0.116f, -0.009f, -0.007f, -0.113f, -0.0175f, -0.006f, 0.000f},
    {-.038f, -0.910f, -0.175f, -0.037f, -0.112f, -0.166f, -0.2800f, -0.024f, 0.000f},
    {-.132f, -0.312f, -0.186f, -0.038f, -0.087f, -0.169f, -0.2175f, -0.05f, 0.000f},
    {-.132f, -0.312f, -0.116f, -0.009f, -0.007f, -0.113f, -0.0175f, -0.006f, 0.000f},
    {-.132f, -0.312f, -0.116f, -0.009f, -0.007f, -0.113f, -0.0175f, -0.006f, 0.000f},
    {-.021f, -0.281f, -0.018f, 0.005f, -.0036f, -0.017f, -0.0090f, 0.021f, 0.000f},
    {0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0.008f, 0.216f, 0.012f, 0.018f, 0.013f, 0.004f, 0.0325f, 0.016f, 1.000f}};
const float rad_tab[18][9] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0},
    {2.0f, 2.0f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 2.0f},
    {1.55f, 1.55f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.5f},
    {1.75f, 1.75f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.85f},
    {1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f},
    {1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f},
    {1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f, 1.4f},
    {1.55f, 1.55f, 1.7f, 1.7f, 1.7f, 1.7f, 1.7f, 1.7f, 1.5f},
    {1.55f, 1.55f, 1.7f, 1.7f, 1.7f, 1.7f, 1.7f, 1.7f, 1.5f},
    {1.55f, 1.55f, 1.7f, 1.7f, 1.7f, 1.7f, 1.7f, 1.7f, 1.5f},
    {2.0f, 2.0f, 1.8f, 1.8f, 1.8f, 1.8f, 1.8f, 1.8f, 1.85f},
    {0, 0, 0, 0, 0, 0, 0, 0, 0},
    {2.0f, 2.0f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 2.0f}};
constexpr double ehm = 362.55;          // init_energy.f:380
constexpr double rwater = (double)1.4f; // INCL.H:70 (REAL literal in a DOUBLE parameter)
}  // namespace

Assembly::Assembly() {
  auto I = [](std::vector<int>& v, int n, int val = 0) { v.assign(n + 2, val); };
  auto D = [](std::vector<double>& v, int n) { v.assign(n + 2, 0.0); };
  I(iatrs1, MXRS); I(iatrs2, MXRS); I(ixatrs, MXRS); I(ivrrs1, MXRS); I(nvrrs, MXRS);
  seq.assign(MXRS + 2, "    ");
  I(ityat, MXAT); I(iowat, MXAT); I(iyowat, MXAT); I(nbdat, MXAT); I(ixmsat, MXAT);
  ibdat.assign((MXAT + 2) * 4, 0); iybdat.assign((MXAT + 2) * 4, 1);
  D(cgat, MXAT); D(xbaat, MXAT); D(ybaat, MXAT); D(zbaat, MXAT); D(baat, MXAT);
  D(snbaat, MXAT); D(csbaat, MXAT); D(xtoat, MXAT); D(ytoat, MXAT); D(ztoat, MXAT);
  D(toat, MXAT); D(sntoat, MXAT); D(cstoat, MXAT); D(blat, MXAT);
  xat_.assign(MXAT + 4, 0.0); yat_.assign(MXAT + 4, 0.0); zat_.assign(MXAT + 4, 0.0);
  nmat.assign(MXAT + 2, "    ");
  D(rvdw, MXAT); D(sigma, MXAT);
  D(olvlvr, MXVR); D(vlvr, MXVR); D(axvr, MXVR);
  I(iatvr, MXVR); I(ityvr, MXVR); I(iclvr, MXVR); I(iorvr, MXVR); I(imsvr1, MXVR);
  I(imsvr2, MXVR); I(latms1, MXMS); I(latms2, MXMS); I(iadvr1, MXVR); I(iadvr2, MXVR);
  I(ladvr, MXVR); I(idvr, MXVR);
  nmvr.assign(MXVR + 2, "   ");
  fxvr.assign(MXVR + 2, 0);
  I(ivwat1, MXAT); I(ivwat2, MXAT); I(i14at1, MXAT); I(i14at2, MXAT);
  I(lvwat1, MXVW); I(lvwat2, MXVW); I(ixatvw, MXVW); I(l14at, MX14); I(ixat14, MX14);
  D(surfres, MXRS);
  std::memset(gbpr, 0, sizeof gbpr);
  std::memset(irsml1, 0, sizeof irsml1);
  std::memset(irsml2, 0, sizeof irsml2);
  std::memset(nvrml, 0, sizeof nvrml);
  std::memset(ivrml1, 0, sizeof ivrml1);
}

// init_energy.f:14-103 (ECEPP branch; FLEX and Lund are outside this path).
void Assembly::init_energy(const std::string& libdir) {
  if (ientyp != 0) fail("init_energy: only ientyp=0 (ECEPP) is on this path");
  flex = false;
  std::string reslib = libdir + (sh2 ? "lib.sh2" : "lib.sh3");
  std::ifstream f(reslib);
  if (!f) fail("init_energy: cannot open residue library " + reslib);
  lib.lines.clear();
  std::string l;
  while (std::getline(f, l)) {
    if (!l.empty() && l.back() == '\r') l.pop_back();
    lib.lines.push_back(l);
  }
  setpar();
  int its = std::abs(itysol);
  if (its > 0 && its <= MXTYSOL) {
    tessel(libdir + "tes.dat");
  } else if (itysol != 0) {
    fail("init_energy: undefined solvent type");
  }
}

// setpar, ECEPP branch (init_energy.f:106-313).
void Assembly::setpar() {
  double atpl[19], efel[19], rmin[19];
  bool dof[19], acf[19];
  conv = 332.0 / 2.0;   // conv=conv/eps_s (:164), conv=332, eps_s=2
  plt = 78.0;
  slp = 0.3;
  for (int i = 1; i <= MXTYAT; ++i) {
    atpl[i] = (double)atpl_s[i - 1] / 100;
    efel[i] = (double)efel_s[i - 1] / 100;
    rmin[i] = (double)rmin_s[i - 1] / 100;
  }
  for (int i = 1; i <= MXTYAT; ++i) {
    double ri = rmin[i], ai = atpl[i];
    double aei = std::sqrt(ai / efel[i]);
    double aic = ai * ehm;
    cij[i][i] = aic * ai / (aei + aei);
    double ri2 = ri * ri, ri6 = ri2 * ri2 * ri2;
    double a = .5 * cij[i][i] * ri6;
    aij[i][i] = a;
    a14[i][i] = .5 * a;
    for (int j = i + 1; j <= MXTYAT; ++j) {
      double aj = atpl[j];
      double c = aic * aj / (aei + std::sqrt(aj / efel[j]));
      cij[i][j] = c;
      cij[j][i] = c;
      double rij = .5 * (ri + rmin[j]);
      double r2 = rij * rij, r6 = r2 * r2 * r2;
      a = .5 * c * r6;
      aij[i][j] = a;
      aij[j][i] = a;
      a = .5 * a;
      a14[i][j] = a;
      a14[j][i] = a;
    }
    dof[i] = do_s[i - 1];
    acf[i] = ac_s[i - 1];
  }
  for (int i = 1; i <= MXTYAT; ++i) {
    cij[i][i] = cdiag[i - 1];
    aij[i][i] = adiag[i - 1];
  }
  for (int i = 1; i <= MXTYAT; ++i) a14[i][i] = .5 * aij[i][i];
  auto hbc = [](int d, int a) { return (double)chb_s[(a - 1) * 4 + (d - 1)]; };
  auto hba = [](int d, int a) { return (double)ahb_s[(a - 1) * 4 + (d - 1)]; };
  for (int i = 1; i <= MXTYTO; ++i) {
    e0to[i] = (double)e0to_s[i - 1] / 2.;
    sgto[i] = sgto_s[i - 1];
    rnto[i] = rnto_s[i - 1];
  }
  for (int i = 1; i <= MXTYAT; ++i)
    for (int j = 1; j <= MXTYAT; ++j) {
      ihbty[i][j] = 0;
      chb[i][j] = 0.;
      ahb[i][j] = 0.;
    }
  int iac = 0, ido = 0;
  for (int i = 1; i <= MXTYAT; ++i) {
    if (dof[i]) {
      ++ido;
      int jac = 0;
      for (int j = 1; j <= i - 1; ++j)
        if (acf[j]) {
          ++jac;
          ihbty[i][j] = 1;
          ihbty[j][i] = -1;
          chb[i][j] = chb[j][i] = hbc(ido, jac);
          ahb[i][j] = ahb[j][i] = hba(ido, jac);
        }
    } else if (acf[i]) {
      ++iac;
      int jdo = 0;
      for (int j = 1; j <= i - 1; ++j)
        if (dof[j]) {
          ++jdo;
          ihbty[i][j] = -1;
          ihbty[j][i] = 1;
          chb[i][j] = chb[j][i] = hbc(jdo, iac);
          ahb[i][j] = ahb[j][i] = hba(jdo, iac);
        }
    }
  }
  for (int i = 1; i <= MXTYTO; ++i) esnto[i] = e0to[i] * sgto[i] * rnto[i];
  for (int t = 1; t <= MXTYAT; ++t)
    for (int s = 1; s <= MXTYSOL; ++s) {
      coef_sl[s][t] = (double)coef_tab[t - 1][s - 1];
      rad_vdw[s][t] = (double)rad_tab[t - 1][s - 1];
    }
}

// tessel (enysol.f:341-365): unit-sphere points of the SASA test.
void Assembly::tessel(const std::string& path) {
  std::ifstream f(path);
  if (!f) fail("Cannot open the file with surface points " + path);
  std::string lin;
  std::getline(f, lin);
  while (!lin.empty() && lin[0] == '!') std::getline(f, lin);
  npnt = (int)read_int_field(sub(lin, 1, 5));
  if (npnt <= 0 || npnt > MXPOINT) fail("tessel: bad number of points");
  spoint.assign(3 * npnt, 0.0);
  for (int i = 1; i <= npnt; ++i) {
    std::getline(f, lin);
    for (int k = 0; k < 3; ++k)
      spoint[(i - 1) * 3 + k] = read_real_field(sub(lin, 1 + 20 * k, 20 + 20 * k), 10);
  }
}

// redseq.f:13-214.
void Assembly::redseq(const std::string& seqfile) {
  std::ifstream f(seqfile);
  if (!f) fail("redseq> ERROR opening sequence file: " + seqfile);
  int nrs = ntlml > 0 ? irsml2[ntlml] : 0;
  std::string line;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    int lg = iendst(line);
    if (lg <= 0) continue;
    int ic = index1(sub(line, 1, lg), '#');
    if (ic > 0) {
      if (ntlml > 0) {
        irsml2[ntlml] = nrs;
        if (nrs - irsml1[ntlml] + 1 == 0) --ntlml;
      }
      ++ntlml;
      if (ntlml > MXML) fail("redseq> NUMBER of molecules too large");
      irsml1[ntlml] = nrs + 1;
      std::string hl = sub(line, ic + 1, lg);
      int i1 = ibegst(hl);
      if (i1 > 0)
        nmml[ntlml] = hl.substr(i1 - 1, iendst(hl) - i1 + 1);
      else {
        char b[8];
        std::snprintf(b, sizeof b, "%4d", ntlml);
        nmml[ntlml] = b;
      }
    } else {
      if (ntlml == 0) {
        ntlml = 1;
        nmml[1] = "   1";
        irsml1[1] = nrs + 1;
      }
      size_t p = 0;
      while (p < line.size()) {
        while (p < line.size() && line[p] == ' ') ++p;
        if (p >= line.size()) break;
        size_t q = p;
        while (q < line.size() && line[q] != ' ') ++q;
        std::string name = line.substr(p, q - p);
        if (name.size() > 4) fail("redseq> INVALID residue NAME >" + name + "<");
        ++nrs;
        if (nrs > MXRS) fail("redseq> NUMBER of residues too large");
        seq[nrs] = pad(name, 4);
        p = q;
      }
    }
  }
  if (nrs == 0) fail("redseq> no residues found");
  for (int i = 1; i <= ntlml; ++i) {
    int ifirs = irsml1[i];
    if (!flex) {
      std::string res = lower(seq[ifirs]);
      if (res.substr(0, 3) == "pro") seq[irsml1[i]] = "pron";
    }
    if (i == ntlml) {
      if (nrs - ifirs + 1 == 0) {
        --ntlml;
        if (ntlml == 0) fail("redseq> no residues found");
        return;
      }
      irsml2[i] = nrs;
    }
  }
}

// redres (getmol.f:253-460): read the atoms and variables of one residue.
void Assembly::redres(const std::string& res, int& nat, int& nxt, int& nvrr) {
  std::string resl = lower(pad(res, 4));
  size_t ln = 0;
  for (; ln < lib.lines.size(); ++ln) {
    const std::string& line = lib.lines[ln];
    if (iendst(line) >= 13 && line[0] == '#' && sub(line, 2, 5) == resl) break;
  }
  if (ln >= lib.lines.size()) fail("redres> residue >" + resl + "< NOT FOUND");
  const std::string& hdr = lib.lines[ln];
  nat = (int)read_int_field(sub(hdr, 6, 9));
  nxt = (int)read_int_field(sub(hdr, 10, 13));
  if (nat > MXATH) fail("redres> number of atoms > mxath");
  nvrr = 0;
  for (int i = 1; i <= nat; ++i) {
    if (ln + i >= lib.lines.size()) fail("redres> ERROR reading library");
    const std::string& a = lib.lines[ln + i];
    nmath[i] = sub(a, 1, 4);
    int icl[4];
    char fix[4];
    std::string nm[4];
    double val[4];
    for (int j = 1; j <= 3; ++j) {
      int b = 4 + (j - 1) * 16;   // 0-based column of the 1x blank
      icl[j] = (int)read_int_field(sub(a, b + 2, b + 3));
      fix[j] = sub(a, b + 4, b + 4)[0];
      nm[j] = sub(a, b + 5, b + 7);
      val[j] = read_real_field(sub(a, b + 8, b + 16), 3);
    }
    blath[i] = val[1];
    double ba = val[2], to = val[3];
    cgath[i] = read_real_field(sub(a, 53, 59), 4);
    int ity = (int)read_int_field(sub(a, 60, 63));
    int iow = (int)read_int_field(sub(a, 64, 67));
    int ibd[4];
    for (int j = 1; j <= 3; ++j) ibd[j] = (int)read_int_field(sub(a, 64 + 4 * j, 67 + 4 * j));
    if (ity <= 0 || ity > MXTYAT) fail("redres> unknown type");
    ityath[i] = ity;
    int jow = std::abs(iow);
    int iexcp = (lower(res).substr(0, 3) == "ace" && i == 1) ? 1 : 0;
    if (iexcp == 0 && i <= jow) fail("redres> atom order error in " + resl);
    iowath[i] = jow;
    iyowath[i] = iow >= 0 ? 1 : -1;
    int ib1 = std::abs(ibd[1]), ib2 = std::abs(ibd[2]), ib3 = std::abs(ibd[3]);
    auto bad = [&]() { fail("redres> Incorrect order of bonds for atom " + nmath[i] + " of " + resl); };
    if (ib1 == i || ib2 == i || ib3 == i) bad();
    if (ib1 == 0) {
      if (ib2 != 0 || ib3 != 0) bad();
      nbdath[i] = 0;
    } else {
      if (ib1 == jow) bad();
      if (ib2 == 0) {
        if (ib3 != 0) bad();
        nbdath[i] = 1;
      } else {
        if (ib2 == jow || ib2 == ib1 || (ib2 > i && ib2 < ib1)) bad();
        if (ib3 == 0) {
          nbdath[i] = 2;
        } else {
          if (ib3 == jow || ib3 == ib1 || ib3 == ib2 || (ib3 > i && (ib3 < ib1 || ib3 < ib2)))
            bad();
          nbdath[i] = 3;
        }
      }
    }
    for (int j = 1; j <= MXBD; ++j) {
      ibdath[j][i] = std::abs(ibd[j]);
      iybdath[j][i] = ibd[j] >= 0 ? 1 : -1;
    }
    baath[i] = ba * cdr;
    toath[i] = to * cdr;
    for (int j = 1; j <= 3; ++j) {
      if (fix[j] != ' ') {
        ++nvrr;
        if (nvrr > MXATH) fail("redres> number of variables > mxvrh");
        int ic = icl[j];
        if (ic <= 0 || (j == 3 && ic > MXTYTO) || (j == 2 && ic > 0) || (j == 1 && ic > 0))
          fail("redres> unknown class");
        ityvrh[nvrr] = j;
        iclvrh[nvrr] = ic;
        iatvrh[nvrr] = i;
        nmvrh[nvrr] = nm[j];
      }
    }
  }
}

// getmol (getmol.f:14-250): assemble molecule nml from the library.
void Assembly::getmol(int nml) {
  int ntlat, ntlvr;
  if (nml == 1) {
    ntlat = 0;
    ntlvr = 0;
  } else {
    int i = irsml2[nml - 1];
    ntlat = iatrs2[i];
    ntlvr = ivrrs1[i] + nvrrs[i] - 1;
  }
  ivrml1[nml] = ntlvr + 1;
  int ilars = irsml2[nml], ifirs = irsml1[nml];
  for (int nrs = ifirs; nrs <= ilars; ++nrs) {
    std::string res = lower(seq[nrs]);
    if (res.substr(0, 3) == "nme" && nrs != ilars) fail("getmol> nme allowed at C-terminus only");
    if (res.substr(0, 3) == "ace" && nrs != ifirs) fail("getmol> ace allowed at N-terminus only");
    int nat, nxt, nvrl;
    redres(res, nat, nxt, nvrl);
    if (nat + ntlat > MXAT) fail("getmol> number of atoms > mxat");
    if (nvrl + ntlvr > MXVR) fail("getmol> number of variables > mxvr");
    for (int i = 1; i <= nat; ++i) {
      int n = i + ntlat;
      nmat[n] = nmath[i];
      ityat[n] = ityath[i];
      cgat[n] = cgath[i];
      blat[n] = blath[i];
      double ba = baath[i];
      baat[n] = ba;
      csbaat[n] = std::cos(ba);
      snbaat[n] = std::sin(ba);
      double to = toath[i];
      toat[n] = to;
      cstoat[n] = std::cos(to);
      sntoat[n] = std::sin(to);
      int iow = iowath[i];
      if (iow == 0) {
        if (nrs == ifirs) {
          iowat[n] = ibdath[1][i] + ntlat;
          iyowat[n] = iybdath[1][i];
          for (int j = 1; j <= MXBD - 1; ++j) {
            ibdath[j][i] = ibdath[j + 1][i];
            iybdath[j][i] = iybdath[j + 1][i];
          }
          ibdath[MXBD][i] = 0;
          iybdath[MXBD][i] = 1;
          nbdath[i] = nbdath[i] - 1;
        } else {
          int nh = ixatrs[nrs - 1];
          iowat[n] = nh;
          iyowat[n] = 1;
          int nbd = nbdat[nh];
          if (nbd == MXBD) fail("getmol> too many bonds to connect residues");
          for (int j = 1; j <= nbd; ++j) {
            int nj = IBD(j, nh);
            double t = toat[nj];
            if (t == 0.0) fail("getmol> DIHEDRAL should be PHASE angle");
            t = t + to;
            if (std::fabs(t) > pi) t = t - fsign(pi2, t);
            toat[nj] = t;
            cstoat[nj] = std::cos(t);
            sntoat[nj] = std::sin(t);
          }
          int nbd1 = nbd + 1;
          IBD(nbd1, nh) = n;
          IYBD(nbd1, nh) = 1;
          nbdat[nh] = nbd1;
        }
      } else {
        iowat[n] = ntlat + iow;
        iyowat[n] = iyowath[i];
      }
      nbdat[n] = nbdath[i];
      for (int j = 1; j <= MXBD; ++j) {
        int ibd = ibdath[j][i];
        if (ibd != 0) {
          IBD(j, n) = ibd + ntlat;
          IYBD(j, n) = iybdath[j][i];
        } else {
          IBD(j, n) = 0;
          IYBD(j, n) = 1;
        }
      }
    }
    ivrrs1[nrs] = ntlvr + 1;
    int mvr = 0;
    for (int i = 1; i <= nvrl; ++i) {
      if (nrs == ifirs) {
        int iat = iatvrh[i];
        if (iat == 1 || (iowath[iat] == 1 && ityvrh[i] == 3)) continue;
      }
      ++mvr;
      ++ntlvr;
      ityvr[ntlvr] = ityvrh[i];
      iclvr[ntlvr] = iclvrh[i];
      iatvr[ntlvr] = iatvrh[i] + ntlat;
      nmvr[ntlvr] = nmvrh[i];
    }
    nvrrs[nrs] = mvr;
    iatrs1[nrs] = ntlat + 1;
    ixatrs[nrs] = ntlat + nxt;
    ntlat = ntlat + nat;
    iatrs2[nrs] = ntlat;
  }
  nvrml[nml] = (nml == 1) ? ntlvr : ntlvr - ivrml1[nml] + 1;
}

// addend (addend.f:13-159): put the requested end groups on molecule nml.
void Assembly::addend(int nml, const std::string& grpn, const std::string& grpc) {
  std::string grn = lower(pad(grpn, 4)), grc = lower(pad(grpc, 4));
  auto h3 = [](const std::string& s) { return s.substr(0, 3); };
  if (h3(grn) == "ace" || h3(grc) == "ace" || h3(grn) == "nme" || h3(grc) == "nme")
    fail("addend> ace/nme belong in the SEQUENCE file");
  int ifirs = irsml1[nml];
  std::string res = lower(seq[ifirs]);
  std::string sbrs;
  if (h3(res) != "ace") {
    if (h3(grn) == "nh2") {
      if (h3(res) == "hyp" && !flex) {
        if (sh2) sbrs = "nh2+";
        else fail("addend> No N-terminal Hyp possible with ECEPP/3 dataset");
      } else if (h3(res) == "pro") {
        sbrs = "nh1 ";
      } else if (h3(res) == "gly" && !flex) {
        sbrs = sh2 ? "nh2 " : "nh2g";
      } else {
        sbrs = "nh2 ";
      }
    } else if (grn == "nh3+") {
      if (h3(res) == "pro" && !flex) sbrs = "nh2+";
      else if (h3(res) == "gly" && !flex) sbrs = "nh3g";
      else sbrs = "nh3+";
    } else {
      fail("addend> Can add only nh2 or nh3+ to N-terminus");
    }
    rplgrp(nml, ifirs, "n   ", sbrs);
  }
  int ilars = irsml2[nml];
  res = lower(seq[ilars]);
  if (h3(res) != "nme") {
    if (grc == "cooh") {
      sbrs = (h3(res) == "gly" && !sh2) ? "gooh" : "cooh";
    } else if (grc == "coo-") {
      sbrs = (h3(res) == "gly" && !sh2) ? "goo-" : "coo-";
    } else {
      fail("addend> Can add only cooh or coo- to C-terminus");
    }
    rplgrp(nml, ilars, "c   ", sbrs);
  }
}

// rplgrp (addend.f:161-592): replace the group rooted at atom rpat of residue
// nrs by the group rooted at rpat of library residue sbrs.
void Assembly::rplgrp(int nml, int nrs, const std::string& rpat, const std::string& sbrs) {
  int ifirs = irsml1[nml], ilars = irsml2[nml];
  int nxt = ixatrs[nrs], nfi = iatrs1[nrs], nla = iatrs2[nrs];
  int nfirp = 0;
  for (int i = nfi; i <= nla; ++i)
    if (rpat == nmat[i]) {
      nfirp = i;
      break;
    }
  if (nfirp == 0) fail("rplgrp> cannot find atom to be replaced");
  int nlarp, irng1, irng2;
  bool bb;
  fndbrn(nml, nrs, nfirp, nlarp, irng1, irng2, bb);
  if (irng1 > 0) fail("rplgrp> Cannot replace atoms inside a ring");
  bool ntbb = false;
  int ibd[MXBD + 2], iybd[MXBD + 2];
  int ibdrg = 0, iybdrg = 1, nxtbb1 = 0, nxtbb2 = 0, isgbb1 = 1;
  bool toL3 = false;
  if (bb) {
    if (!(nfirp == nxt && nrs == ilars)) {
      if (nfirp == nfi && nrs == ifirs) {
        ntbb = true;
        ibd[1] = iowat[nfirp];
        iybd[1] = iyowat[nfirp];
        for (int i = 1; i <= MXBD; ++i) {
          ibd[i + 1] = IBD(i, nfirp);
          iybd[i + 1] = IYBD(i, nfirp);
        }
        ibdrg = 0;
        iybdrg = 1;
        for (int i = 1; i <= nbdat[nfirp] + 1; ++i) {
          if (iowat[ibd[i]] != nfirp) {
            if (ibdrg != 0) fail("rplgrp> Can handle only simple ring at 1st atom");
            ibdrg = ibd[i];
            iybdrg = iybd[i];
          }
        }
        nxtbb1 = nlarp + 1;
        isgbb1 = iyowat[nxtbb1];
        bool found = false;
        if (nxtbb1 == nxt) {
          if (nrs < ilars) {
            nxtbb2 = iatrs1[nrs + 1];
            found = true;
          }
        } else {
          for (int i = nxt; i >= nxtbb1 + 1; --i)
            if (iowat[i] == nxtbb1) {
              nxtbb2 = i;
              found = true;
              break;
            }
        }
        if (!found) fail("rplgrp> necessary 2 previous atoms are not available");
        toL3 = true;
      } else {
        fail("rplgrp> Cannot replace BACKBONE atom");
      }
    }
  }
  if (!toL3) {   // label 2: previous atoms
    if (nfirp == nfi && nrs == ifirs) fail("rplgrp> 2 previous atoms are not available");
    nxtbb1 = iowat[nfirp];
    if (nxtbb1 == nfi && nrs == ifirs) fail("rplgrp> 2 previous atoms are not available");
    nxtbb2 = iowat[nxtbb1];
  }
  // label 3: data of the substituent
  int natsb, nxtsb, nvrsb;
  redres(sbrs, natsb, nxtsb, nvrsb);
  int nfisb = 0;
  for (int i = 1; i <= natsb; ++i)
    if (rpat == nmath[i]) {
      nfisb = i;
      break;
    }
  if (nfisb == 0) fail("rplgrp> Cannot find atom in substituent residue");
  int nlasb = nfisb;
  for (int i = 1; i <= nbdath[nfisb]; ++i) {
    int ib = ibdath[i][nfisb];
    if (iowath[ib] < nfisb) fail("rplgrp> Cannot replace atoms inside a ring");
    for (int j = ib; j <= natsb; ++j) {
      if (j > ib && iowath[j] < ib) break;
      for (int k = 1; k <= nbdath[j]; ++k)
        if (ibdath[k][j] < nfisb) fail("rplgrp> Cannot replace atoms inside a ring");
      nlasb = j;
    }
  }
  double x1, x2, x3, y1, y2, y3, z1, z2, z3;
  setsys(nxtbb1, nfirp, nxtbb2, x1, x2, x3, y1, y2, y3, z1, z2, z3);
  xtoat[nfirp] = x1;
  ytoat[nfirp] = x2;
  ztoat[nfirp] = x3;
  xbaat[nfirp] = z1;
  ybaat[nfirp] = z2;
  zbaat[nfirp] = z3;
  if (ntbb) {   // virtual atoms 0 and -1
    double ct = cstoat[nxtbb2], st = sntoat[nxtbb2];
    double ca = csbaat[nxtbb1], sa = snbaat[nxtbb1];
    double h2 = -sa * ct, h3 = -sa * st;
    x1 = -ca * x1 + h2 * y1 + h3 * z1;
    x2 = -ca * x2 + h2 * y2 + h3 * z2;
    x3 = -ca * x3 + h2 * y3 + h3 * z3;
    double dx = 1.0 / std::sqrt(x1 * x1 + x2 * x2 + x3 * x3);
    x1 = x1 * dx;
    x2 = x2 * dx;
    x3 = x3 * dx;
    xat(0) = xat(nfirp) + x1;
    yat(0) = yat(nfirp) + x2;
    zat(0) = zat(nfirp) + x3;
    z1 = -st * y1 + ct * z1;
    z2 = -st * y2 + ct * z2;
    z3 = -st * y3 + ct * z3;
    double dz = 1.0 / std::sqrt(z1 * z1 + z2 * z2 + z3 * z3);
    z1 = z1 * dz;
    z2 = z2 * dz;
    z3 = z3 * dz;
    ct = cstoat[nxtbb1];
    st = sntoat[nxtbb1];
    xat(-1) = xat(0) - ct * (z2 * x3 - z3 * x2) - st * z1;
    yat(-1) = yat(0) - ct * (z3 * x1 - z1 * x3) - st * z2;
    zat(-1) = zat(0) - ct * (z1 * x2 - z2 * x1) - st * z3;
  }
  // shift atom data
  int nrp = nlarp - nfirp, nsb = nlasb - nfisb, nsh;
  if (nrp != nsb) {
    nsh = nsb - nrp;
    for (int i = nfi; i <= nfirp - 1; ++i)
      for (int j = 1; j <= MXBD; ++j) {
        int ib = IBD(j, i);
        if (ib > nlarp && ib <= nla) IBD(j, i) = ib + nsh;
      }
    int ilaat = iatrs2[irsml2[ntlml]];
    int i1, i2, i3;
    if (nrp > nsb) {
      i1 = nlarp + 1;
      i2 = ilaat;
      i3 = 1;
    } else {
      if (ilaat + nsh > MXAT) fail("rplgrp> number of atoms > mxat");
      i1 = ilaat;
      i2 = nlarp + 1;
      i3 = -1;
    }
    for (int i = i1; i3 > 0 ? i <= i2 : i >= i2; i += i3) {
      int ii = i + nsh;
      nbdat[ii] = nbdat[i];
      ibd[1] = iowat[i];
      iybd[1] = iyowat[i];
      for (int j = 1; j <= MXBD; ++j) {
        ibd[j + 1] = IBD(j, i);
        iybd[j + 1] = IYBD(j, i);
      }
      for (int j = 1; j <= MXBD + 1; ++j)
        if (ibd[j] > nfirp) ibd[j] = ibd[j] + nsh;
      iowat[ii] = ibd[1];
      iyowat[ii] = iybd[1];
      for (int j = 1; j <= MXBD; ++j) {
        IBD(j, ii) = ibd[j + 1];
        IYBD(j, ii) = iybd[j + 1];
      }
      ityat[ii] = ityat[i];
      nmat[ii] = nmat[i];
      cgat[ii] = cgat[i];
      blat[ii] = blat[i];
      baat[ii] = baat[i];
      snbaat[ii] = snbaat[i];
      csbaat[ii] = csbaat[i];
      toat[ii] = toat[i];
      sntoat[ii] = sntoat[i];
      cstoat[ii] = cstoat[i];
      xat(ii) = xat(i);
      yat(ii) = yat(i);
      zat(ii) = zat(i);
      xtoat[ii] = xtoat[i];
      ytoat[ii] = ytoat[i];
      ztoat[ii] = ztoat[i];
      xbaat[ii] = xbaat[i];
      ybaat[ii] = ybaat[i];
      zbaat[ii] = zbaat[i];
    }
    for (int i = nrs + 1; i <= irsml2[ntlml]; ++i) {
      iatrs1[i] += nsh;
      iatrs2[i] += nsh;
      ixatrs[i] += nsh;
    }
    iatrs2[nrs] = nla + nsh;
    if (nxt > nlarp) ixatrs[nrs] = nxt + nsh;
  } else {
    nsh = 0;
  }
  // correct data of nfirp
  int ish = nfirp - nfisb;
  ityat[nfirp] = ityath[nfisb];
  if (!sh2) cgat[nfirp] = cgath[nfisb];
  int nb = nbdath[nfisb];
  for (int i = 1; i <= MXBD; ++i) {
    int ib = ibdath[i][nfisb];
    if (ib != 0) {
      ibd[i] = ib + ish;
      iybd[i] = iybdath[i][nfisb];
    } else {
      ibd[i] = 0;
      iybd[i] = 1;
    }
  }
  if (ntbb) {
    ibd[MXBD + 1] = 0;
    iybd[MXBD + 1] = 1;
    ibd[nb + 1] = nxtbb1 + nsh;
    iybd[nb + 1] = isgbb1;
    if (ibdrg != 0) {
      ++nb;
      if (nb > MXBD) fail("rplgrp> need more bonds than mxbd");
      ibd[nb + 1] = ibdrg + nsh;
      iybd[nb + 1] = iybdrg;
    }
    iowat[nfirp] = ibd[1];
    iyowat[nfirp] = iybd[1];
    for (int i = 1; i <= MXBD; ++i) {
      IBD(i, nfirp) = ibd[i + 1];
      IYBD(i, nfirp) = iybd[i + 1];
    }
  } else {
    for (int i = 1; i <= MXBD; ++i) {
      IBD(i, nfirp) = ibd[i];
      IYBD(i, nfirp) = iybd[i];
    }
  }
  nbdat[nfirp] = nb;
  // add data for substituent
  int ii = nfirp;
  for (int i = nfisb + 1; i <= nlasb; ++i) {
    ++ii;
    nbdat[ii] = nbdath[i];
    int iow = iowath[i] + ish;
    iowat[ii] = iow;
    iyowat[ii] = iyowath[i];
    for (int j = 1; j <= MXBD; ++j) {
      int ib = ibdath[j][i];
      IBD(j, ii) = ib >= nfisb ? ib + ish : ib;
      IYBD(j, ii) = iybdath[j][i];
    }
    ityat[ii] = ityath[i];
    nmat[ii] = nmath[i];
    cgat[ii] = cgath[i];
    blat[ii] = blath[i];
    double ba = baath[i];
    baat[ii] = ba;
    csbaat[ii] = std::cos(ba);
    snbaat[ii] = std::sin(ba);
    double to = toath[i];
    toat[ii] = to;
    cstoat[ii] = std::cos(to);
    sntoat[ii] = std::sin(to);
    eyring(ii, iow);
    if (ntbb) {
      if (iow == nfirp) {
        ba = valang(0, nfirp, ii);
        baat[ii] = ba;
        csbaat[ii] = std::cos(ba);
        snbaat[ii] = std::sin(ba);
        to = dihedr(-1, 0, nfirp, ii);
        toat[ii] = to;
        cstoat[ii] = std::cos(to);
        sntoat[ii] = std::sin(to);
      } else if (iowat[iow] == nfirp) {
        to = dihedr(0, nfirp, iow, ii);
        toat[ii] = to;
        cstoat[ii] = std::cos(to);
        sntoat[ii] = std::sin(to);
      }
    }
  }
  // variables
  int ilavr = ivrml1[ntlml] + nvrml[ntlml] - 1;
  int ifivr = ivrrs1[nrs];
  int ivrrp = 0, lvrrp = 0;
  for (int i = ifivr; i <= ifivr + nvrrs[nrs] - 1; ++i) {
    int iat = iatvr[i];
    if (nfirp < iat && iat <= nlarp) {
      ++ivrrp;
      lvrrp = i;
    }
  }
  if (ivrrp == 0) {
    bool got = false;
    for (int i = ifivr; i <= ilavr; ++i)
      if (iatvr[i] > nlarp) {
        lvrrp = i - 1;
        got = true;
        break;
      }
    if (!got) lvrrp = ilavr;
  }
  int ivrsb = 0;
  for (int i = 1; i <= nvrsb; ++i) {
    int iat = iatvrh[i];
    if (nfisb < iat && iat <= nlasb) {
      int ity = ityvrh[i];
      if (ntbb && iowath[iat] == nfisb && ity > 2) continue;
      ++ivrsb;
      nmvrh[ivrsb] = nmvrh[i];
      ityvrh[ivrsb] = ityvrh[i];
      iclvrh[ivrsb] = iclvrh[i];
      iatvrh[ivrsb] = iat;
    }
  }
  if (nsh != 0)
    for (int i = lvrrp + 1; i <= ilavr; ++i) iatvr[i] += nsh;
  if (ivrrp != ivrsb) {
    int jsh = ivrsb - ivrrp;
    int i1, i2, i3;
    if (ivrrp > ivrsb) {
      i1 = lvrrp + 1;
      i2 = ilavr;
      i3 = 1;
    } else {
      if (ilavr + jsh > MXVR) fail("rplgrp> number of variables > mxvr");
      i1 = ilavr;
      i2 = lvrrp + 1;
      i3 = -1;
    }
    for (int i = i1; i3 > 0 ? i <= i2 : i >= i2; i += i3) {
      int k = i + jsh;
      ityvr[k] = ityvr[i];
      iclvr[k] = iclvr[i];
      nmvr[k] = nmvr[i];
      iatvr[k] = iatvr[i];
    }
    for (int i = nrs + 1; i <= irsml2[ntlml]; ++i) ivrrs1[i] += jsh;
    nvrrs[nrs] += jsh;
    nvrml[nml] += jsh;
    for (int i = nml + 1; i <= ntlml; ++i) ivrml1[i] += jsh;
  }
  ii = lvrrp - ivrrp;
  for (int i = 1; i <= ivrsb; ++i) {
    ++ii;
    nmvr[ii] = nmvrh[i];
    ityvr[ii] = ityvrh[i];
    iclvr[ii] = iclvrh[i];
    iatvr[ii] = iatvrh[i] + ish;
  }
}

// fndbrn (setmvs.f:414-492): atom range of the branch starting at ifirg.
void Assembly::fndbrn(int nml, int nrs, int ifirg, int& ilarg, int& irg1, int& irg2, bool& bb) {
  ilarg = ifirg;
  bb = false;
  irg1 = 0;
  int ifi = iatrs1[nrs], ila = iatrs2[nrs], ixt = ixatrs[nrs];
  if (ifirg == ifi) {
    bb = true;
    if (nrs != irsml1[nml]) {
      ilarg = ila;
    } else {
      int ibd[5] = {0, iowat[ifirg], IBD(1, ifirg), IBD(2, ifirg), IBD(3, ifirg)};
      int il = 0;
      for (int i = 1; i <= nbdat[ifirg] + 1; ++i) {
        int ib = ibd[i];
        if (ib > il && iowat[ib] == ifirg) il = ib;
      }
      if (il > 0) ilarg = il - 1;
    }
  } else {
    if (ifirg == ixt) bb = true;
    for (int i = 1; i <= nbdat[ifirg]; ++i) {
      int ib = IBD(i, ifirg);
      if (iowat[ib] == ifirg) {
        for (int j = ib; j <= ila; ++j) {
          if (j > ib && iowat[j] < ib) break;
          if (j == ixt) bb = true;
          for (int k = 1; k <= nbdat[j]; ++k) {
            int jb = IBD(k, j);
            if (jb < ifirg) {
              irg1 = j;
              irg2 = jb;
            }
          }
          ilarg = j;
        }
      } else if (ib < ifirg) {
        irg1 = ifirg;
        irg2 = ib;
      }
    }
  }
}

int Assembly::nursvr(int ivr) {   // nursvr.f:11-40
  for (int i = ntlml; i >= 1; --i) {
    int ifirs = irsml1[i];
    if (ivr >= ivrrs1[ifirs] && nvrml[i] > 0)
      for (int j = irsml2[i]; j >= ifirs; --j)
        if (ivr >= ivrrs1[j] && nvrrs[j] > 0) return j;
  }
  fail("nursvr> Cannot find variable");
}

int Assembly::nursat(int iat) {   // nursvr.f:42-76
  for (int i = 1; i <= ntlml; ++i) {
    int ifirs = irsml1[i], ilars = irsml2[i];
    if (iat >= iatrs1[ifirs] && iat <= iatrs2[ilars])
      for (int j = ifirs; j <= ilars; ++j)
        if (iat >= iatrs1[j] && iat <= iatrs2[j]) return j;
  }
  fail("nursat> Cannot find atom");
}

// setmvs (setmvs.f:13-412): variable order and non-overlapping moving sets.
void Assembly::setmvs(int nml) {
  int ntlvr = nvrml[nml];
  int nms, nad;
  if (nml == 1) {
    imsml1[1] = 1;
    nms = 0;
    iadml1[1] = 1;
    nad = 0;
  } else {
    imsml1[nml] = imsml1[nml - 1] + nmsml[nml - 1];
    nms = imsml1[nml] - 1;
    iadml1[nml] = iadml1[nml - 1] + nadml[nml - 1];
    nad = iadml1[nml] - 1;
  }
  if (ntlvr == 0) {
    nmsml[nml] = 0;
    nadml[nml] = 0;
    return;
  }
  int ifirs = irsml1[nml], ilars = irsml2[nml];
  int ifivr = ivrml1[nml], ilavr = ifivr + ntlvr - 1;
  int ifiat = iatrs1[ifirs], ilaat = iatrs2[ilars];
  // sort keys: primary atom *10 + (0 torsion / 1 angle / 2 length)
  for (int n = ifirs; n <= ilars; ++n) {
    int ib = ivrrs1[n];
    for (int i = ib; i <= ib + nvrrs[n] - 1; ++i) {
      int ia = iatvr[i], io = iowat[ia], it = ityvr[i];
      if (it == 3) {
        for (int j = 1; j <= nbdat[io]; ++j) {
          int ii = IBD(j, io);
          if (iowat[ii] == io) ia = std::min(ia, ii);
        }
        iadvr1[i] = ia * 10;
      } else if (it == 2) {
        iadvr1[i] = ia * 10 + 1;
      } else if (it == 1) {
        iadvr1[i] = ia * 10 + 2;
      }
      iorvr[i] = i;
    }
  }
  // heapsort of iorvr by key (setmvs.f:118-157)
  {
    int k = ilavr, l = ifivr + ntlvr / 2, ii = ifivr - 1;
    int io, n, i, j;
    for (;;) {
      if (l > ifivr) {
        --l;
        io = iorvr[l];
        n = iadvr1[io];
      } else {
        io = iorvr[k];
        n = iadvr1[io];
        iorvr[k] = iorvr[ifivr];
        --k;
        if (k == ifivr) {
          iorvr[k] = io;
          break;
        }
      }
      i = l;
      j = l + l - ii;
      while (j <= k) {
        if (j < k)
          if (iadvr1[iorvr[j]] < iadvr1[iorvr[j + 1]]) ++j;
        if (n < iadvr1[iorvr[j]]) {
          iorvr[i] = iorvr[j];
          i = j;
          j = j + j - ii;
        } else {
          j = k + 1;
        }
      }
      iorvr[i] = io;
    }
  }
  // moving sets (setmvs.f:158-280)
  nms = imsml1[nml] - 1;
  for (int io = ifivr; io <= ilavr; ++io) {
    int iv = iorvr[io];
    int ir = nursvr(iv);
    int ia = iatvr[iv];
    int ib = iowat[ia];
    int it = ityvr[iv];
    int i1 = 0, i2 = 0;
    if (it == 3) {
      i1 = 0;
      for (int i = 1; i <= nbdat[ib]; ++i) {
        int j = IBD(i, ib);
        if (iowat[j] == ib) {
          int k, irg1, irg2;
          bool bb;
          fndbrn(nml, ir, j, k, irg1, irg2, bb);
          if (bb) k = ilaat;
          if (i1 != 0) {
            if (j > i2 + 1 || k < i1 - 1) fail("setmvs> Cannot combine disjunct ranges");
            if (j < i1) i1 = j;
            if (k > i2) i2 = k;
          } else {
            i1 = j;
            i2 = k;
          }
        }
      }
    } else if (it == 2 || it == 1) {
      i1 = ia;
      int irg1, irg2;
      bool bb;
      fndbrn(nml, ir, i1, i2, irg1, irg2, bb);
      if (bb) i2 = ilaat;
    }
    if (nms + 1 > MXMS) fail("setmvs> Number of moving sets > mxms");
    imsvr1[iv] = nms + 1;
    imsvr2[iv] = nms + 1;
    for (int jo = ifivr; jo <= io - 1; ++jo) {
      int jv = iorvr[jo];
      int j1s = imsvr1[jv];
      int jns = imsvr2[jv] - j1s + 1;
      int j = j1s;
      while (j < j1s + jns) {
        int j1 = latms1[j], j2 = latms2[j];
        if (i1 <= j2 && i2 >= j1) {
          int ja = 0;
          if (i1 > j1) {
            if (i2 > j2) fail("setmvs> atom ranges overlap only PARTLY");
            ja = 1;
            latms2[j] = i1 - 1;
          }
          if (i2 < j2) {
            if (i1 < j1) fail("setmvs> atom ranges overlap only PARTLY");
            if (ja > 0) {
              ++nms;
              if (nms > MXMS) fail("setmvs> Number of moving sets > mxms");
              ++jns;
              for (int k = nms; k >= j + 2; --k) {
                latms1[k] = latms1[k - 1];
                latms2[k] = latms2[k - 1];
              }
              for (int ko = jo + 1; ko <= io; ++ko) {
                int k = iorvr[ko];
                ++imsvr1[k];
                ++imsvr2[k];
              }
              latms2[j + 1] = j2;
            }
            latms1[j + ja] = i2 + 1;
            ++ja;
          }
          if (ja == 0) {
            --nms;
            --jns;
            for (int k = j; k <= nms; ++k) {
              latms1[k] = latms1[k + 1];
              latms2[k] = latms2[k + 1];
            }
            for (int ko = jo + 1; ko <= io; ++ko) {
              int k = iorvr[ko];
              --imsvr1[k];
              --imsvr2[k];
            }
          } else {
            j += ja;
          }
        } else {
          ++j;
        }
      }
      imsvr2[jv] = j1s + jns - 1;
    }
    ++nms;
    latms1[nms] = i1;
    latms2[nms] = i2;
  }
  nmsml[nml] = nms - imsml1[nml] + 1;
  for (int ia = ifiat; ia <= ilaat; ++ia) ixmsat[ia] = 0;
  for (int is = imsml1[nml]; is <= nms; ++is)
    for (int ia = latms1[is]; ia <= latms2[is]; ++ia) ixmsat[ia] = is;
  // 'added' variables (setmvs.f:294-369)
  int i = iorvr[ifivr];
  int ii = imsvr1[i];
  for (int io = ifivr; io <= ilavr - 1; ++io) {
    int ic = i, ia = iatvr[i], ib = iowat[ia], it = ityvr[i], is = ii;
    int n = nad + 1;
    iadvr1[i] = n;
    i = iorvr[io + 1];
    ii = imsvr1[i];
    auto registered = [&](int ja) {
      for (int k = n; k <= nad; ++k)
        if (iatvr[ladvr[k]] == ja) return true;
      return false;
    };
    for (int jo = io + 1; jo <= ilavr; ++jo) {
      int j = iorvr[jo], ja = iatvr[j], jb = iowat[ja];
      if (it == 3 && jb == ib) {
        if (!registered(ja)) {
          ++nad;
          if (nad > MXVR) fail("setmvs> Number of added variables > mxvr");
          ladvr[nad] = j;
        }
      }
      if (is < ii) {
        for (int k = is; k <= ii - 1; ++k)
          if (latms1[k] <= jb && jb <= latms2[k]) {
            if (!registered(ja)) {
              ++nad;
              if (nad > MXVR) fail("setmvs> Number of added variables > mxvr");
              ladvr[nad] = j;
            }
          }
      } else {
        if (ja == ia && !registered(ja)) {
          ++nad;
          if (nad > MXVR) fail("setmvs> Number of added variables > mxvr");
          ladvr[nad] = j;
        }
      }
    }
    iadvr2[ic] = nad;
  }
  iadvr1[i] = nad + 1;
  iadvr2[i] = nad;
  nadml[nml] = nad - iadml1[nml] + 1;
}

namespace {
// quench (mklist.f:305-372): remove range [i1,i2] from the list of ranges;
// true if anything overlapped.
constexpr int MXH = 50;
bool quench(int i1, int i2, int& n, int* l1, int* l2) {
  bool q = false;
  int j = 1;
  while (j <= n) {
    int j1 = l1[j], j2 = l2[j];
    if (i1 <= j2 && i2 >= j1) {
      q = true;
      int ja = 0;
      if (i1 > j1) {
        ja = 1;
        l2[j] = i1 - 1;
      }
      if (i2 < j2) {
        if (ja > 0) {
          ++n;
          if (n > MXH) throw std::runtime_error("quench> too many sets");
          for (int k = n; k >= j + 2; --k) {
            l1[k] = l1[k - 1];
            l2[k] = l2[k - 1];
          }
          l2[j + 1] = j2;
        }
        l1[j + ja] = i2 + 1;
        ++ja;
      }
      if (ja == 0) {
        --n;
        for (int k = j; k <= n; ++k) {
          l1[k] = l1[k + 1];
          l2[k] = l2[k + 1];
        }
      } else {
        j += ja;
      }
    } else {
      ++j;
    }
  }
  return q;
}
}  // namespace

// mklist (mklist.f:12-303): vdW-domain and 1-4 interaction lists.
void Assembly::mklist(int nml) {
  constexpr int MX2 = 50;
  int l1st1[MXH + 2], l1st2[MXH + 2], l2nd1[MXH + 2], l2nd2[MXH + 2], l1i[MXBD + 2],
      l2i[MX2 + 2];
  if (nml == 1) {
    ivwml1[1] = 1;
    i14ml1[1] = 1;
  } else {
    ivwml1[nml] = ivwml1[nml - 1] + nvwml[nml - 1];
    i14ml1[nml] = i14ml1[nml - 1] + n14ml[nml - 1];
  }
  int ntlms = nmsml[nml];
  if (ntlms == 0) {
    nvwml[nml] = 0;
    n14ml[nml] = 0;
    return;
  }
  int nvw = ivwml1[nml] - 1, n14 = i14ml1[nml] - 1;
  int ifiat = iatrs1[irsml1[nml]], ilaat = iatrs2[irsml2[nml]];
  int ifivr = ivrml1[nml], ilavr = ifivr + nvrml[nml] - 1;
  for (int i = ifiat; i <= ilaat; ++i) {
    ivwat1[i] = 0;
    i14at1[i] = 0;
  }
  int n1st = 1;
  l1st1[1] = ifiat;
  l1st2[1] = ilaat;
  int i1s = imsml1[nml] + ntlms;
  auto push2 = [&](int& n2i, int v) {
    ++n2i;
    if (n2i > MX2) fail("mklist> too many atoms in list L2I");
    l2i[n2i] = v;
  };
  for (int io = ilavr; io >= ifivr; --io) {
    int iv = iorvr[io], it = ityvr[iv];
    int i2s = i1s - 1;
    i1s = imsvr1[iv];
    if (i2s - i1s + 1 <= 0) continue;
    for (int is = i1s; is <= i2s; ++is) quench(latms1[is], latms2[is], n1st, l1st1, l1st2);
    for (int i = 1; i <= n1st; ++i) {
      l2nd1[i] = l1st1[i];
      l2nd2[i] = l1st2[i];
    }
    int n2nd = n1st;
    int ib = iowat[iatvr[iv]];
    quench(ib, ib, n2nd, l2nd1, l2nd2);
    bool ovlp = false;
    int iob = iowat[ib];
    int n2i = 0;
    if (iob > 0) {
      ovlp = quench(iob, iob, n2nd, l2nd1, l2nd2);
      for (int i = 1; i <= nbdat[iob]; ++i) {
        int ibd = IBD(i, iob);
        if (ibd != ib && iowat[ibd] == iob && quench(ibd, ibd, n2nd, l2nd1, l2nd2))
          push2(n2i, ibd);
      }
      int cnt = n2i;   // Fortran DO: trip count fixed at loop entry
      for (int i = 1; i <= cnt; ++i) {
        int ia = l2i[i], im = ixmsat[ia];
        if (im > 0)
          for (int j = latms1[im]; j <= latms2[im]; ++j)
            if (ia != j && quench(j, j, n2nd, l2nd1, l2nd2)) push2(n2i, j);
      }
      int ioiob = iowat[iob];
      if (ioiob > 0) {
        if (quench(ioiob, ioiob, n2nd, l2nd1, l2nd2)) push2(n2i, ioiob);
      }
    } else {
      iob = -10;
    }
    int n1i = 0;
    for (int i = 1; i <= nbdat[ib]; ++i) {
      int ibd = IBD(i, ib);
      if (iowat[ibd] == ib && quench(ibd, ibd, n2nd, l2nd1, l2nd2)) {
        ++n1i;
        if (n1i > MXBD) fail("mklist> too many atoms bound to base");
        l1i[n1i] = ibd;
        for (int j = 1; j <= nbdat[ibd]; ++j) {
          int jbd = IBD(j, ibd);
          if (iowat[jbd] == ibd && quench(jbd, jbd, n2nd, l2nd1, l2nd2)) push2(n2i, jbd);
        }
      }
    }
    int im = ixmsat[ib];
    if (im > 0)
      for (int i = latms1[im]; i <= latms2[im]; ++i)
        if (quench(i, i, n2nd, l2nd1, l2nd2)) push2(n2i, i);
    for (int is = i1s; is <= i2s; ++is) {
      for (int i = latms1[is]; i <= latms2[is]; ++i) {
        if (nvw + n2nd > MXVW) fail("mklist> Number of vdw-domains > mxvw");
        ivwat1[i] = nvw + 1;
        ivwat2[i] = nvw + n2nd;
        for (int j = 1; j <= n2nd; ++j) {
          ++nvw;
          ixatvw[nvw] = i;
          lvwat1[nvw] = l2nd1[j];
          lvwat2[nvw] = l2nd2[j];
        }
        if (n14 + n2i > MX14) fail("mklist> Number of 1-4 interactions > mx14");
        i14at1[i] = n14 + 1;
        for (int j = 1; j <= n2i; ++j) {
          ++n14;
          ixat14[n14] = i;
          l14at[n14] = l2i[j];
        }
        int iow = iowat[i];
        if (iow != ib) {
          if (n14 + n1i > MX14) fail("mklist> Number of 1-4 interactions > mx14");
          for (int j = 1; j <= n1i; ++j) {
            ++n14;
            ixat14[n14] = i;
            l14at[n14] = l1i[j];
          }
          if (ovlp && (it == 1 || it == 2)) {
            ++n14;
            ixat14[n14] = i;
            l14at[n14] = iob;
          }
          if (iowat[iow] != ib && it == 1) {
            ++n14;
            ixat14[n14] = i;
            l14at[n14] = ib;
          }
        }
        i14at2[i] = n14;
      }
    }
  }
  nvwml[nml] = nvw - ivwml1[nml] + 1;
  n14ml[nml] = n14 - i14ml1[nml] + 1;
  for (int i = ifiat; i <= ilaat; ++i) {
    if (ivwat1[i] <= 0) {
      ivwat1[i] = 1;
      ivwat2[i] = 0;
    }
    if (i14at1[i] <= 0) {
      i14at1[i] = 1;
      i14at2[i] = 0;
    }
  }
}

// redvar (redvar.f:13-648): read a .var file, set and fix variables, rebuild.
void Assembly::redvar(const std::string& varfile) {
  const int maxfld = 4, maxide = 30, ilrg = 1000000;
  int ntlvr = ivrml1[ntlml] + nvrml[ntlml] - 1;
  if (ntlvr == 0) return;
  std::ifstream f(varfile);
  if (!f) fail("redvar> ERROR opening file to set variables: " + varfile);
  std::vector<char> forml(MXML + 2, 1), forrs(MXRS + 2, 1), forvr(MXVR + 2, 1),
      stvr(MXVR + 2, 0);
  std::vector<double> vlvrx(MXVR + 2, 0.0);
  for (int i = 1; i <= ntlvr; ++i) {
    fxvr[i] = 0;
    forvr[i] = 1;
    stvr[i] = 0;
    int it = ityvr[i];
    double vr;
    if (it == 3) vr = toat[iatvr[i]];
    else if (it == 2) vr = baat[iatvr[i]];
    else if (it == 1) vr = blat[iatvr[i]];
    else fail("redvar> unknown variable type");
    vlvrx[i] = vr;
  }
  std::string raw;
  while (std::getline(f, raw)) {
    if (!raw.empty() && raw.back() == '\r') raw.pop_back();
    std::string line = pad(raw, 132);
    int ile = iendst(line);
    if (ile <= 0 || index1(sub(line, 1, ile), '#') > 0) continue;
    int ilb = index1(sub(line, 1, ile), '@') + 1;
    if (ilb >= 2) {   // global parameters of a molecule
      int nml = 1;
      std::string lincmd;
      int l;
      if (index1(sub(line, ilb, ile), ':') > 0) {
        extstr(':', ilb, ile, line, lincmd, l);
        if (iredin(lincmd, nml) <= 0 || nml <= 0 || nml > ntlml)
          fail("redvar> Incorrect molecule number");
      }
      l = ile - ilb + 1;
      if (l <= 0) fail("redvar> line with global parameters must contain 6 numbers");
      lincmd = pad(sub(line, ilb, ile), 132);
      int k = 1;
      double rn[7];
      std::string linh;
      int n;
      for (int i = 1; i <= 5; ++i) {
        extstr(',', k, l, lincmd, linh, n);
        if (k > l || iredrl(linh, rn[i]) <= 0)
          fail("redvar> line with global parameters must contain 6 numbers");
      }
      n = l - k + 1;
      if (n <= 0) fail("redvar> line with global parameters must contain 6 numbers");
      linh = pad(sub(lincmd, k, l), 132);
      if (iredrl(linh, rn[6]) <= 0) fail("redvar> line with global parameters");
      if (std::fabs(rn[4]) > 1.8e2 + 1e-6 || std::fabs(rn[5]) > 9e1 + 1e-6 ||
          std::fabs(rn[6]) > 1.8e2 + 1e-6)
        fail("redvar> global angles out of range");
      for (int i = 1; i <= 3; ++i) gbpr[i][nml] = rn[i];
      for (int i = 4; i <= 6; ++i) gbpr[i][nml] = rn[i] * cdr;
      continue;
    }
    ilb = 1;
    while (ilb <= ile) {
      std::string lincmd;
      int ice;
      extstr(';', ilb, ile, line, lincmd, ice);
      if (ice <= 0) continue;
      bool fix;
      int ifx = index1(sub(lincmd, 1, ice), '&');
      if (ifx > 0) {
        fix = true;
        lincmd[ifx - 1] = ' ';
        if (ifx == ice) {
          --ice;
          if (ice == 0) {
            ice = 1;
            lincmd[0] = '*';
          }
        }
      } else {
        fix = false;
      }
      std::string linfld[maxfld + 1];
      int ifdend[maxfld + 1];
      int nfld = 0, icb = 1;
      while (icb <= ice) {
        ++nfld;
        if (nfld > maxfld) fail("redvar> Cannot interpret command");
        extstr(':', icb, ice, lincmd, linfld[nfld], ifdend[nfld]);
        if (ifdend[nfld] <= 0) {
          linfld[nfld][0] = '*';
          ifdend[nfld] = 1;
        }
      }
      for (int i = 1; i <= nfld - 1; ++i) {
        int ii = i, ifld = nfld - i;
        if (ifld == 3) {
          for (int j = 1; j <= ntlml; ++j) forml[j] = 0;
        } else if (ifld == 2) {
          for (int j = 1; j <= ntlml; ++j)
            for (int k = irsml1[j]; k <= irsml2[j]; ++k) forrs[k] = 0;
        } else if (ifld == 1) {
          for (int j = 1; j <= ntlvr; ++j) forvr[j] = 0;
        }
        int nide = 0, ifb = 1, ife = ifdend[i];
        while (ifb <= ife) {
          ++nide;
          if (nide > maxide) fail("redvar> too many identifiers");
          std::string linide;
          int ide;
          extstr(',', ifb, ife, linfld[ii], linide, ide);
          if (ide <= 0 || linide[0] == '*') {
            if (ifld == 3) {
              for (int j = 1; j <= ntlml; ++j) forml[j] = 1;
            } else if (ifld == 2) {
              for (int j = 1; j <= ntlml; ++j)
                if (forml[j])
                  for (int k = irsml1[j]; k <= irsml2[j]; ++k) forrs[k] = 1;
            } else if (ifld == 1) {
              for (int j = 1; j <= ntlml; ++j)
                if (forml[j])
                  for (int k = irsml1[j]; k <= irsml2[j]; ++k)
                    if (forrs[k])
                      for (int l = ivrrs1[k]; l <= ivrrs1[k] + nvrrs[k] - 1; ++l) forvr[l] = 1;
            }
            continue;
          }
          int ihy = index1(sub(linide, 1, ide), '-');
          if (ihy <= 0) {
            int inum;
            if (iredin(linide, inum) > 0) {
              if (ifld == 3) {
                if (inum <= 0 || inum > ntlml) fail("redvar> Error in identifier");
                forml[inum] = 1;
              } else if (ifld == 2) {
                for (int j = 1; j <= ntlml; ++j)
                  if (forml[j]) {
                    int nfi = irsml1[j], k = inum + nfi - 1;
                    if (k < nfi || k > irsml2[j]) fail("redvar> Error in identifier");
                    forrs[k] = 1;
                  }
              } else if (ifld == 1) {
                for (int j = 1; j <= ntlml; ++j)
                  if (forml[j])
                    for (int k = irsml1[j]; k <= irsml2[j]; ++k)
                      if (forrs[k]) {
                        int nfi = ivrrs1[k], l = inum + nfi - 1;
                        if (l < nfi || l > nfi + nvrrs[k] - 1) fail("redvar> Error in identifier");
                        forvr[l] = 1;
                      }
              }
            } else {   // name, exact or with trailing wild card
              int id;
              bool exa;
              if (linide[ide - 1] == '*') {
                id = ide - 1;
                exa = false;
              } else {
                id = ide;
                exa = true;
              }
              auto match = [&](const std::string& nm) {
                int ib = ibegst(nm);
                if (ib <= 0) return false;
                int ieh = iendst(nm);
                int ieh1 = ieh - ib + 1;
                std::string linh = nm.substr(ib - 1, ieh1);
                return ((exa && ieh1 == id) || (!exa && ieh1 >= id)) &&
                       linh.substr(0, id) == linide.substr(0, id);
              };
              if (ifld == 3) {
                for (int j = 1; j <= ntlml; ++j)
                  if (match(nmml[j])) forml[j] = 1;
              } else if (ifld == 2) {
                for (int j = 1; j <= ntlml; ++j)
                  if (forml[j])
                    for (int k = irsml1[j]; k <= irsml2[j]; ++k)
                      if (match(seq[k])) forrs[k] = 1;
              } else if (ifld == 1) {
                for (int j = 1; j <= ntlml; ++j)
                  if (forml[j])
                    for (int k = irsml1[j]; k <= irsml2[j]; ++k)
                      if (forrs[k])
                        for (int l = ivrrs1[k]; l <= ivrrs1[k] + nvrrs[k] - 1; ++l)
                          if (match(nmvr[l])) forvr[l] = 1;
              }
            }
          } else {   // zone n1-n2
            if (ide == 1 && ihy == ide) fail("redvar> Error in identifier");
            int ibz, iez;
            if (ihy == 1) {
              ibz = 1;
            } else {
              std::string linh = pad(sub(linide, 1, ihy - 1), 132);
              if (iredin(linh, ibz) <= 0 || ibz <= 0) fail("redvar> Error in identifier");
            }
            if (ihy == ide) {
              iez = ilrg;
            } else {
              std::string linh = pad(sub(linide, ihy + 1, ide), 132);
              if (iredin(linh, iez) <= 0 || iez <= 0 || iez < ibz)
                fail("redvar> Error in identifier");
            }
            if (ifld == 3) {
              if (iez > ntlml) iez = ntlml;
              for (int j = ibz; j <= iez; ++j) forml[j] = 1;
            } else if (ifld == 2) {
              for (int j = 1; j <= ntlml; ++j)
                if (forml[j]) {
                  int kbz = irsml1[j] + ibz - 1, kez = irsml1[j] + iez - 1;
                  int kk = kez > irsml2[j] ? irsml2[j] : kez;
                  for (int k = kbz; k <= kk; ++k) forrs[k] = 1;
                }
            } else if (ifld == 1) {
              for (int j = 1; j <= ntlml; ++j)
                if (forml[j])
                  for (int k = irsml1[j]; k <= irsml2[j]; ++k) {
                    int kv = nvrrs[k];
                    if (forrs[k] && kv > 0) {
                      int ll = ivrrs1[k], lbz = ll + ibz - 1;
                      int lez = iez > kv ? ll + kv - 1 : ll + iez - 1;
                      for (int l = lbz; l <= lez; ++l) forvr[l] = 1;
                    }
                  }
            }
          }
        }
      }
      double val;
      if (iredrl(linfld[nfld], val) > 0) {
        for (int i = 1; i <= ntlvr; ++i)
          if (forvr[i]) {
            vlvrx[i] = val;
            fxvr[i] = fix;
            stvr[i] = 1;
          }
      } else {
        fail("redvar> Cannot read value from >" + lincmd.substr(0, ice) + "<");
      }
    }
  }
  int iv = 0;
  for (int i = 1; i <= ntlml; ++i) {
    for (int j = 1; j <= 6; ++j)
      if (gbpr[j][i] != 0.0) {
        setvar(i, vlvrx.data());
        break;
      }
    if (nvrml[i] > 0) {
      bool did = false;
      for (int j = irsml1[i]; j <= irsml2[i]; ++j)
        for (int k = ivrrs1[j]; k <= ivrrs1[j] + nvrrs[j] - 1; ++k) {
          ++iv;
          if (stvr[iv]) {
            did = true;
            int ity = ityvr[iv];
            if (ity == 3 || ity == 2) vlvrx[iv] = vlvrx[iv] * cdr;
          }
        }
      if (did) setvar(i, vlvrx.data());
    }
  }
}

// init_molecule (init_molecule.f:13-221), ab-initio branch (iabin=1).
void Assembly::init_molecule(const std::string& seqfile, const std::string& varfile,
                         const std::string& grpn, const std::string& grpc) {
  int ontlml = ntlml > 0 ? ntlml + 1 : 1;
  redseq(seqfile);
  int ntl = ntlml;
  for (int i = ontlml; i <= ntl; ++i) {
    getmol(i);
    for (int j = 1; j <= 6; ++j) gbpr[j][i] = 0.0;
    bldmol(i);
    ntlml = i;
    addend(i, grpn, grpc);
    setmvs(i);
    mklist(i);
  }
  if (ibegst(varfile) > 0) redvar(varfile);
  nvr = 0;
  for (int i = 1; i <= ivrml1[ntlml] + nvrml[ntlml] - 1; ++i) {
    if (!fxvr[i]) {
      ++nvr;
      idvr[nvr] = i;
    }
    int it = ityvr[i];
    if (it == 3) vlvr[i] = toat[iatvr[i]];
    else if (it == 2) vlvr[i] = baat[iatvr[i]];
    else if (it == 1) vlvr[i] = blat[iatvr[i]];
    olvlvr[i] = vlvr[i];
  }
  for (int i = 1; i <= ivrml1[ntlml] + nvrml[ntlml] - 1; ++i)
    axvr[i] = (ityvr[i] == 3 && !fxvr[i]) ? pi2 : 0.0;   // both branches give 2*pi (:157-190)
  if (itysol != 0) {
    int i1 = iatrs1[irsml1[1]], i2 = iatrs2[irsml2[ntlml]];
    int its = std::abs(itysol);
    for (int i = i1; i <= i2; ++i) {
      int it = ityat[i];
      sigma[i] = coef_sl[its][it];
      rvdw[i] = rad_vdw[its][it];
      if (nmat[i][0] != 'h') rvdw[i] = rvdw[i] + rwater;
    }
  }
}

}  // namespace smmpb200
