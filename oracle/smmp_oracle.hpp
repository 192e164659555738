// CPU oracle for the SMMP energy-and-sweep path -- TEST INFRASTRUCTURE ONLY.
//
// This is a C++17 FP64 restatement of the Fortran reference (SMMP trunk) used
// as the parity checker for the CUDA product path.  Only tests/, the smoke()
// check and bench.py's CPU-baseline leg may load it; the product library never
// links it.  Every routine cites the reference file:line it follows.  Arrays
// are 1-based (index 0 unused, xat/yat/zat also carry the two virtual atoms
// -1 and 0 used by rplgrp) so that the index arithmetic of the setup code
// (getmol/addend/setmvs/mklist) can be checked line by line.
//
// Floating point: compiled with -ffp-contract=off so that every + and * is a
// separately rounded IEEE operation in the reference's evaluation order.
#pragma once
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace oracle {

// Capacities (INCL.H:14-36 holds the reference's compile-time caps; these are
// larger so that the 60-residue synthetic protein fits).
constexpr int MXML = 10;
constexpr int MXRS = 512;
constexpr int MXAT = 8192;
constexpr int MXBD = 3;
constexpr int MXATH = 100;
constexpr int MXVR = MXRS * 8;
constexpr int MXMS = MXVR * 3;
constexpr int MXVW = MXAT * 32;
constexpr int MX14 = MXAT * 16;
constexpr int MXTYAT = 18;
constexpr int MXTYTO = 19;
constexpr int MXHBDO = 4;
constexpr int MXHBAC = 6;
constexpr int MXTYSOL = 9;
constexpr int MXPOINT = 2000;

struct Library {            // text of a residue library (lib.sh3 / lib.sh2)
  std::vector<std::string> lines;
};

struct Smmp {
  // ------------------------------------------------ switches (INCL.H:224,327)
  bool sh2 = false, epsd = false, flex = false;
  int ientyp = 0, itysol = 0;
  bool rndord = false;
  int upchswitch = 0;
  double beta = 0.0;

  // ------------------------------------------------ force field (setpar)
  double cij[MXTYAT + 1][MXTYAT + 1], aij[MXTYAT + 1][MXTYAT + 1];
  double a14[MXTYAT + 1][MXTYAT + 1], chb[MXTYAT + 1][MXTYAT + 1];
  double ahb[MXTYAT + 1][MXTYAT + 1];
  int ihbty[MXTYAT + 1][MXTYAT + 1];
  double e0to[MXTYTO + 1], sgto[MXTYTO + 1], rnto[MXTYTO + 1], esnto[MXTYTO + 1];
  double conv = 0, plt = 0, slp = 0;

  // ------------------------------------------------ solvation (tessel, sol)
  int npnt = 0;
  std::vector<double> spoint;   // [(il-1)*3 + k], il 1..npnt, k 0..2
  double coef_sl[MXTYSOL + 1][MXTYAT + 1], rad_vdw[MXTYSOL + 1][MXTYAT + 1];

  Library lib;

  // ------------------------------------------------ molecules
  int ntlml = 0;
  int irsml1[MXML + 1], irsml2[MXML + 1], ivrml1[MXML + 1], nvrml[MXML + 1];
  int imsml1[MXML + 1], nmsml[MXML + 1], iadml1[MXML + 1], nadml[MXML + 1];
  int ixrfpt[4][MXML + 1];
  int nvwml[MXML + 1], ivwml1[MXML + 1], n14ml[MXML + 1], i14ml1[MXML + 1];
  double gbpr[7][MXML + 1], rfpt[4][MXML + 1];
  double xrfax[4][MXML + 1], yrfax[4][MXML + 1], zrfax[4][MXML + 1];
  std::string nmml[MXML + 1];

  // ------------------------------------------------ residues
  std::vector<int> iatrs1, iatrs2, ixatrs, ivrrs1, nvrrs;
  std::vector<std::string> seq;   // 4-char padded names

  // ------------------------------------------------ atoms
  std::vector<int> ityat, iowat, iyowat, nbdat, ixmsat;
  std::vector<int> ibdat, iybdat;                 // [(i)*4 + j], j 1..3
  std::vector<double> cgat, xbaat, ybaat, zbaat, baat, snbaat, csbaat;
  std::vector<double> xtoat, ytoat, ztoat, toat, sntoat, cstoat, blat;
  std::vector<double> xat_, yat_, zat_;           // offset by 2 (index -1..)
  std::vector<std::string> nmat;
  std::vector<double> rvdw, sigma;

  // ------------------------------------------------ variables
  int nvr = 0;
  std::vector<double> olvlvr, vlvr, axvr;
  std::vector<int> iatvr, ityvr, iclvr, iorvr, imsvr1, imsvr2, latms1, latms2;
  std::vector<int> iadvr1, iadvr2, ladvr, idvr;
  std::vector<std::string> nmvr;
  std::vector<char> fxvr;

  // ------------------------------------------------ interaction lists
  std::vector<int> ivwat1, ivwat2, i14at1, i14at2, lvwat1, lvwat2, l14at;
  std::vector<int> ixatvw, ixat14;

  // ------------------------------------------------ energies
  double eyel = 0, eyvw = 0, eyhb = 0, eyvr = 0, eysm = 0, eysl = 0;
  double asa = 0, vdvol = 0, eyslh = 0, eyslp = 0, asap = 0, asah = 0;
  std::vector<double> surfres;

  // ------------------------------------------------ help arrays (redres)
  std::string nmath[MXATH + 1], nmvrh[MXATH + 1];
  int ityath[MXATH + 1], iowath[MXATH + 1], iyowath[MXATH + 1], nbdath[MXATH + 1];
  int ibdath[MXBD + 2][MXATH + 1], iybdath[MXBD + 2][MXATH + 1];
  int ityvrh[MXATH + 1], iclvrh[MXATH + 1], iatvrh[MXATH + 1];
  double blath[MXATH + 1], baath[MXATH + 1], toath[MXATH + 1], cgath[MXATH + 1];

  // ------------------------------------------------ MT19937 (twister.f /myblock/)
  uint32_t mt[624];
  int mti = 625;

  // ------------------------------------------------ acceptance statistics
  long long ncalls = 0, nacalls = 0;

  Smmp();

  double& xat(int i) { return xat_[i + 2]; }
  double& yat(int i) { return yat_[i + 2]; }
  double& zat(int i) { return zat_[i + 2]; }
  int& IBD(int j, int i) { return ibdat[i * 4 + j]; }
  int& IYBD(int j, int i) { return iybdat[i * 4 + j]; }

  // setup
  void init_energy(const std::string& libdir);
  void setpar();
  void tessel(const std::string& path);
  void init_molecule(const std::string& seqfile, const std::string& varfile,
                     const std::string& grpn, const std::string& grpc);
  void redseq(const std::string& seqfile);
  void getmol(int nml);
  void redres(const std::string& res, int& nat, int& nxt, int& nvrr);
  void addend(int nml, const std::string& grpn, const std::string& grpc);
  void rplgrp(int nml, int nrs, const std::string& rpat, const std::string& sbrs);
  void setmvs(int nml);
  void fndbrn(int nml, int nrs, int ifirg, int& ilarg, int& irg1, int& irg2, bool& bb);
  void mklist(int nml);
  void redvar(const std::string& varfile);
  int nursvr(int ivr);
  int nursat(int iat);

  // rebuild
  void setvar(int nml, const double* vlvrx);
  void bldmol(int nml);
  void fnd3ba(int nml, int& i1, int& i2, int& i3);
  void eyring(int i, int ia);
  void setsys(int i1, int i2, int i3, double& x1, double& x2, double& x3,
              double& y1, double& y2, double& y3, double& z1, double& z2, double& z3);
  void setgbl(int nml, int i1, int i2, int i3, double* xg, double* zg);
  double valang(int i1, int i2, int i3);
  double dihedr(int i1, int i2, int i3, int i4);

  // energy
  double energy();
  double enyshe(int nml);
  double enysol(int nmol);
  double esolan(int nmol);
  // gradient (gradient.f, opeshe.f): energy and gdeyvr[iv] = dE/dvlvr[iv]
  double opeshe(int nml);
  double gradient();
  std::vector<double> gdeyvr;
  void gradient_by_sums(int nml, std::vector<double>& gd);   // order-free form (tests)
  // atoms moved by each variable of nml: its moving sets and, recursively,
  // those of the variables added to it (setmvs.f)
  std::vector<std::vector<int>> moved_atoms(int nml);
  // opesol.f: eysl and gdeysl[iv] = d(eysl)/d(variable iv) (itysol < 0)
  void opesol(int nml, std::vector<double>& gdeysl);
  // minimisation (minim.f imin = 1, minqsn.f); log: (energy, |grad|^2) per call
  int minim(int imin, int maxit, double eps, std::vector<double>* log);
  int minqsn(int n, double* x, double& f, double* g, const double* scal, double acur,
             int maxfun, std::vector<double>* log);
  void minim_move(int n, double& f, const double* x, double* g, std::vector<double>* log);
  int mincjg(int n, double* x, double& f, double* g, double acur, int maxfun,
             std::vector<double>* log);

  // random numbers
  void sgrnd(int32_t seed);
  double grnd();

  // sampling
  enum WeightKind { W_CANON = 0, W_MUCA = 1, W_MUCA2 = 2 };
  struct Weight {
    int kind = W_CANON;
    const double* b = nullptr;      // indexed [k - kmin]
    const double* alpha = nullptr;
    int kmin = 0, kmax = 0;
    double ebin = 1.0;
  };
  double weight(const Weight& w, double x) const;
  void metropolis(double& eol1, double& acz, const Weight& w);
};

// esolan.f:12-1050 over atoms 1..numat (1-based arrays; radii with the water
// probe added); returns sum_i sigma_i A_i, the areas A_i in As_out[1..numat]
// and gradan[3j + k] = sum_i sigma_i dA_i/dr_jk (esolan.f:1034-1042) when
// those are not null.  grnd draws the re-orientation angles from the
// caller's stream.
double esolan_areas(int numat, const double* x, const double* y, const double* z,
                    const double* rvdw, const double* sigma, const std::function<double()>& grnd,
                    double* As_out, double* gradan = nullptr);

// enysol.f:107-330 over the spheres 1..numat (1-based arrays, radii > 0 take
// part): asa and vdvol of the numerical surface; per_atom(k, area, icount)
// for each sphere in the reference's box order.
void enysol_spheres(int numat, const double* x, const double* y, const double* z,
                    const double* rv, const double* spoint, int npnt, double& asa, double& vdvol,
                    const std::function<void(int, double, int)>& per_atom);

// mulcan_par_mod.f90:93-145 and :163-168: the multicanonical weight
// recursion (arrays indexed k - kmin; ihist zeroed by the update).
void muca_update(int kmin, int kmax, double ebin, double beta, int* ihist, double* xhist,
                 double* g1, double* b, double* alpha, double* ent);
void muca_finish(int kmin, int kmax, double ebin, double beta, double* b, double* alpha);

// Angle helpers (difang.f:12-60): results wrapped into (-pi, pi].
double difang(double a1, double a2);
double addang(double a1, double a2);

}  // namespace oracle
