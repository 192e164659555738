// ECEPP/3 (and /2) force-field parameters for the energy kernels.
//
// The numbers below are the force field (init_energy.f:315-610, BLOCK DATA);
// they must equal the reference's to reproduce its energies.  Values the
// reference writes as default-REAL literals are kept as float and widened,
// as its DATA statements do.  The derived tables (12-6 and 10-12 constants
// per type pair, torsion constants) follow the combination rules of
// init_energy.f:106-313 (setpar), computed here from the per-type data.
#include <cmath>
#include <fstream>
#include <stdexcept>
#include <string>

#include "molbuild.hpp"

namespace smmpb200 {

namespace {

constexpr int kTypes = 18;     // atom classes
constexpr int kTorClasses = 19;
constexpr int kSolModels = 9;

// Per atom class: polarisability (x100), effective electrons (x100), r_min (x100).
const float kPolar[kTypes] = {42., 42., 42., 42., 42., 42., 93., 151., 115., 59., 84., 59.,
                              93., 93., 93., 220., 42., 93.};
const float kElectrons[kTypes] = {85., 85., 85., 85., 85., 85., 520., 520., 520., 700., 700.,
                                  700., 610., 610., 610., 1480., 85., 520.};
const float kRmin[kTypes] = {292., 293., 268., 268., 283., 293., 412., 374., 370., 324., 312.,
                             324., 351., 351., 351., 415., 248., 412.};
// Hydrogen-bond donors and acceptors among the classes.
const bool kDonor[kTypes] = {0, 0, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
const bool kAcceptor[kTypes] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 0, 0, 0};
// 10-12 constants by (donor rank 1..4, acceptor rank 1..6), donor fastest.
const float kHbC[24] = {2624., 2624., 4610., 0., 4014., 4014., 5783., 0.,
                        2624., 2624., 4610., 0., 8244., 8244., 8244., 0.,
                        8244., 8244., 8244., 0., 8244., 8244., 8244., 0.};
const float kHbA[24] = {5890., 5890., 11220., 0., 12040., 12040., 16583., 0.,
                        5890., 5890., 11220., 0., 32897., 32897., 32897., 0.,
                        32897., 32897., 32897., 0., 32897., 32897., 32897., 0.};
// Torsion potential e0 (x2), sign, periodicity per torsion class.
const float kTorE0[kTorClasses] = {20., 0., 0., 2.7f, .6f, 1.8f, 1.8f, 0., 0., 0., 0., 0., 2.,
                                   1.5f, 3.5f, 8., 18., 20., 15.};
const float kTorSign[kTorClasses] = {-1., 0., 0., 1., 1., 1., 1., 0., 0., 0., 0., 0., 1., 1.,
                                     -1., -1., -1., -1., -1.};
const float kTorN[kTorClasses] = {2., 0., 0., 3., 3., 3., 3., 0., 0., 0., 0., 0., 3., 3., 2.,
                                  2., 2., 2., 2.};
// Like-pair constants that replace the combination rule (C, A per class).
const double kSelfC[kTypes] = {45.5, 45.5, 45.5, 45.5, 45.5, 45.5, 370.5, 766.6, 509.5, 217.2,
                               369.0, 217.2, 401.3, 401.3, 401.3, 2274.4, 45.5, 370.5};
const double kSelfA[kTypes] = {14090.0, 14380.0, 8420.0, 8420.0, 11680.0, 14380.0, 906100.0,
                               1049000.0, 653600.0, 125600.0, 170200.0, 125600.0, 375200.0,
                               375200.0, 375200.0, 5809000.0, 5340.0, 909000.0};
// Solvation coefficient and radius per (atom class, solvation model 1..9).
const float kSolCoef[kTypes][kSolModels] = {
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
const float kSolRadius[kTypes][kSolModels] = {
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
constexpr double kHalfElectronMass = 362.55;   // the London constant of the C_ij rule
constexpr double kCoulomb = 332.0;             // kcal/mol * A / e^2
constexpr double kEpsS = 2.0;                  // constant dielectric
constexpr double kProbe = (double)1.4f;        // water probe radius (a REAL literal)

// Squared distance below which a term of the pair can exceed `g` kcal/mol.
double guard_r2(double a, double c, int hb, double g) {
  double r2a = a > 0 ? std::pow(a / g, 1.0 / 6.0) : 0.0;   // A/r^12 > g
  double r2c = 0.0;
  if (c > 0) r2c = hb ? std::pow(c / g, 1.0 / 5.0)          // C/r^10 > g
                      : std::pow(c / g, 1.0 / 3.0);         // C/r^6  > g
  return std::max(r2a, r2c);
}

// Unit-sphere points of the numerical SASA (tes.dat: '!' comment lines, the
// point count in columns 1-5, then x, y, z in 20-column fields).
void read_sphere_points(const std::string& path, ForceField& ff) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("Cannot open the file with surface points " + path);
  std::string line;
  do {
    if (!std::getline(f, line)) throw std::runtime_error("tes.dat: no point count");
  } while (!line.empty() && line[0] == '!');
  const int n = std::stoi(line.substr(0, 5));
  if (n <= 0 || n > 2000) throw std::runtime_error("tes.dat: bad number of points");
  ff.spoint.assign(3 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i) {
    if (!std::getline(f, line)) throw std::runtime_error("tes.dat: too few points");
    line.resize(60, ' ');
    for (int k = 0; k < 3; ++k) ff.spoint[3 * i + k] = std::stod(line.substr(20 * k, 20));
  }
  ff.npnt = n;
}

}  // namespace

std::string library_path(const std::string& libdir, bool sh2) {
  std::string d = libdir;
  if (!d.empty() && d.back() != '/') d += '/';
  return d + (sh2 ? "lib.sh2" : "lib.sh3");
}

ForceField ecepp_forcefield(const std::string& libdir, bool sh2, bool epsd, int itysol) {
  (void)sh2;   // ECEPP/2 and /3 share the parameter set; their libraries differ
  ForceField ff;
  double A[kTypes][kTypes], C[kTypes][kTypes], A14[kTypes][kTypes];
  double alpha[kTypes], ne[kTypes], r0[kTypes];
  for (int t = 0; t < kTypes; ++t) {
    alpha[t] = (double)kPolar[t] / 100;
    ne[t] = (double)kElectrons[t] / 100;
    r0[t] = (double)kRmin[t] / 100;
  }
  // Slater-Kirkwood C_ij, A_ij from C_ij and the mean r_min (A = C r^6 / 2),
  // 1-4 repulsion halved.
  for (int i = 0; i < kTypes; ++i) {
    const double si = std::sqrt(alpha[i] / ne[i]);
    const double ki = alpha[i] * kHalfElectronMass;
    for (int j = i; j < kTypes; ++j) {
      const double sj = (j == i) ? si : std::sqrt(alpha[j] / ne[j]);
      const double c = ki * alpha[j] / (si + sj);
      const double r = (j == i) ? r0[i] : .5 * (r0[i] + r0[j]);
      const double r2 = r * r, r6 = r2 * r2 * r2;
      const double a = .5 * c * r6;
      C[i][j] = C[j][i] = c;
      A[i][j] = A[j][i] = a;
      A14[i][j] = A14[j][i] = .5 * a;
    }
  }
  for (int i = 0; i < kTypes; ++i) {
    C[i][i] = kSelfC[i];
    A[i][i] = kSelfA[i];
    A14[i][i] = .5 * A[i][i];
  }
  // 10-12 terms between a donor and an acceptor class, by their ranks.
  int rank[kTypes];
  int nd = 0, na = 0;
  for (int t = 0; t < kTypes; ++t) rank[t] = kDonor[t] ? nd++ : (kAcceptor[t] ? na++ : -1);
  double hbA[kTypes][kTypes] = {}, hbC[kTypes][kTypes] = {};
  int hb[kTypes][kTypes] = {};
  for (int i = 0; i < kTypes; ++i)
    for (int j = 0; j < kTypes; ++j) {
      const bool da = kDonor[i] && !kDonor[j] && kAcceptor[j];
      const bool ad = kDonor[j] && !kDonor[i] && kAcceptor[i];
      if (!da && !ad) continue;
      const int d = da ? rank[i] : rank[j], a = da ? rank[j] : rank[i];
      hb[i][j] = 1;
      hbC[i][j] = (double)kHbC[a * 4 + d];
      hbA[i][j] = (double)kHbA[a * 4 + d];
    }
  const double g = 100.0;   // FP32 guard energy (kcal/mol), see PairTable
  for (int i = 0; i < kTypes; ++i)
    for (int j = 0; j < kTypes; ++j) {
      const int k = i * kTypes + j;
      ff.pair.hb[k] = hb[i][j];
      ff.pair.a[k] = hb[i][j] ? hbA[i][j] : A[i][j];
      ff.pair.a14[k] = hb[i][j] ? hbA[i][j] : A14[i][j];
      ff.pair.c[k] = hb[i][j] ? hbC[i][j] : C[i][j];
      ff.pair.guard_r2[k] =
          guard_r2(std::max(ff.pair.a[k], ff.pair.a14[k]), ff.pair.c[k], hb[i][j], g);
    }
  ff.conv = kCoulomb / kEpsS;
  ff.plt = 78.0;
  ff.slp = 0.3;
  ff.epsd = epsd ? 1 : 0;
  ff.itysol = itysol;
  ff.tor_e0.assign(kTorClasses + 1, 0.0);
  ff.tor_sg.assign(kTorClasses + 1, 0.0);
  ff.tor_rn.assign(kTorClasses + 1, 0.0);
  for (int c = 1; c <= kTorClasses; ++c) {
    ff.tor_e0[c] = (double)kTorE0[c - 1] / 2.;
    ff.tor_sg[c] = kTorSign[c - 1];
    ff.tor_rn[c] = kTorN[c - 1];
  }
  const int model = std::abs(itysol);
  if (model > kSolModels) throw std::runtime_error("init_energy: undefined solvent type");
  ff.sol_sigma.assign(kTypes + 1, 0.0);
  ff.sol_radius.assign(kTypes + 1, 0.0);
  ff.probe = kProbe;
  if (model > 0) {
    for (int t = 1; t <= kTypes; ++t) {
      ff.sol_sigma[t] = (double)kSolCoef[t - 1][model - 1];
      ff.sol_radius[t] = (double)kSolRadius[t - 1][model - 1];
    }
    std::string d = libdir;
    if (!d.empty() && d.back() != '/') d += '/';
    read_sphere_points(d + "tes.dat", ff);
  }
  return ff;
}

}  // namespace smmpb200
