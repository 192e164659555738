// Flattened, 0-based topology of one molecule as the GPU kernels read it.
//
// build_topology() (molbuild.hpp) emits:
//  * rebuild data: parent atom, bond length, cos/sin of the valence angle, the
//    atoms grouped by depth below the first backbone atom (one parallel
//    Eyring step per depth level, bldmol.f:64-78);
//  * variables: primary atom, base atom, the sibling atoms whose dihedral the
//    variable shifts (setvar.f:40-56), the contiguous atom range that rotates
//    with it (setmvs.f:168-199, the range before overlaps are removed), and the
//    torsion-potential constants (enyshe.f:79-80);
//  * pair work: the dense pair list (every mklist.f pair once, ordered by
//    listing atom then partner, 1-4 pairs flagged), used by the sweep; and
//    the same pairs as every (atom, vdW domain) cut into chunks of at most 8
//    consecutive partners plus the 1-4 partners as explicit pairs, used by
//    the gradient kernel and the host checks;
//  * solvation radii and coefficients (init_molecule.f:194-210).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace smmpb200 {

constexpr int kNumTypes = 18;     // ECEPP atom classes (INCL.H mxtyat)
constexpr int kChunk = 8;         // partners per vdW chunk
constexpr int kMaxAtoms = 16383;  // 14-bit atom index in the packed pair words
constexpr int kNearWindow = 64;   // pairs (i, i+1..i+64) carry explicit flags

// Per type-pair constants, [ti*18+tj].  A/C of the 12-6 (or 12-10 hydrogen
// bond) term, the halved repulsion of 1-4 pairs, and the squared distance
// beyond which every van der Waals / H-bond term is below the FP32 guard
// energy of 100 kcal/mol (closer pairs are evaluated in FP64 in the mixed
// mode).
struct PairTable {
  double a[kNumTypes * kNumTypes];
  double a14[kNumTypes * kNumTypes];
  double c[kNumTypes * kNumTypes];
  int hb[kNumTypes * kNumTypes];
  double guard_r2[kNumTypes * kNumTypes];
};

struct ForceField {
  PairTable pair;
  double conv = 166.0;     // 332/eps_s
  double plt = 78.0, slp = 0.3;
  int epsd = 0;
  int itysol = 0;
  std::vector<double> spoint;   // npnt*3 unit-sphere points
  int npnt = 0;
  // torsion constants per torsion class (index 1..19): e0, sign, periodicity
  std::vector<double> tor_e0, tor_sg, tor_rn;
  // solvation coefficient and radius per atom class (index 1..18) of the
  // chosen model, and the probe radius added to heavy atoms
  std::vector<double> sol_sigma, sol_radius;
  double probe = 0.0;
};

struct MolTopo {
  int natoms = 0, nvar = 0, nfree = 0;
  int i1 = 0, i2 = 0, i3 = 0;          // first three backbone atoms
  double gbpr[6] = {0, 0, 0, 0, 0, 0};
  // atoms
  std::vector<int> iow;                // parent atom (-1 for i1)
  std::vector<uint8_t> type;           // 0-based ECEPP class
  std::vector<double> charge, blen, cba, sba, toat0;
  std::vector<double> rvdw, sigma;
  std::vector<int> level_atoms, level_off;   // CSR by depth (level 0 = i1 only)
  std::vector<int> residue_of_atom;
  // variables (all torsions of the molecule, fixed ones included)
  std::vector<int> var_atom, var_base, var_lo, var_hi, var_class, var_fixed;
  std::vector<int> sib_off, sib;       // CSR of atoms shifted by each variable
  std::vector<double> var_e0, var_sg, var_rn, axvr, vlvr0;
  std::vector<int> idvr;               // free variables (0-based var index)
  std::vector<std::string> var_name, atom_name;
  std::vector<int> var_residue;
  // pair work
  std::vector<uint32_t> chunks;        // i | j0<<14 | (len-1)<<28
  std::vector<uint32_t> pairs14;       // i | j<<14
  // every pair of the lists once, by listing atom then partner:
  // i | j<<14 | is14<<28 (the sweep's dense pair loop)
  std::vector<uint32_t> flat;
  long long npairs = 0;                // pair terms per full evaluation
  std::vector<int> var_cross;          // pairs across each variable's bond (one atom in its range)
  // For molecules of at most 65,535 pairs: per free variable, the indices
  // into `flat` of the pairs whose distance its turn changes (one atom in
  // its range, neither on its axis), CSR by variable (empty for fixed ones).
  std::vector<int> cross_off;
  std::vector<uint16_t> cross_idx;
  // The same pair set by rows: for atom i, bit k of near_mask[i] / near14[i]
  // marks pair (i, i+1+k) as a normal / 1-4 pair.  rows_ok is set when every
  // pair more than kNearWindow apart is a normal pair and no pair is listed
  // twice (checked), so row i is the two masked 32-atom windows after i and
  // then every later atom.
  std::vector<uint64_t> near_mask, near14;
  bool rows_ok = false;
  // solvation
  std::vector<int> heavy;              // atoms with rvdw > 0
  int nres = 0;
  // output (outpdb.f): residue names (seq, lower case), first atom of each
  // residue, and CSR of each atom's bonded partners after it, in outpdb order
  std::vector<std::string> res_name;
  std::vector<int> res_atom0;
  std::vector<int> conect_off, conect;
};

// outvar.f:50-121 (outvbs) for one molecule: the text outvar writes for the
// variables vlvr (radians, all t.nvar of them), with molecule number iml in
// each line's prefix.
std::string outvar_text(const MolTopo& t, const double* vlvr, int iml);
// outpdb.f:12-185 for the only molecule of a system: PDB text (80-column
// lines: ATOM/HETATM, TER, CONECT, END) of coordinates xyz[3*natoms].
std::string outpdb_text(const MolTopo& t, const double* xyz);

}  // namespace smmpb200
