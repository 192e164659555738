// Molecule builder: residue library, sequence and variable files -> MolTopo.
//
// This is the product's own construction of the chain the GPU kernels read.
// It builds the covalent tree residue by residue from the library templates,
// puts the terminal groups in place while assembling, and derives every list
// the sweep needs from that tree:
//
//  * a torsion variable turns the subtrees hanging from its base atom (the
//    parent of its primary atom) about the bond base -> parent(base); those
//    subtrees are one contiguous atom range [lo, hi] (checked);
//  * every atom belongs to the rigid group of the innermost variable whose
//    range holds it; the pair set is every pair whose distance some variable
//    changes: an atom of a variable's group with any atom of a group whose
//    range starts earlier, except the two atoms on the variable's axis (its
//    base and the base's parent);
//  * a pair is a 1-4 pair when its partner holds the axis's outer atom: the
//    outer atom's other children with the rest of their contiguous group
//    runs, the outer atom's parent, and the base's own run (the reference's
//    rule; every such pair depends on that one variable alone);
//  * each pair is listed under the atom of the innermost-moved rigid group
//    (the group whose variable's range starts later), partners as runs of
//    consecutive atoms.
//
// What has to stay alike with the reference, because existing input decks
// and the reference's energies depend on it: the residue library's fixed
// columns (getmol.f:263-276), the sequence file (redseq.f), the variable
// file's command language (redvar.f:13-62), the phase convention of
// dihedrals bonded to the same atom (getmol.f:146-170, setvar.f:40-56), the
// choice and geometry of the terminal groups (addend.f:13-160, the internal
// coordinates of groups on the first backbone atom re-expressed against two
// virtual atoms, addend.f:318-357, 523-547), and the ECEPP parameter tables.
#pragma once
#include <map>
#include <string>
#include <vector>

#include "topology.hpp"

namespace smmpb200 {

// One atom line of a residue template (0-based indices inside the template;
// angles in radians).
struct TemplateAtom {
  std::string name;            // 4 characters, blank padded
  int type = 0;                // ECEPP class 1..18
  double charge = 0, blen = 0, bang = 0, tors = 0;
  int parent = -1;             // -1: first atom of the residue
  std::vector<int> bonds;      // bonded atoms listed on this line, in order
};

struct TemplateVar {
  int kind = 3;                // 1 bond length, 2 bond angle, 3 torsion
  int cls = 0;                 // torsion class (e0/sg/rn row)
  int atom = 0;                // primary atom (template index)
  std::string name;            // 3 characters, blank padded
};

struct ResidueTemplate {
  std::string name;            // 4 characters, lower case, blank padded
  int link = 0;                // atom that bonds to the following residue
  std::vector<TemplateAtom> atoms;
  std::vector<TemplateVar> vars;
};

class ResidueLibrary {
 public:
  // Reads every residue of a library file (lib.sh3 / lib.sh2 layout).
  explicit ResidueLibrary(const std::string& path);
  // The template of a residue name (case-insensitive); throws if absent.
  const ResidueTemplate& get(const std::string& name) const;
  const std::string& path() const { return path_; }

 private:
  ResidueTemplate parse(size_t header_line) const;
  std::string path_;
  std::vector<std::string> lines_;
  std::map<std::string, size_t> header_;                  // name -> residue line
  mutable std::map<std::string, ResidueTemplate> cache_;  // parsed on first use
};

// Settings that shape a molecule (the f2py module's epar_l / isolty switches).
struct BuildOptions {
  bool sh2 = false;            // ECEPP/2 library and charges
  int itysol = 0;              // solvation model (0 none, >0 numerical, <0 analytic)
  std::string grpn = "nh2", grpc = "cooh";   // terminal groups
};

// Residue names of the one molecule of a sequence file, as written there
// (a leading Pro becomes "pron"), and the molecule's name.
struct SequenceFile {
  std::string name;
  std::vector<std::string> residues;
};
SequenceFile read_sequence(const std::string& path);

// The molecule as built: topology plus the per-atom bond lists (outpdb) and
// the state the variable file leaves.
MolTopo build_topology(const ResidueLibrary& lib, const ForceField& ff, const BuildOptions& opt,
                       const std::string& seqfile, const std::string& varfile);

// ECEPP/3 (or /2) force field with the solvation model's sphere points read
// from libdir/tes.dat when itysol != 0.
ForceField ecepp_forcefield(const std::string& libdir, bool sh2, bool epsd, int itysol);
// Path of the residue library init_energy selects (libdir + lib.sh2/lib.sh3).
std::string library_path(const std::string& libdir, bool sh2);

// Angle helpers (difang.f:12-60): results wrapped into (-pi, pi].
double difang(double a1, double a2);
double addang(double a1, double a2);

}  // namespace smmpb200
