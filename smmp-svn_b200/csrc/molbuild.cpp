// Molecule builder (see molbuild.hpp for the design).
#include "molbuild.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <stdexcept>

namespace smmpb200 {

namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kDegToRad = 1.745329251994330e-2;   // the reference's literal, not pi/180
constexpr int kMaxTorsionClass = 19;

[[noreturn]] void fail(const std::string& m) { throw std::runtime_error(m); }

std::string lower(std::string s) {
  for (char& c : s)
    if (c >= 'A' && c <= 'Z') c = char(c - 'A' + 'a');
  return s;
}
std::string pad(std::string s, size_t n) {
  s.resize(n, ' ');
  return s;
}
std::string trim(const std::string& s) {
  const size_t b = s.find_first_not_of(" \t");
  if (b == std::string::npos) return "";
  const size_t e = s.find_last_not_of(" \t");
  return s.substr(b, e - b + 1);
}
std::string column(const std::string& line, size_t from, size_t width) {
  if (from >= line.size()) return std::string(width, ' ');
  return pad(line.substr(from, width), width);
}
// Fortran I edit descriptor on input: blanks ignored, empty field is 0.
int read_int(const std::string& field) {
  std::string t;
  for (char c : field)
    if (c != ' ') t += c;
  if (t.empty()) return 0;
  char* end = nullptr;
  const long v = std::strtol(t.c_str(), &end, 10);
  if (*end) fail("bad integer field >" + field + "<");
  return (int)v;
}
// Fortran F/D edit descriptor on input: a field without a decimal point has
// `decimals` implied fraction digits.
double read_real(const std::string& field, int decimals) {
  std::string t;
  for (char c : field)
    if (c != ' ') t += (c == 'd' || c == 'D') ? 'e' : c;
  if (t.empty()) return 0.0;
  char* end = nullptr;
  double v = std::strtod(t.c_str(), &end);
  if (*end) fail("bad real field >" + field + "<");
  if (t.find('.') == std::string::npos) v /= std::pow(10.0, decimals);
  return v;
}

// --------------------------------------------------------------------- geometry
struct V3 {
  double x = 0, y = 0, z = 0;
};
V3 operator-(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 cross(const V3& a, const V3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
V3 unit(const V3& a) {
  const double s = 1.0 / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return {a.x * s, a.y * s, a.z * s};
}
// Local frame of an atom: x along the bond from its parent, z normal to the
// plane of the parent's bond (Eyring's construction).
struct Frame {
  V3 pos, x, z;
};
// Atom placed from its parent's frame by bond length, valence angle and
// dihedral (Eyring's method).
Frame place(const Frame& p, double blen, double bang, double tors) {
  const double ct = std::cos(tors), st = std::sin(tors);
  const double ca = std::cos(bang), sa = std::sin(bang);
  const V3 y = cross(p.z, p.x);
  const double h2 = -sa * ct, h3 = -sa * st;
  Frame f;
  f.x = unit({-ca * p.x.x + h2 * y.x + h3 * p.z.x, -ca * p.x.y + h2 * y.y + h3 * p.z.y,
              -ca * p.x.z + h2 * y.z + h3 * p.z.z});
  f.z = unit({-st * y.x + ct * p.z.x, -st * y.y + ct * p.z.y, -st * y.z + ct * p.z.z});
  f.pos = {p.pos.x + f.x.x * blen, p.pos.y + f.x.y * blen, p.pos.z + f.x.z * blen};
  return f;
}
double valence_angle(const V3& a, const V3& vertex, const V3& b) {
  const V3 u = a - vertex, w = b - vertex;
  const double uu = u.x * u.x + u.y * u.y + u.z * u.z, ww = w.x * w.x + w.y * w.y + w.z * w.z;
  double c = (u.x * w.x + u.y * w.y + u.z * w.z) / std::sqrt(uu * ww);
  c = std::min(1.0, std::max(-1.0, c));
  return std::acos(c);
}
double dihedral(const V3& a, const V3& b, const V3& c, const V3& d) {
  const V3 b1 = b - a, b2 = c - b, b3 = d - c;
  const V3 n1 = cross(b1, b2), n2 = cross(b2, b3);
  const double nn = (n1.x * n1.x + n1.y * n1.y + n1.z * n1.z) * (n2.x * n2.x + n2.y * n2.y + n2.z * n2.z);
  if (nn == 0.0) fail("dihedral of collinear atoms");
  double c0 = (n1.x * n2.x + n1.y * n2.y + n1.z * n2.z) / std::sqrt(nn);
  c0 = std::min(1.0, std::max(-1.0, c0));
  double t = std::acos(c0);
  const V3 m = cross(n1, n2);
  if (m.x * b2.x + m.y * b2.y + m.z * b2.z < 0.0) t = -t;
  return t;
}
// Frame of the first backbone atom for global angles (0, 0, 0): x along the
// bond to the second backbone atom, z normal to the plane of the first two
// bonds (setgbl.f's construction with the identity orientation).
Frame first_frame(double ba2, double t2, double t3) {
  const double ct2 = std::cos(t2), st2 = std::sin(t2), sa2 = std::sin(ba2);
  V3 x = unit({-std::cos(ba2), -sa2 * ct2, -sa2 * st2});
  const double ct3 = std::cos(t3), st3 = std::sin(t3);
  V3 z = unit({-st3 * (st2 * x.z + ct2 * x.y), st3 * ct2 * x.x + ct3 * st2,
               st3 * st2 * x.x - ct3 * ct2});
  const V3 y = cross(z, x);
  Frame f;
  f.x = unit({x.x, y.x, z.x});
  f.z = unit({x.z, y.z, z.z});
  return f;
}

// ------------------------------------------------------------ residue pieces
// A residue while the chain is assembled: atoms with residue-local parents
// and bonds (-1: the residue's first atom has its parent in the previous
// residue), and its variables.
struct Piece {
  std::vector<TemplateAtom> atoms;
  std::vector<TemplateVar> vars;
  int link = 0;
};

Piece piece_of(const ResidueTemplate& t) {
  Piece p;
  p.atoms = t.atoms;
  p.vars = t.vars;
  p.link = t.link;
  return p;
}

int find_atom(const Piece& p, const std::string& name) {
  for (size_t i = 0; i < p.atoms.size(); ++i)
    if (p.atoms[i].name == name) return (int)i;
  return -1;
}

// Last atom of the subtree of atom `a` inside a piece (atoms of a subtree
// are consecutive; checked).
int subtree_end(const Piece& p, int a) {
  int end = a;
  for (size_t j = a + 1; j < p.atoms.size(); ++j) {
    int q = p.atoms[j].parent;
    while (q > a) q = p.atoms[q].parent;
    if (q != a) break;
    end = (int)j;
  }
  return end;
}

// The group rooted at atom `root` of `host` (root..host_end) replaced by the
// group rooted at the atom of the same name in `sub`.  The root keeps the
// host's internal coordinates, takes the substituent's class (and charge,
// unless `keep_charge`) and bonds; `extra_bonds` (host indices) follow them.
// Variables of the removed atoms give way to the substituent's, which
// `skip_var` can drop.  Returns the map host index -> new index (-1 removed).
template <class SkipVar>
std::vector<int> replace_group(Piece& host, int root, int host_end, const ResidueTemplate& sub,
                               bool keep_charge, const std::vector<int>& extra_bonds,
                               SkipVar skip_var, std::vector<int>* sub_index) {
  Piece s = piece_of(sub);
  const int sroot = find_atom(s, host.atoms[root].name);
  if (sroot < 0) fail("terminal group " + sub.name + " has no atom " + host.atoms[root].name);
  const int send = subtree_end(s, sroot);
  for (int j = sroot + 1; j <= send; ++j)
    for (int b : s.atoms[j].bonds)
      if (b < sroot) fail("terminal group " + sub.name + ": ring back into the residue");
  const int n_host = (int)host.atoms.size();
  const int n_sub = send - sroot;   // substituent atoms after its root
  std::vector<int> hmap(n_host, -1), smap(s.atoms.size(), -1);
  for (int i = 0; i <= root; ++i) hmap[i] = i;
  for (int j = sroot; j <= send; ++j) smap[j] = root + (j - sroot);
  for (int i = host_end + 1; i < n_host; ++i) hmap[i] = i - (host_end - root) + n_sub;
  Piece out;
  out.link = hmap[host.link] >= 0 ? hmap[host.link] : root;
  for (int i = 0; i <= root; ++i) out.atoms.push_back(host.atoms[i]);
  TemplateAtom& r = out.atoms[root];
  r.type = s.atoms[sroot].type;
  if (!keep_charge) r.charge = s.atoms[sroot].charge;
  r.bonds.clear();
  for (int b : s.atoms[sroot].bonds) r.bonds.push_back(smap.at(b));
  for (int b : extra_bonds) r.bonds.push_back(hmap.at(b));
  for (int j = sroot + 1; j <= send; ++j) {
    TemplateAtom a = s.atoms[j];
    a.parent = smap.at(a.parent);
    for (int& b : a.bonds) b = smap.at(b);
    out.atoms.push_back(a);
  }
  for (int i = host_end + 1; i < n_host; ++i) {
    TemplateAtom a = host.atoms[i];
    if (a.parent >= 0) {
      if (hmap[a.parent] < 0) fail("terminal group: an atom hangs from a replaced atom");
      a.parent = hmap[a.parent];
    }
    for (int& b : a.bonds) {
      if (hmap[b] < 0) fail("terminal group: a bond to a replaced atom");
      b = hmap[b];
    }
    out.atoms.push_back(a);
  }
  for (int i = 0; i < root; ++i)
    for (int& b : out.atoms[i].bonds) {
      if (hmap[b] < 0) fail("terminal group: a bond to a replaced atom");
      b = hmap[b];
    }
  // variables: host's up to the root, the substituent's, host's after the group
  for (const TemplateVar& v : host.vars)
    if (v.atom <= root) out.vars.push_back(v);
  for (const TemplateVar& v : s.vars) {
    if (v.atom <= sroot || v.atom > send || skip_var(s, sroot, v)) continue;
    TemplateVar w = v;
    w.atom = smap[v.atom];
    out.vars.push_back(w);
  }
  for (const TemplateVar& v : host.vars)
    if (v.atom > host_end) {
      TemplateVar w = v;
      w.atom = hmap[v.atom];
      out.vars.push_back(w);
    }
  if (sub_index) *sub_index = smap;
  host = out;
  return hmap;
}

// N-terminal group (addend.f:55-100, rplgrp's first-backbone-atom case).
void put_n_terminus(Piece& p, const ResidueTemplate& sub, bool sh2) {
  const int root = find_atom(p, "n   ");
  if (root != 0) fail("rplgrp> cannot replace the N-terminal atom n of the first residue");
  // children of the first atom; the group replaced ends before its last child
  int last_child = -1, ring = -1;
  for (int b : p.atoms[0].bonds) {
    if (p.atoms[b].parent == 0)
      last_child = std::max(last_child, b);
    else if (ring < 0)
      ring = b;
    else
      fail("rplgrp> can handle only a simple ring at the first atom");
  }
  if (last_child < 0) fail("rplgrp> first atom without a following backbone atom");
  const int host_end = last_child - 1;
  const int bb1 = host_end + 1;   // next backbone atom
  int bb2 = -1;                   // the backbone atom after it
  if (bb1 == p.link) fail("rplgrp> N-terminal group on a residue whose second atom links on");
  for (int i = p.link; i > bb1; --i)
    if (p.atoms[i].parent == bb1) {
      bb2 = i;
      break;
    }
  if (bb2 < 0) fail("rplgrp> cannot find the backbone atom after the first two");
  // The first three backbone atoms as the library builds them (first atom at
  // the origin, identity global orientation), then the frame of the first
  // atom that the substituent's internal coordinates refer to: x from the
  // second backbone atom to the first, z normal to the plane with the third.
  const TemplateAtom &A1 = p.atoms[bb1], &A2 = p.atoms[bb2];
  Frame f0 = first_frame(A1.bang, A1.tors, A2.tors);
  const Frame f1 = place(f0, A1.blen, A1.bang, A1.tors);
  const Frame f2 = place(f1, A2.blen, A2.bang, A2.tors);
  const V3 n = f0.pos, xr = n - f1.pos, yr = n - f2.pos;
  Frame root_frame;
  root_frame.pos = n;
  root_frame.x = unit(xr);
  root_frame.z = unit(cross(xr, yr));
  const V3 yv = cross(root_frame.z, root_frame.x);
  // two virtual atoms before the first one, so that the first atom's
  // children get internal coordinates in the chain's convention
  V3 v0, vm1;
  {
    const double ct = std::cos(A2.tors), st = std::sin(A2.tors);
    const double ca = std::cos(A1.bang), sa = std::sin(A1.bang);
    const V3 &X = root_frame.x, &Z = root_frame.z;
    const double h2 = -sa * ct, h3 = -sa * st;
    const V3 x = unit({-ca * X.x + h2 * yv.x + h3 * Z.x, -ca * X.y + h2 * yv.y + h3 * Z.y,
                       -ca * X.z + h2 * yv.z + h3 * Z.z});
    v0 = {n.x + x.x, n.y + x.y, n.z + x.z};
    const V3 z = unit({-st * yv.x + ct * Z.x, -st * yv.y + ct * Z.y, -st * yv.z + ct * Z.z});
    const double ct1 = std::cos(A1.tors), st1 = std::sin(A1.tors);
    const V3 zx = cross(z, x);
    vm1 = {v0.x - ct1 * zx.x - st1 * z.x, v0.y - ct1 * zx.y - st1 * z.y,
           v0.z - ct1 * zx.z - st1 * z.z};
  }
  std::vector<int> extra = {bb1};
  if (ring >= 0) extra.push_back(ring);
  std::vector<int> smap;
  const int old_n = (int)p.atoms.size();
  (void)old_n;
  auto skip = [](const Piece& s, int sroot, const TemplateVar& v) {
    return v.kind == 3 && s.atoms[v.atom].parent == sroot;   // torsions about the first atom
  };
  replace_group(p, 0, host_end, sub, sh2, extra, skip, &smap);
  // substituent atoms re-expressed against the virtual atoms
  const int nsub = (int)std::count_if(smap.begin(), smap.end(), [](int x) { return x > 0; });
  std::vector<Frame> fr(p.atoms.size());
  fr[0] = root_frame;
  for (int k = 1; k <= nsub; ++k) {
    TemplateAtom& a = p.atoms[k];
    fr[k] = place(fr[a.parent], a.blen, a.bang, a.tors);
    if (a.parent == 0) {
      a.bang = valence_angle(v0, n, fr[k].pos);
      a.tors = dihedral(vm1, v0, n, fr[k].pos);
    } else if (p.atoms[a.parent].parent == 0) {
      a.tors = dihedral(v0, n, fr[a.parent].pos, fr[k].pos);
    }
  }
}

// C-terminal group (addend.f:102-143, rplgrp's last-backbone-atom case).
void put_c_terminus(Piece& p, const ResidueTemplate& sub, bool sh2) {
  const int root = find_atom(p, "c   ");
  if (root < 0) fail("rplgrp> cannot find atom c to be replaced");
  if (root != p.link) fail("rplgrp> cannot replace backbone atom c that is not the link atom");
  if (p.atoms[root].parent <= 0)
    fail("rplgrp> the C-terminal atom hangs from the first atom of the molecule");
  const int host_end = subtree_end(p, root);
  auto keep = [](const Piece&, int, const TemplateVar&) { return false; };
  replace_group(p, root, host_end, sub, sh2, {}, keep, nullptr);
}

// ------------------------------------------------------------ variable file
struct VarSettings {
  std::vector<char> set, fixed;
  std::vector<double> value;   // as read (degrees for angles)
  double gbpr[6] = {0, 0, 0, 0, 0, 0};
};

// Up to the next separator: the piece (blanks trimmed) and the position after it.
std::string next_token(const std::string& s, size_t& pos, char sep) {
  const size_t q = s.find(sep, pos);
  std::string tok = s.substr(pos, q == std::string::npos ? std::string::npos : q - pos);
  pos = (q == std::string::npos) ? s.size() : q + 1;
  return trim(tok);
}
bool parse_count(const std::string& s, int& v) {   // digits only, fewer than 10
  const std::string t = trim(s);
  if (t.empty() || t.size() > 9) return false;
  for (char c : t)
    if (c < '0' || c > '9') return false;
  v = std::atoi(t.c_str());
  return true;
}
bool parse_value(const std::string& s, double& v) {   // <= 17 chars, <= 6 decimals
  const std::string t = trim(s);
  if (t.empty() || t.find(',') != std::string::npos) return false;
  const size_t dot = t.find('.');
  if (dot != std::string::npos) {
    if (!(t.size() <= 17 && dot < 11 && t.size() - 1 - dot <= 6)) return false;
  } else if (!(t.size() < 11)) {
    return false;
  }
  char* end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return *end == 0;
}
bool name_matches(const std::string& name, const std::string& ident) {
  const std::string nm = trim(name);
  if (!ident.empty() && ident.back() == '*') {
    const std::string pre = ident.substr(0, ident.size() - 1);
    return nm.size() >= pre.size() && nm.compare(0, pre.size(), pre) == 0;
  }
  return nm == ident;
}

struct VarFileContext {
  std::string mol_name;
  std::vector<std::string> res_names;   // as in the sequence file
  std::vector<int> res_var_first, res_var_count;
  std::vector<std::string> var_names;
};

// The variable file's commands (redvar.f:13-62): "mol : res : var : value"
// with fields counted from the right, ',' between identifiers, ';' between
// commands, '&' fixing, '*' wildcards, 'n1-n2' zones; '@' lines set the six
// global parameters.  A field left out keeps the previous command's choice.
VarSettings read_var_file(const std::string& path, const VarFileContext& c) {
  std::ifstream f(path);
  if (!f) fail("redvar> ERROR opening file to set variables: " + path);
  const int nres = (int)c.res_names.size(), nvar = (int)c.var_names.size();
  VarSettings out;
  out.set.assign(nvar, 0);
  out.fixed.assign(nvar, 0);
  out.value.assign(nvar, 0.0);
  bool for_mol = true;
  std::vector<char> for_res(nres, 1), for_var(nvar, 1);
  std::string line;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    const size_t last = line.find_last_not_of(' ');
    if (last == std::string::npos) continue;
    line = line.substr(0, last + 1);
    if (line.find('#') != std::string::npos) continue;
    const size_t at = line.find('@');
    if (at != std::string::npos) {   // global parameters
      std::string rest = line.substr(at + 1);
      const size_t colon = rest.find(':');
      if (colon != std::string::npos) {
        int m = 0;
        if (!parse_count(rest.substr(0, colon), m) || m != 1)
          fail("redvar> Incorrect molecule number in >" + line + "<");
        rest = rest.substr(colon + 1);
      }
      double rn[6];
      size_t pos = 0;
      for (int k = 0; k < 5; ++k) {
        if (pos >= rest.size() || !parse_value(next_token(rest, pos, ','), rn[k]))
          fail("redvar> line with global parameters must contain 6 numbers: " + line);
      }
      if (pos >= rest.size() || !parse_value(rest.substr(pos), rn[5]))
        fail("redvar> line with global parameters must contain 6 numbers: " + line);
      if (std::fabs(rn[3]) > 180.0 + 1e-6 || std::fabs(rn[4]) > 90.0 + 1e-6 ||
          std::fabs(rn[5]) > 180.0 + 1e-6)
        fail("redvar> global angles outside [-180,180], [-90,90], [-180,180]: " + line);
      for (int k = 0; k < 3; ++k) out.gbpr[k] = rn[k];
      for (int k = 3; k < 6; ++k) out.gbpr[k] = rn[k] * kDegToRad;
      continue;
    }
    size_t pos = 0;
    while (pos < line.size()) {
      std::string cmd = next_token(line, pos, ';');
      if (cmd.empty()) continue;
      bool fix = false;
      const size_t amp = cmd.find('&');
      if (amp != std::string::npos) {
        fix = true;
        if (amp + 1 == cmd.size()) {
          cmd.erase(amp);
          if (trim(cmd).empty()) cmd = "*";
        } else {
          cmd[amp] = ' ';
        }
      }
      std::vector<std::string> fields;
      size_t fp = 0;
      while (fp < cmd.size()) {
        std::string fld = next_token(cmd, fp, ':');
        fields.push_back(fld.empty() ? "*" : fld);
        if (fields.size() > 4) fail("redvar> Cannot interpret command >" + cmd + "<");
      }
      const int nfld = (int)fields.size();
      for (int i = 0; i + 1 < nfld; ++i) {
        const int level = nfld - 1 - i;   // 3 molecule, 2 residue, 1 variable
        if (level == 3) for_mol = false;
        if (level == 2) std::fill(for_res.begin(), for_res.end(), 0);
        if (level == 1) std::fill(for_var.begin(), for_var.end(), 0);
        size_t ip = 0;
        int nid = 0;
        const std::string& fld = fields[i];
        while (ip < fld.size()) {
          if (++nid > 30) fail("redvar> too many identifiers in >" + fld + "<");
          const std::string id = next_token(fld, ip, ',');
          auto bad = [&] { fail("redvar> Error in identifier >" + id + "< of command >" + cmd + "<"); };
          auto all_vars_of = [&](int r) {
            for (int v = c.res_var_first[r]; v < c.res_var_first[r] + c.res_var_count[r]; ++v)
              for_var[v] = 1;
          };
          if (id.empty() || id[0] == '*') {
            if (level == 3) for_mol = true;
            if (level == 2 && for_mol) std::fill(for_res.begin(), for_res.end(), 1);
            if (level == 1 && for_mol)
              for (int r = 0; r < nres; ++r)
                if (for_res[r]) all_vars_of(r);
            continue;
          }
          const size_t hy = id.find('-');
          int num = 0;
          if (hy == std::string::npos && parse_count(id, num)) {   // an index
            if (level == 3) {
              if (num != 1) bad();
              for_mol = true;
            } else if (level == 2 && for_mol) {
              if (num < 1 || num > nres) bad();
              for_res[num - 1] = 1;
            } else if (level == 1 && for_mol) {
              for (int r = 0; r < nres; ++r)
                if (for_res[r]) {
                  if (num < 1 || num > c.res_var_count[r]) bad();
                  for_var[c.res_var_first[r] + num - 1] = 1;
                }
            }
          } else if (hy == std::string::npos) {   // a name
            if (level == 3) {
              if (name_matches(c.mol_name, id)) for_mol = true;
            } else if (level == 2 && for_mol) {
              for (int r = 0; r < nres; ++r)
                if (name_matches(c.res_names[r], id)) for_res[r] = 1;
            } else if (level == 1 && for_mol) {
              for (int r = 0; r < nres; ++r)
                if (for_res[r])
                  for (int v = c.res_var_first[r]; v < c.res_var_first[r] + c.res_var_count[r]; ++v)
                    if (name_matches(c.var_names[v], id)) for_var[v] = 1;
            }
          } else {   // a zone n1-n2, -n2 or n1-
            if (id.size() == 1) bad();
            int lo = 1, hi = 1000000;
            if (hy > 0 && (!parse_count(id.substr(0, hy), lo) || lo <= 0)) bad();
            if (hy + 1 < id.size() && (!parse_count(id.substr(hy + 1), hi) || hi <= 0 || hi < lo))
              bad();
            if (level == 3) {
              if (lo <= 1 && hi >= 1) for_mol = true;
            } else if (level == 2 && for_mol) {
              for (int r = lo - 1; r < std::min(hi, nres); ++r) for_res[r] = 1;
            } else if (level == 1 && for_mol) {
              for (int r = 0; r < nres; ++r) {
                const int kv = c.res_var_count[r];
                if (!for_res[r] || kv <= 0) continue;
                for (int k = lo; k <= std::min(hi, kv); ++k) for_var[c.res_var_first[r] + k - 1] = 1;
              }
            }
          }
        }
      }
      double val = 0.0;
      if (!parse_value(fields.back(), val)) fail("redvar> Cannot read value from >" + cmd + "<");
      for (int v = 0; v < nvar; ++v)
        if (for_var[v]) {
          out.value[v] = val;
          out.fixed[v] = fix ? 1 : 0;
          out.set[v] = 1;
        }
    }
  }
  return out;
}

}  // namespace

// ---------------------------------------------------------------- angles
double difang(double a1, double a2) {
  const double d = std::fmod(a2 - a1, kTwoPi);
  return std::fabs(d) <= kPi ? d : d - std::copysign(kTwoPi, d);
}
double addang(double a1, double a2) {
  const double d = std::fmod(a1 + a2, kTwoPi);
  return std::fabs(d) <= kPi ? d : d - std::copysign(kTwoPi, d);
}

// ---------------------------------------------------------------- library
ResidueLibrary::ResidueLibrary(const std::string& path) : path_(path) {
  std::ifstream f(path);
  if (!f) fail("init_energy: cannot open residue library " + path);
  std::string l;
  while (std::getline(f, l)) {
    if (!l.empty() && l.back() == '\r') l.pop_back();
    lines_.push_back(l);
  }
  // Residue lines: '#', the name in columns 2-5, at least 13 columns.  The
  // first line of a name is the one used.
  for (size_t li = 0; li < lines_.size(); ++li) {
    const std::string& h = lines_[li];
    const size_t last = h.find_last_not_of(' ');
    if (h.empty() || h[0] != '#' || last == std::string::npos || last + 1 < 13) continue;
    const std::string nm = lower(column(h, 1, 4));
    if (!header_.count(nm)) header_[nm] = li;
  }
}

// Residue line: '#', name (4), atom count and link atom (2i4).  Atom line:
// name (a4), three (1x,i2,a1,a3,f9.3) groups for bond length, valence angle
// and dihedral (class, '*' when it is a variable, variable name, value),
// charge (f7.4), class (i4), parent and three bonds (4i4); a negative parent
// or bond only marks the bond order.
ResidueTemplate ResidueLibrary::parse(size_t li) const {
  const std::string& h = lines_[li];
  ResidueTemplate t;
  t.name = lower(column(h, 1, 4));
  const int nat = read_int(column(h, 5, 4));
  t.link = read_int(column(h, 9, 4)) - 1;
  if (nat <= 0 || li + (size_t)nat >= lines_.size())
    fail("redres> ERROR reading residue " + t.name + " in " + path_);
  if (t.link < 0 || t.link >= nat) fail("redres> bad link atom in residue " + t.name);
  for (int i = 0; i < nat; ++i) {
    const std::string& a = lines_[li + 1 + i];
    TemplateAtom at;
    at.name = column(a, 0, 4);
    double val[3];
    for (int k = 0; k < 3; ++k) {
      const size_t b = 4 + 16 * k;
      const int cls = read_int(column(a, b + 1, 2));
      const char fix = column(a, b + 3, 1)[0];
      const std::string vname = column(a, b + 4, 3);
      val[k] = read_real(column(a, b + 7, 9), 3);
      if (fix != ' ') {
        if (cls <= 0 || (k == 2 && cls > kMaxTorsionClass))
          fail("redres> unknown class for variable " + vname + " in residue " + t.name);
        TemplateVar v;
        v.kind = k + 1;
        v.cls = cls;
        v.atom = i;
        v.name = vname;
        t.vars.push_back(v);
      }
    }
    at.blen = val[0];
    at.bang = val[1] * kDegToRad;
    at.tors = val[2] * kDegToRad;
    at.charge = read_real(column(a, 52, 7), 4);
    at.type = read_int(column(a, 59, 4));
    if (at.type <= 0 || at.type > 18)
      fail("redres> unknown type for atom " + at.name + " in residue " + t.name);
    const int par = std::abs(read_int(column(a, 63, 4)));
    const bool ace_first = t.name.compare(0, 3, "ace") == 0 && i == 0;
    if (!ace_first && par > i)
      fail("redres> atom " + at.name + " of " + t.name + " should be placed AFTER atom #" +
           std::to_string(par));
    at.parent = par - 1;   // -1: first atom (ace's first atom names its first hydrogen)
    for (int k = 0; k < 3; ++k) {
      const int b = std::abs(read_int(column(a, 67 + 4 * k, 4)));
      if (b == 0) break;
      if (b == i + 1 || b == par)
        fail("redres> Incorrect order of bonds for atom " + at.name + " of " + t.name);
      at.bonds.push_back(b - 1);
    }
    t.atoms.push_back(at);
  }
  return t;
}

const ResidueTemplate& ResidueLibrary::get(const std::string& name) const {
  const std::string nm = lower(pad(name, 4));
  auto c = cache_.find(nm);
  if (c != cache_.end()) return c->second;
  auto it = header_.find(nm);
  if (it == header_.end()) fail("redres> residue >" + name + "< NOT FOUND in " + path_);
  return cache_.emplace(nm, parse(it->second)).first->second;
}

// ---------------------------------------------------------------- sequence
SequenceFile read_sequence(const std::string& path) {
  std::ifstream f(path);
  if (!f) fail("redseq> ERROR opening sequence file: " + path);
  std::vector<SequenceFile> mols;
  std::string line;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (trim(line).empty()) continue;
    const size_t hash = line.find('#');
    if (hash != std::string::npos) {   // a new molecule, named by the rest of the line
      if (!mols.empty() && mols.back().residues.empty()) mols.pop_back();
      SequenceFile m;
      m.name = trim(line.substr(hash + 1));
      if (m.name.size() > 80) m.name.resize(80);
      if (m.name.empty()) {
        char b[16];
        std::snprintf(b, sizeof b, "%4d", (int)(mols.size() % 10000) + 1);
        m.name = b;
      }
      mols.push_back(m);
      continue;
    }
    if (mols.empty()) mols.push_back({"   1", {}});
    size_t p = 0;
    while (p < line.size()) {
      while (p < line.size() && line[p] == ' ') ++p;
      if (p >= line.size()) break;
      size_t q = line.find(' ', p);
      if (q == std::string::npos) q = line.size();
      const std::string nm = line.substr(p, q - p);
      if (nm.size() > 4) fail("redseq> INVALID residue NAME >" + nm + "< in " + path);
      mols.back().residues.push_back(nm);
      p = q;
    }
  }
  if (!mols.empty() && mols.back().residues.empty()) mols.pop_back();
  if (mols.empty()) fail("redseq> no residues found in " + path);
  if (mols.size() != 1) fail("build_molecule: one molecule per sequence file");
  SequenceFile m = mols[0];
  if (lower(m.residues[0]).compare(0, 3, "pro") == 0) m.residues[0] = "pron";
  return m;
}

// ---------------------------------------------------------------- molecule
MolTopo build_topology(const ResidueLibrary& lib, const ForceField& ff, const BuildOptions& opt,
                       const std::string& seqfile, const std::string& varfile) {
  const SequenceFile sq = read_sequence(seqfile);
  const int nres = (int)sq.residues.size();
  const std::string gn = lower(opt.grpn), gc = lower(opt.grpc);
  if (gn.compare(0, 3, "ace") == 0 || gc.compare(0, 3, "ace") == 0 || gn.compare(0, 3, "nme") == 0 ||
      gc.compare(0, 3, "nme") == 0)
    fail("addend> N-Acetyl (ace) or N-Methylamide (nme) should be put in SEQUENCE file");

  // atoms of the whole chain
  std::vector<TemplateAtom> atoms;   // global indices
  std::vector<int> res_of_atom, res_first(nres), res_link(nres);
  std::vector<TemplateVar> vars;
  std::vector<int> res_var_first(nres), res_var_count(nres);
  for (int r = 0; r < nres; ++r) {
    const std::string nm = lower(pad(sq.residues[r], 4));
    if (nm.compare(0, 3, "nme") == 0 && r != nres - 1)
      fail("getmol> residue >" + nm + "< allowed at C-terminus only !");
    if (nm.compare(0, 3, "ace") == 0 && r != 0)
      fail("getmol> residue >" + nm + "< allowed at N-terminus only !");
    Piece p = piece_of(lib.get(nm));
    if (r == 0) {   // no variable of the first atom, no torsion about it
      std::vector<TemplateVar> keep;
      for (const TemplateVar& v : p.vars)
        if (!(v.atom == 0 || (v.kind == 3 && p.atoms[v.atom].parent == 0))) keep.push_back(v);
      p.vars = keep;
    }
    const std::string h3 = nm.substr(0, 3);
    if (r == 0 && h3 != "ace") {
      std::string s;
      if (gn.compare(0, 3, "nh2") == 0) {
        if (h3 == "hyp") {
          if (!opt.sh2) fail("addend> No N-terminal Hyp possible with ECEPP/3 dataset");
          s = "nh2+";
        } else if (h3 == "pro") {
          s = "nh1 ";
        } else if (h3 == "gly") {
          s = opt.sh2 ? "nh2 " : "nh2g";
        } else {
          s = "nh2 ";
        }
      } else if (pad(gn, 4) == "nh3+") {
        s = h3 == "pro" ? "nh2+" : (h3 == "gly" ? "nh3g" : "nh3+");
      } else {
        fail("addend> Can add only nh2 or nh3+ to N-terminus");
      }
      put_n_terminus(p, lib.get(s), opt.sh2);
    }
    if (r == nres - 1 && h3 != "nme") {
      std::string s;
      if (pad(gc, 4) == "cooh")
        s = (h3 == "gly" && !opt.sh2) ? "gooh" : "cooh";
      else if (pad(gc, 4) == "coo-")
        s = (h3 == "gly" && !opt.sh2) ? "goo-" : "coo-";
      else
        fail("addend> Can add only cooh or coo- to C-terminus");
      put_c_terminus(p, lib.get(s), opt.sh2);
    }
    const int base = (int)atoms.size();
    res_first[r] = base;
    res_link[r] = base + p.link;
    for (size_t i = 0; i < p.atoms.size(); ++i) {
      TemplateAtom a = p.atoms[i];
      for (int& b : a.bonds) b += base;
      if (i == 0) {
        if (r == 0) {
          a.parent = -1;
          if (p.atoms[0].parent > 0) a.bonds.insert(a.bonds.begin(), base + p.atoms[0].parent);
        } else {
          // bonded to the previous residue's link atom; the dihedrals of
          // atoms already bonded there are phases relative to this one
          const int nh = res_link[r - 1];
          for (int nj : atoms[nh].bonds) {
            if (atoms[nj].tors == 0.0)
              fail("getmol> DIHEDRAL for atom " + atoms[nj].name + " should be a PHASE angle");
            double t = atoms[nj].tors + a.tors;
            if (std::fabs(t) > kPi) t -= std::copysign(kTwoPi, t);
            atoms[nj].tors = t;
          }
          if (atoms[nh].bonds.size() >= 3) fail("getmol> need a 4th bond to connect residues");
          atoms[nh].bonds.push_back(base);
          a.parent = nh;
        }
      } else {
        a.parent += base;
      }
      atoms.push_back(a);
      res_of_atom.push_back(r);
    }
    res_var_first[r] = (int)vars.size();
    for (TemplateVar v : p.vars) {
      if (v.kind != 3) fail("build_molecule: only torsion variables exist in the ECEPP libraries");
      v.atom += base;
      vars.push_back(v);
    }
    res_var_count[r] = (int)vars.size() - res_var_first[r];
  }
  const int n = (int)atoms.size();
  const int nv = (int)vars.size();
  if (n > kMaxAtoms) fail("build_molecule: more atoms than the packed pair words hold");

  // tree: children and subtree ends (atoms of a subtree are consecutive)
  std::vector<std::vector<int>> children(n);
  for (int i = 1; i < n; ++i) {
    if (atoms[i].parent < 0 || atoms[i].parent >= i) fail("build_molecule: atom built before its parent");
    children[atoms[i].parent].push_back(i);
  }
  std::vector<int> sub_end(n), sub_size(n, 1);
  for (int i = n - 1; i >= 0; --i) {
    sub_end[i] = i;
    for (int c : children[i]) {
      sub_end[i] = std::max(sub_end[i], sub_end[c]);
      sub_size[i] += sub_size[c];
    }
    if (sub_end[i] - i + 1 != sub_size[i]) fail("build_molecule: a branch is not a run of atoms");
  }

  // variable file
  std::vector<char> fixed(nv, 0);
  double gbpr[6] = {0, 0, 0, 0, 0, 0};
  auto set_torsions = [&](const std::vector<double>& target) {   // setvar.f:40-56
    for (int v = 0; v < nv; ++v) {
      const int base = atoms[vars[v].atom].parent;
      const double shift = difang(atoms[vars[v].atom].tors, target[v]);
      for (int c : children[base]) {
        double t = atoms[c].tors + shift;
        if (std::fabs(t) > kPi) t -= std::copysign(kTwoPi, t);
        atoms[c].tors = t;
      }
    }
  };
  if (!trim(varfile).empty()) {
    VarFileContext ctx;
    ctx.mol_name = sq.name;
    ctx.res_names = sq.residues;
    ctx.res_var_first = res_var_first;
    ctx.res_var_count = res_var_count;
    for (const TemplateVar& v : vars) ctx.var_names.push_back(v.name);
    const VarSettings vs = read_var_file(varfile, ctx);
    std::vector<double> target(nv);
    bool any_set = false;
    for (int v = 0; v < nv; ++v) {
      target[v] = vs.set[v] ? vs.value[v] : atoms[vars[v].atom].tors;
      fixed[v] = vs.fixed[v];
      any_set = any_set || vs.set[v];
    }
    bool any_gbpr = false;
    for (int k = 0; k < 6; ++k) {
      gbpr[k] = vs.gbpr[k];
      any_gbpr = any_gbpr || gbpr[k] != 0.0;
    }
    // The reference applies the variables once before converting the values
    // it read to radians when global parameters are given (redvar.f:557-567),
    // and once after; the second pass sets every target, the first only
    // leaves its rounding in the phases.
    if (any_gbpr) set_torsions(target);
    if (any_set) {
      for (int v = 0; v < nv; ++v)
        if (vs.set[v]) target[v] = vs.value[v] * kDegToRad;
      set_torsions(target);
    }
  }

  // ---- flattened topology
  MolTopo t;
  t.natoms = n;
  t.nvar = nv;
  t.i1 = 0;
  t.i2 = children[0].empty() ? -1 : *std::max_element(children[0].begin(), children[0].end());
  if (t.i2 < 0) fail("fnd3ba> the first atom has no following atom");
  {
    const int link0 = res_link[0];
    t.i3 = -1;
    if (t.i2 == link0) {
      if (nres > 1) t.i3 = res_first[1];
    } else {
      for (int i = link0; i > t.i2; --i)
        if (atoms[i].parent == t.i2) {
          t.i3 = i;
          break;
        }
    }
    if (t.i3 < 0) fail("fnd3ba> Cannot find the third backbone atom");
  }
  for (int k = 0; k < 6; ++k) t.gbpr[k] = gbpr[k];
  t.iow.resize(n);
  t.type.resize(n);
  t.charge.resize(n);
  t.blen.resize(n);
  t.cba.resize(n);
  t.sba.resize(n);
  t.toat0.resize(n);
  t.rvdw.assign(n, 0.0);
  t.sigma.assign(n, 0.0);
  t.atom_name.resize(n);
  t.residue_of_atom = res_of_atom;
  for (int i = 0; i < n; ++i) {
    const TemplateAtom& a = atoms[i];
    t.iow[i] = a.parent;
    t.type[i] = uint8_t(a.type - 1);
    t.charge[i] = a.charge;
    t.blen[i] = a.blen;
    t.cba[i] = std::cos(a.bang);
    t.sba[i] = std::sin(a.bang);
    t.toat0[i] = a.tors;
    t.atom_name[i] = a.name;
    if (ff.itysol != 0) {   // init_molecule.f:194-210
      t.sigma[i] = ff.sol_sigma.at(a.type);
      t.rvdw[i] = ff.sol_radius.at(a.type);
      if (a.name[0] != 'h') t.rvdw[i] += ff.probe;
    }
    if (t.rvdw[i] > 0.0) t.heavy.push_back(i);
  }
  t.nres = nres;
  // bonded partners after each atom (outpdb.f:137-176); the first atom lists
  // all of its partners when it has more than one
  t.conect_off.assign(1, 0);
  for (int r = 0; r < nres; ++r) {
    t.res_name.push_back(pad(sq.residues[r], 4));
    t.res_atom0.push_back(res_first[r]);
  }
  for (int i = 0; i < n; ++i) {
    const bool listed = (i == 0) ? atoms[0].bonds.size() >= 2 : !atoms[i].bonds.empty();
    if (listed)
      for (int b : atoms[i].bonds)
        if (b > i) t.conect.push_back(b);
    t.conect_off.push_back((int)t.conect.size());
  }
  // depth levels (every atom but the first is placed from its parent)
  std::vector<int> depth(n, 0);
  int maxd = 0;
  for (int i = 1; i < n; ++i) maxd = std::max(maxd, depth[i] = depth[atoms[i].parent] + 1);
  t.level_off.assign(maxd + 2, 0);
  for (int i = 0; i < n; ++i) t.level_off[depth[i] + 1]++;
  for (int d = 0; d <= maxd; ++d) t.level_off[d + 1] += t.level_off[d];
  t.level_atoms.assign(n, 0);
  {
    std::vector<int> fill(t.level_off.begin(), t.level_off.end() - 1);
    for (int i = 0; i < n; ++i) t.level_atoms[fill[depth[i]]++] = i;
  }
  // variables: the base's children turn; their subtrees form one run.  A
  // base carries one torsion (setmvs.f:15-17): the sweep relies on it, since
  // a variable's replayed setvar then moves no other variable's atom.
  {
    std::vector<int> seen(n, -1);
    for (int v = 0; v < nv; ++v) {
      const int base = atoms[vars[v].atom].parent;
      if (seen[base] >= 0) fail("setmvs> two torsion variables turn about one base atom");
      seen[base] = v;
    }
  }
  std::vector<int> axis_o(nv);
  t.sib_off.push_back(0);
  for (int v = 0; v < nv; ++v) {
    const TemplateVar& var = vars[v];
    const int base = atoms[var.atom].parent;
    if (base == 0) fail("build_molecule: a variable turns about the first backbone atom");
    axis_o[v] = atoms[base].parent;
    int lo = n, hi = -1, count = 0;
    for (int c : children[base]) {
      t.sib.push_back(c);
      lo = std::min(lo, c);
      hi = std::max(hi, sub_end[c]);
      count += sub_size[c];
    }
    if (hi - lo + 1 != count) fail("setmvs> Cannot combine disjunct ranges of atoms for " + var.name);
    t.sib_off.push_back((int)t.sib.size());
    t.var_atom.push_back(var.atom);
    t.var_base.push_back(base);
    t.var_lo.push_back(lo);
    t.var_hi.push_back(hi);
    t.var_class.push_back(var.cls);
    t.var_e0.push_back(ff.tor_e0.at(var.cls));
    t.var_sg.push_back(ff.tor_sg.at(var.cls));
    t.var_rn.push_back(ff.tor_rn.at(var.cls));
    t.var_fixed.push_back(fixed[v]);
    t.axvr.push_back(fixed[v] ? 0.0 : kTwoPi);   // init_molecule.f:152-186
    t.vlvr0.push_back(atoms[var.atom].tors);
    t.var_name.push_back(pad(var.name, 3));
    int rv = 0;
    while (rv + 1 < nres && v >= res_var_first[rv + 1]) ++rv;
    t.var_residue.push_back(rv);
    if (!fixed[v]) t.idvr.push_back(v);
  }
  t.nfree = (int)t.idvr.size();

  // ---- pair set.  Every atom belongs to the rigid group of the innermost
  // variable whose range holds it (none: the group of the first atom); a
  // group's key is the first atom of that range.  An atom of a group with
  // variable v pairs with every atom of a group with a smaller key except
  // the two atoms on v's axis: exactly the pairs whose distance some
  // variable changes (the geometric check in the tests).  Its 1-4 partners
  // (mklist.f:96-207) are the atoms that hold the axis's outer atom o: o's
  // other children with the rest of their contiguous same-group runs, o's
  // parent, and the run of the base's own group.
  std::vector<int> own(n, -1), key(n, -1), own_len(n, n + 1);
  for (int v = 0; v < nv; ++v) {
    const int lo = t.var_lo[v], hi = t.var_hi[v];
    for (int i = lo; i <= hi; ++i)
      if (hi - lo < own_len[i]) {
        own_len[i] = hi - lo;
        own[i] = v;
        key[i] = lo;
      }
  }
  std::vector<int> run_lo(n), run_hi(n);   // maximal runs of one group
  for (int i = 0; i < n; ++i)
    run_lo[i] = (i > 0 && own[i - 1] == own[i]) ? run_lo[i - 1] : i;
  for (int i = n - 1; i >= 0; --i)
    run_hi[i] = (i + 1 < n && own[i + 1] == own[i]) ? run_hi[i + 1] : i;
  std::vector<std::vector<int>> members(nv);
  for (int i = 0; i < n; ++i)
    if (own[i] >= 0) members[own[i]].push_back(i);
  std::vector<char> is14(n, 0);
  for (int v = 0; v < nv; ++v) {
    if (members[v].empty()) continue;
    const int b = t.var_base[v], o = axis_o[v], kv = t.var_lo[v];
    auto avail = [&](int j) { return j >= 0 && key[j] < kv && j != b && j != o; };
    std::vector<int> ext;
    auto take = [&](int j) {
      if (avail(j) && !is14[j]) {
        is14[j] = 1;
        ext.push_back(j);
      }
    };
    auto take_run = [&](int a) {
      if (own[a] < 0) return;
      for (int j = run_lo[a]; j <= run_hi[a]; ++j) take(j);
    };
    // o's following bonds (the first atom's first bond stands for its parent)
    const std::vector<int>& ob = atoms[o].bonds;
    std::vector<int> sibs;
    for (size_t k = (o == 0 ? 1 : 0); k < ob.size(); ++k)
      if (ob[k] != b && atoms[ob[k]].parent == o && avail(ob[k]) && !is14[ob[k]]) {
        take(ob[k]);
        sibs.push_back(ob[k]);
      }
    for (int c : sibs) take_run(c);
    const int up = (o == 0) ? (ob.empty() ? -1 : ob[0]) : atoms[o].parent;
    take(up);
    take_run(b);
    std::vector<int> normal, one4;
    for (int j = 0; j < n; ++j)
      if (avail(j)) (is14[j] ? one4 : normal).push_back(j);
    for (int i : members[v]) {
      for (size_t k = 0; k < normal.size();) {   // runs of consecutive partners
        size_t e = k;
        while (e + 1 < normal.size() && normal[e + 1] == normal[e] + 1) ++e;
        for (int j0 = normal[k]; j0 <= normal[e]; j0 += kChunk) {
          const int len = std::min(kChunk, normal[e] - j0 + 1);
          t.chunks.push_back(uint32_t(i) | (uint32_t(j0) << 14) | (uint32_t(len - 1) << 28));
          t.npairs += len;
        }
        k = e + 1;
      }
      for (int j : one4) {
        t.pairs14.push_back(uint32_t(i) | (uint32_t(j) << 14));
        t.npairs += 1;
      }
    }
    for (int j : ext) is14[j] = 0;
  }
  // chunk and 1-4 words in atom order of the listing atom
  auto by_atom = [](uint32_t x, uint32_t y) { return (x & 0x3fffu) < (y & 0x3fffu); };
  std::stable_sort(t.chunks.begin(), t.chunks.end(), by_atom);
  std::stable_sort(t.pairs14.begin(), t.pairs14.end(), by_atom);
  // the dense list: every pair once, by listing atom, then partner
  {
    std::vector<uint64_t> keyed;
    keyed.reserve((size_t)t.npairs);
    for (uint32_t w : t.chunks) {
      const uint32_t i = w & 0x3fffu, j0 = (w >> 14) & 0x3fffu, len = ((w >> 28) & 7u) + 1;
      for (uint32_t j = j0; j < j0 + len; ++j) keyed.push_back(((uint64_t)i << 32) | (j << 1));
    }
    for (uint32_t w : t.pairs14)
      keyed.push_back(((uint64_t)(w & 0x3fffu) << 32) | ((w >> 14) << 1) | 1u);
    std::sort(keyed.begin(), keyed.end());
    t.flat.reserve(keyed.size());
    for (uint64_t k : keyed)
      t.flat.push_back(uint32_t(k >> 32) | (uint32_t((k & 0xffffffffu) >> 1) << 14) |
                       (uint32_t(k & 1u) << 28));
  }
  // pair kind per unordered pair: 0 none, 1 one-four, 2 normal
  if ((long long)n * n > (1ll << 26)) fail("build_molecule: molecule too large for the pair table");
  std::vector<uint8_t> cnt((size_t)n * n, 0);
  for (uint32_t w : t.chunks) {
    const int i = int(w & 0x3fffu), j0 = int((w >> 14) & 0x3fffu), len = int((w >> 28) & 7u) + 1;
    for (int j = j0; j < j0 + len; ++j) cnt[(size_t)std::min(i, j) * n + std::max(i, j)] = 2;
  }
  for (uint32_t w : t.pairs14) {
    const int i = int(w & 0x3fffu), j = int(w >> 14);
    cnt[(size_t)std::min(i, j) * n + std::max(i, j)] = 1;
  }
  // pairs across each variable's bond (exactly one atom in its range): the
  // pair terms an incremental proposal sums before and after the move
  {
    std::vector<std::pair<int, int>> pl;
    pl.reserve((size_t)t.npairs);
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (cnt[(size_t)i * n + j]) pl.emplace_back(i, j);
    for (int v = 0; v < nv; ++v) {
      const int lo = t.var_lo[v], hi = t.var_hi[v];
      int c = 0;
      for (const auto& q : pl) c += ((q.first >= lo && q.first <= hi) != (q.second >= lo && q.second <= hi));
      t.var_cross.push_back(c);
    }
  }
  // the same, as indices into the dense list, for each free variable, less
  // the pairs with an atom on the variable's axis (their distance does not
  // change when the range turns about that axis)
  t.cross_off.assign(nv + 1, 0);
  if (t.flat.size() <= 65535) {
    std::vector<char> is_free(nv, 0);
    for (int v : t.idvr) is_free[v] = 1;
    for (int v = 0; v < nv; ++v) {
      t.cross_off[v] = (int)t.cross_idx.size();
      if (!is_free[v]) continue;
      const int lo = t.var_lo[v], hi = t.var_hi[v], b = t.var_base[v], a = t.iow[b];
      for (size_t k = 0; k < t.flat.size(); ++k) {
        const int i = int(t.flat[k] & 0x3fffu), j = int((t.flat[k] >> 14) & 0x3fffu);
        if (i == a || i == b || j == a || j == b) continue;
        if ((i >= lo && i <= hi) != (j >= lo && j <= hi)) t.cross_idx.push_back((uint16_t)k);
      }
    }
    t.cross_off[nv] = (int)t.cross_idx.size();
  }
  // the same pair set by rows (every pair once, 1-4 pairs within the window)
  t.near_mask.assign(n, 0);
  t.near14.assign(n, 0);
  bool ok = true;
  for (int i = 0; i < n && ok; ++i)
    for (int j = i + 1; j < n; ++j) {
      const uint8_t c = cnt[(size_t)i * n + j];
      const int d = j - i;
      if (d <= kNearWindow) {
        if (c == 1) t.near14[i] |= 1ull << (d - 1);
        if (c >= 2) t.near_mask[i] |= 1ull << (d - 1);
      } else if (c != 2) {
        ok = false;   // a distant pair that is not a normal pair
        break;
      }
    }
  t.rows_ok = ok && n <= 4096;
  return t;
}

}  // namespace smmpb200
