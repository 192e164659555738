// Text output of a molecule: outvar and outpdb formats (see topology.hpp).
#include "topology.hpp"

#include <algorithm>
#include <cstdio>
#include <string>
#include <cmath>
#include <stdexcept>

namespace smmpb200 {

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
