// Multicanonical weight recursion of mulcan_par (mulcan_par_mod.f90), host
// side; see muca.cpp.
#pragma once

namespace smmpb200 {

struct MucaBins {
  int kmin, kmax;   // energy bins kmin..kmax of width ebin
  double ebin;
  double beta;      // 1 / (k_B T) of the run
};

// One update from the histogram ihist of the last nup sweeps (then zeroed):
// xhist, g1, b, alpha, ent as mulcan_par keeps them (mulcan_par_mod.f90:93-145).
void muca_update(const MucaBins& q, int* ihist, double* xhist, double* g1, double* b,
                 double* alpha, double* ent);
// The weights written at the end of the run (mulcan_par_mod.f90:163-168):
// beta folded into b, alpha recomputed, for muca_weight2.
void muca_finish(const MucaBins& q, double* b, double* alpha);

}  // namespace smmpb200
