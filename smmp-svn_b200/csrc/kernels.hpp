// Launch wrappers of the sm_100a kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"

namespace smmpb200 {

size_t sweep_smem_bytes(const DMolSet& set);
// Shared-memory pool a molecule needs when its topology is staged.
size_t stage_bytes_of(const DMol& d, bool lists);

cudaError_t launch_seed(uint32_t* mt, const int* seeds, int nslots, cudaStream_t st);
cudaError_t launch_draw(uint32_t* mt, int slot, int n, double* out, cudaStream_t st);
cudaError_t launch_random_start(const DMolSet& set, const DChains& ch, const int* order, int n,
                                cudaStream_t st);
cudaError_t launch_energy(const DMolSet& set, const DChains& ch, int first, int count, bool fp32,
                          cudaStream_t st);
cudaError_t launch_sweep(const DMolSet& set, const DChains& ch, const DWeight& w, int first,
                         int count, int nsweeps, int flags, double check_tol, cudaStream_t st);
// Fused parallel tempering: nsweeps rounds of (one sweep of every chain, one
// exchange) in one cooperative launch over chains [0, count).
cudaError_t launch_sweep_pt(const DMolSet& set, const DChains& ch, const DWeight& w, int count,
                            int nsweeps, int flags, double check_tol, const DPTFused& pt,
                            cudaStream_t st);
// Metropolis steps of the analytic SASA model, driven from the host: the
// proposal p of chains [first, first+n), the decision after its energy(),
// the closing check; eolc holds the tracked energies.
cudaError_t launch_propose(const DMolSet& set, const DChains& ch, int first, int n, int p,
                           int rndord, double* vold, int* jvar, cudaStream_t st);
cudaError_t launch_decide(const DChains& ch, const DWeight& w, int first, int n,
                          const double* vold, const int* jvar, double* eolc, cudaStream_t st);
cudaError_t launch_close(const DChains& ch, int first, int n, const double* eolc, int check,
                         double check_tol, cudaStream_t st);
cudaError_t launch_copy_eol(const DChains& ch, int first, int n, double* eolc, cudaStream_t st);
// Analytic SASA (esolan.cu): k_esolan over chains [first, first+count) adds
// eysl to eol and terms; ch.coords must hold the chains' rebuilt coordinates.
// scratch: esolan_scratch_bytes(count); area: nchains * tstride doubles.
constexpr int kEsolanBatch = 16;
size_t esolan_scratch_bytes(int count);
cudaError_t launch_esolan(const DMolSet& set, const DChains& ch, int first, int count,
                          double* scratch, double* area, cudaStream_t st);
// gradient.f / opeshe.f: dE/dv of every variable of chains [first,
// first+count) into grad[chain * vstride + v], energies into ch.eol/terms.
cudaError_t launch_gradient(const DMolSet& set, const DChains& ch, int first, int count,
                            double* grad, cudaStream_t st);
cudaError_t launch_exchange(const DChains& ch, int* temp_chain, const double* betas, int n,
                            uint32_t* mt, int* iswitch, int wrap, unsigned long long* stats,
                            cudaStream_t st);

// The sweeps of the 384-thread build of kernels.cu (small molecules: less
// register spilling per thread, and their pair work needs no more warps).
namespace t384 {
size_t sweep_smem_bytes(const DMolSet& set);
cudaError_t launch_sweep(const DMolSet& set, const DChains& ch, const DWeight& w, int first,
                         int count, int nsweeps, int flags, double check_tol, cudaStream_t st);
cudaError_t launch_sweep_pt(const DMolSet& set, const DChains& ch, const DWeight& w, int count,
                            int nsweeps, int flags, double check_tol, const DPTFused& pt,
                            cudaStream_t st);
}  // namespace t384

}  // namespace smmpb200
