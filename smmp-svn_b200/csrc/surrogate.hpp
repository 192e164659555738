// Learned energy surrogate: a per-sequence MLP on the sin/cos of the free
// dihedrals (3 hidden layers of 256, SiLU), BF16 weights with FP32
// accumulation, trained on the GPU with the project's own tensor-core
// kernels (mma.sync m16n8k16 BF16, FP32 accumulators) and Adam.  It has no
// counterpart in the reference; the sweep uses it as the first stage of a
// two-stage (delayed-acceptance) Metropolis step.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device.cuh"

namespace smmpb200 {

constexpr int kHidden = 256;
// Size of the fixed scratch array of Surrogate::predict_noalloc (held by
// every GPU that loads the library, until the process exits).
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;

// Offsets (in floats) of the parameters in the flat FP32 vector, for an
// input width nin_pad (a multiple of 16):
//   W1 [nin_pad][H], b1 [H], W2 [H][H], b2 [H], W3 [H][H], b3 [H], w4 [H], b4 [1].
struct MlpLayout {
  int nin = 0, nin_pad = 0;
  size_t w1 = 0, b1 = 0, w2 = 0, b2 = 0, w3 = 0, b3 = 0, w4 = 0, b4 = 0, n = 0;
  explicit MlpLayout(int nin_ = 0);
};

class Surrogate {
 public:
  Surrogate(int nang, uint64_t seed);
  ~Surrogate();
  Surrogate(const Surrogate&) = delete;
  Surrogate& operator=(const Surrogate&) = delete;

  int nang() const { return nang_; }
  int device() const { return device_; }   // the GPU that holds the parameters
  const MlpLayout& layout() const { return L_; }
  void set_stream(cudaStream_t s) { stream_ = s; }

  // Training set: n conformations of nang free dihedrals (radians, FP64) and
  // their energies.  Energies above `clip` are clipped; targets are
  // normalised by the set's mean and standard deviation.
  void set_data(const double* ang, const double* energy, int n, double clip);
  // Minibatch Adam over the training set; returns the mean squared error (in
  // normalised units) of the last epoch.
  double train(int epochs, int batch, double lr, uint64_t shuffle_seed);
  // Batched forward pass (tensor-core GEMMs); energies in kcal/mol.
  void predict(const double* ang, int n, double* out);
  // Loss and gradients of one batch (no update), in normalised units:
  // loss = mean (y - t)^2 with t = (clip(E) - mu) / sigma.
  double gradients(const double* ang, const double* energy, int n, float* grad_out);
  void get_params(float* out) const;
  void set_params(const float* in);
  void set_norm(float mu, float sigma) { mu_ = mu, sigma_ = sigma; }
  float mu() const { return mu_; }
  float sigma() const { return sigma_; }
  // Device view for the sweep kernels (builds the transposed weight copies).
  DSurrogate device_view();
  // Forward pass that allocates nothing (for callers that cannot allocate
  // device memory): device-resident inputs and outputs, scratch in a fixed
  // file-scope device array (kNoAllocScratchBytes).  The surrogate's own GPU
  // (device()) must be current; another current device is rejected with
  // std::invalid_argument before anything is launched.  See surrogate.cu.
  void predict_noalloc(const float* ang_dev, int n, double* energy_dev, cudaStream_t st) const;
  static int noalloc_max_rows(int nin_pad);

 private:
  void ensure_scratch(int batch);
  void upload_angles(const double* ang, int n, float* dst);
  void forward(int B, const float* ang, const int* idx);
  double backward(int B, const float* target, const int* tidx, bool accumulate_loss);
  void refresh_bf16();
  void sync();

  int nang_;
  int device_ = 0;
  MlpLayout L_;
  cudaStream_t stream_ = nullptr;
  float mu_ = 0.f, sigma_ = 1.f;
  double clip_ = 1e30;
  // parameters: FP32 master, Adam moments, gradients, BF16 copies of weights
  float *P_ = nullptr, *G_ = nullptr, *M_ = nullptr, *V_ = nullptr;
  __nv_bfloat16* Wb_ = nullptr;   // W1 | W2 | W3 | w4
  __nv_bfloat16* Wt_ = nullptr;   // W1^T | W2^T | W3^T ([256][K] each)
  size_t wb1_ = 0, wb2_ = 0, wb3_ = 0, wb4_ = 0, nwb_ = 0;
  long long step_ = 0;
  // training set
  float* ang_ = nullptr;   // [n][nang]
  float* tgt_ = nullptr;   // [n], normalised
  int ndata_ = 0;
  // scratch for one batch
  int cap_ = 0;
  __nv_bfloat16 *X_ = nullptr, *H1_ = nullptr, *H2_ = nullptr, *H3_ = nullptr, *dA_ = nullptr,
                *dB_ = nullptr;
  float *Z1_ = nullptr, *Z2_ = nullptr, *Z3_ = nullptr, *y_ = nullptr, *dy_ = nullptr,
        *loss_ = nullptr, *tbuf_ = nullptr, *abuf_ = nullptr;
  int* idx_ = nullptr;
};

}  // namespace smmpb200
