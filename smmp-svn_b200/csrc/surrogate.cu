// Surrogate MLP: tensor-core GEMMs (mma.sync m16n8k16, BF16 in, FP32
// accumulate) with fused bias/SiLU epilogues, the output layer, MSE loss,
// backward pass and Adam.  See surrogate.hpp.
#include "surrogate.hpp"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>

namespace smmpb200 {

using bf16 = __nv_bfloat16;

void check_cuda(cudaError_t e, const char* what);   // runtime.cu

MlpLayout::MlpLayout(int nin_) : nin(nin_), nin_pad((nin_ + 15) / 16 * 16) {
  const size_t H = kHidden;
  w1 = 0;
  b1 = w1 + (size_t)nin_pad * H;
  w2 = b1 + H;
  b2 = w2 + H * H;
  w3 = b2 + H;
  b3 = w3 + H * H;
  w4 = b3 + H;
  b4 = w4 + H;
  n = b4 + 1;
}

namespace {

constexpr int BM = 64, BN = 64, BK = 32, PADK = 8, GT = 128;

__device__ __forceinline__ float sigm(float z) { return 1.f / (1.f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigm(z);
  return s * (1.f + z * (1.f - s));
}

__device__ __forceinline__ uint32_t ld32(const bf16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}

__device__ __forceinline__ void mma16816(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

enum { kEpiHidden = 0, kEpiStore = 1, kEpiSiluGrad = 2 };

// C[M][N] = A[M][K] * B[K][N] on a 64x64 tile per block (4 warps of 32x32),
// K in steps of 32.  LA = 0: A stored [M][K] (row stride lda); LA = 1: A
// stored [K][M].  LB = 0: B stored [K][N]; LB = 1: B stored [N][K].  Tiles are
// staged in shared memory as [m][k] and [n][k] (K contiguous) whatever the
// global layout, and read as mma fragments.  Epilogues:
//   kEpiHidden:   Zf = acc + bias[n]; Cb = bf16(silu(Zf))      (forward layer)
//   kEpiStore:    Cf += acc (atomic; K may be split over gridDim.z)  (weight gradient)
//   kEpiSiluGrad: Cb = bf16(acc * silu'(Zp))                    (backward layer)
template <int LA, int LB, int EPI>
__global__ void __launch_bounds__(GT) k_gemm(int M, int N, int K, const bf16* __restrict__ A,
                                             int lda, const bf16* __restrict__ B, int ldb,
                                             const float* __restrict__ bias,
                                             const float* __restrict__ Zp, float* Cf, bf16* Cb,
                                             int ldc) {
  __shared__ __align__(16) bf16 As[BM][BK + PADK];
  __shared__ __align__(16) bf16 Bs[BN][BK + PADK];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kchunk = (K + gridDim.z * BK - 1) / (gridDim.z * BK) * BK;
  const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
  const bf16 zero = __float2bfloat16(0.f);
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    for (int e = tid; e < BM * BK; e += GT) {
      int r, c;
      if (LA == 0) {
        r = e / BK;
        c = e % BK;
      } else {
        c = e / BM;
        r = e % BM;
      }
      const int gm = m0 + r, gk = k0 + c;
      bf16 v = zero;
      if (gm < M && gk < kend) v = LA == 0 ? A[(size_t)gm * lda + gk] : A[(size_t)gk * lda + gm];
      As[r][c] = v;
    }
    for (int e = tid; e < BN * BK; e += GT) {
      int r, c;
      if (LB == 1) {
        r = e / BK;
        c = e % BK;
      } else {
        c = e / BN;
        r = e % BN;
      }
      const int gn = n0 + r, gk = k0 + c;
      bf16 v = zero;
      if (gn < N && gk < kend) v = LB == 1 ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
      Bs[r][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t a[2][4], b[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int r = wm * 32 + mt * 16 + g;
        a[mt][0] = ld32(&As[r][kk + 2 * t]);
        a[mt][1] = ld32(&As[r + 8][kk + 2 * t]);
        a[mt][2] = ld32(&As[r][kk + 2 * t + 8]);
        a[mt][3] = ld32(&As[r + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int c = wn * 32 + nt * 8 + g;
        b[nt][0] = ld32(&Bs[c][kk + 2 * t]);
        b[nt][1] = ld32(&Bs[c][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma16816(acc[mt][nt], a[mt], b[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int r = m0 + wm * 32 + mt * 16 + g + 8 * h;
          const int c = n0 + wn * 32 + nt * 8 + 2 * t + q;
          if (r >= M || c >= N) continue;
          const float v = acc[mt][nt][2 * h + q];
          const size_t o = (size_t)r * ldc + c;
          if (EPI == kEpiHidden) {
            const float z = v + bias[c];
            Cf[o] = z;
            Cb[o] = __float2bfloat16(silu(z));
          } else if (EPI == kEpiStore) {
            atomicAdd(&Cf[o], v);
          } else {
            Cb[o] = __float2bfloat16(v * dsilu(Zp[o]));
          }
        }
}

// X[b][2k], X[b][2k+1] = sin, cos of dihedral k of conformation idx[b]
// (b itself when idx is null); columns past 2*nang are zero.
__global__ void k_features(const float* __restrict__ ang, const int* __restrict__ idx, int B,
                           int nang, int nin_pad, bf16* __restrict__ X) {
  const int b = blockIdx.x;
  if (b >= B) return;
  const size_t src = (size_t)(idx ? idx[b] : b) * nang;
  for (int c = threadIdx.x; c < nin_pad; c += blockDim.x) {
    float v = 0.f;
    if (c < 2 * nang) {
      float sn, cs;
      sincosf(ang[src + (c >> 1)], &sn, &cs);
      v = (c & 1) ? cs : sn;
    }
    X[(size_t)b * nin_pad + c] = __float2bfloat16(v);
  }
}

// y[b] = H3[b] . w4 + b4 (one warp per row).
__global__ void k_out_fwd(int B, const bf16* __restrict__ H3, const bf16* __restrict__ w4,
                          const float* __restrict__ b4, float* __restrict__ y) {
  const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= B) return;
  float s = 0.f;
  for (int n = lane; n < kHidden; n += 32)
    s += __bfloat162float(H3[(size_t)b * kHidden + n]) * __bfloat162float(w4[n]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[b] = s + b4[0];
}

// Loss and output-layer backward: dy[b] = 2 (y - t) / B, loss += (y - t)^2,
// dZ3[b][n] = bf16(dy w4[n] silu'(Z3[b][n])).
__global__ void k_out_bwd(int B, const float* __restrict__ y, const float* __restrict__ tall,
                          const int* __restrict__ tidx, const bf16* __restrict__ w4,
                          const float* __restrict__ Z3, bf16* __restrict__ dZ3,
                          float* __restrict__ dy, float* loss) {
  const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= B) return;
  const float tb = tall[tidx ? tidx[b] : b];
  const float d = y[b] - tb;
  const float g = 2.f * d / (float)B;
  if (lane == 0) {
    dy[b] = g;
    atomicAdd(loss, d * d);
  }
  for (int n = lane; n < kHidden; n += 32) {
    const size_t o = (size_t)b * kHidden + n;
    dZ3[o] = __float2bfloat16(g * __bfloat162float(w4[n]) * dsilu(Z3[o]));
  }
}

// out[n] += sum over rows b of D[b][n] * (w ? w[b] : 1), rows split over blocks.
template <class T>
__global__ void k_colsum(int B, int N, const T* __restrict__ D, const float* __restrict__ w,
                         float* __restrict__ out) {
  const int n = threadIdx.x;
  if (n >= N) return;
  const int r0 = blockIdx.x * 256, r1 = min(B, r0 + 256);
  float s = 0.f;
  for (int b = r0; b < r1; ++b) {
    float v;
    if constexpr (sizeof(T) == 2)
      v = __bfloat162float(D[(size_t)b * N + n]);
    else
      v = (float)D[(size_t)b * N + n];
    s += w ? v * w[b] : v;
  }
  atomicAdd(&out[n], s);
}

__global__ void k_adam(size_t n, float* __restrict__ P, const float* __restrict__ G,
                       float* __restrict__ M, float* __restrict__ V, float lr, float b1, float b2,
                       float eps, float bc1, float bc2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
  }
}

// dst[n][k] = bf16(src[k][n]) for a [K][256] FP32 matrix.
__global__ void k_transpose_bf16(int K, const float* __restrict__ src, bf16* __restrict__ dst) {
  const int n = blockIdx.x, k0 = threadIdx.x;
  for (int k = k0; k < K; k += blockDim.x)
    dst[(size_t)n * K + k] = __float2bfloat16(src[(size_t)k * kHidden + n]);
}

__global__ void k_to_bf16(size_t n, const float* __restrict__ src, bf16* __restrict__ dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    dst[i] = __float2bfloat16(src[i]);
}

template <class T>
T* dmalloc(size_t n) {
  void* p = nullptr;
  check_cuda(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc (surrogate)");
  return static_cast<T*>(p);
}

template <int LA, int LB, int EPI>
void gemm(cudaStream_t st, int M, int N, int K, const bf16* A, int lda, const bf16* B, int ldb,
          const float* bias, const float* Zp, float* Cf, bf16* Cb, int ldc) {
  // weight gradients reduce over the batch: split that K over enough blocks
  // to cover the GPU
  const int tiles = ((N + BN - 1) / BN) * ((M + BM - 1) / BM);
  int splits = 1;
  if (EPI == kEpiStore) splits = std::max(1, std::min((K + 255) / 256, 296 / std::max(tiles, 1)));
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, splits);
  k_gemm<LA, LB, EPI><<<grid, GT, 0, st>>>(M, N, K, A, lda, B, ldb, bias, Zp, Cf, Cb, ldc);
  check_cuda(cudaGetLastError(), "surrogate GEMM launch");
}

}  // namespace

// ============================================================================ Surrogate

Surrogate::Surrogate(int nang, uint64_t seed) : nang_(nang), L_(2 * nang) {
  if (nang <= 0) throw std::invalid_argument("Surrogate: no free dihedrals");
  check_cuda(cudaGetDevice(&device_), "cudaGetDevice");
  const int H = kHidden;
  wb1_ = 0;
  wb2_ = wb1_ + (size_t)L_.nin_pad * H;
  wb3_ = wb2_ + (size_t)H * H;
  wb4_ = wb3_ + (size_t)H * H;
  nwb_ = wb4_ + H;
  P_ = dmalloc<float>(L_.n);
  G_ = dmalloc<float>(L_.n);
  M_ = dmalloc<float>(L_.n);
  V_ = dmalloc<float>(L_.n);
  Wb_ = dmalloc<bf16>(nwb_);
  loss_ = dmalloc<float>(1);
  // Kaiming-uniform weights (bound sqrt(6 / fan_in)), zero biases; padded
  // input rows of W1 are zero.
  std::vector<float> p(L_.n, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](size_t off, int fan_in, int rows, int cols, int valid_rows) {
    std::uniform_real_distribution<float> u(-std::sqrt(6.f / fan_in), std::sqrt(6.f / fan_in));
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < cols; ++c) p[off + (size_t)r * cols + c] = r < valid_rows ? u(rng) : 0.f;
  };
  fill(L_.w1, L_.nin, L_.nin_pad, H, L_.nin);
  fill(L_.w2, H, H, H, H);
  fill(L_.w3, H, H, H, H);
  fill(L_.w4, H, H, 1, H);
  check_cuda(cudaMemcpy(P_, p.data(), L_.n * sizeof(float), cudaMemcpyHostToDevice), "H2D params");
  check_cuda(cudaMemset(M_, 0, L_.n * sizeof(float)), "memset");
  check_cuda(cudaMemset(V_, 0, L_.n * sizeof(float)), "memset");
  refresh_bf16();
  sync();
}

Surrogate::~Surrogate() {
  for (void* q : {(void*)P_, (void*)G_, (void*)M_, (void*)V_, (void*)Wb_, (void*)Wt_, (void*)loss_,
                  (void*)ang_, (void*)tgt_, (void*)X_, (void*)H1_, (void*)H2_, (void*)H3_,
                  (void*)dA_, (void*)dB_, (void*)Z1_, (void*)Z2_, (void*)Z3_, (void*)y_,
                  (void*)dy_, (void*)tbuf_, (void*)abuf_, (void*)idx_})
    if (q) cudaFree(q);
}

void Surrogate::sync() { check_cuda(cudaStreamSynchronize(stream_), "surrogate sync"); }

void Surrogate::refresh_bf16() {
  const int H = kHidden;
  auto conv = [&](size_t src, size_t dst, size_t n) {
    k_to_bf16<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, stream_>>>(n, P_ + src,
                                                                                      Wb_ + dst);
  };
  conv(L_.w1, wb1_, (size_t)L_.nin_pad * H);
  conv(L_.w2, wb2_, (size_t)H * H);
  conv(L_.w3, wb3_, (size_t)H * H);
  conv(L_.w4, wb4_, H);
  check_cuda(cudaGetLastError(), "surrogate bf16 refresh");
}

void Surrogate::ensure_scratch(int batch) {
  if (batch <= cap_) return;
  for (void* q : {(void*)X_, (void*)H1_, (void*)H2_, (void*)H3_, (void*)dA_, (void*)dB_,
                  (void*)Z1_, (void*)Z2_, (void*)Z3_, (void*)y_, (void*)dy_, (void*)tbuf_,
                  (void*)abuf_, (void*)idx_})
    if (q) cudaFree(q);
  const size_t B = batch, H = kHidden;
  X_ = dmalloc<bf16>(B * L_.nin_pad);
  H1_ = dmalloc<bf16>(B * H);
  H2_ = dmalloc<bf16>(B * H);
  H3_ = dmalloc<bf16>(B * H);
  dA_ = dmalloc<bf16>(B * H);
  dB_ = dmalloc<bf16>(B * H);
  Z1_ = dmalloc<float>(B * H);
  Z2_ = dmalloc<float>(B * H);
  Z3_ = dmalloc<float>(B * H);
  y_ = dmalloc<float>(B);
  dy_ = dmalloc<float>(B);
  tbuf_ = dmalloc<float>(B);
  abuf_ = dmalloc<float>(B * nang_);
  idx_ = dmalloc<int>(B);
  cap_ = batch;
}

void Surrogate::upload_angles(const double* ang, int n, float* dst) {
  std::vector<float> f((size_t)n * nang_);
  for (size_t i = 0; i < f.size(); ++i) f[i] = (float)ang[i];
  check_cuda(cudaMemcpyAsync(dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice,
                             stream_),
             "H2D angles");
  sync();
}

void Surrogate::forward(int B, const float* ang, const int* idx) {
  const int H = kHidden, K1 = L_.nin_pad;
  k_features<<<B, 128, 0, stream_>>>(ang, idx, B, nang_, K1, X_);
  gemm<0, 0, kEpiHidden>(stream_, B, H, K1, X_, K1, Wb_ + wb1_, H, P_ + L_.b1, nullptr, Z1_, H1_, H);
  gemm<0, 0, kEpiHidden>(stream_, B, H, H, H1_, H, Wb_ + wb2_, H, P_ + L_.b2, nullptr, Z2_, H2_, H);
  gemm<0, 0, kEpiHidden>(stream_, B, H, H, H2_, H, Wb_ + wb3_, H, P_ + L_.b3, nullptr, Z3_, H3_, H);
  k_out_fwd<<<(B + 7) / 8, 256, 0, stream_>>>(B, H3_, Wb_ + wb4_, P_ + L_.b4, y_);
  check_cuda(cudaGetLastError(), "surrogate forward");
}

// Gradients of the mean squared error of the batch into G_ (overwritten).
double Surrogate::backward(int B, const float* target, const int* tidx, bool accumulate_loss) {
  const int H = kHidden, K1 = L_.nin_pad;
  check_cuda(cudaMemsetAsync(G_, 0, L_.n * sizeof(float), stream_), "memset grads");
  if (!accumulate_loss) check_cuda(cudaMemsetAsync(loss_, 0, sizeof(float), stream_), "memset");
  k_out_bwd<<<(B + 7) / 8, 256, 0, stream_>>>(B, y_, target, tidx, Wb_ + wb4_, Z3_, dA_, dy_, loss_);
  const unsigned rb = (unsigned)((B + 255) / 256);
  k_colsum<bf16><<<rb, 256, 0, stream_>>>(B, H, H3_, dy_, G_ + L_.w4);      // dw4
  k_colsum<float><<<rb, 1, 0, stream_>>>(B, 1, dy_, nullptr, G_ + L_.b4);  // db4
  // layer 3: dW3 = H2^T dZ3, db3, dZ2 = (dZ3 W3^T) silu'(Z2)
  gemm<1, 0, kEpiStore>(stream_, H, H, B, H2_, H, dA_, H, nullptr, nullptr, G_ + L_.w3, nullptr, H);
  k_colsum<bf16><<<rb, 256, 0, stream_>>>(B, H, dA_, nullptr, G_ + L_.b3);
  gemm<0, 1, kEpiSiluGrad>(stream_, B, H, H, dA_, H, Wb_ + wb3_, H, nullptr, Z2_, nullptr, dB_, H);
  // layer 2
  gemm<1, 0, kEpiStore>(stream_, H, H, B, H1_, H, dB_, H, nullptr, nullptr, G_ + L_.w2, nullptr, H);
  k_colsum<bf16><<<rb, 256, 0, stream_>>>(B, H, dB_, nullptr, G_ + L_.b2);
  gemm<0, 1, kEpiSiluGrad>(stream_, B, H, H, dB_, H, Wb_ + wb2_, H, nullptr, Z1_, nullptr, dA_, H);
  // layer 1 (no input gradient)
  gemm<1, 0, kEpiStore>(stream_, K1, H, B, X_, K1, dA_, H, nullptr, nullptr, G_ + L_.w1, nullptr, H);
  k_colsum<bf16><<<rb, 256, 0, stream_>>>(B, H, dA_, nullptr, G_ + L_.b1);
  check_cuda(cudaGetLastError(), "surrogate backward");
  return 0.0;
}

void Surrogate::set_data(const double* ang, const double* energy, int n, double clip) {
  if (n <= 0) throw std::invalid_argument("Surrogate::set_data: empty training set");
  clip_ = clip;
  double s = 0.0, s2 = 0.0;
  std::vector<float> t(n);
  for (int i = 0; i < n; ++i) {
    const double e = std::min(energy[i], clip);
    s += e;
    s2 += e * e;
  }
  const double mean = s / n, var = std::max(s2 / n - mean * mean, 1e-12);
  mu_ = (float)mean;
  sigma_ = (float)std::sqrt(var);
  for (int i = 0; i < n; ++i) t[i] = (float)((std::min(energy[i], clip) - mean) / sigma_);
  if (ang_) cudaFree(ang_);
  if (tgt_) cudaFree(tgt_);
  ang_ = dmalloc<float>((size_t)n * nang_);
  tgt_ = dmalloc<float>(n);
  upload_angles(ang, n, ang_);
  check_cuda(cudaMemcpy(tgt_, t.data(), n * sizeof(float), cudaMemcpyHostToDevice), "H2D targets");
  ndata_ = n;
}

double Surrogate::train(int epochs, int batch, double lr, uint64_t shuffle_seed) {
  if (ndata_ <= 0) throw std::invalid_argument("Surrogate::train: no training set");
  if (batch <= 0 || epochs <= 0) throw std::invalid_argument("Surrogate::train: bad batch/epochs");
  batch = std::min(batch, ndata_);
  ensure_scratch(batch);
  std::vector<int> perm(ndata_);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937_64 rng(shuffle_seed);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  double last = 0.0;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    check_cuda(cudaMemsetAsync(loss_, 0, sizeof(float), stream_), "memset");
    const int nb = ndata_ / batch;   // full batches only
    for (int k = 0; k < nb; ++k) {
      check_cuda(cudaMemcpyAsync(idx_, perm.data() + (size_t)k * batch, batch * sizeof(int),
                                 cudaMemcpyHostToDevice, stream_),
                 "H2D batch index");
      forward(batch, ang_, idx_);
      backward(batch, tgt_, idx_, true);
      ++step_;
      const float bc1 = 1.f - std::pow(b1, (float)step_), bc2 = 1.f - std::pow(b2, (float)step_);
      k_adam<<<1024, 256, 0, stream_>>>(L_.n, P_, G_, M_, V_, (float)lr, b1, b2, eps, bc1, bc2);
      refresh_bf16();
      // the index buffer is reused by the next batch: keep the host copy alive
      sync();
    }
    float l = 0.f;
    check_cuda(cudaMemcpy(&l, loss_, sizeof(float), cudaMemcpyDeviceToHost), "D2H loss");
    last = (double)l / ((double)nb * batch);
  }
  return last;
}

void Surrogate::predict(const double* ang, int n, double* out) {
  const int chunk = 4096;
  ensure_scratch(std::min(chunk, std::max(n, 1)));
  std::vector<float> y;
  for (int b0 = 0; b0 < n; b0 += cap_) {
    const int B = std::min(cap_, n - b0);
    upload_angles(ang + (size_t)b0 * nang_, B, abuf_);
    forward(B, abuf_, nullptr);
    y.resize(B);
    check_cuda(cudaMemcpyAsync(y.data(), y_, B * sizeof(float), cudaMemcpyDeviceToHost, stream_),
               "D2H predictions");
    sync();
    for (int i = 0; i < B; ++i) out[b0 + i] = (double)mu_ + (double)sigma_ * (double)y[i];
  }
}

double Surrogate::gradients(const double* ang, const double* energy, int n, float* grad_out) {
  ensure_scratch(n);
  upload_angles(ang, n, abuf_);
  std::vector<float> t(n);
  for (int i = 0; i < n; ++i) t[i] = (float)((std::min(energy[i], clip_) - mu_) / sigma_);
  check_cuda(cudaMemcpyAsync(tbuf_, t.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream_),
             "H2D targets");
  forward(n, abuf_, nullptr);
  backward(n, tbuf_, nullptr, false);
  float l = 0.f;
  check_cuda(cudaMemcpyAsync(grad_out, G_, L_.n * sizeof(float), cudaMemcpyDeviceToHost, stream_),
             "D2H grads");
  check_cuda(cudaMemcpyAsync(&l, loss_, sizeof(float), cudaMemcpyDeviceToHost, stream_), "D2H loss");
  sync();
  return (double)l / n;
}

void Surrogate::get_params(float* out) const {
  check_cuda(cudaMemcpy(out, P_, L_.n * sizeof(float), cudaMemcpyDeviceToHost), "D2H params");
}

void Surrogate::set_params(const float* in) {
  check_cuda(cudaMemcpy(P_, in, L_.n * sizeof(float), cudaMemcpyHostToDevice), "H2D params");
  refresh_bf16();
  sync();
}

DSurrogate Surrogate::device_view() {
  const int H = kHidden;
  if (!Wt_) Wt_ = dmalloc<bf16>((size_t)L_.nin_pad * H + 2 * (size_t)H * H);
  bf16* w1t = Wt_;
  bf16* w2t = w1t + (size_t)L_.nin_pad * H;
  bf16* w3t = w2t + (size_t)H * H;
  k_transpose_bf16<<<H, 256, 0, stream_>>>(L_.nin_pad, P_ + L_.w1, w1t);
  k_transpose_bf16<<<H, 256, 0, stream_>>>(H, P_ + L_.w2, w2t);
  k_transpose_bf16<<<H, 256, 0, stream_>>>(H, P_ + L_.w3, w3t);
  check_cuda(cudaGetLastError(), "surrogate transpose");
  sync();
  DSurrogate d;
  d.w1t = w1t;
  d.w2t = w2t;
  d.w3t = w3t;
  d.w1 = Wb_ + wb1_;
  d.w2 = Wb_ + wb2_;
  d.w3 = Wb_ + wb3_;
  d.w4 = Wb_ + wb4_;
  d.b1 = P_ + L_.b1;
  d.b2 = P_ + L_.b2;
  d.b3 = P_ + L_.b3;
  d.b4 = P_ + L_.b4;
  d.nin = L_.nin;
  d.nin_pad = L_.nin_pad;
  d.mu = mu_;
  d.sigma = sigma_;
  return d;
}

// ============================================================================ no-alloc forward
//
// Some callers cannot allocate device memory at the point where they need a
// prediction: code that runs while a framework's caching allocator owns the
// device memory budget, a real-time loop whose allocations are forbidden, or
// a host thread that must not take the driver's allocation locks.  For them,
// predict_noalloc runs the same forward kernels as predict() on
// device-resident inputs and outputs, with its intermediate activations in
// the fixed array below instead of cudaMalloc'd buffers.
//
// * The array is kNoAllocScratchBytes (16 MiB) and lives on every GPU that
//   loads the library until the process exits.  A call needs per row
//   2*nin_pad + 18*256 + 4 bytes (plus 256-byte alignment per sub-buffer);
//   noalloc_max_rows() gives the limit and larger n is rejected.
// * Host code cannot pass the array's name to a kernel: on the host it names
//   a host-side stand-in, not device memory.  The device address is looked up
//   with cudaGetSymbolAddress once per device, on the first call made while
//   that device is current; make that first call before any stream capture.
// * Nothing in the array must start at zero: every scratch byte a call reads
//   was written earlier in the same call.  Every call shares the one array
//   and it keeps the last call's contents, so calls that overlap on the GPU
//   (concurrent streams, or concurrent host threads) race; serialise them.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

__global__ void k_denorm(int n, const float* __restrict__ y, float mu, float sigma,
                         double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)mu + (double)sigma * (double)y[i];
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Scratch layout of one call: X | Z1 Z2 Z3 | H1 H2 H3 | y, each 256-aligned.
struct NoAllocLayout {
  size_t x, z1, z2, z3, h1, h2, h3, y, total;
  NoAllocLayout(int n, int nin_pad) {
    const size_t H = kHidden;
    x = 0;
    z1 = align256(x + (size_t)n * nin_pad * sizeof(bf16));
    z2 = align256(z1 + (size_t)n * H * sizeof(float));
    z3 = align256(z2 + (size_t)n * H * sizeof(float));
    h1 = align256(z3 + (size_t)n * H * sizeof(float));
    h2 = align256(h1 + (size_t)n * H * sizeof(bf16));
    h3 = align256(h2 + (size_t)n * H * sizeof(bf16));
    y = align256(h3 + (size_t)n * H * sizeof(bf16));
    total = y + (size_t)n * sizeof(float);
  }
};

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once
// per device).
unsigned char* noalloc_scratch() {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("predict_noalloc: device index");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch),
               "cudaGetSymbolAddress (no-alloc scratch)");
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
  }
  return g_noalloc_ptr[dev];
}

}  // namespace

int Surrogate::noalloc_max_rows(int nin_pad) {
  int lo = 0, hi = 1 << 22;
  while (lo < hi) {   // largest n whose layout fits
    const int mid = lo + (hi - lo + 1) / 2;
    if (NoAllocLayout(mid, nin_pad).total <= kNoAllocScratchBytes)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

void Surrogate::predict_noalloc(const float* ang_dev, int n, double* energy_dev,
                                cudaStream_t st) const {
  int dev = -1;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev != device_)
    throw std::invalid_argument("smmp_sur_predict_noalloc: device " + std::to_string(dev) +
                                " is current, but the surrogate's parameters are on device " +
                                std::to_string(device_) + "; make that device current");
  if (n <= 0) return;
  const int maxn = noalloc_max_rows(L_.nin_pad);
  if (n > maxn)
    throw std::invalid_argument("smmp_sur_predict_noalloc: " + std::to_string(n) +
                                " rows exceed the fixed scratch (at most " +
                                std::to_string(maxn) + " rows for this network)");
  unsigned char* base = noalloc_scratch();
  const NoAllocLayout lay(n, L_.nin_pad);
  bf16* X = reinterpret_cast<bf16*>(base + lay.x);
  float* Z1 = reinterpret_cast<float*>(base + lay.z1);
  float* Z2 = reinterpret_cast<float*>(base + lay.z2);
  float* Z3 = reinterpret_cast<float*>(base + lay.z3);
  bf16* H1 = reinterpret_cast<bf16*>(base + lay.h1);
  bf16* H2 = reinterpret_cast<bf16*>(base + lay.h2);
  bf16* H3 = reinterpret_cast<bf16*>(base + lay.h3);
  float* y = reinterpret_cast<float*>(base + lay.y);
  const int H = kHidden, K1 = L_.nin_pad;
  k_features<<<n, 128, 0, st>>>(ang_dev, nullptr, n, nang_, K1, X);
  gemm<0, 0, kEpiHidden>(st, n, H, K1, X, K1, Wb_ + wb1_, H, P_ + L_.b1, nullptr, Z1, H1, H);
  gemm<0, 0, kEpiHidden>(st, n, H, H, H1, H, Wb_ + wb2_, H, P_ + L_.b2, nullptr, Z2, H2, H);
  gemm<0, 0, kEpiHidden>(st, n, H, H, H2, H, Wb_ + wb3_, H, P_ + L_.b3, nullptr, Z3, H3, H);
  k_out_fwd<<<(n + 7) / 8, 256, 0, st>>>(n, H3, Wb_ + wb4_, P_ + L_.b4, y);
  k_denorm<<<(n + 255) / 256, 256, 0, st>>>(n, y, mu_, sigma_, energy_dev);
  check_cuda(cudaGetLastError(), "predict_noalloc launch");
}

}  // namespace smmpb200
