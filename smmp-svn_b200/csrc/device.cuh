// Device-side data structures shared by the kernels and the host runtime.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace smmpb200 {

constexpr int kTypes = 18;
constexpr int kTP = kTypes * kTypes;
// Threads per chain (one CTA per chain).  kernels.cu is built twice: with 512
// threads, and with 384 for the sweeps of small molecules (its kernels and
// launchers then sit in namespace smmpb200::t384; SMMP_THREADS and
// SMMP_BLOCK_VARIANT set by the build).
#ifndef SMMP_THREADS
#define SMMP_THREADS 512
#endif
constexpr int kThreads = SMMP_THREADS;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxNeighbours = 96;       // SASA neighbours per atom (per-warp buffer)
constexpr int kSasaQueue = 64;           // SASA neighbour candidates queued per warp
// Speculative window of the sweep (k_sweep): up to this many consecutive
// proposals evaluated at once from the same state.
constexpr int kMaxWindow = 8;

// An MT19937 stream slot: 624 state words, mti, the head and tail counters
// of a queue of tempered values already drawn from the state but not yet
// consumed, padding, then the queue (64 doubles).  The stream a slot yields is
// the queue in order, then grnd() of the state (twister.f:104-177).
constexpr int kMTWords = 768;
constexpr int kQueue = 64;
constexpr int kMTIdx = 624, kQHead = 625, kQTail = 626, kQOff = 640;

// One molecule, GPU resident (all indices 0-based, see topology.hpp).
struct DMol {
  int natoms, nvar, nfree, nchunks, n14, nheavy, nlevels, nres, nsib;
  int i1, i2, i3;
  double gbpr[6];
  double ag[9];        // global axes of the first frame from gbpr[3..5], [row * 3 + col]
  const int* iow;
  const uint8_t* type;
  const double* charge;
  const double* blen;
  const double* cba;
  const double* sba;
  const double* toat0;
  const double* rvdw;
  const double* sigma;
  const int* level_atoms;
  const int* level_off;
  const int* var_atom;
  const int* var_base;
  const int* var_lo;
  const int* var_hi;
  const int* sib_off;
  const int* sib;
  const double* var_e0;
  const double* var_sg;
  const double* var_rn;
  const double* axvr;
  const int* idvr;
  const uint32_t* chunks;
  const uint32_t* pairs14;
  const int* heavy;
  const int* residue_of_atom;
  // dense pair set (topology.hpp)
  const unsigned long long* near_mask;   // row form of the pair set (rows != 0)
  const unsigned long long* near14;
  int rows;
  int npairs;                            // pair terms of a full evaluation
  const uint32_t* flat;                  // every pair once: i | j<<14 | is14<<28
  const int* var_cross;                  // pair terms across each variable's bond
  // pairs each free variable's turn changes, as indices into flat (CSR by
  // variable; cache = 0 when the molecule has none: over 65,535 pairs)
  const int* cross_off;
  const uint16_t* cross_idx;
  int ncross, cross_max;
  int cache;
};

// Force field constants read by every chain (copied to shared memory).
struct DForceField {
  double a[kTP], a14[kTP], c[kTP], guard_r2[kTP];
  int hb[kTP];
  double conv, plt, slp;
  int epsd, itysol, npnt;
  const double* spoint;    // device, npnt*3
};

// Scalars of the force field every pair term reads.
struct FFScalars {
  double conv, plt, slp;
  int epsd, itysol, npnt;
};

// Everything a launch needs to know about the molecules of its chains.
struct DMolSet {
  const DMol* mols;          // device array
  int nmols;
  int max_atoms, max_vars;   // shared-memory sizing
  int stage_bytes;           // shared-memory pool for the staged topology
  int stage_lists;           // 1: the pair lists are staged too (they fit)
  int any_rows;              // 1: some molecule evaluates its pairs by rows
  int da;                    // 1: shared memory for the surrogate's first stage
  int window;                // proposals per speculative window (<= 1: one at a time)
  int cache_pairs;           // > 0: shared memory for the cached pair terms of this many
  int cache_cross;           //      pairs and the new terms of this many crossing pairs
  const DForceField* ff;     // device
  FFScalars f;
};

// Sampling weight (canon.f can_weight; mulcan_par_mod.f90 muca_weight*).
enum WeightKind : int { kWeightCanon = 0, kWeightMuca = 1, kWeightMuca2 = 2 };
struct DWeight {
  int kind;
  int kmin, kmax;
  double ebin;
  const double* b;       // [kmax-kmin+1]
  const double* alpha;
};

// Mutable state of a set of chains (replicas).
// Device view of a trained energy surrogate (an MLP on the sin/cos of the
// free dihedrals, 3 hidden layers of 256, SiLU), BF16 weights.
struct DSurrogate {
  const __nv_bfloat16* w1;   // [nin_pad][256]
  const __nv_bfloat16* w2;   // [256][256]
  const __nv_bfloat16* w3;   // [256][256]
  const __nv_bfloat16* w4;   // [256]
  const __nv_bfloat16* w1t;  // [256][nin_pad]  (transposed copies: K contiguous)
  const __nv_bfloat16* w2t;  // [256][256]
  const __nv_bfloat16* w3t;  // [256][256]
  const float* b1;
  const float* b2;
  const float* b3;
  const float* b4;
  int nin, nin_pad;          // nin = 2 * free dihedrals
  float mu, sigma;           // energy = mu + sigma * output
};

struct DChains {
  int nchains;
  const int* mol_of_chain;
  double* vlvr;          // [chain * vstride + var]
  int vstride;
  double* toat;          // [slot * tstride + atom]  (phase-constant dihedral state)
  int tstride;
  const int* toat_slot;
  uint32_t* mt;          // [slot * kMTWords] stream slots
  const int* mt_slot;
  double* beta;          // current inverse temperature of each chain
  double* eol;           // energy of the current conformation
  double* terms;         // [chain*6]: eyel eyvw eyhb eyvr eysl eysm (last full evaluation)
  unsigned long long* nacc;
  unsigned long long* nprop;
  unsigned long long* pterms;   // pair terms evaluated by the sweeps (FP32-issue roofline)
  int* err;              // first error of each chain (0 = none)
  double* coords;        // optional [chain * 3 * tstride] coordinates after the call
  // delayed acceptance (surrogate first stage), on when sur.w1 != nullptr
  DSurrogate sur;
  float da_floor;        // a chain whose stage-2 acceptance falls below this ...
  int da_min;            // ... after this many stage-1 acceptances takes plain steps
  unsigned long long* da_n1;   // [chain] proposals that passed stage 1
  unsigned long long* da_n2;   // [chain] proposals accepted at stage 2
};

// Parallel tempering fused into one cooperative sweep launch: after every
// sweep all blocks meet at a grid barrier, block 0 runs the exchange step
// (partem_s.f:210-232) and every chain takes up its new inverse temperature.
// on == 0 for ordinary launches.
struct DPTFused {
  int on;
  int n;                       // temperature labels (= chains of the launch)
  int wrap;
  int* temp_chain;             // [n] chain at each label
  const double* betas;         // [n] inverse temperature of each label
  uint32_t* mt;                // exchange stream slot (kMTWords)
  double* lq;                  // [kQueue] scratch of the exchange stream's refills
  int* iswitch;
  unsigned long long* stats;   // [2n]
  unsigned* bar;               // [2] grid barrier: arrivals, generation
  unsigned long long timeout_ns;   // a barrier wait longer than this sets kErrTimeout
  unsigned extra;              // arrivals beyond the launch's blocks (0; >0 only in tests:
                               // the barrier then never opens and every wait runs out)
  int master;                  // 1: the launch's last block runs no chain but the
                               // exchanges (set by the launcher)
};

enum SweepFlags : int {
  kFlagRndOrd = 1,        // random variable order (rndord)
  kFlagFP32 = 2,          // FP32 pair terms with FP64 guard and accumulation
  kFlagExtraSetvar = 4,   // one extra setvar+rebuild before the sweep (partem_s)
  kFlagNoCheck = 8,       // skip the end-of-sweep consistency check
};

enum ErrorCode : int {
  kErrNone = 0,
  kErrNonFinite = 1,      // NaN/Inf energy
  kErrConsistency = 2,    // |E_incremental - E_fresh| above tolerance at sweep end
  kErrNeighbours = 3,     // reserved: a crowded SASA atom is scanned directly instead
  kErrTimeout = 4,        // a bounded wait gave up
};

}  // namespace smmpb200
