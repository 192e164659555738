// Host runtime of the SMMP energy-and-sweep path: molecules assembled on the
// host, uploaded once, and ensembles of chains (replicas) whose whole state
// lives on the GPU.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "device.cuh"
#include "topology.hpp"

namespace smmpb200 {

// Switches of the reference's COMMON blocks epar_l, isolty and updchois.
struct Config {
  int sh2 = 0, epsd = 0, itysol = 0, ientyp = 0, rndord = 0, upchswitch = 0;
};

void check_cuda(cudaError_t e, const char* what);

// A molecule assembled from a residue library, a sequence and a .var file.
struct Molecule {
  MolTopo topo;
  ForceField ff;
  Config cfg;
};
std::shared_ptr<Molecule> build_molecule(const std::string& libdir, const Config& cfg,
                                         const std::string& seqfile, const std::string& varfile,
                                         const std::string& grpn, const std::string& grpc);

// Device copies of a list of molecules sharing one force field.
class DeviceSet {
 public:
  explicit DeviceSet(const std::vector<std::shared_ptr<Molecule>>& mols);
  ~DeviceSet();
  DeviceSet(const DeviceSet&) = delete;
  DeviceSet& operator=(const DeviceSet&) = delete;
  const DMolSet& set() const { return set_; }
  // reserve shared memory for the surrogate's first stage (re-sizes staging)
  void set_da(bool on);
  // pair-work form of the molecules that allow rows: 0 pair lists, 1 rows,
  // -1 the size-based default
  void set_rows(int mode);
  int any_rows_possible() const;
  // proposals per speculative window of the sweep (1: one at a time); the
  // window's buffers take up to 64 KB of shared memory, which caps it for
  // large molecules, and SASA sweeps run one at a time.  Returns the size set.
  int set_window(int k);
  int window() const { return set_.window >= 2 ? set_.window : 1; }

 private:
  void size_staging();
  size_t with_lists_ = 0, without_ = 0;
  int cache_pairs_ = 0, cache_cross_ = 0;   // cached pair terms, when they fit
  std::vector<DMol> dm_;
  std::vector<int> rows_ok_;
  DMol* dmols_ = nullptr;
  template <class T>
  const T* upload(const std::vector<T>& v);
  std::vector<void*> allocs_;
  DMolSet set_{};
};

// Parallel-tempering bookkeeping (partem_s.f ipoi / pbe).
struct PTState {
  int n = 0;            // number of temperature labels
  int wrap = 1;         // replica n pairs with replica 1 (partem_s.f:222)
  int* temp_chain = nullptr;          // device [n]
  double* betas = nullptr;            // device [n], beta of each label
  uint32_t* mt = nullptr;             // device stream slot (kMTWords) of the exchanges
  int* iswitch = nullptr;             // device
  unsigned long long* stats = nullptr;   // device [2n] attempts/accepts per pair
  double* lq = nullptr;               // device [kQueue] refill scratch of the fused exchange
  unsigned* bar = nullptr;            // device [2] grid barrier of the fused launch
  bool fused = true;                  // batched runs: one cooperative launch when possible
  double timeout_s = 30.0;            // bound on one grid-barrier wait
  unsigned barrier_extra = 0;         // tests only: arrivals that never come
};

// An ensemble of chains; every chain is an independent copy of one molecule.
class Ensemble {
 public:
  // shared_stream: all chains consume one MT19937 stream and one dihedral
  // state in turn, as partem_s.f does (serial compatibility mode).
  Ensemble(std::vector<std::shared_ptr<Molecule>> mols, std::vector<int> chain_mol,
           std::vector<int> seeds, std::vector<double> betas, bool shared_stream);
  ~Ensemble();
  Ensemble(const Ensemble&) = delete;
  Ensemble& operator=(const Ensemble&) = delete;

  int nchains() const { return n_; }
  void set_stream(cudaStream_t s);   // nullptr: own stream
  // Delayed acceptance with a trained surrogate as the first stage (nullptr:
  // plain Metropolis).  A chain whose stage-2 acceptance falls below `floor`
  // after min_stage1 stage-1 passes takes plain steps.  The surrogate's
  // device memory must outlive its use here.
  void set_surrogate(const DSurrogate* view, float floor, int min_stage1);
  void da_stats(std::vector<unsigned long long>& n1, std::vector<unsigned long long>& n2) const;
  // Autotuner: times one sweep of all chains with each pair-work form (0 pair
  // lists, 1 row passes, 2 rows for molecules of 128+ atoms) from the same
  // saved state, keeps the fastest and restores the state.  Returns the
  // winner; ms_out[3] the three times.
  int autotune(int flags, double* ms_out);
  // The speculative window the autotuner chose (1: none) and the times of
  // one sweep with windows of 2, 4 and 8 proposals on the row form (0: not
  // timed); set_window fixes it by hand.
  int window() const { return dev_->window(); }
  int set_window(int k);
  const double* window_ms() const { return window_ms_; }
  // pair-work form by hand (as autotune's choice: 0 pair lists, 1 rows,
  // 2 rows for molecules of 128+ atoms)
  void set_pair_work(int form);
  cudaStream_t stream() const { return stream_; }
  const DChains& chains() const { return ch_; }
  const DMolSet& set() const { return dev_->set(); }
  const Molecule& molecule_of(int c) const { return *mols_[chain_mol_[c]]; }

  void random_start();                       // canon.f:60-67 for every chain
  void energy(bool fp32);                    // energy() of every chain
  // gradient.f (vacuum): dE/dv of every variable of every chain into
  // g[chain * vstride + v] (FP64), energies as energy() leaves them
  void gradient(std::vector<double>& g);
  void sweeps(int nsweeps, int flags, const DWeight& w);   // metropolis, no exchange
  void sweeps_chain(int c, int nsweeps, int flags, const DWeight& w);
  void energy_chain(int c, bool fp32);
  void equilibrate(int nequi, int flags);   // partem_s.f:134-162

  void set_pt(const std::vector<double>& betas, int wrap, int exchange_seed);
  // nsweeps of (all chains one sweep, then one exchange); serial=true visits
  // the chains one by one in temperature order as partem_s.f does.
  void pt_sweeps(int nsweeps, int flags, bool serial, int graph_chunk);
  void pt_map(std::vector<int>& temp_chain) const;
  void pt_stats(std::vector<unsigned long long>& s) const;
  // exchange state for checkpoints: map, parity switch, exchange stream
  bool has_pt() const { return pt_.n == n_; }
  // Fused cooperative launch for batched parallel tempering (on by default);
  // off, or when the chains cannot all be resident, runs take the graph path.
  // barrier_extra > 0 (tests of the bounded wait) makes every barrier wait
  // for arrivals that never come: every chain ends with kErrTimeout.
  void set_pt_fused(bool on, double timeout_s, unsigned barrier_extra = 0);
  bool pt_fused_last() const { return pt_fused_last_; }
  void pt_get_state(std::vector<int>& tc, int& iswitch, std::vector<uint32_t>& mt,
                    std::vector<double>& betas) const;
  void pt_set_state(const std::vector<int>& tc, int iswitch, const std::vector<uint32_t>& mt,
                    const std::vector<double>& betas);

  // host <-> device state
  void get_vlvr(std::vector<double>& v) const;    // [chain*vstride]
  void set_vlvr(const std::vector<double>& v);
  void get_eol(std::vector<double>& e) const;
  void get_terms(std::vector<double>& t) const;
  void get_acceptance(std::vector<unsigned long long>& acc,
                      std::vector<unsigned long long>& prop) const;
  void get_errors(std::vector<int>& e) const;
  // pair terms the sweeps evaluated per chain (full sums and the pairs across
  // each incremental proposal's bond, before and after the move)
  void get_pair_terms(std::vector<unsigned long long>& p) const;
  void set_acceptance(const std::vector<unsigned long long>& acc,
                      const std::vector<unsigned long long>& prop);
  void get_coords(std::vector<double>& xyz);       // [chain*3*tstride]
  void get_betas(std::vector<double>& b) const;
  void set_betas(const std::vector<double>& b);
  void get_mt(std::vector<uint32_t>& mt) const;   // [slot*kMTWords]
  void set_mt(const std::vector<uint32_t>& mt);
  void get_toat(std::vector<double>& t) const;
  void set_toat(const std::vector<double>& t);
  void draw(int slot, int n, std::vector<double>& out);
  int vstride() const { return ch_.vstride; }
  int tstride() const { return ch_.tstride; }
  int nslots_mt() const { return nmt_; }
  int nslots_toat() const { return ntoat_; }
  double check_tol = 1e-6;        // FP64 consistency tolerance (metropolis.f:173)
  double check_tol_fp32 = 1e-2;   // FP32 pair terms

 private:
  void launch_sweep_range(int first, int count, int nsweeps, int flags, const DWeight& w);
  std::vector<std::shared_ptr<Molecule>> mols_;
  std::vector<int> chain_mol_;
  std::unique_ptr<DeviceSet> dev_;
  int n_ = 0, nmt_ = 0, ntoat_ = 0;
  DChains ch_{};
  std::vector<void*> allocs_;
  cudaStream_t stream_ = nullptr;
  cudaStream_t own_stream_ = nullptr;
  PTState pt_;
  cudaGraphExec_t graph_ = nullptr;
  int graph_len_ = 0, graph_flags_ = -1;
  bool pt_fused_last_ = false;   // the last batched pt_sweeps ran the fused launch
  double window_ms_[3] = {0.0, 0.0, 0.0};
  double* coords_buf_ = nullptr;
  double* grad_buf_ = nullptr;
  // analytic SASA (itysol < 0): per-thread scratch of k_esolan for
  // kEsolanBatch chains, the per-atom areas of every chain
  double* esolan_scratch_ = nullptr;
  double* esolan_area_ = nullptr;
  // host-driven sweeps of the analytic model: old value, variable and
  // tracked energy of each chain's current proposal
  double* an_vold_ = nullptr;
  int* an_jvar_ = nullptr;
  double* an_eolc_ = nullptr;
  void energy_launch(int first, int count, bool fp32, bool want_coords);
  void sweeps_analytic(int first, int count, int nsweeps, int flags, const DWeight& w);
};

}  // namespace smmpb200
