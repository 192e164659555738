// Host runtime: molecule upload, chain ensembles, sweeps, replica exchange.
#include "runtime.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>

#include "kernels.hpp"
#include "molbuild.hpp"

namespace smmpb200 {

// The part of the first frame (setgbl, bldmol.f:303-420) that depends only
// on the molecule's global angles gbpr[3..5]: three normalised axes, column
// c of ag[r * 3 + c].  A constant of the molecule, so computed here once.
static void global_axes(const double* gbpr, double* ag) {
  const double ca = std::cos(gbpr[3]), sa = std::sin(gbpr[3]);
  const double cb = std::cos(gbpr[4]), sb = std::sin(gbpr[4]);
  const double cg = std::cos(gbpr[5]), sg = std::sin(gbpr[5]);
  const double x1 = ca * cg - sa * sb * sg, x2 = sa * cg + ca * sb * sg, x3 = -cb * sg;
  double d = std::sqrt(x1 * x1 + x2 * x2 + x3 * x3);
  ag[0] = x1 / d;
  ag[3] = x2 / d;
  ag[6] = x3 / d;
  const double y1 = -sa * cb, y2 = ca * cb, y3 = sb;
  d = std::sqrt(y1 * y1 + y2 * y2 + y3 * y3);
  ag[1] = y1 / d;
  ag[4] = y2 / d;
  ag[7] = y3 / d;
  const double z1 = ca * sg + sa * sb * cg, z2 = sa * sg - ca * sb * cg, z3 = cb * cg;
  d = std::sqrt(z1 * z1 + z2 * z2 + z3 * z3);
  ag[2] = z1 / d;
  ag[5] = z2 / d;
  ag[8] = z3 / d;
}

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {
template <class T>
T* dalloc(std::vector<void*>& owner, size_t n) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  check_cuda(cudaMalloc(&p, bytes), "cudaMalloc");
  owner.push_back(p);
  // zeroed, so that the unused words of a stream slot (and with them a
  // checkpoint) do not depend on what the memory held before
  check_cuda(cudaMemset(p, 0, bytes), "cudaMemset");
  check_cuda(cudaStreamSynchronize(nullptr), "cudaMemset sync");   // before any other stream
  return static_cast<T*>(p);
}
template <class T>
void h2d(T* d, const std::vector<T>& h) {
  if (!h.empty()) check_cuda(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "H2D");
}
template <class T>
void d2h(std::vector<T>& h, const T* d, size_t n) {
  h.resize(n);
  if (n) check_cuda(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost), "D2H");
}
}  // namespace

std::shared_ptr<Molecule> build_molecule(const std::string& libdir, const Config& cfg,
                                         const std::string& seqfile, const std::string& varfile,
                                         const std::string& grpn, const std::string& grpc) {
  if (cfg.ientyp != 0) throw std::runtime_error("init_energy: only ientyp=0 (ECEPP) is on this path");
  auto m = std::make_shared<Molecule>();
  m->ff = ecepp_forcefield(libdir, cfg.sh2 != 0, cfg.epsd != 0, cfg.itysol);
  const ResidueLibrary lib(library_path(libdir, cfg.sh2 != 0));
  BuildOptions opt;
  opt.sh2 = cfg.sh2 != 0;
  opt.itysol = cfg.itysol;
  opt.grpn = grpn;
  opt.grpc = grpc;
  m->topo = build_topology(lib, m->ff, opt, seqfile, varfile);
  m->cfg = cfg;
  return m;
}

// ---------------------------------------------------------------------------- DeviceSet

template <class T>
const T* DeviceSet::upload(const std::vector<T>& v) {
  T* d = dalloc<T>(allocs_, v.size());
  h2d(d, v);
  return d;
}

DeviceSet::DeviceSet(const std::vector<std::shared_ptr<Molecule>>& mols) {
  if (mols.empty()) throw std::runtime_error("DeviceSet: no molecules");
  const ForceField& ff = mols[0]->ff;
  DForceField h{};
  std::memcpy(h.a, ff.pair.a, sizeof h.a);
  std::memcpy(h.a14, ff.pair.a14, sizeof h.a14);
  std::memcpy(h.c, ff.pair.c, sizeof h.c);
  std::memcpy(h.guard_r2, ff.pair.guard_r2, sizeof h.guard_r2);
  std::memcpy(h.hb, ff.pair.hb, sizeof h.hb);
  h.conv = ff.conv;
  h.plt = ff.plt;
  h.slp = ff.slp;
  h.epsd = ff.epsd;
  h.itysol = ff.itysol;
  h.npnt = ff.npnt;
  h.spoint = upload(ff.spoint.empty() ? std::vector<double>{0.0} : ff.spoint);
  DForceField* dff = dalloc<DForceField>(allocs_, 1);
  check_cuda(cudaMemcpy(dff, &h, sizeof h, cudaMemcpyHostToDevice), "H2D ff");
  std::vector<DMol> dm;
  int max_atoms = 0, max_vars = 0;
  for (auto& mp : mols) {
    const MolTopo& t = mp->topo;
    if (mp->ff.itysol != ff.itysol || mp->ff.epsd != ff.epsd)
      throw std::runtime_error("DeviceSet: molecules of one ensemble must share the force field");
    if (ff.itysol > 0 && ff.npnt > 128)
      throw std::runtime_error("DeviceSet: the SASA kernel takes at most 128 sphere points");
    if (ff.itysol > 0 && !t.heavy.empty()) {
      // The SASA kernel tests surface points in FP32 with a 1e-4 margin; that
      // bounds the FP32 error while neighbour offsets stay below 3 radii,
      // i.e. while no radius exceeds twice another.
      double lo = 1e300, hi = 0.0;
      for (int k : t.heavy) {
        lo = std::min(lo, t.rvdw[k]);
        hi = std::max(hi, t.rvdw[k]);
      }
      if (hi > 2.0 * lo)
        throw std::runtime_error("DeviceSet: SASA radii differ by more than a factor of 2");
    }
    DMol d{};
    d.natoms = t.natoms;
    d.nvar = t.nvar;
    d.nfree = t.nfree;
    d.nchunks = (int)t.chunks.size();
    d.n14 = (int)t.pairs14.size();
    d.nheavy = (int)t.heavy.size();
    d.nlevels = (int)t.level_off.size() - 1;
    d.nres = t.nres;
    d.nsib = (int)t.sib.size();
    d.i1 = t.i1;
    d.i2 = t.i2;
    d.i3 = t.i3;
    for (int k = 0; k < 6; ++k) d.gbpr[k] = t.gbpr[k];
    global_axes(t.gbpr, d.ag);
    d.iow = upload(t.iow);
    d.type = upload(t.type);
    d.charge = upload(t.charge);
    d.blen = upload(t.blen);
    d.cba = upload(t.cba);
    d.sba = upload(t.sba);
    d.toat0 = upload(t.toat0);
    d.rvdw = upload(t.rvdw);
    d.sigma = upload(t.sigma);
    d.level_atoms = upload(t.level_atoms);
    d.level_off = upload(t.level_off);
    d.var_atom = upload(t.var_atom);
    d.var_base = upload(t.var_base);
    d.var_lo = upload(t.var_lo);
    d.var_hi = upload(t.var_hi);
    d.var_cross = upload(t.var_cross);
    d.cross_off = upload(t.cross_off);
    d.cross_idx = upload(t.cross_idx.empty() ? std::vector<uint16_t>{0} : t.cross_idx);
    d.ncross = (int)t.cross_idx.size();
    d.cross_max = 0;
    for (int v = 0; v < t.nvar; ++v)
      d.cross_max = std::max(d.cross_max, t.cross_off[v + 1] - t.cross_off[v]);
    d.cache = t.cross_idx.empty() ? 0 : 1;
    d.flat = upload(t.flat.empty() ? std::vector<uint32_t>{0} : t.flat);
    d.npairs = (int)t.npairs;
    d.sib_off = upload(t.sib_off);
    d.sib = upload(t.sib.empty() ? std::vector<int>{0} : t.sib);
    d.var_e0 = upload(t.var_e0);
    d.var_sg = upload(t.var_sg);
    d.var_rn = upload(t.var_rn);
    d.axvr = upload(t.axvr);
    d.idvr = upload(t.idvr.empty() ? std::vector<int>{0} : t.idvr);
    d.chunks = upload(t.chunks.empty() ? std::vector<uint32_t>{0} : t.chunks);
    d.pairs14 = upload(t.pairs14.empty() ? std::vector<uint32_t>{0} : t.pairs14);
    d.heavy = upload(t.heavy.empty() ? std::vector<int>{0} : t.heavy);
    d.residue_of_atom = upload(t.residue_of_atom);
    {
      std::vector<unsigned long long> nm(t.near_mask.begin(), t.near_mask.end()),
          n14(t.near14.begin(), t.near14.end());
      d.near_mask = upload(nm);
      d.near14 = upload(n14);
    }
    // Default pair-work form before any autotuning: rows from about a
    // hundred atoms on (measured: Met-enkephalin, 75 atoms, is faster with
    // the pair lists; Ace-Ala40-NMe, 412 atoms, with rows).
    d.rows = (t.rows_ok && t.natoms >= 128) ? 1 : 0;
    rows_ok_.push_back(t.rows_ok ? 1 : 0);
    dm.push_back(d);
    max_atoms = std::max(max_atoms, t.natoms);
    max_vars = std::max(max_vars, t.nvar);
  }
  DMol* dmols = dalloc<DMol>(allocs_, dm.size());
  h2d(dmols, dm);
  dmols_ = dmols;
  dm_ = dm;
  set_.mols = dmols;
  set_.nmols = (int)dm.size();
  set_.max_atoms = max_atoms;
  set_.max_vars = max_vars;
  set_.ff = dff;
  set_.f = FFScalars{ff.conv, ff.plt, ff.slp, ff.epsd, ff.itysol, ff.npnt};
  set_.any_rows = 0;
  for (const DMol& d : dm) set_.any_rows |= d.rows;
  set_.da = 0;
  cache_pairs_ = cache_cross_ = 0;
  for (const DMol& d : dm)
    if (d.cache) {
      cache_pairs_ = std::max(cache_pairs_, d.npairs);
      cache_cross_ = std::max(cache_cross_, d.cross_max);
    }
  with_lists_ = without_ = 0;
  for (const DMol& d : dm) {
    with_lists_ = std::max(with_lists_, stage_bytes_of(d, true));
    without_ = std::max(without_, stage_bytes_of(d, false));
  }
  size_staging();
}

int DeviceSet::any_rows_possible() const {
  int any = 0;
  for (int r : rows_ok_) any |= r;
  return any;
}

void DeviceSet::set_rows(int mode) {
  for (size_t k = 0; k < dm_.size(); ++k) {
    const bool big = dm_[k].natoms >= 128;
    dm_[k].rows = rows_ok_[k] && (mode == 1 || (mode < 0 && big)) ? 1 : 0;
  }
  h2d(dmols_, dm_);
  set_.any_rows = 0;
  for (const DMol& d : dm_) set_.any_rows |= d.rows;
  with_lists_ = without_ = 0;
  for (const DMol& d : dm_) {
    with_lists_ = std::max(with_lists_, stage_bytes_of(d, true));
    without_ = std::max(without_, stage_bytes_of(d, false));
  }
  size_staging();
}

int DeviceSet::set_window(int k) {
  k = std::max(1, std::min(k, kMaxWindow));
  if (set_.f.itysol > 0) k = 1;
  const size_t per = (size_t)std::max(set_.max_atoms, 1) * (3 * 8 + 2 * 16);   // FP64 + hi/lo
  while (k >= 2 && (size_t)k * per > 64 * 1024) --k;
  set_.window = k >= 2 ? k : 0;
  size_staging();
  return k;
}

void DeviceSet::set_da(bool on) {
  set_.da = on ? 1 : 0;
  size_staging();
}

void DeviceSet::size_staging() {
  const size_t with_lists = with_lists_, without = without_;
  // stage the pair lists too when the largest molecule's copy fits
  // (and keep the cached pair terms of list-form molecules when that fits too)
  const size_t budget = 200 * 1024;
  set_.stage_lists = 1;
  set_.stage_bytes = (int)with_lists;
  set_.cache_pairs = cache_pairs_;
  set_.cache_cross = cache_cross_;
  if (sweep_smem_bytes(set_) > budget) set_.cache_pairs = set_.cache_cross = 0;
  if (sweep_smem_bytes(set_) > budget) {
    set_.stage_lists = 0;
    set_.stage_bytes = (int)without;
  }
  // A large molecule stages only the leading topology arrays that fit; the
  // kernel reads the rest from global memory (stage_mol stops at the first
  // array past the end of the pool).
  const size_t limit = 227 * 1024;
  set_.stage_bytes = 0;
  size_t state = sweep_smem_bytes(set_);
  if (state > limit)
    throw std::runtime_error("DeviceSet: molecule too large for one CTA's shared memory");
  set_.stage_bytes = (int)std::min(set_.stage_lists ? with_lists : without, limit - state);
}

DeviceSet::~DeviceSet() {
  for (void* p : allocs_) cudaFree(p);
}

// ---------------------------------------------------------------------------- Ensemble

namespace {
// Sweeps of ensembles whose molecules have at most 128 atoms run the
// 384-thread build of the sweep kernel: with fewer threads each thread keeps
// its state in registers (the 512-thread build spills), and the pair work of
// a small molecule does not need the extra warps (measured: Met-enkephalin
// 4 % faster; the 256-chain poly-Ala batch and the 60-residue protein 11 %
// and 17 % slower with 384 threads, so they keep 512).  Delayed acceptance
// keeps 512 threads (its surrogate batches were measured at half the speed
// with 384).
bool small_molecules(const DMolSet& set, const DChains& ch) {
  return set.max_atoms <= 128 && ch.sur.w1 == nullptr;
}

cudaError_t sweep_launch(const DMolSet& set, const DChains& ch, const DWeight& w, int first,
                         int count, int nsweeps, int flags, double check_tol, cudaStream_t st) {
  return small_molecules(set, ch)
             ? t384::launch_sweep(set, ch, w, first, count, nsweeps, flags, check_tol, st)
             : launch_sweep(set, ch, w, first, count, nsweeps, flags, check_tol, st);
}
cudaError_t sweep_launch_pt(const DMolSet& set, const DChains& ch, const DWeight& w, int count,
                            int nsweeps, int flags, double check_tol, const DPTFused& pt,
                            cudaStream_t st) {
  return small_molecules(set, ch)
             ? t384::launch_sweep_pt(set, ch, w, count, nsweeps, flags, check_tol, pt, st)
             : launch_sweep_pt(set, ch, w, count, nsweeps, flags, check_tol, pt, st);
}
}  // namespace

Ensemble::Ensemble(std::vector<std::shared_ptr<Molecule>> mols, std::vector<int> chain_mol,
                   std::vector<int> seeds, std::vector<double> betas, bool shared_stream)
    : mols_(std::move(mols)), chain_mol_(std::move(chain_mol)) {
  n_ = (int)chain_mol_.size();
  if (n_ <= 0) throw std::runtime_error("Ensemble: no chains");
  for (int m : chain_mol_)
    if (m < 0 || m >= (int)mols_.size()) throw std::runtime_error("Ensemble: bad molecule index");
  if ((int)betas.size() != n_) throw std::runtime_error("Ensemble: one beta per chain");
  dev_.reset(new DeviceSet(mols_));
  check_cuda(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "stream");
  stream_ = own_stream_;
  int vstride = dev_->set().max_vars, tstride = dev_->set().max_atoms;
  nmt_ = shared_stream ? 1 : n_;
  ntoat_ = shared_stream ? 1 : n_;
  if ((int)seeds.size() != nmt_) throw std::runtime_error("Ensemble: one seed per stream");
  ch_.nchains = n_;
  ch_.vstride = vstride;
  ch_.tstride = tstride;
  int* mol_of = dalloc<int>(allocs_, n_);
  h2d(mol_of, chain_mol_);
  ch_.mol_of_chain = mol_of;
  ch_.vlvr = dalloc<double>(allocs_, (size_t)n_ * vstride);
  ch_.toat = dalloc<double>(allocs_, (size_t)ntoat_ * tstride);
  std::vector<int> tslot(n_), mslot(n_);
  for (int c = 0; c < n_; ++c) {
    tslot[c] = shared_stream ? 0 : c;
    mslot[c] = shared_stream ? 0 : c;
  }
  int* dts = dalloc<int>(allocs_, n_);
  int* dms = dalloc<int>(allocs_, n_);
  h2d(dts, tslot);
  h2d(dms, mslot);
  ch_.toat_slot = dts;
  ch_.mt_slot = dms;
  ch_.mt = dalloc<uint32_t>(allocs_, (size_t)nmt_ * kMTWords);
  ch_.beta = dalloc<double>(allocs_, n_);
  ch_.eol = dalloc<double>(allocs_, n_);
  ch_.terms = dalloc<double>(allocs_, (size_t)n_ * 6);
  ch_.nacc = dalloc<unsigned long long>(allocs_, n_);
  ch_.nprop = dalloc<unsigned long long>(allocs_, n_);
  ch_.pterms = dalloc<unsigned long long>(allocs_, n_);
  ch_.err = dalloc<int>(allocs_, n_);
  ch_.coords = nullptr;
  ch_.sur = DSurrogate{};
  ch_.da_floor = 0.2f;
  ch_.da_min = 64;
  ch_.da_n1 = dalloc<unsigned long long>(allocs_, n_);
  ch_.da_n2 = dalloc<unsigned long long>(allocs_, n_);
  check_cuda(cudaMemset(ch_.da_n1, 0, n_ * sizeof(unsigned long long)), "memset");
  check_cuda(cudaMemset(ch_.da_n2, 0, n_ * sizeof(unsigned long long)), "memset");
  check_cuda(cudaMemset(ch_.nacc, 0, n_ * sizeof(unsigned long long)), "memset");
  check_cuda(cudaMemset(ch_.nprop, 0, n_ * sizeof(unsigned long long)), "memset");
  check_cuda(cudaMemset(ch_.err, 0, n_ * sizeof(int)), "memset");
  check_cuda(cudaMemset(ch_.eol, 0, n_ * sizeof(double)), "memset");
  check_cuda(cudaMemset(ch_.terms, 0, (size_t)n_ * 6 * sizeof(double)), "memset");
  // initial variables and dihedral state from the assembled molecules
  std::vector<double> vl((size_t)n_ * vstride, 0.0), to((size_t)ntoat_ * tstride, 0.0);
  for (int c = 0; c < n_; ++c) {
    const MolTopo& t = mols_[chain_mol_[c]]->topo;
    std::copy(t.vlvr0.begin(), t.vlvr0.end(), vl.begin() + (size_t)c * vstride);
  }
  for (int sl = 0; sl < ntoat_; ++sl) {
    const MolTopo& t = mols_[chain_mol_[sl]]->topo;
    std::copy(t.toat0.begin(), t.toat0.end(), to.begin() + (size_t)sl * tstride);
  }
  h2d(ch_.vlvr, vl);
  h2d(ch_.toat, to);
  h2d(ch_.beta, betas);
  int* dseed = dalloc<int>(allocs_, nmt_);
  h2d(dseed, seeds);
  check_cuda(launch_seed(ch_.mt, dseed, nmt_, stream_), "seed");
  check_cuda(cudaStreamSynchronize(stream_), "seed sync");
}

Ensemble::~Ensemble() {
  if (graph_) cudaGraphExecDestroy(graph_);
  if (stream_) cudaStreamSynchronize(stream_);
  if (own_stream_ && stream_ != own_stream_) cudaStreamSynchronize(own_stream_);
  for (void* p : allocs_) cudaFree(p);
  if (coords_buf_) cudaFree(coords_buf_);
  if (esolan_scratch_) cudaFree(esolan_scratch_);
  if (esolan_area_) cudaFree(esolan_area_);
  if (an_vold_) cudaFree(an_vold_);
  if (an_jvar_) cudaFree(an_jvar_);
  if (an_eolc_) cudaFree(an_eolc_);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Ensemble::set_surrogate(const DSurrogate* view, float floor, int min_stage1) {
  check_cuda(cudaStreamSynchronize(stream_), "set_surrogate sync");
  if (view) {
    if (view->w1 == nullptr) throw std::invalid_argument("set_surrogate: empty surrogate");
    for (int c = 0; c < n_; ++c)
      if (2 * molecule_of(c).topo.nfree != view->nin)
        throw std::invalid_argument("set_surrogate: the surrogate's input width does not match "
                                    "every chain's free dihedrals");
    if (floor < 0.f || floor > 1.f || min_stage1 < 0)
      throw std::invalid_argument("set_surrogate: floor in [0,1], min_stage1 >= 0");
    ch_.sur = *view;
    ch_.da_floor = floor;
    ch_.da_min = min_stage1;
  } else {
    ch_.sur = DSurrogate{};
  }
  dev_->set_da(view != nullptr);
  check_cuda(cudaMemset(ch_.da_n1, 0, n_ * sizeof(unsigned long long)), "memset");
  check_cuda(cudaMemset(ch_.da_n2, 0, n_ * sizeof(unsigned long long)), "memset");
  if (graph_) cudaGraphExecDestroy(graph_);   // kernel arguments changed
  graph_ = nullptr;
  graph_len_ = 0;
}

void Ensemble::gradient(std::vector<double>& g) {
  if (set().f.itysol != 0)
    throw std::invalid_argument("the GPU gradient is for the vacuum energy (itysol 0)");
  if (!grad_buf_) grad_buf_ = dalloc<double>(allocs_, (size_t)n_ * ch_.vstride);
  check_cuda(launch_gradient(set(), ch_, 0, n_, grad_buf_, stream_), "gradient launch");
  check_cuda(cudaStreamSynchronize(stream_), "gradient sync");
  d2h(g, grad_buf_, (size_t)n_ * ch_.vstride);
}

void Ensemble::set_pair_work(int form) {
  if (form < 0 || form > 2) throw std::invalid_argument("pair-work form must be 0, 1 or 2");
  const int rows_mode[3] = {0, 1, -1};
  dev_->set_rows(rows_mode[form]);
  if (graph_) cudaGraphExecDestroy(graph_);   // kernel arguments changed
  graph_ = nullptr;
  graph_len_ = 0;
}

int Ensemble::set_window(int k) {
  const int got = dev_->set_window(k);
  if (graph_) cudaGraphExecDestroy(graph_);   // kernel arguments changed
  graph_ = nullptr;
  graph_len_ = 0;
  return got;
}

// Autotuner: time one sweep of every chain with each pair-work form (0:
// pair lists; 1: 32-partner row passes; 2: row passes for molecules of 128
// atoms or more, lists for the rest), then the row form with speculative
// windows of 2, 4 and 8 proposals, each from the same saved state (best of
// three timed sweeps after a warm-up), keep the fastest, and put the state
// back.  The timed sweeps leave no trace.
int Ensemble::autotune(int flags, double* ms_out) {
  window_ms_[0] = window_ms_[1] = window_ms_[2] = 0.0;
  if (!dev_->any_rows_possible()) {
    if (ms_out) ms_out[0] = ms_out[1] = ms_out[2] = 0.0;
    set_window(1);
    return 0;
  }
  check_cuda(cudaStreamSynchronize(stream_), "autotune sync");
  const size_t nv = (size_t)n_ * ch_.vstride, nt = (size_t)ntoat_ * ch_.tstride,
               nm = (size_t)nmt_ * kMTWords;
  std::vector<double> v, t, e, tr;
  std::vector<uint32_t> mt;
  std::vector<unsigned long long> a, p, d1, d2, pt;
  std::vector<int> er;
  d2h(v, ch_.vlvr, nv);
  d2h(t, ch_.toat, nt);
  d2h(mt, ch_.mt, nm);
  d2h(e, ch_.eol, n_);
  d2h(tr, ch_.terms, (size_t)n_ * 6);
  d2h(a, ch_.nacc, n_);
  d2h(p, ch_.nprop, n_);
  d2h(pt, ch_.pterms, n_);
  d2h(d1, ch_.da_n1, n_);
  d2h(d2, ch_.da_n2, n_);
  d2h(er, ch_.err, n_);
  auto restore = [&] {
    h2d(ch_.vlvr, v);
    h2d(ch_.toat, t);
    h2d(ch_.mt, mt);
    h2d(ch_.eol, e);
    h2d(ch_.terms, tr);
    h2d(ch_.nacc, a);
    h2d(ch_.nprop, p);
    h2d(ch_.pterms, pt);
    h2d(ch_.da_n1, d1);
    h2d(ch_.da_n2, d2);
    h2d(ch_.err, er);
  };
  DWeight w{kWeightCanon, 0, 0, 1.0, nullptr, nullptr};
  cudaEvent_t e0, e1;
  check_cuda(cudaEventCreate(&e0), "event");
  check_cuda(cudaEventCreate(&e1), "event");
  auto time_sweep = [&]() {
    restore();
    launch_sweep_range(0, n_, 1, flags | kFlagNoCheck, w);   // warm-up
    check_cuda(cudaStreamSynchronize(stream_), "autotune sync");
    double best_ms = 1e300;
    for (int rep = 0; rep < 3; ++rep) {
      restore();
      check_cuda(cudaEventRecord(e0, stream_), "event");
      launch_sweep_range(0, n_, 1, flags | kFlagNoCheck, w);
      check_cuda(cudaEventRecord(e1, stream_), "event");
      check_cuda(cudaEventSynchronize(e1), "event sync");
      float f = 0.f;
      check_cuda(cudaEventElapsedTime(&f, e0, e1), "event time");
      best_ms = std::min(best_ms, (double)f);
    }
    return best_ms;
  };
  double ms[3] = {0.0, 0.0, 0.0};
  const int rows_mode[3] = {0, 1, -1};   // DeviceSet::set_rows argument of each form
  dev_->set_window(1);
  for (int mode = 0; mode < 3; ++mode) {
    dev_->set_rows(rows_mode[mode]);
    ms[mode] = time_sweep();
  }
  int best = 0;
  for (int mode = 1; mode < 3; ++mode)
    if (ms[mode] < ms[best]) best = mode;
  double best_ms = ms[best];
  int best_window = 1;
  const int windows[3] = {2, 4, 8};
  for (int k = 0; k < 3; ++k) {   // speculative windows need the row form
    dev_->set_rows(1);
    if (dev_->set_window(windows[k]) != windows[k]) break;
    window_ms_[k] = time_sweep();
    if (window_ms_[k] < best_ms) {
      best_ms = window_ms_[k];
      best = 1;
      best_window = windows[k];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dev_->set_window(best_window);
  dev_->set_rows(rows_mode[best]);
  restore();
  if (graph_) cudaGraphExecDestroy(graph_);   // kernel arguments changed
  graph_ = nullptr;
  graph_len_ = 0;
  if (ms_out) {
    ms_out[0] = ms[0];
    ms_out[1] = ms[1];
    ms_out[2] = ms[2];
  }
  return best;
}

void Ensemble::da_stats(std::vector<unsigned long long>& n1,
                        std::vector<unsigned long long>& n2) const {
  d2h(n1, ch_.da_n1, n_);
  d2h(n2, ch_.da_n2, n_);
}

void Ensemble::set_stream(cudaStream_t s) {
  check_cuda(cudaStreamSynchronize(stream_), "set_stream sync");
  stream_ = s ? s : own_stream_;
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  graph_len_ = 0;
}

void Ensemble::random_start() {
  std::vector<int> order(n_);
  std::iota(order.begin(), order.end(), 0);
  int* d = nullptr;
  check_cuda(cudaMallocAsync(&d, n_ * sizeof(int), stream_), "malloc");
  check_cuda(cudaMemcpyAsync(d, order.data(), n_ * sizeof(int), cudaMemcpyHostToDevice, stream_), "H2D");
  check_cuda(launch_random_start(set(), ch_, d, n_, stream_), "random_start");
  check_cuda(cudaFreeAsync(d, stream_), "free");
  check_cuda(cudaStreamSynchronize(stream_), "random_start sync");
}

// energy() of chains [first, first+count) (energy.f:12-119): setvar, rebuild
// and the ECEPP/3 terms in k_energy, with the numerical SASA there when
// itysol > 0; with itysol < 0 the rebuilt coordinates go to a buffer and
// k_esolan adds the analytic solvation term (energy.f:79-82), a batch of
// chains at a time.
void Ensemble::energy_launch(int first, int count, bool fp32, bool want_coords) {
  const bool analytic = set().f.itysol < 0;
  DChains c2 = ch_;
  if (analytic || want_coords) {
    if (!coords_buf_)
      check_cuda(cudaMalloc(&coords_buf_, (size_t)n_ * 3 * ch_.tstride * sizeof(double)), "malloc");
    c2.coords = coords_buf_;
  }
  check_cuda(launch_energy(set(), c2, first, count, fp32, stream_), "energy");
  if (!analytic) return;
  if (!esolan_scratch_) {
    check_cuda(cudaMalloc(&esolan_scratch_, esolan_scratch_bytes(kEsolanBatch)), "malloc");
    check_cuda(cudaMalloc(&esolan_area_, (size_t)n_ * ch_.tstride * sizeof(double)), "malloc");
  }
  for (int b = first; b < first + count; b += kEsolanBatch)
    check_cuda(launch_esolan(set(), c2, b, std::min(kEsolanBatch, first + count - b),
                             esolan_scratch_, esolan_area_, stream_),
               "esolan");
}

// Metropolis sweeps with the analytic SASA model (itysol < 0) for chains
// [first, first+count): metropolis.f:13-184 with one energy() per proposal,
// as the reference calls it, because esolan may draw from the chain's stream
// between a proposal's numbers and its acceptance number.  Each proposal is
// three launches over all chains: k_propose, energy(), k_decide.
void Ensemble::sweeps_analytic(int first, int count, int nsweeps, int flags, const DWeight& w) {
  if (flags & kFlagExtraSetvar)
    throw std::runtime_error("the serial PT schedule is not built for the analytic SASA model");
  if (ch_.sur.w1 != nullptr)
    throw std::runtime_error("delayed acceptance is not built for the analytic SASA model");
  int nfree = -1;
  for (int c = first; c < first + count; ++c) {   // no chain may see an extra energy()
    const int nf = mols_[chain_mol_[c]]->topo.nfree;
    if (nfree >= 0 && nf != nfree)
      throw std::runtime_error("analytic SASA sweeps: chains of one launch need the same free "
                               "dihedrals");
    nfree = nf;
  }
  if (!an_vold_) {
    check_cuda(cudaMalloc(&an_vold_, n_ * sizeof(double)), "malloc");
    check_cuda(cudaMalloc(&an_jvar_, n_ * sizeof(int)), "malloc");
    check_cuda(cudaMalloc(&an_eolc_, n_ * sizeof(double)), "malloc");
  }
  const bool fp32 = (flags & kFlagFP32) != 0;
  const int rnd = (flags & kFlagRndOrd) ? 1 : 0;
  const double tol = fp32 ? check_tol_fp32 : check_tol;
  for (int sw = 0; sw < nsweeps; ++sw) {
    energy_launch(first, count, fp32, false);   // metropolis.f:35
    check_cuda(launch_copy_eol(ch_, first, count, an_eolc_, stream_), "copy eol");
    for (int p = 0; p < nfree; ++p) {
      check_cuda(launch_propose(set(), ch_, first, count, p, rnd, an_vold_, an_jvar_, stream_),
                 "propose");
      energy_launch(first, count, fp32, false);
      check_cuda(launch_decide(ch_, w, first, count, an_vold_, an_jvar_, an_eolc_, stream_),
                 "decide");
    }
    energy_launch(first, count, fp32, false);   // metropolis.f:172-179
    check_cuda(launch_close(ch_, first, count, an_eolc_, (flags & kFlagNoCheck) ? 0 : 1, tol,
                            stream_),
               "close");
  }
}

void Ensemble::energy(bool fp32) {
  energy_launch(0, n_, fp32, false);
  check_cuda(cudaStreamSynchronize(stream_), "energy sync");
}

void Ensemble::energy_chain(int c, bool fp32) { energy_launch(c, 1, fp32, false); }

void Ensemble::launch_sweep_range(int first, int count, int nsweeps, int flags, const DWeight& w) {
  if (set().f.itysol < 0) {
    sweeps_analytic(first, count, nsweeps, flags, w);
    return;
  }
  double tol = (flags & kFlagFP32) ? check_tol_fp32 : check_tol;
  check_cuda(sweep_launch(set(), ch_, w, first, count, nsweeps, flags, tol, stream_), "sweep");
}

void Ensemble::sweeps(int nsweeps, int flags, const DWeight& w) {
  if (nmt_ == 1 && n_ > 1) {   // shared stream: chains strictly one after another
    for (int c = 0; c < n_; ++c) launch_sweep_range(c, 1, nsweeps, flags, w);
  } else {
    launch_sweep_range(0, n_, nsweeps, flags, w);
  }
  check_cuda(cudaStreamSynchronize(stream_), "sweeps sync");
}

void Ensemble::sweeps_chain(int c, int nsweeps, int flags, const DWeight& w) {
  launch_sweep_range(c, 1, nsweeps, flags, w);
}

void Ensemble::equilibrate(int nequi, int flags) {
  DWeight w{kWeightCanon, 0, 0, 1.0, nullptr, nullptr};
  bool fp32 = (flags & kFlagFP32) != 0;
  if (nmt_ == 1 && n_ > 1) {
    for (int c = 0; c < n_; ++c) {
      energy_chain(c, fp32);
      if (nequi > 0) launch_sweep_range(c, 1, nequi, flags, w);
    }
  } else {
    check_cuda(launch_energy(set(), ch_, 0, n_, fp32, stream_), "energy");
    if (nequi > 0) launch_sweep_range(0, n_, nequi, flags, w);
  }
  check_cuda(cudaStreamSynchronize(stream_), "equilibrate sync");
}

void Ensemble::set_pt(const std::vector<double>& betas, int wrap, int exchange_seed) {
  if ((int)betas.size() != n_) throw std::runtime_error("set_pt: one temperature per chain");
  pt_.n = n_;
  pt_.wrap = wrap;
  pt_.temp_chain = dalloc<int>(allocs_, n_);
  pt_.betas = dalloc<double>(allocs_, n_);
  pt_.mt = dalloc<uint32_t>(allocs_, kMTWords);
  pt_.iswitch = dalloc<int>(allocs_, 1);
  pt_.stats = dalloc<unsigned long long>(allocs_, 2 * n_);
  pt_.lq = dalloc<double>(allocs_, kQueue);
  pt_.bar = dalloc<unsigned>(allocs_, 2);
  std::vector<int> tc(n_);
  std::iota(tc.begin(), tc.end(), 0);
  h2d(pt_.temp_chain, tc);
  h2d(pt_.betas, betas);
  h2d(ch_.beta, betas);
  std::vector<int> one{1};
  h2d(pt_.iswitch, one);
  check_cuda(cudaMemset(pt_.stats, 0, 2 * n_ * sizeof(unsigned long long)), "memset");
  if (nmt_ == 1) {
    pt_.mt = ch_.mt;   // partem_s: the exchange draws from the same stream
  } else {
    int* ds = dalloc<int>(allocs_, 1);
    std::vector<int> sd{exchange_seed};
    h2d(ds, sd);
    check_cuda(launch_seed(pt_.mt, ds, 1, stream_), "seed");
  }
  check_cuda(cudaStreamSynchronize(stream_), "set_pt sync");
}

void Ensemble::set_pt_fused(bool on, double timeout_s, unsigned barrier_extra) {
  if (!(timeout_s > 0.0)) throw std::runtime_error("set_pt_fused: timeout must be positive");
  pt_.fused = on;
  pt_.timeout_s = timeout_s;
  pt_.barrier_extra = barrier_extra;
}

void Ensemble::pt_sweeps(int nsweeps, int flags, bool serial, int graph_chunk) {
  if (pt_.n != n_) throw std::runtime_error("pt_sweeps: call set_pt first");
  DWeight w{kWeightCanon, 0, 0, 1.0, nullptr, nullptr};
  pt_fused_last_ = false;
  if (serial) {
    std::vector<int> tc;
    for (int s = 0; s < nsweeps; ++s) {
      d2h(tc, pt_.temp_chain, n_);
      for (int k = 0; k < n_; ++k) launch_sweep_range(tc[k], 1, 1, flags | kFlagExtraSetvar, w);
      check_cuda(launch_exchange(ch_, pt_.temp_chain, pt_.betas, n_, pt_.mt, pt_.iswitch, pt_.wrap,
                                 pt_.stats, stream_),
                 "exchange");
      check_cuda(cudaStreamSynchronize(stream_), "pt sync");
    }
    return;
  }
  if (set().f.itysol < 0) {   // analytic SASA: host-driven sweeps, then the exchange
    for (int s = 0; s < nsweeps; ++s) {
      launch_sweep_range(0, n_, 1, flags, w);
      check_cuda(launch_exchange(ch_, pt_.temp_chain, pt_.betas, n_, pt_.mt, pt_.iswitch, pt_.wrap,
                                 pt_.stats, stream_),
                 "exchange");
    }
    check_cuda(cudaStreamSynchronize(stream_), "pt sync");
    return;
  }
  double tol = (flags & kFlagFP32) ? check_tol_fp32 : check_tol;
  if (pt_.fused && nmt_ != 1 && nsweeps > 0) {
    // every chain resident at once: sweeps and exchanges in one launch, the
    // rounds separated by grid barriers
    check_cuda(cudaMemsetAsync(pt_.bar, 0, 2 * sizeof(unsigned), stream_), "memset");
    DPTFused f{1,          n_,        pt_.wrap,   pt_.temp_chain, pt_.betas,
               pt_.mt,     pt_.lq,    pt_.iswitch, pt_.stats,     pt_.bar,
               (unsigned long long)(pt_.timeout_s * 1e9), pt_.barrier_extra};
    cudaError_t e = sweep_launch_pt(set(), ch_, w, n_, nsweeps, flags, tol, f, stream_);
    if (e == cudaSuccess) {
      pt_fused_last_ = true;
      check_cuda(cudaStreamSynchronize(stream_), "pt sync");
      return;
    }
    if (e != cudaErrorCooperativeLaunchTooLarge && e != cudaErrorNotSupported)
      check_cuda(e, "fused pt launch");
    (void)cudaGetLastError();   // not possible here: take the graph path
  }
  auto enqueue = [&](int k) {
    for (int i = 0; i < k; ++i) {
      check_cuda(sweep_launch(set(), ch_, w, 0, n_, 1, flags, tol, stream_), "sweep");
      check_cuda(launch_exchange(ch_, pt_.temp_chain, pt_.betas, n_, pt_.mt, pt_.iswitch, pt_.wrap,
                                 pt_.stats, stream_),
                 "exchange");
    }
  };
  if (graph_chunk <= 1) {
    enqueue(nsweeps);
  } else {
    if (!graph_ || graph_len_ != graph_chunk || graph_flags_ != flags) {
      if (graph_) cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
      // attribute calls happen outside the capture
      check_cuda(sweep_launch(set(), ch_, w, 0, 0, 0, flags, tol, stream_), "prep");
      cudaGraph_t g;
      check_cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
      enqueue(graph_chunk);
      check_cuda(cudaStreamEndCapture(stream_, &g), "end capture");
      check_cuda(cudaGraphInstantiate(&graph_, g, 0), "instantiate");
      cudaGraphDestroy(g);
      graph_len_ = graph_chunk;
      graph_flags_ = flags;
    }
    int full = nsweeps / graph_chunk, rest = nsweeps % graph_chunk;
    for (int i = 0; i < full; ++i) check_cuda(cudaGraphLaunch(graph_, stream_), "graph launch");
    enqueue(rest);
  }
  check_cuda(cudaStreamSynchronize(stream_), "pt sync");
}

void Ensemble::pt_map(std::vector<int>& tc) const { d2h(tc, pt_.temp_chain, pt_.n); }
void Ensemble::pt_stats(std::vector<unsigned long long>& s) const { d2h(s, pt_.stats, 2 * pt_.n); }

void Ensemble::pt_get_state(std::vector<int>& tc, int& iswitch, std::vector<uint32_t>& mt,
                            std::vector<double>& betas) const {
  d2h(tc, pt_.temp_chain, pt_.n);
  std::vector<int> sw;
  d2h(sw, pt_.iswitch, 1);
  iswitch = sw[0];
  d2h(mt, pt_.mt, kMTWords);
  d2h(betas, pt_.betas, pt_.n);
}
void Ensemble::pt_set_state(const std::vector<int>& tc, int iswitch,
                            const std::vector<uint32_t>& mt, const std::vector<double>& betas) {
  if ((int)tc.size() != pt_.n || mt.size() != (size_t)kMTWords || (int)betas.size() != pt_.n)
    throw std::runtime_error("pt_set_state: size");
  h2d(pt_.temp_chain, tc);
  h2d(pt_.iswitch, std::vector<int>{iswitch});
  h2d(pt_.mt, mt);
  h2d(pt_.betas, betas);
}

void Ensemble::get_vlvr(std::vector<double>& v) const { d2h(v, ch_.vlvr, (size_t)n_ * ch_.vstride); }
void Ensemble::set_vlvr(const std::vector<double>& v) {
  if (v.size() != (size_t)n_ * ch_.vstride) throw std::runtime_error("set_vlvr: size");
  h2d(ch_.vlvr, v);
}
void Ensemble::get_eol(std::vector<double>& e) const { d2h(e, ch_.eol, n_); }
void Ensemble::get_terms(std::vector<double>& t) const { d2h(t, ch_.terms, (size_t)n_ * 6); }
void Ensemble::get_acceptance(std::vector<unsigned long long>& a,
                              std::vector<unsigned long long>& p) const {
  d2h(a, ch_.nacc, n_);
  d2h(p, ch_.nprop, n_);
}
void Ensemble::get_errors(std::vector<int>& e) const { d2h(e, ch_.err, n_); }
void Ensemble::get_pair_terms(std::vector<unsigned long long>& p) const { d2h(p, ch_.pterms, n_); }
void Ensemble::set_acceptance(const std::vector<unsigned long long>& acc,
                              const std::vector<unsigned long long>& prop) {
  if ((int)acc.size() != n_ || (int)prop.size() != n_) throw std::runtime_error("set_acceptance: size");
  h2d(ch_.nacc, acc);
  h2d(ch_.nprop, prop);
}
void Ensemble::get_betas(std::vector<double>& b) const { d2h(b, ch_.beta, n_); }
void Ensemble::set_betas(const std::vector<double>& b) {
  if ((int)b.size() != n_) throw std::runtime_error("set_betas: size");
  h2d(ch_.beta, b);
}
void Ensemble::get_mt(std::vector<uint32_t>& m) const { d2h(m, ch_.mt, (size_t)nmt_ * kMTWords); }
void Ensemble::set_mt(const std::vector<uint32_t>& m) {
  if (m.size() != (size_t)nmt_ * kMTWords) throw std::runtime_error("set_mt: size");
  h2d(ch_.mt, m);
}
void Ensemble::get_toat(std::vector<double>& t) const { d2h(t, ch_.toat, (size_t)ntoat_ * ch_.tstride); }
void Ensemble::set_toat(const std::vector<double>& t) {
  if (t.size() != (size_t)ntoat_ * ch_.tstride) throw std::runtime_error("set_toat: size");
  h2d(ch_.toat, t);
}

void Ensemble::get_coords(std::vector<double>& xyz) {
  // a full rebuild of every chain into a coordinate buffer (state unchanged
  // apart from the setvar call the reference's energy() also makes)
  energy_launch(0, n_, false, true);
  check_cuda(cudaStreamSynchronize(stream_), "coords sync");
  d2h(xyz, coords_buf_, (size_t)n_ * 3 * ch_.tstride);
}

void Ensemble::draw(int slot, int n, std::vector<double>& out) {
  double* d = nullptr;
  check_cuda(cudaMalloc(&d, std::max(n, 1) * sizeof(double)), "malloc");
  check_cuda(launch_draw(ch_.mt, slot, n, d, stream_), "draw");
  check_cuda(cudaStreamSynchronize(stream_), "draw sync");
  d2h(out, d, n);
  cudaFree(d);
}

}  // namespace smmpb200
