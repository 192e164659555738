/*
 * smmp_b200.h -- C ABI of the B200 implementation of SMMP's energy-and-sweep
 * path (libsmmp_b200.so).
 *
 * Two layers:
 *
 *  1. The reference-facing layer.  One global system, as SMMP keeps its state
 *     in COMMON blocks; each entry point replaces the f2py binding of the
 *     reference routine cited beside it (trunk/smmp.pyf, trunk/<file>.f).
 *     Angles are radians, energies kcal/mol, variables 0-based arrays over
 *     all variables of the system (the reference's vlvr(1..ntlvr)).
 *
 *  2. The batched layer.  Independent molecules (smmp_mol_*) and ensembles of
 *     chains / replicas (smmp_ens_*) whose whole state stays on the GPU; this
 *     has no single counterpart in the reference -- it replaces the loops of
 *     partem_s.f and canon.f over many replicas.
 *
 * Every function returning int returns 0 on success and a nonzero status on
 * failure; smmp_last_error() then describes the failure (thread-local).  The
 * library never aborts the process where the reference would STOP.
 */
#ifndef SMMP_B200_H
#define SMMP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define SMMP_OK 0
#define SMMP_ERR_ARG 1       /* invalid argument or call order */
#define SMMP_ERR_INPUT 2     /* unreadable / inconsistent input files */
#define SMMP_ERR_CUDA 3      /* CUDA runtime error or no usable GPU */
#define SMMP_ERR_KERNEL 4    /* a kernel reported an error word (see below) */

/* Per-chain error words reported by the kernels (smmp_ens_errors). */
#define SMMP_KERR_NONFINITE 1     /* NaN/Inf energy */
#define SMMP_KERR_CONSISTENCY 2   /* |E_incremental - E_fresh| > tolerance at sweep end */
#define SMMP_KERR_NEIGHBOURS 3    /* reserved, never set: an atom with more SASA neighbours than the per-warp buffer holds is scanned directly */
#define SMMP_KERR_TIMEOUT 4       /* a bounded wait gave up */

/* Switches of the reference's COMMON blocks /epar_l/ (sh2, epsd, ientyp),
 * /isolty/ (itysol) and /updchois/ (rndord, upchswitch); INCL.H:224-327.
 * Only ientyp=0 (ECEPP/2-3), itysol in {-9..9}, upchswitch=0 are on this path
 * (itysol < 0, the analytic SASA of esolan.f, for energy evaluations only). */
typedef struct smmp_config {
  int sh2;        /* 1: ECEPP/2 library (lib.sh2), 0: ECEPP/3 (lib.sh3) */
  int epsd;       /* 1: sigmoidal distance-dependent dielectric */
  int itysol;     /* 0: vacuum, 1..9: numerical SASA model (enysol.f),
                     -1..-9: analytic SASA, same parameter sets (esolan.f) */
  int ientyp;     /* must be 0 (ECEPP) */
  int rndord;     /* 1: random variable order in a sweep */
  int upchswitch; /* must be 0 (no biased Gaussian steps) */
} smmp_config_t;

/* Sampling weight W(E) of metropolis (its `dummy` callback argument,
 * smmp.pyf:3-10): kind 0 = can_weight beta*E (canon.f:135-149);
 * 1 = muca_weight (beta+b[k])*E+alpha[k]; 2 = muca_weight2 b[k]*E+alpha[k]
 * (mulcan_par_mod.f90:380-410), k = int(clamp(E/ebin+sign(1/2,E),kmin,kmax)),
 * b and alpha indexed k-kmin; 3 = host callback (callback(E, user)). */
typedef double (*smmp_weight_fn)(double energy, void* user);
typedef struct smmp_weight {
  int kind;
  int kmin, kmax;
  double ebin;
  const double* b;
  const double* alpha;
  smmp_weight_fn callback;
  void* user;
} smmp_weight_t;

const char* smmp_last_error(void);
/* 1 if a CUDA device is usable by this library. */
int smmp_gpu_available(void);

/* ---------------------------------------------------------------- layer 1 */

/* Drop the global system (molecule, GPU state, switches, stream), as a
 * fresh process of the reference starts from its BLOCK DATA defaults. */
int smmp_reset(void);

int smmp_set_config(const smmp_config_t* cfg);   /* write the COMMON switches */
int smmp_get_config(smmp_config_t* cfg);

/* init_energy(libdir): smmp.pyf:4404, init_energy.f:14.  libdir holds
 * lib.sh3 / lib.sh2 and tes.dat. */
int smmp_init_energy(const char* libdir);

/* init_molecule(iabin, grpn, grpc, seqfile, varfile): smmp.pyf:5011-5016,
 * init_molecule.f:13.  iabin must be 1 (sequence + variables); PDB input is
 * outside this path.  varfile may be NULL or blank. */
int smmp_init_molecule(int iabin, const char* grpn, const char* grpc, const char* seqfile,
                       const char* varfile);

/* energy(): smmp.pyf:380, energy.f:12.  Uses the current variables (as
 * written by smmp_set_vlvr or a previous call) and updates the dihedral
 * state as setvar does. */
int smmp_energy(double* e_out);
/* Terms of the last energy evaluation: eyel, eyvw, eyhb, eyvr, eysl, eysm
 * (COMMON /eny_r/, INCL.H:343-349). */
int smmp_energy_terms(double terms[6]);

/* enysol(nmol=0): smmp.pyf:664-665, enysol.f:13.  The numerical solvation
 * energy eysl of the current conformation (nmol 0 or 1: the one molecule).
 * The reference sums it over the coordinates of the last rebuild; here the
 * conformation is rebuilt from the current variables (as energy() does) and
 * its eysl returned; the energy terms are updated as by smmp_energy.  Needs a
 * numerical SASA model (itysol 1..9), else SMMP_ERR_ARG. */
int smmp_enysol(int nmol, double* eysl);

/* setvar(nml, vlvrx): smmp.pyf:949-950, setvar.f:13.  Sets the variables of
 * molecule nml (1-based) and rebuilds its coordinates. */
int smmp_setvar(int nml, const double* vlvrx);

/* metropolis(eol1, acz, dummy): smmp.pyf:22-25, metropolis.f:13.  One sweep;
 * eol and acz are updated in place as the f2py intent(in,out) arguments. */
int smmp_metropolis(double* eol, double* acz, const smmp_weight_t* w);

/* Multicanonical weight recursion of mulcan_par (mulcan_par_mod.f90:93-145),
 * host only: the histogram ihist of the last sweeps (zeroed on return)
 * updates xhist, g1, b, alpha, ent for bins kmin..kmax (arrays of
 * kmax-kmin+1, index k-kmin); beta = 1/(k_B T).  smmp_muca_finish folds beta
 * into b and recomputes alpha (mulcan_par_mod.f90:163-168), the weights of
 * muca_weight2 (smmp_weight_t kind 2). */
int smmp_muca_update(int kmin, int kmax, double ebin, double beta, int* ihist, double* xhist,
                     double* g1, double* b, double* alpha, double* ent);
int smmp_muca_finish(int kmin, int kmax, double ebin, double beta, double* b, double* alpha);

/* outvar(nml, fileName): outvar.f:12.  The current variables in the .var
 * command language; fileName "" (or blanks): standard output.  nml 0 or 1. */
int smmp_outvar(int nml, const char* fileName);
/* outpdb(nml, fileName): outpdb.f:12.  The current conformation (rebuilt
 * from the variables) in PDB format; fileName "" (or blanks): standard output. */
int smmp_outpdb(int nml, const char* fileName);

/* gradient(): gradient.f:13 (opeshe.f:12-317), vacuum energy (itysol 0).
 * Sets the variables and rebuilds (as setvar), then gdeyvr[ntlvr] = dE/dv of
 * every variable (COMMON /eny_r/ gdeyvr) and *eysm the energy; the terms as
 * smmp_energy_terms gives them.  FP64 on the GPU. */
int smmp_gradient(double* gdeyvr, double* eysm);
/* minim(imin, maxit, eps): smmp.pyf:1234, minim.f:13.  Minimises the energy
 * over the free variables with the GPU gradient: imin 1 quasi-Newton (BFGS),
 * 2 conjugate gradients (Polak-Ribiere+), each with a strong-Wolfe line
 * search; stops when the squared gradient is below eps, after maxit energy
 * and gradient evaluations, or when a line search makes no progress.  The
 * variables are left at the minimum (wrapped into (-pi, pi]) and the energy
 * re-evaluated; *nop (if not NULL) = evaluations used.  The search path is
 * this library's own, not minqsn.f's: the same minimum, not the same steps.
 * Vacuum energy (itysol 0) only. */
int smmp_minim(int imin, int maxit, double eps, int* nop);

/* sgrnd(seed) / grnd(): smmp.pyf:5620, twister.f:64 and :104. */
int smmp_sgrnd(int32_t seed);
double smmp_grnd(void);

/* canon(nequi, nswp, nmes, temp, lrand): smmp.pyf:3522-3527, canon.f:12.
 * Energies after every nmes-th sweep are written to trace (if not NULL,
 * nswp/nmes+1 values); out[0..2] = energy after equilibration, acceptance
 * rate, last energy (if out is not NULL). */
int smmp_canon(int nequi, int nswp, int nmes, double temp, int lrand, double* trace,
               double* out);

/* anneal(nequi, nswp, nmes, tmax, tmin, lrand): smmp.pyf:2663, anneal.f:13.
 * out[0..5] = start energy, energy after equilibration, acceptance, last
 * energy, lowest energy, sweep of the lowest energy. */
int smmp_anneal(int nequi, int nswp, int nmes, double tmax, double tmin, int lrand, double* out);

/* COMMON views: /bet/ beta, /mol_par/ nvr, /var_r/ vlvr axvr, /var_i/ idvr. */
int smmp_set_beta(double beta);
double smmp_get_beta(void);
int smmp_get_sizes(int* natoms, int* ntlvr, int* nvr);
int smmp_get_vlvr(double* vlvr);          /* [ntlvr] */
int smmp_set_vlvr(const double* vlvr);    /* [ntlvr] */
int smmp_get_idvr(int* idvr);             /* [nvr], 1-based variable indices */
int smmp_get_axvr(double* axvr);          /* [ntlvr] */
int smmp_get_coords(double* xyz);         /* [natoms*3] after a rebuild */
int smmp_get_acceptance(long long* ncalls, long long* nacalls);   /* /updstats/ */

/* ---------------------------------------------------------------- layer 2 */

typedef struct smmp_mol smmp_mol_t;
typedef struct smmp_ens smmp_ens_t;

/* Assemble one molecule (init_energy + init_molecule on a private system). */
smmp_mol_t* smmp_mol_build(const char* libdir, const smmp_config_t* cfg, const char* seqfile,
                           const char* varfile, const char* grpn, const char* grpc);
void smmp_mol_free(smmp_mol_t* m);
/* info[0..5] = natoms, nvar (all), nvr (free), pair terms per evaluation,
 * number of heavy (SASA) atoms, residues. */
int smmp_mol_info(const smmp_mol_t* m, long long info[6]);

/* 0-based indices (into the molecule's variables) of its free dihedrals, in
 * idvr order (redvar.f); info[2] of them. */
int smmp_mol_idvr(const smmp_mol_t* m, int* idvr);
/* The molecule's variables as built (library values, then the .var file's
 * settings; redvar.f): vlvr[nvar] in radians. */
int smmp_mol_vlvr0(const smmp_mol_t* m, double* vlvr);
/* The atoms each variable moves, as the contiguous 0-based range
 * [lo[v], hi[v]] of the molecule's atom order (nvar entries each). */
int smmp_mol_var_ranges(const smmp_mol_t* m, int* lo, int* hi);
/* The atoms as built (init_molecule.f:60-136: getmol, addend, redvar), 0-based:
 * parent[i] (-1 for the first atom), ECEPP class type[i] (1..18), charge[i],
 * and geom[4*i..4*i+3] = bond length, valence angle, dihedral (radians; the
 * dihedral state the variable file leaves), solvation radius. */
int smmp_mol_atoms(const smmp_mol_t* m, int* parent, int* type, double* charge, double* geom);
/* The variables (getmol.f:206-232, addend.f:583-660, redvar.f): per variable
 * info[4*v..4*v+3] = primary atom (0-based), torsion class, 1 if fixed by the
 * variable file, residue (0-based); nvar rows. */
int smmp_mol_vars(const smmp_mol_t* m, int* info);
/* The interaction lists (mklist.f:12-303): pairs[3*k..3*k+2] = listing atom,
 * partner, 1 for a 1-4 pair (0 normal), for the info[3] pair terms of one
 * energy evaluation, each pair once. */
int smmp_mol_pairs(const smmp_mol_t* m, int* pairs);
/* outvar.f:50-121 (outvbs) for one molecule, host only: the text outvar
 * writes for variables vlvr (radians, all variables of the molecule), with
 * molecule number iml in the line prefix.  buf NULL: *len = the bytes needed
 * (final NUL included); else *len is buf's size on entry. */
int smmp_mol_outvar(const smmp_mol_t* m, const double* vlvr, int iml, char* buf, uint64_t* len);
/* outpdb.f:12-185 for one molecule, host only: PDB text (80-column ATOM/HETATM,
 * TER, CONECT and END lines) of coordinates xyz[3*natoms] (Angstrom).  buf
 * and *len as for smmp_mol_outvar. */
int smmp_mol_outpdb(const smmp_mol_t* m, const double* xyz, char* buf, uint64_t* len);
/* An ensemble of nchains chains; chain c is a copy of mols[chain_mol[c]].
 * betas[c] is its inverse temperature.  shared_stream=0: chain c draws from
 * its own MT19937 stream seeded seeds[c]; shared_stream=1: all chains share
 * one stream (seeds[0]) and one dihedral state, visited in turn as partem_s.f
 * does.  flags: SMMP_ENS_FP32 selects FP32 pair terms (FP64 guard and
 * accumulation); otherwise pair terms are FP64. */
#define SMMP_ENS_FP32 2
#define SMMP_ENS_RNDORD 1
smmp_ens_t* smmp_ens_create(smmp_mol_t* const* mols, int nmols, const int* chain_mol,
                            int nchains, const int* seeds, const double* betas,
                            int shared_stream, int flags);
void smmp_ens_free(smmp_ens_t* e);
/* Launch the ensemble's work on a caller's cudaStream_t (NULL: the
 * ensemble's own stream), e.g. to time it with events on that stream. */
int smmp_ens_set_stream(smmp_ens_t* e, void* stream);
int smmp_ens_random_start(smmp_ens_t* e);          /* canon.f:60-67 per chain */
int smmp_ens_energy(smmp_ens_t* e, double* eol);   /* energy() of every chain */
/* Per-chain start of partem_s.f:134-162: energy() then nequi sweeps of
 * each chain at its own beta, chains in order (one after another when they
 * share a stream). */
int smmp_ens_equilibrate(smmp_ens_t* e, int nequi);
/* nsweeps metropolis sweeps of every chain with weight w (NULL: canonical). */
int smmp_ens_sweeps(smmp_ens_t* e, int nsweeps, const smmp_weight_t* w);
/* Parallel tempering: betas[k] of temperature label k (chain k starts at
 * label k); wrap=1 pairs label n with 1 (partem_s.f:222). */
int smmp_ens_set_pt(smmp_ens_t* e, const double* betas, int wrap, int exchange_seed);
/* nsweeps of (one sweep of every chain, then one exchange).  serial=1 visits
 * chains one at a time in label order (the partem_s.f schedule); serial=0
 * runs all chains at once, captured in CUDA graphs of graph_chunk sweeps. */
int smmp_ens_pt_sweeps(smmp_ens_t* e, int nsweeps, int serial, int graph_chunk);
/* Batched runs (serial=0) go as one cooperative launch when every chain can
 * be resident at once (on by default): each sweep ends at a grid barrier, one
 * warp exchanges, a second barrier hands out the new temperatures.  A barrier
 * wait longer than timeout_s seconds ends the run with error code 4.  Results
 * are bit-identical to the graph path.  barrier_extra is 0 except in tests of
 * that bounded wait: the barriers then wait for arrivals that never come.
 * No counterpart in the reference. */
int smmp_ens_set_pt_fused(smmp_ens_t* e, int on, double timeout_s, int barrier_extra);
int smmp_ens_pt_fused_last(smmp_ens_t* e, int* fused);   /* 1: last run was fused */
int smmp_ens_pt_map(smmp_ens_t* e, int* temp_chain);   /* ipoi, 0-based chains */
/* Exchange statistics since smmp_ens_set_pt: stats[2k] attempts and
 * stats[2k+1] accepted exchanges of the label pair (k, k+1) (k = n-1: the
 * periodic pair (n-1, 0)); partem_s.f:210-232. */
int smmp_ens_pt_stats(smmp_ens_t* e, uint64_t* stats);
/* Pair terms the sweeps of each chain have evaluated (no counterpart in the
 * reference, which sums every pair at every energy() call): full sums at the
 * sweep's opening and closing evaluations and re-sums, every pair of a
 * proposal summed in full, and twice the pairs across a proposal's bond in
 * the incremental mode.  Delayed-acceptance sweeps are not counted. */
int smmp_ens_pair_terms(smmp_ens_t* e, uint64_t* terms);
/* gradient.f (vacuum) for every chain: grad[chain * vstride + v] = dE/dv of
 * every variable (FP64), energies[chain] the energy (may be NULL).  The chains'
 * dihedral states go through setvar as in the reference. */
int smmp_ens_gradient(smmp_ens_t* e, double* grad, double* energies);
int smmp_ens_sizes(smmp_ens_t* e, int* nchains, int* vstride, int* tstride);
int smmp_ens_get_energies(smmp_ens_t* e, double* eol);          /* [nchains] */
int smmp_ens_get_terms(smmp_ens_t* e, double* terms);           /* [nchains*6] */
int smmp_ens_get_vlvr(smmp_ens_t* e, double* vlvr);             /* [nchains*vstride] */
int smmp_ens_set_vlvr(smmp_ens_t* e, const double* vlvr);
int smmp_ens_get_betas(smmp_ens_t* e, double* betas);
int smmp_ens_get_coords(smmp_ens_t* e, double* xyz);            /* [nchains*3*tstride] */
int smmp_ens_acceptance(smmp_ens_t* e, unsigned long long* acc, unsigned long long* prop);
int smmp_ens_errors(smmp_ens_t* e, int* err);                   /* [nchains] */
/* Draw n numbers from MT stream slot (grnd of that stream). */
int smmp_ens_draw(smmp_ens_t* e, int slot, int n, double* out);
/* Checkpoint: variables, dihedral state, MT19937 states, betas, energies and
 * the PT map, so that a restored ensemble continues bit-identically.
 * smmp_ens_checkpoint with buf=NULL returns the size in *bytes. */
int smmp_ens_checkpoint(smmp_ens_t* e, void* buf, uint64_t* bytes);
int smmp_ens_restore(smmp_ens_t* e, const void* buf, uint64_t bytes);

/* ---------------------------------------------------------------- surrogate
 * Learned energy surrogate (no counterpart in the reference): an MLP on the
 * sin/cos of the nang free dihedrals, 3 hidden layers of 256 with SiLU, BF16
 * weights and FP32 accumulation, trained on the GPU by the library's own
 * tensor-core forward/backward kernels with Adam.  Angles are [n*nang]
 * radians (FP64, row-major), energies kcal/mol. */
typedef struct smmp_sur smmp_sur_t;
smmp_sur_t* smmp_sur_create(int nang, uint64_t seed);
void smmp_sur_free(smmp_sur_t* s);
/* nin = 2*nang inputs, padded to nin_pad; nparams FP32 parameters in the
 * order W1[nin_pad][256] b1 W2[256][256] b2 W3[256][256] b3 w4[256] b4. */
int smmp_sur_sizes(smmp_sur_t* s, int* nin, int* nin_pad, int64_t* nparams);
/* Training set; energies above clip are clipped, targets normalised by the
 * set's mean and standard deviation (kept as {mu, sigma}). */
int smmp_sur_set_data(smmp_sur_t* s, const double* ang, const double* energy, int n, double clip);
/* epochs of minibatch Adam; *loss = mean squared error of the last epoch in
 * normalised units. */
int smmp_sur_train(smmp_sur_t* s, int epochs, int batch, double lr, uint64_t shuffle_seed,
                   double* loss);
int smmp_sur_predict(smmp_sur_t* s, const double* ang, int n, double* energy_out);
/* Gradient of the batch's mean squared error (normalised units) with respect
 * to every parameter, without an update. */
int smmp_sur_gradients(smmp_sur_t* s, const double* ang, const double* energy, int n,
                       float* grad_out, double* loss);
/* The forward pass of smmp_sur_predict for callers that cannot allocate
 * device memory when they need a prediction (a framework's caching allocator
 * owns the memory budget, or allocation is forbidden in a real-time loop).
 * No counterpart in the reference.  It allocates nothing: ang_dev
 * ([n*nang] FP32 radians) and energy_dev ([n] FP64) are device pointers the
 * caller owns, and the intermediate activations live in one fixed 16 MiB
 * device array that every GPU loading the library holds until exit.  n above
 * the rows that fit (3,563 for 24 dihedrals, 2,757 for 365) is
 * rejected with SMMP_ERR_ARG.  The GPU on which the surrogate was created
 * (it holds the weights) must be the current device; a call made while
 * another device is current is rejected with SMMP_ERR_ARG before anything
 * runs.  The first call on a device looks up the
 * array's device address; make it before any stream capture.  Calls share
 * the array: calls that overlap on the GPU race. stream: a cudaStream_t or
 * NULL (the default stream). */
int smmp_sur_predict_noalloc(smmp_sur_t* s, const float* ang_dev, int n, double* energy_dev,
                             void* stream);
/* Delayed acceptance (no counterpart in the reference): sweeps of the
 * ensemble screen each proposal with the surrogate first (stage 1) and
 * evaluate the exact energy only for proposals that pass; the second stage
 * corrects with the exact energy, so the stationary distribution is that of
 * the plain sweep.  A chain whose stage-2 acceptance falls below `floor`
 * after min_stage1 stage-1 passes takes plain steps from its next sweep on.
 * All chains must be one molecule whose free dihedrals the surrogate takes;
 * the surrogate must outlive the ensemble's use of it.  s = NULL: plain
 * sweeps again.  Stage counters restart at zero. */
int smmp_ens_set_surrogate(smmp_ens_t* e, smmp_sur_t* s, double floor, int min_stage1);
/* Autotuner (no counterpart in the reference): times one sweep of every
 * chain with each pair-work decomposition the molecules allow (0: 8-partner
 * chunks of the mklist lists; 1: 32-partner passes over rows of the pair
 * triangle; 2: rows for molecules of 128 atoms or more, lists for the rest)
 * from the same saved state, keeps the fastest for later sweeps and restores
 * the state, so the call leaves no trace in the trajectory.  *choice = the
 * winner; ms[3] = the three times in milliseconds (zeros when no molecule
 * allows rows). */
int smmp_ens_autotune(smmp_ens_t* e, int* choice, double* ms);
/* Speculative windows (no counterpart in the reference): in the sweep's
 * incremental mode (FP32 pair terms, row-form pair work, relaxed states, no
 * SASA) up to `window` consecutive proposals are evaluated at once from the
 * same state, each as if the earlier ones had been rejected, and the first
 * accepted one is kept -- the same trajectory bit for bit as one proposal at
 * a time, with fewer block barriers.  smmp_ens_autotune also times the row
 * form with windows of 2, 4 and 8 and keeps a window when it is faster.
 * smmp_ens_set_window sets it by hand (1: one proposal at a time; larger
 * molecules get a smaller window, see *applied).  smmp_ens_window reports the
 * window in use and ms[3], the autotuner's times of one sweep with windows of
 * 2, 4 and 8 (0: not timed). */
int smmp_ens_set_window(smmp_ens_t* e, int window, int* applied);
int smmp_ens_window(smmp_ens_t* e, int* window, double* ms);
/* The pair-work form by hand, as smmp_ens_autotune's choice (0 chunk lists,
 * 1 rows, 2 rows for molecules of 128+ atoms; molecules without the row
 * form keep the lists). */
int smmp_ens_set_pair_work(smmp_ens_t* e, int form);
/* Per chain: proposals that passed stage 1, and that were then accepted. */
int smmp_ens_da_stats(smmp_ens_t* e, uint64_t* stage1, uint64_t* stage2);
/* Parameters and normalisation norm[2] = {mu, sigma}. */
int smmp_sur_get_params(smmp_sur_t* s, float* params, float* norm);
int smmp_sur_set_params(smmp_sur_t* s, const float* params, const float* norm);

#ifdef __cplusplus
}
#endif
#endif /* SMMP_B200_H */
