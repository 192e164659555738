"""Benchmark: MC sweeps/s of the energy-and-sweep path on one B200.

Default workload (the headline configuration): parallel tempering of 64
replicas of Met-enkephalin (Tyr-Gly-Gly-Phe-Met, nh2/cooh ends, 75 atoms, 24
free dihedrals), ECEPP/3 in vacuum, temperatures geometric 100-1000 K,
neighbour exchange after every sweep, seeded uniform random start.  Inputs are
synthetic (seeded random starts of the reference's own Met-enkephalin deck).

A step is one CUDA-graph launch of 16 parallel-tempering sweeps (each: one
sweep of every replica, then one exchange).  value = replica sweeps per second
of the whole job.  Every step is timed with CUDA events on the stream the
kernels run on; L2 is flushed (a 256 MiB write) between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pt_enkefa64|polyala256|protein60_pt128]

The other workloads measure the larger configurations with the same timing
rules: 256 independent Ace-Ala_n-NMe chains (n uniform in 10..40, seeded) with
SASA solvation at 300 K, and parallel tempering of a 60-residue protein drawn
from the natural amino-acid composition (926 atoms, 365 dihedrals) with SASA,
128 replicas geometric 250-600 K.

--impl reference times the reference's algorithm on the host cores: the CPU
oracle (a C++ restatement of the Fortran, which no Fortran compiler here can
build) running the same chains with all host threads.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "smmp-svn_b200"))
DATA = os.path.join(ROOT, "tests", "golden", "smmp_data") + "/"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle_smmp.so")

METRIC = "MC sweeps/s (all replicas, 1 B200): plain vs batched+surrogate, ΔE≤1e-3"
GAS = 1.98773e-3


def geometric(tmin, tmax, n):
    return [tmin * (tmax / tmin) ** (k / (n - 1)) for k in range(n)]


# ------------------------------------------------------------------ workloads
class Workload:
    """One benchmark configuration: its molecules, chains, temperatures and
    what one timed step does."""
    name = ""
    sweeps_per_step = 1
    pt = False
    itysol = 0

    def molecule_files(self):
        """[(seqfile, varfile or None)] of the distinct molecules."""
        raise NotImplementedError

    def chain_mol(self):
        raise NotImplementedError

    def temperatures(self):
        raise NotImplementedError

    def seeds(self, rank):
        return [31433 + 1000 * k + 100000 * rank for k in range(len(self.chain_mol()))]

    def describe(self):
        raise NotImplementedError


class PTEnkefa64(Workload):
    name = "pt_enkefa64"
    sweeps_per_step = 16
    pt = True

    def molecule_files(self):
        return [(DATA + "enkefa.seq", DATA + "enkefa.var")]

    def chain_mol(self):
        return [0] * 64

    def temperatures(self):
        return geometric(100.0, 1000.0, 64)

    def describe(self):
        return {"workload": "parallel tempering, Met-enkephalin (75 atoms, 24 dihedrals), "
                            "64 replicas 100-1000 K geometric, ECEPP/3 vacuum, exchange every sweep",
                "replicas": 64, "sweeps_per_step": self.sweeps_per_step, "atoms": 75,
                "dihedrals": 24, "pair_terms_per_evaluation": 2498}


class Polyala256(Workload):
    name = "polyala256"
    sweeps_per_step = 4
    itysol = 1

    def __init__(self):
        from smmp.sequences import polyala_lengths
        self.lengths = polyala_lengths(256, seed=12345)
        self.distinct = sorted(set(self.lengths))

    def molecule_files(self):
        from smmp.sequences import polyala, write_seq
        d = tempfile.mkdtemp(prefix="smmp_bench_")
        return [(write_seq(os.path.join(d, "ala%d.seq" % n), polyala(n), "ala%d" % n), None)
                for n in self.distinct]

    def chain_mol(self):
        return [self.distinct.index(n) for n in self.lengths]

    def temperatures(self):
        return [300.0] * 256

    def describe(self):
        return {"workload": "256 independent chains Ace-Ala_n-NMe, n uniform 10-40 (seed 12345), "
                            "ECEPP/3 + SASA solvation (itysol 1), 300 K canonical",
                "chains": 256, "sweeps_per_step": self.sweeps_per_step,
                "mean_residues": sum(self.lengths) / 256.0}


class Protein60PT128(Workload):
    name = "protein60_pt128"
    sweeps_per_step = 2
    pt = True
    itysol = 1

    def molecule_files(self):
        from smmp.sequences import natural_protein, write_seq
        d = tempfile.mkdtemp(prefix="smmp_bench_")
        return [(write_seq(os.path.join(d, "protein60.seq"), natural_protein(60), "protein60"),
                 None)]

    def chain_mol(self):
        return [0] * 128

    def temperatures(self):
        return geometric(250.0, 600.0, 128)

    def describe(self):
        return {"workload": "parallel tempering, 60-residue protein of natural composition "
                            "(seed 2024; 926 atoms, 365 dihedrals), ECEPP/3 + SASA solvation, "
                            "128 replicas 250-600 K geometric, exchange every sweep",
                "replicas": 128, "sweeps_per_step": self.sweeps_per_step, "atoms": 926,
                "dihedrals": 365, "pair_terms_per_evaluation": 425508}


WORKLOADS = {w.name: w for w in (PTEnkefa64, Polyala256, Protein60PT128)}


def config(wl, extra=None):
    c = wl.describe()
    c.update({"pair_precision": "fp32 terms, fp64 guard+sum",
              "l2": "flushed (256 MiB write) between timed steps", "parallelism": "replicas"})
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.out = ""

    def summary(self):
        rows = []
        for line in (getattr(self, "out", "") or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ CPU baseline
def oracle_lib():
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle")],
                              stdout=subprocess.DEVNULL)
    L = ctypes.CDLL(ORACLE_SO)
    L.orc_create.restype = ctypes.c_void_p
    L.orc_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.orc_bench_chains.restype = ctypes.c_double
    L.orc_bench_chains.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double)]
    return L


class OracleChains:
    """The reference algorithm (CPU oracle, FP64) on the workload's chains,
    every host thread busy: one handle per distinct molecule, seeded random
    start."""

    def __init__(self, wl, files):
        self.L = oracle_lib()
        self.cores = os.cpu_count() or 1
        self.handles = []
        for seq, var in files:
            h = ctypes.c_void_p(self.L.orc_create(DATA.encode(), 0, 0, wl.itysol))
            rc = self.L.orc_init_molecule(h, seq.encode(), (var or " ").encode(), b"nh2", b"cooh")
            assert rc == 0
            self.L.orc_sgrnd(h, ctypes.c_int(31433))
            self.L.orc_random_start(h)
            self.handles.append(h)
        self.cm = wl.chain_mol()
        self.temps = wl.temperatures()

    def run(self, mol, nchains, nsweeps):
        """Seconds for nchains chains of molecule `mol` x nsweeps on all threads."""
        chains = [c for c, m in enumerate(self.cm) if m == mol]
        chains = (chains * (1 + nchains // max(1, len(chains))))[:nchains]
        seeds = (ctypes.c_int * nchains)(*[31433 + 1000 * c for c in chains])
        betas = (ctypes.c_double * nchains)(*[1.0 / (self.temps[c] * GAS) for c in chains])
        out = (ctypes.c_double * nchains)()
        return self.L.orc_bench_chains(self.handles[mol], nchains, seeds, betas, nsweeps,
                                       self.cores, out)

    def sample(self, target_seconds):
        """(chain sweeps per second, description, seconds) from one bounded
        sample.  One molecule: all chains for as many sweeps as fit
        target_seconds.  Several: for each molecule, `cores` chains (every
        thread busy) for one sweep; each molecule's per-chain-sweep cost is
        weighted by its number of chains in the workload."""
        n = len(self.handles)
        nchains = len(self.cm)
        if n == 1:
            probe = self.run(0, min(self.cores, nchains), 1)
            per_round = probe * max(1, nchains // self.cores)
            nsw = max(1, int(target_seconds / max(per_round, 1e-6)))
            t = self.run(0, nchains, nsw)
            return nchains * nsw / t, "%d chains x %d sweeps, %.1f s" % (nchains, nsw, t), t
        cost = 0.0
        total = 0.0
        for m in range(n):
            t = self.run(m, self.cores, 1)
            total += t
            cost += self.cm.count(m) * t / self.cores
        return nchains / cost, ("%d chains x 1 sweep of each of %d molecules, weighted by the "
                                "workload's chain counts, %.1f s" % (self.cores, n, total)), total


def cpu_baseline(wl, files, target_seconds=15.0):
    oc = OracleChains(wl, files)
    value, sample, _ = oc.sample(target_seconds)
    return {"value": value, "unit": "sweeps/s", "cores": oc.cores, "kind": "port",
            "sample": sample + " (no exchanges)"}


def max_over_ranks(values, world, device=None):
    """Element-wise max of per-rank timings (the job takes as long as its
    slowest rank)."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def job_rate(units_per_rank, world, ms):
    """Whole-job throughput: units all ranks processed / slowest rank's time."""
    return units_per_rank * world / (ms / 1000.0)


# ------------------------------------------------------------------ our arm
def run_ours(args, rank, world):
    import torch
    from smmp.ensemble import Ensemble, Molecule

    wl = WORKLOADS[args.workload]()
    spp = wl.sweeps_per_step
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    files = wl.molecule_files()
    mols = [Molecule(seq, var, libdir=DATA, itysol=wl.itysol) for seq, var in files]
    cm = wl.chain_mol()
    nch = len(cm)
    betas = [1.0 / (t * GAS) for t in wl.temperatures()]
    ens = Ensemble(mols, cm, wl.seeds(rank), betas, fp32=True)
    stream = torch.cuda.Stream()
    ens.set_stream(stream.cuda_stream)
    ens.random_start()
    if wl.pt:
        ens.set_pt(betas, wrap=False, exchange_seed=4711 + rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        if wl.pt:
            ens.pt_sweeps(spp, graph_chunk=spp)
        else:
            ens.sweeps(spp)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    # the autotuner picks the pair-work decomposition (state left unchanged)
    form, (ms_lists, ms_rows, ms_size) = ens.autotune()
    tuned = {"pair_work": form, "sweep_ms_lists": ms_lists, "sweep_ms_rows": ms_rows,
             "sweep_ms_rows_128plus": ms_size}
    # ---- device-timed region: K steps, each bracketed by events on the stream
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    with Clocks(dev) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            step()
            ends[k].record(stream)
        barrier()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    # batched PT runs each step as one cooperative launch of spp (sweep,
    # exchange) rounds when every chain is resident at once
    fused = bool(wl.pt and ens.pt_fused_last())
    # ---- roofline: the sweep kernel alone, one launch per sweep, event-timed
    n_roof = 50 if wl.name == "pt_enkefa64" else 8
    rs = [torch.cuda.Event(enable_timing=True) for _ in range(n_roof)]
    re_ = [torch.cuda.Event(enable_timing=True) for _ in range(n_roof)]
    for k in range(n_roof):
        with torch.cuda.stream(stream):
            flush.zero_()
            rs[k].record(stream)
        ens.sweeps(1)
        re_[k].record(stream)
    torch.cuda.synchronize()
    sweep_kernel_ms = statistics.mean(a.elapsed_time(b) for a, b in zip(rs, re_))
    # ---- end-to-end through the C ABI with host buffers every step
    vl = torch.empty((nch, ens.vstride), dtype=torch.float64, pin_memory=True).numpy()
    vl[:] = ens.vlvr()
    e2e_steps = max(10, args.steps // 4) if wl.name == "pt_enkefa64" else max(3, args.steps // 4)
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(e2e_steps):
        ens.set_vlvr(vl)                                   # H2D of the step's state
        step()
        ens.energies()                                     # D2H of the result
        vl[:] = ens.vlvr()                                 # D2H of the new state
    t1.record(stream)
    barrier()
    e2e_ms = t0.elapsed_time(t1)
    errors = ens.errors()
    if errors.any():
        raise SystemExit("kernel error words: %s" % errors.tolist())

    # max over ranks
    ms, e2e_ms, sweep_kernel_ms = max_over_ranks([ms, e2e_ms, sweep_kernel_ms], world, "cuda")
    value = job_rate(nch * spp * args.steps, world, ms)
    e2e_value = job_rate(nch * spp * e2e_steps, world, e2e_ms)

    # roofline: algorithmic HBM bytes per launch of the sweep kernel
    # (16 B coordinates per atom + 8 B per dihedral + 8 B energy, per
    # evaluation; one evaluation per free dihedral per sweep; every chain)
    bytes_per_sweep = sum(mols[m].nvr * (16 * mols[m].natoms + 8 * mols[m].nvr + 8) for m in cm)
    if fused:   # the timed step is that one launch (and an 8-byte memset)
        roof_kernel, roof_ms, bytes_per_launch = "k_sweep<true> (fused PT)", ms / args.steps, \
            bytes_per_sweep * spp
    else:
        roof_kernel, roof_ms, bytes_per_launch = "k_sweep<true>", sweep_kernel_ms, bytes_per_sweep
    achieved = bytes_per_launch / (roof_ms / 1000.0) / 1e9
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(PEAKS):
        try:
            peak = float(json.load(open(PEAKS))["hbm_gbs"])
            peak_src = "measured"
        except Exception:
            pass
    traffic = None
    tf = os.path.join(ROOT, "profiles", "k_sweep_traffic.json")
    if wl.name == "pt_enkefa64" and os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get("fused_bytes_per_launch" if fused
                                              else "bytes_per_launch")
        except Exception:
            traffic = None
    line = {
        "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 pair terms / f64 rebuild+acceptance",
        "data": ("synthetic (seeded random starts of the reference's Met-enkephalin deck)"
                 if wl.name == "pt_enkefa64"
                 else "synthetic (seeded sequences, seeded random starts)"),
        "config": config(wl, {"autotune": tuned}),
        "e2e": {"value": e2e_value, "unit": "sweeps/s",
                "h2d_bytes_per_step": int(vl.nbytes),
                "d2h_bytes_per_step": int(vl.nbytes + 8 * nch)},
        "gpu_launches": args.steps * (1 if fused or not wl.pt else spp * 2),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_src, "kernel": roof_kernel,
                     "kernel_ms_per_launch": roof_ms,
                     "bytes_per_launch": bytes_per_launch,
                     "single_sweep_launch_ms": sweep_kernel_ms},
        "clocks": clk.summary(),
    }
    if wl.name == "pt_enkefa64" and not args.no_surrogate:
        line["plain_single_replica"] = single_replica(mols[0], spp, stream)
        line["surrogate"] = surrogate_leg(ens, mols[0], betas, spp, stream, flush)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(wl, files)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def single_replica(mol, spp, stream):
    """The plain method on one replica (one chain, same kernel): the GPU
    baseline the batched throughput is compared with."""
    import torch
    from smmp.ensemble import Ensemble
    one = Ensemble([mol], [0], [31433], [1.0 / (300.0 * GAS)], fp32=True)
    one.set_stream(stream.cuda_stream)
    one.random_start()
    one.sweeps(20)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    n = 400
    t0.record(stream)
    for _ in range(n // spp):
        one.sweeps(spp)
    t1.record(stream)
    torch.cuda.synchronize()
    return {"value": n / (t0.elapsed_time(t1) / 1000.0), "unit": "sweeps/s",
            "config": "1 chain, 300 K, same kernel, %d sweeps per launch" % spp}


def surrogate_leg(ens, mol, betas, spp, stream, flush):
    """Train the energy surrogate on the run's own PT states and time the
    delayed-acceptance sweeps (surrogate first stage, exact second stage).
    Training time is reported separately, as the metric asks."""
    import numpy as np
    import torch
    from smmp.ensemble import Ensemble
    from smmp.surrogate import Surrogate, collect_samples
    nch = len(betas)
    t0 = time.time()
    ang, e = collect_samples(ens, mol, 500)                  # 32,000 states
    t_collect = time.time() - t0
    # FP64 labels from the GPU's FP64 energy kernel (parity-tested against the
    # FP64 oracle to 1e-10); the sampler's own energies are FP32-pair sums
    lab = Ensemble([mol], [0] * len(e), [1] * len(e), [1.0] * len(e))
    V = np.zeros((len(e), lab.vstride))
    V[:] = ens.vlvr()[0]
    V[:, mol.idvr] = ang
    lab.set_vlvr(V)
    e64 = lab.energy()
    del lab
    rng = np.random.default_rng(0)
    order = rng.permutation(len(e))
    nt = len(e) // 10
    test, train = order[:nt], order[nt:]
    clip = float(np.percentile(e64, 99))
    sur = Surrogate(mol.nvr, seed=2)
    sur.set_data(ang[train], e64[train], clip=clip)
    epochs, batch = 40, 512
    torch.cuda.synchronize()
    t0 = time.time()
    sur.train(epochs, batch=batch, lr=1e-3)
    t_train = time.time() - t0
    pred = sur.predict(ang[test])
    keep = e64[test] < clip
    rmse = float(np.sqrt(np.mean((pred[keep] - e64[test][keep]) ** 2)))
    flops = 3 * 2 * (2 * mol.nvr * 256 + 2 * 256 * 256 + 256) * (len(train) // batch) * batch * epochs
    peak = 1590.0
    if os.path.exists(PEAKS):
        try:
            peak = float(json.load(open(PEAKS))["bf16_tflops"])
        except Exception:
            pass
    out = {"train_states": int(len(train)), "collect_s": t_collect, "train_s": t_train,
           "epochs": epochs, "batch": batch,
           "heldout_rmse_kcal": rmse, "heldout_energy_std_kcal": float(e64[test][keep].std()),
           "labels": "FP64 GPU energies (parity-tested to 1e-10 against the FP64 oracle)",
           "train_roofline": {"bound": "tensor", "achieved": flops / t_train / 1e12, "peak": peak,
                              "unit": "TFLOP/s", "frac": flops / t_train / 1e12 / peak}}
    # delayed-acceptance PT sweeps on the same replicas, timed like the plain arm
    res = {}
    for mode in ("plain", "delayed"):
        ens.set_surrogate(sur if mode == "delayed" else None, floor=0.2, min_stage1=64)
        ens.pt_sweeps(spp, graph_chunk=spp)
        a0, p0 = ens.acceptance()
        s0 = ens.da_stats()
        k = 20
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ms = 0.0
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.zero_()
                ev0.record(stream)
            ens.pt_sweeps(spp, graph_chunk=spp)
            ev1.record(stream)
            torch.cuda.synchronize()
            ms += ev0.elapsed_time(ev1)
        a, p = ens.acceptance()
        s1 = ens.da_stats()
        accepted = float((a - a0).sum())
        exact = float((s1[0] - s0[0]).sum()) if mode == "delayed" else float((p - p0).sum())
        res[mode] = {"value": nch * spp * k / (ms / 1000.0), "unit": "sweeps/s",
                     "acceptance": accepted / float((p - p0).sum()),
                     "exact_evaluations_per_accepted_move": exact / max(accepted, 1.0)}
        if mode == "delayed":
            res[mode]["stage1_pass"] = float((s1[0] - s0[0]).sum()) / float((p - p0).sum())
            res[mode]["stage2_acceptance"] = float((s1[1] - s0[1]).sum()) / max(
                float((s1[0] - s0[0]).sum()), 1.0)
    ens.set_surrogate(None)
    out["pt_plain"] = res["plain"]
    out["pt_delayed_acceptance"] = res["delayed"]
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]()
    files = wl.molecule_files()
    oc = OracleChains(wl, files)
    nch = len(wl.chain_mol())
    enk = wl.name == "pt_enkefa64"
    # each step: a bounded sample of the workload (every replica 20 sweeps for
    # Met-enkephalin; the per-molecule sample of OracleChains otherwise)
    for _ in range(args.warmup if enk else 0):
        oc.run(0, nch, 1)
    total = 0.0
    units = 0.0
    sample = ""
    for _ in range(args.steps):
        if enk:
            per = 20
            total += oc.run(0, nch, per)
            units += nch * per
            sample = "%d replicas x %d sweeps per step, %d steps" % (nch, per, args.steps)
        else:
            rate, sample, t = oc.sample(5.0)
            total += t
            units += rate * t
    value = units / total
    extra = {"pair_precision": "fp64 (reference arithmetic)"}
    if enk:
        extra["sweeps_per_step"] = 20
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "sweeps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total * 1000.0 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(wl, extra),
        "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": oc.cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pt_enkefa64", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the surrogate training / delayed-acceptance leg")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world)


if __name__ == "__main__":
    main()
