"""Benchmark: MC sweeps/s of the energy-and-sweep path on one B200.

Default workload (the headline configuration): parallel tempering of 64
replicas of Met-enkephalin (Tyr-Gly-Gly-Phe-Met, nh2/cooh ends, 75 atoms, 24
free dihedrals), ECEPP/3 in vacuum, temperatures geometric 100-1000 K,
neighbour exchange after every sweep, seeded uniform random start.  Inputs are
synthetic (seeded random starts of the reference's own Met-enkephalin deck).

A step is one cooperative launch of 16 parallel-tempering rounds (each: one
sweep of every replica, then one exchange).  value = replica sweeps per second
of the whole job.  Every step is timed with CUDA events on the stream the
kernels run on; L2 is flushed (a 256 MiB write) between steps.  e2e times the
same steps from the same starting state through the C ABI with the state
copied from and to pinned host memory every step.  The default run also
measures the other two configurations with a few steps each
(other_workloads).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pt_enkefa64|polyala256|protein60_pt128]

The other workloads measure the larger configurations with the same timing
rules: 256 independent Ace-Ala_n-NMe chains (n uniform in 10..40, seeded) with
SASA solvation at 300 K, and parallel tempering of a 60-residue protein drawn
from the natural amino-acid composition (926 atoms, 365 dihedrals) with SASA,
128 replicas geometric 250-600 K.

--impl reference times the reference's algorithm on the host cores: the CPU
oracle (a C++ restatement of the Fortran, which no Fortran compiler here can
build), compiled for the host's CPU (-O2 -march=native), running the same
chains, temperatures and exchanges with all host threads; its chains persist
from step to step.
"""
import argparse
import ctypes
import hashlib
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
def _cpu_model():
    model, flags = "", ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if not model and line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                if not flags and line.startswith("flags"):
                    flags = line.split(":", 1)[1].strip()
                if model and flags:
                    break
    except OSError:
        pass
    return model, hashlib.sha1((model + "|" + flags).encode()).hexdigest()[:12]


def oracle_lib(native=False):
    """The CPU oracle as a library: the checker build (oracle/liboracle_smmp.so)
    or, for timing, a build for this host's own CPU (-O2 -march=native, made
    on first use under oracle/_native/<cpu>/; still no contraction and no
    fast-math, so its arithmetic is the checker's)."""
    if native:
        _, key = _cpu_model()
        d = os.path.join(ROOT, "oracle", "_native", key)
        path = os.path.join(d, "liboracle_smmp.so")
        if not os.path.exists(path):
            os.makedirs(d, exist_ok=True)
            odir = os.path.join(ROOT, "oracle")
            srcs = sorted(os.path.join(odir, f) for f in os.listdir(odir) if f.endswith(".cpp"))
            tmp = path + ".%d" % os.getpid()
            subprocess.check_call([os.environ.get("CXX", "g++"), "-O2", "-march=native",
                                   "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                                   "-shared", "-o", tmp] + srcs + ["-lpthread"])
            os.replace(tmp, path)
    else:
        path = ORACLE_SO
        if not os.path.exists(path):
            subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle")],
                                  stdout=subprocess.DEVNULL)
    L = ctypes.CDLL(path)
    L.orc_create.restype = ctypes.c_void_p
    L.orc_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.orc_init_molecule.argtypes = [ctypes.c_void_p] + [ctypes.c_char_p] * 4
    L.orc_pt_create.restype = ctypes.c_void_p
    L.orc_pt_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int]
    L.orc_pt_run.restype = ctypes.c_double
    L.orc_pt_run.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.orc_pt_free.argtypes = [ctypes.c_void_p]
    L.orc_last_error.restype = ctypes.c_char_p
    return L


class CpuChains:
    """The reference algorithm (the CPU oracle, FP64) on the workload's chains
    with every host thread busy: one persistent ensemble per distinct
    molecule, each chain with its own stream and random start, parallel
    tempering workloads exchanging after every round as the GPU arm does.
    Successive samples continue the trajectories.  A workload of several
    molecules keeps `cores` chains of each and weights each molecule's
    per-chain-sweep cost by its number of chains in the workload."""

    def __init__(self, wl, files, native=True):
        self.L = oracle_lib(native)
        self.cores = os.cpu_count() or 1
        self.cpu = _cpu_model()[0]
        self.build = "-O2 -march=native" if native else "-O2"
        self.cm = wl.chain_mol()
        temps = wl.temperatures()
        self.nch = len(self.cm)
        self.objs = []
        for m, (seq, var) in enumerate(files):
            h = ctypes.c_void_p(self.L.orc_create(DATA.encode(), 0, 0, wl.itysol))
            rc = self.L.orc_init_molecule(h, seq.encode(), (var or " ").encode(), b"nh2", b"cooh")
            assert rc == 0, self.L.orc_last_error()
            chains = [c for c in range(self.nch) if self.cm[c] == m]
            if len(files) > 1:
                chains = (chains * (1 + self.cores // len(chains)))[:self.cores]
            n = len(chains)
            betas = (ctypes.c_double * n)(*[1.0 / (temps[c] * GAS) for c in chains])
            seeds = (ctypes.c_int * n)(*[31433 + 1000 * c + 7 * k for k, c in enumerate(chains)])
            pt = self.L.orc_pt_create(h, n, betas, seeds, 4711, 0, self.cores, 1 if wl.pt else 0)
            assert pt, self.L.orc_last_error()
            self.objs.append((h, ctypes.c_void_p(pt), n, self.cm.count(m)))

    def rounds(self, m, n):
        t = self.L.orc_pt_run(self.objs[m][1], int(n))
        if t < 0:
            raise RuntimeError(self.L.orc_last_error().decode())
        return t

    def sample(self, target_seconds):
        """(chain sweeps per second, description, seconds): one warm-up round,
        then as many rounds as fit target_seconds (one molecule), or one
        round of each molecule (several)."""
        if len(self.objs) == 1:
            probe = self.rounds(0, 1)
            if probe > 0.25 * target_seconds:   # a large molecule: the probe is the sample
                return self.nch / probe, "%d chains x 1 round, %.1f s" % (self.nch, probe), probe
            nr = max(1, int(target_seconds / max(probe, 1e-6)))
            t = self.rounds(0, nr)
            return self.nch * nr / t, "%d chains x %d rounds, %.1f s" % (self.nch, nr, t), t
        cost = total = 0.0
        for m, (_, _, n, count) in enumerate(self.objs):
            self.rounds(m, 1)
            t = self.rounds(m, 1)
            total += t
            cost += count * t / n
        return self.nch / cost, ("%d chains of each of %d molecules x 1 round, weighted by the "
                                 "workload's chain counts, %.1f s" % (self.cores, len(self.objs),
                                                                      total)), total

    def close(self):
        for h, pt, _, _ in self.objs:
            self.L.orc_pt_free(pt)
        self.objs = []


def cpu_baseline(wl, files, target_seconds=12.0):
    oc = CpuChains(wl, files)
    value, sample, _ = oc.sample(target_seconds)
    oc.close()
    return {"value": value, "unit": "sweeps/s", "cores": oc.cores, "kind": "port",
            "cpu": oc.cpu, "build": oc.build,
            "sample": sample + ("" if not wl.pt else " with an exchange after every round")}


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
def fp32_peak_tflops():
    """FP32 FMA issue peak of the device (148 SMs x 128 lanes x 2 flops at
    the measured maximum SM clock; no measured FP32 peak exists)."""
    mhz = 1965.0
    if os.path.exists(PEAKS):
        try:
            mhz = float(json.load(open(PEAKS)).get("sm_max_mhz", mhz))
        except Exception:
            pass
    return 148 * 128 * 2 * mhz * 1e6 / 1e12


def max_dE_vs_oracle(ens, files, wl, mols, nsample=16):
    """Largest |E_GPU - E_FP64 oracle| (kcal/mol) over a sample of chains:
    the GPU's tracked energy of each chain's current conformation against the
    oracle's FP64 energy() of the same variables."""
    L = oracle_lib(False)
    L.orc_energy.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                             ctypes.POINTER(ctypes.c_double)]
    L.orc_set_vlvr.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    L.orc_destroy.argtypes = [ctypes.c_void_p]
    cm = wl.chain_mol()
    V, E = ens.vlvr(), ens.energies()
    handles = {}
    worst = 0.0
    picks = sorted(set(int(round(x)) for x in
                       [k * (len(cm) - 1) / max(1, nsample - 1) for k in range(nsample)]))
    for c in picks:
        m = cm[c]
        if m not in handles:
            h = ctypes.c_void_p(L.orc_create(DATA.encode(), 0, 0, wl.itysol))
            seq, var = files[m]
            assert L.orc_init_molecule(h, seq.encode(), (var or " ").encode(), b"nh2",
                                       b"cooh") == 0
            handles[m] = h
        v = (ctypes.c_double * mols[m].nvar)(*V[c, :mols[m].nvar])
        L.orc_set_vlvr(handles[m], v)
        e, t = ctypes.c_double(), (ctypes.c_double * 6)()
        assert L.orc_energy(handles[m], ctypes.byref(e), t) == 0
        worst = max(worst, abs(E[c] - e.value))
    for h in handles.values():
        L.orc_destroy(h)
    return worst, len(picks)


def measure(wl, args, rank, world, dev, stream, flush, steps, warmup, headline):
    """Our arm on one workload: the device-timed region (steps x one step of
    spp sweeps, L2 flushed before each), the kernel's own launches, the same
    steps end to end through the C ABI from the same starting state, and the
    checks and rooflines that explain them."""
    import torch
    from smmp.ensemble import Ensemble, Molecule
    spp = wl.sweeps_per_step
    files = wl.molecule_files()
    mols = [Molecule(seq, var, libdir=DATA, itysol=wl.itysol) for seq, var in files]
    cm = wl.chain_mol()
    nch = len(cm)
    betas = [1.0 / (t * GAS) for t in wl.temperatures()]
    ens = Ensemble(mols, cm, wl.seeds(rank), betas, fp32=True)
    ens.set_stream(stream.cuda_stream)
    ens.random_start()
    if wl.pt:
        ens.set_pt(betas, wrap=False, exchange_seed=4711 + rank)

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

    for _ in range(warmup):
        step()
    # the autotuner picks the pair-work decomposition and the speculative
    # window (state left unchanged)
    form, (ms_lists, ms_rows, ms_size) = ens.autotune()
    win, (w2, w4, w8) = ens.window()
    tuned = {"pair_work": form, "window": win, "sweep_ms_lists": ms_lists,
             "sweep_ms_rows": ms_rows, "sweep_ms_rows_128plus": ms_size,
             "sweep_ms_rows_window2": w2, "sweep_ms_rows_window4": w4,
             "sweep_ms_rows_window8": w8}
    start = ens.checkpoint()
    # ---- device-timed region: K steps, each bracketed by events on the stream
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    pt0 = int(ens.pair_terms().sum())
    barrier()
    with Clocks(dev) as clk:
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            step()
            ends[k].record(stream)
        barrier()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    pterms = int(ens.pair_terms().sum()) - pt0
    fused = bool(wl.pt and ens.pt_fused_last())
    errors = ens.errors()
    if errors.any():
        raise SystemExit("kernel error words: %s" % errors.tolist())
    dE, nde = max_dE_vs_oracle(ens, files, wl, mols)
    # ---- the sweep kernel alone, one launch per sweep, event-timed
    n_roof = 50 if headline else 4
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
    # ---- end to end through the C ABI with host buffers every step, the same
    # steps from the same starting state as the timed region
    ens.restore(start)
    vl = torch.empty((nch, ens.vstride), dtype=torch.float64, pin_memory=True).numpy()
    vl[:] = ens.vlvr()
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        ens.set_vlvr(vl)                                   # H2D of the step's state
        step()
        ens.energies()                                     # D2H of the result
        vl[:] = ens.vlvr()                                 # D2H of the new state
    t1.record(stream)
    barrier()
    e2e_ms = t0.elapsed_time(t1)
    if ens.errors().any():
        raise SystemExit("kernel error words: %s" % ens.errors().tolist())
    ms, e2e_ms, sweep_kernel_ms = max_over_ranks([ms, e2e_ms, sweep_kernel_ms], world, "cuda")
    value = job_rate(nch * spp * steps, world, ms)
    e2e_value = job_rate(nch * spp * steps, world, e2e_ms)
    # HBM roofline (north_star's figure): algorithmic bytes per launch of the
    # sweep kernel (16 B coordinates per atom + 8 B per dihedral + 8 B energy,
    # per evaluation; one evaluation per free dihedral per sweep; every chain)
    bytes_per_sweep = sum(mols[m].nvr * (16 * mols[m].natoms + 8 * mols[m].nvr + 8) for m in cm)
    if fused:   # the timed step is that one launch (and an 8-byte memset)
        roof_kernel, roof_ms, bytes_per_launch = "k_sweep<true> (fused PT)", ms / steps, \
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
    if headline and os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get("fused_bytes_per_launch" if fused
                                              else "bytes_per_launch")
        except Exception:
            traffic = None
    # FP32 issue roofline (the pair terms the sweeps evaluated, 30 flops each)
    tflops = pterms * 30.0 / (ms / 1000.0) / 1e12
    fpeak = fp32_peak_tflops()
    return {
        "value": value, "unit": "sweeps/s", "ms_per_step": ms / steps,
        "config": config(wl, {"autotune": tuned}),
        "e2e": {"value": e2e_value, "unit": "sweeps/s",
                "h2d_bytes_per_step": int(vl.nbytes),
                "d2h_bytes_per_step": int(vl.nbytes + 8 * nch)},
        "gpu_launches": steps * (1 if fused or not wl.pt else spp * 2),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_src, "kernel": roof_kernel,
                     "kernel_ms_per_launch": roof_ms,
                     "bytes_per_launch": bytes_per_launch,
                     "single_sweep_launch_ms": sweep_kernel_ms},
        "roofline_fp32_issue": {"achieved": tflops, "peak": fpeak, "unit": "TFLOP/s",
                                "frac": tflops / fpeak,
                                "pair_terms_per_sweep": pterms / float(nch * spp * steps),
                                "flops_per_pair_term": 30,
                                "peak_source": "computed (148 SMs x 128 FP32 lanes x 2 x "
                                               "measured max SM clock)"},
        "max_abs_dE_vs_fp64_oracle_kcal": dE, "dE_sample_chains": nde,
        "clocks": clk.summary(), "_ens": ens, "_mols": mols, "_files": files,
        "_betas": betas,
    }


def run_ours(args, rank, world):
    import torch
    wl = WORKLOADS[args.workload]()
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    headline = wl.name == "pt_enkefa64"
    r = measure(wl, args, rank, world, dev, stream, flush, args.steps, args.warmup, headline)
    ens, mols, files, betas = r.pop("_ens"), r.pop("_mols"), r.pop("_files"), r.pop("_betas")
    line = {
        "metric": METRIC, "value": r["value"], "unit": "sweeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 pair terms / f64 rebuild+acceptance",
        "data": ("synthetic (seeded random starts of the reference's Met-enkephalin deck)"
                 if headline else "synthetic (seeded sequences, seeded random starts)"),
    }
    line.update({k: v for k, v in r.items() if k not in line})
    if headline and not args.no_surrogate:
        line["plain_single_replica"] = single_replica(mols[0], wl.sweeps_per_step, stream)
        line["surrogate"] = surrogate_leg(ens, mols[0], betas, wl.sweeps_per_step, stream, flush)
    del ens
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(wl, files)
    if headline and world == 1 and not args.no_extra:
        # the other configurations, bounded: measured with the same rules
        others = {}
        for name in ("polyala256", "protein60_pt128"):
            w2 = WORKLOADS[name]()
            r2 = measure(w2, args, rank, world, dev, stream, flush, 3, 2, False)
            for k in ("_ens", "_mols", "_betas"):
                r2.pop(k)
            f2 = r2.pop("_files")
            if not args.no_cpu:
                r2["cpu_baseline"] = cpu_baseline(w2, f2, target_seconds=8.0)
                r2["e2e_vs_cpu"] = r2["e2e"]["value"] / r2["cpu_baseline"]["value"]
            others[name] = r2
        line["other_workloads"] = others
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
    """The reference algorithm on the host cores (the CPU oracle, FP64, built
    for this CPU), on our arm's workload: the same chains, temperatures and
    exchange schedule, every host thread busy.  A step is a bounded sample:
    20 rounds of all 64 replicas for Met-enkephalin, one sample of
    CpuChains otherwise.  The chains persist from step to step."""
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]()
    files = wl.molecule_files()
    oc = CpuChains(wl, files)
    nch = len(wl.chain_mol())
    enk = wl.name == "pt_enkefa64"
    per = 20
    for _ in range(args.warmup if enk else 0):
        oc.rounds(0, 1)
    total = units = 0.0
    sample = ""
    for _ in range(args.steps):
        if enk:
            total += oc.rounds(0, per)
            units += nch * per
            sample = ("%d replicas x %d rounds (sweep + exchange) per step, %d steps"
                      % (nch, per, args.steps))
        else:
            rate, sample, t = oc.sample(5.0)
            total += t
            units += rate * t
    oc.close()
    value = units / total
    extra = {"pair_precision": "fp64 (reference arithmetic)"}
    if enk:
        extra["sweeps_per_step"] = per
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "sweeps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total * 1000.0 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(wl, extra),
        "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": oc.cores, "kind": "port",
                         "cpu": oc.cpu, "build": oc.build, "sample": sample},
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
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the bounded legs of the other workloads")
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
