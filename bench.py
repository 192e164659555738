"""Benchmark: MC sweeps/s of parallel tempering of Met-enkephalin on one B200.

Workload (the headline configuration): 64 replicas of Met-enkephalin
(Tyr-Gly-Gly-Phe-Met, nh2/cooh ends, 75 atoms, 24 free dihedrals), ECEPP/3 in
vacuum, temperatures geometric 100-1000 K, neighbour exchange after every
sweep, seeded uniform random start.  Inputs are synthetic (seeded random
starts of the reference's own Met-enkephalin deck).

A step is one CUDA-graph launch of SWEEPS_PER_STEP parallel-tempering sweeps
(each: one sweep of every replica, then one exchange).  value = replica sweeps
per second of the whole job.  Every step is timed with CUDA events on the
stream the kernels run on; L2 is flushed (a 256 MiB write) between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's algorithm on the host cores: the CPU
oracle (a C++ restatement of the Fortran, which no Fortran compiler here can
build) running the same replicas with all host threads.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "smmp-svn_b200"))
DATA = os.path.join(ROOT, "tests", "golden", "smmp_data") + "/"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle_smmp.so")

NREP = 64
TMIN, TMAX = 100.0, 1000.0
SWEEPS_PER_STEP = 16
METRIC = "MC sweeps/s (all replicas, 1 B200): plain vs batched+surrogate, ΔE≤1e-3"
GAS = 1.98773e-3


def temperatures(n=NREP):
    return [TMIN * (TMAX / TMIN) ** (k / (n - 1)) for k in range(n)]


def config(extra=None):
    c = {"workload": "parallel tempering, Met-enkephalin (75 atoms, 24 dihedrals), "
                     "64 replicas 100-1000 K geometric, ECEPP/3 vacuum, exchange every sweep",
         "replicas": NREP, "sweeps_per_step": SWEEPS_PER_STEP, "atoms": 75, "dihedrals": 24,
         "pair_terms_per_evaluation": 2498, "pair_precision": "fp32 terms, fp64 guard+sum",
         "l2": "flushed (256 MiB write) between timed steps", "parallelism": "replicas"}
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


def cpu_baseline(target_seconds=15.0):
    """The reference algorithm (CPU oracle, FP64) on the same replicas over all
    host threads, on a bounded number of sweeps per replica."""
    L = oracle_lib()
    h = ctypes.c_void_p(L.orc_create(DATA.encode(), 0, 0, 0))
    rc = L.orc_init_molecule(h, (DATA + "enkefa.seq").encode(), (DATA + "enkefa.var").encode(),
                             b"nh2", b"cooh")
    assert rc == 0
    L.orc_sgrnd(h, ctypes.c_int(31433))
    L.orc_random_start(h)
    cores = os.cpu_count() or 1
    seeds = (ctypes.c_int * NREP)(*[31433 + 1000 * k for k in range(NREP)])
    betas = (ctypes.c_double * NREP)(*[1.0 / (t * GAS) for t in temperatures()])
    out = (ctypes.c_double * NREP)()
    # calibrate on one thread-worth of work, then size the sample
    t = L.orc_bench_chains(h, min(cores, NREP), seeds, betas, 2, cores, out)
    per_sweep_round = t / 2.0 * (NREP / min(cores, NREP))
    nsw = max(2, int(target_seconds / max(per_sweep_round, 1e-6)))
    t = L.orc_bench_chains(h, NREP, seeds, betas, nsw, cores, out)
    value = NREP * nsw / t
    return {"value": value, "unit": "sweeps/s", "cores": cores, "kind": "port",
            "sample": "%d replicas x %d sweeps of the same workload (no exchanges), %.1f s"
                      % (NREP, nsw, t)}


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
    import numpy as np
    import torch
    from smmp.ensemble import Ensemble, Molecule

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)
    temps = temperatures()
    betas = [1.0 / (t * GAS) for t in temps]
    seeds = [31433 + 1000 * k + 100000 * rank for k in range(NREP)]
    ens = Ensemble([mol], [0] * NREP, seeds, betas, fp32=True)
    stream = torch.cuda.Stream()
    ens.set_stream(stream.cuda_stream)
    ens.random_start()
    ens.set_pt(betas, wrap=False, exchange_seed=4711 + rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        ens.pt_sweeps(SWEEPS_PER_STEP, graph_chunk=SWEEPS_PER_STEP)
    # ---- device-timed region: K steps, each bracketed by events on the stream
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    with Clocks(dev) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            ens.pt_sweeps(SWEEPS_PER_STEP, graph_chunk=SWEEPS_PER_STEP)
            ends[k].record(stream)
        barrier()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    # ---- roofline: the sweep kernel alone, one launch per sweep, event-timed
    n_roof = 50
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
    vl = torch.empty((NREP, ens.vstride), dtype=torch.float64, pin_memory=True).numpy()
    vl[:] = ens.vlvr()
    e2e_steps = max(10, args.steps // 4)
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(e2e_steps):
        ens.set_vlvr(vl)                                   # H2D of the step's state
        ens.pt_sweeps(SWEEPS_PER_STEP, graph_chunk=SWEEPS_PER_STEP)
        e_host = ens.energies()                            # D2H of the result
        vl[:] = ens.vlvr()                                 # D2H of the new state
    t1.record(stream)
    barrier()
    e2e_ms = t0.elapsed_time(t1)
    errors = ens.errors()
    if errors.any():
        raise SystemExit("kernel error words: %s" % errors.tolist())

    # max over ranks
    ms, e2e_ms, sweep_kernel_ms = max_over_ranks([ms, e2e_ms, sweep_kernel_ms], world, "cuda")
    value = job_rate(NREP * SWEEPS_PER_STEP * args.steps, world, ms)
    e2e_value = job_rate(NREP * SWEEPS_PER_STEP * e2e_steps, world, e2e_ms)

    # roofline: algorithmic HBM bytes per launch of the sweep kernel
    # (16 B coordinates per atom + 8 B per dihedral + 8 B energy, per
    # evaluation; nvr evaluations per sweep; 64 replicas per launch)
    natoms, nvr = 75, 24
    bytes_per_launch = NREP * nvr * (16 * natoms + 8 * nvr + 8)
    achieved = bytes_per_launch / (sweep_kernel_ms / 1000.0) / 1e9
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(PEAKS):
        try:
            peak = float(json.load(open(PEAKS))["hbm_gbs"])
            peak_src = "measured"
        except Exception:
            pass
    traffic = None
    tf = os.path.join(ROOT, "profiles", "k_sweep_traffic.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get("bytes_per_launch")
        except Exception:
            traffic = None
    line = {
        "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 pair terms / f64 rebuild+acceptance",
        "data": "synthetic (seeded random starts of the reference's Met-enkephalin deck)",
        "config": config(),
        "e2e": {"value": e2e_value, "unit": "sweeps/s",
                "h2d_bytes_per_step": int(vl.nbytes),
                "d2h_bytes_per_step": int(vl.nbytes + 8 * NREP)},
        "gpu_launches": args.steps * SWEEPS_PER_STEP * 2,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_src, "kernel": "k_sweep<true>",
                     "kernel_ms_per_launch": sweep_kernel_ms,
                     "bytes_per_launch": bytes_per_launch},
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    L = oracle_lib()
    h = ctypes.c_void_p(L.orc_create(DATA.encode(), 0, 0, 0))
    assert L.orc_init_molecule(h, (DATA + "enkefa.seq").encode(), (DATA + "enkefa.var").encode(),
                               b"nh2", b"cooh") == 0
    L.orc_sgrnd(h, ctypes.c_int(31433))
    L.orc_random_start(h)
    cores = os.cpu_count() or 1
    seeds = (ctypes.c_int * NREP)(*[31433 + 1000 * k for k in range(NREP)])
    betas = (ctypes.c_double * NREP)(*[1.0 / (t * GAS) for t in temperatures()])
    out = (ctypes.c_double * NREP)()
    # each step: every replica 20 sweeps (a bounded sample of the workload)
    per = 20
    for _ in range(args.warmup):
        L.orc_bench_chains(h, NREP, seeds, betas, 1, cores, out)
    total = 0.0
    for _ in range(args.steps):
        total += L.orc_bench_chains(h, NREP, seeds, betas, per, cores, out)
    value = NREP * per * args.steps / total
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "sweeps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total * 1000.0 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(
            {"sweeps_per_step": per, "pair_precision": "fp64 (reference arithmetic)"}),
        "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": cores, "kind": "port",
                         "sample": "%d replicas x %d sweeps per step, %d steps"
                                   % (NREP, per, args.steps)},
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
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
