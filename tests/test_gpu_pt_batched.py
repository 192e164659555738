"""Batched parallel tempering, the headline workload's mode: every chain
draws from its own stream, the exchanges from a stream of their own, and all
disjoint pairs of a parity step are decided at once (one warp).  The oracle
restates that schedule (orc_partem_batched: per-chain streams, the exchange
step of partem_s.f:210-232 with one draw per pair in pair order).

* FP64 pair terms: after 200 rounds the GPU's temperature map, exchange
  statistics, every chain's variables and energy equal the oracle's.
* FP32 pair terms: the trajectories agree with the FP64 oracle until the
  first decision that the FP32 rounding flips; the round is printed.
* Statistics: per-temperature energy distributions of batched PT and of the
  serial partem_s schedule (one shared stream) agree within statistical error
  over independent runs (mean energy and the fraction below the pooled
  median at every temperature, |z| < 4.5).
"""
import numpy as np
import pytest

from conftest import DATA, Oracle

pytestmark = pytest.mark.gpu

SEQ, VAR = DATA + "enkefa.seq", DATA + "enkefa.var"


def _ladder(n, tmin=100.0, tmax=1000.0):
    from smmp.ensemble import beta_of
    temps = tmin * (tmax / tmin) ** (np.arange(n) / (n - 1))
    return [beta_of(t) for t in temps]


def _gpu(n, betas, seeds, wrap, fp32):
    from smmp.ensemble import Ensemble, Molecule
    mol = Molecule(SEQ, VAR, libdir=DATA)
    ens = Ensemble([mol], [0] * n, seeds, betas, fp32=fp32)
    ens.random_start()
    ens.set_pt(betas, wrap=wrap, exchange_seed=4711)
    return ens


@pytest.mark.parametrize("wrap,rounds", [(False, 200), (True, 100)])
def test_batched_pt_equals_the_oracle_in_fp64(wrap, rounds):
    n = 16
    betas = _ladder(n)
    seeds = [31433 + 1000 * k for k in range(n)]
    o = Oracle(SEQ, VAR)
    tc, eo, vl, (att, acc) = o.partem_batched(betas, seeds, 4711, wrap, rounds)
    ens = _gpu(n, betas, seeds, wrap, fp32=False)
    ens.pt_sweeps(rounds)
    assert ens.pt_fused_last() and not ens.errors().any()
    assert np.array_equal(ens.pt_map(), tc[-1])
    ga, gc = ens.pt_stats()
    assert np.array_equal(ga, att) and np.array_equal(gc, acc)
    assert acc.sum() > 0 and acc.sum() < att.sum()
    idvr = o.idvr() - 1
    assert np.array_equal(ens.vlvr()[:, idvr], vl[-1])
    np.testing.assert_allclose(ens.energies(), eo[-1], rtol=1e-10, atol=1e-9)


def test_batched_pt_fp32_first_decision_flip():
    n, rounds = 16, 200
    betas = _ladder(n)
    seeds = [31433 + 1000 * k for k in range(n)]
    o = Oracle(SEQ, VAR)
    tc, eo, vl, _ = o.partem_batched(betas, seeds, 4711, False, rounds)
    ens = _gpu(n, betas, seeds, False, fp32=True)
    idvr = o.idvr() - 1
    first = None
    for r in range(rounds):
        ens.pt_sweeps(1)
        same = np.array_equal(ens.pt_map(), tc[r]) and \
            np.array_equal(ens.vlvr()[:, idvr], vl[r])
        if not same:
            first = r + 1
            break
        relaxed = np.abs(eo[r]) < 1e4
        assert np.all(np.abs(ens.energies() - eo[r])[relaxed] <= 1e-3)
    print("\nFP32 pair terms, 16 replicas: first decision flip against the FP64 oracle at round",
          first if first else "none within %d rounds" % rounds)
    assert first is None or first > 20


def _label_energies(ens, rounds, serial):
    """Energy at every label after every round (rounds x labels)."""
    out = np.zeros((rounds, ens.nchains))
    for r in range(rounds):
        ens.pt_sweeps(1, serial=serial)
        out[r] = ens.energies()[ens.pt_map()]
    return out


def test_batched_pt_samples_the_serial_schedules_distribution():
    from smmp.ensemble import Ensemble, Molecule
    n, runs, equi, prod = 8, 6, 150, 900
    betas = _ladder(n, 250.0, 1000.0)
    mol = Molecule(SEQ, VAR, libdir=DATA)
    samples = {"batched": [], "serial": []}
    for run in range(runs):
        b = Ensemble([mol], [0] * n, [9000 + 100 * run + k for k in range(n)], betas, fp32=True)
        b.random_start()
        b.set_pt(betas, wrap=True, exchange_seed=77 + run)
        b.pt_sweeps(equi)
        samples["batched"].append(_label_energies(b, prod, serial=False))
        s = Ensemble([mol], [0] * n, [5000 + run], betas, shared_stream=True, fp32=True)
        s.random_start()
        s.set_pt(betas, wrap=True)
        s.pt_sweeps(equi, serial=True)
        samples["serial"].append(_label_energies(s, prod, serial=True))
    pooled = np.concatenate(samples["batched"] + samples["serial"])
    med = np.median(pooled, axis=0)
    worst = 0.0
    for k in range(n):
        for stat in (lambda e: e.mean(), lambda e: (e < med[k]).mean()):
            a = np.array([stat(x[:, k]) for x in samples["batched"]])
            c = np.array([stat(x[:, k]) for x in samples["serial"]])
            se = np.sqrt(a.var(ddof=1) / runs + c.var(ddof=1) / runs)
            z = abs(a.mean() - c.mean()) / max(se, 1e-12)
            worst = max(worst, z)
    print("\nbatched vs serial PT, 8 temperatures, %d runs each: largest |z| = %.2f" % (runs, worst))
    assert worst < 4.5
