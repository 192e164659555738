"""Synthetic sequences for the benchmark configurations.

* Ace-Ala_n-NMe chains with n drawn uniformly from [nmin, nmax] (the uneven
  batch of independent chains).
* A protein of L residues drawn from the natural amino-acid composition,
  without proline at position 1 (an N-terminal proline takes the nh1 end group
  path, which the residue library supports only for ECEPP/3's 'pron').

Composition: UniProtKB/Swiss-Prot release statistics (amino-acid composition
of the reviewed database, percent), rounded to two decimals.
"""
import numpy as np

# residue -> percent (UniProtKB/Swiss-Prot composition)
NATURAL_COMPOSITION = {
    "ala": 8.25, "arg": 5.53, "asn": 4.06, "asp": 5.45, "cys": 1.37,
    "gln": 3.93, "glu": 6.75, "gly": 7.07, "his": 2.27, "ile": 5.96,
    "leu": 9.66, "lys": 5.84, "met": 2.42, "phe": 3.86, "pro": 4.70,
    "ser": 6.56, "thr": 5.34, "trp": 1.08, "tyr": 2.92, "val": 6.87,
}


def polyala_lengths(count, seed=12345, nmin=10, nmax=40):
    rng = np.random.default_rng(seed)
    return rng.integers(nmin, nmax + 1, size=count).tolist()


def polyala(n):
    return ["ace"] + ["ala"] * n + ["nme"]


def natural_protein(length, seed=2024):
    names = sorted(NATURAL_COMPOSITION)
    p = np.array([NATURAL_COMPOSITION[k] for k in names], dtype=np.float64)
    p /= p.sum()
    rng = np.random.default_rng(seed)
    seq = [names[k] for k in rng.choice(len(names), size=length, p=p)]
    while seq[0] == "pro":
        seq[0] = names[rng.choice(len(names), p=p)]
    return seq


def write_seq(path, residues, name="chain"):
    with open(path, "w") as f:
        f.write("# %s\n" % name)
        for k in range(0, len(residues), 15):
            f.write(" ".join(residues[k:k + 15]) + "\n")
    return path
