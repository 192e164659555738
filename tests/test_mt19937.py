"""MT19937 with the reference's seeding (twister.f:64-177).

No golden stream exists in the reference; the stream is pinned by the
annealing trajectory golden and here against numpy's MT19937 core: the
reference differs from the standard generator only in its Knuth-69069
seeding, so loading the seeded state into numpy must give the same words.
"""
import numpy as np
import pytest

from conftest import DATA, Oracle


def knuth_state(seed):
    mt = np.zeros(624, dtype=np.uint64)
    mt[0] = seed & 0xffffffff
    for i in range(1, 624):
        mt[i] = (69069 * int(mt[i - 1])) & 0xffffffff
    return mt.astype(np.uint32)


@pytest.mark.parametrize("seed", [4357, 31433, 81236, -5])
def test_oracle_grnd_equals_numpy_mt19937_with_knuth_seeding(seed):
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    o.sgrnd(seed)
    bg = np.random.MT19937()
    bg.state = {"bit_generator": "MT19937", "state": {"key": knuth_state(seed), "pos": 624}}
    words = bg.random_raw(5000).astype(np.uint64)
    got = np.array([o.grnd() for _ in range(5000)])
    assert np.all(got == words.astype(np.float64) / 4294967295.0)
    assert got.min() >= 0.0 and got.max() <= 1.0


def test_unseeded_stream_uses_4357():
    a = Oracle(DATA + "enkefa.seq")
    b = Oracle(DATA + "enkefa.seq")
    b.sgrnd(4357)
    assert [a.grnd() for _ in range(700)] == [b.grnd() for _ in range(700)]
