"""The parallel-tempering restart files (partem_s.f:100-110, 237-255) on the
CPU: par_R.in's record layout, and a write/read round trip through outvar and
the .var reader."""
import struct

import numpy as np

from conftest import DATA

CRD = 57.2957795130823


def test_par_r_round_trip(tmp_path):
    from smmp.ensemble import Molecule
    from smmp.restart import conf_name, read_par_r, write_par_r
    m = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)
    rng = np.random.default_rng(4)
    rows = np.tile(m.vlvr0, (3, 1))
    rows[:, m.idvr] += rng.uniform(-1.0, 1.0, (3, len(m.idvr)))
    rows = (rows + np.pi) % (2 * np.pi) - np.pi
    eol = np.array([-3.5, 1.25, 17.0])
    write_par_r(str(tmp_path), 5000, eol, rows, m)
    blob = (tmp_path / "par_R.in").read_bytes()
    assert len(blob) == 3 * ((4 + 4 + 4) + (4 + 24 + 4))
    assert struct.unpack_from("<iii", blob, 0) == (4, 5000, 4)
    assert struct.unpack_from("<i3di", blob, 12) == (24, -3.5, 1.25, 17.0, 24)
    for k in range(1, 4):
        assert (tmp_path / conf_name(k)).exists()
    nstart, e, v = read_par_r(str(tmp_path), 3, DATA + "enkefa.seq", libdir=DATA)
    assert nstart == 5000
    assert np.array_equal(e, [-3.5, -3.5, -3.5])   # the reference reads the first value
    d = (v - rows) * CRD
    d = (d + 180.0) % 360.0 - 180.0
    assert np.abs(d).max() <= 5e-4


def test_conf_names():
    from smmp.restart import conf_name
    assert conf_name(1) == "conf_0001.var" and conf_name(11) == "conf_0011.var"
    assert conf_name(10000) == ""
