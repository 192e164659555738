"""Restart files of the serial parallel-tempering driver (partem_s.f:100-110
reads them, :237-255 writes them): ``par_R.in``, a Fortran unformatted
sequential file (each record framed by its 4-byte length) holding for every
replica k a record with the sweep count and a record with the energies, and
``conf_NNNN.var``, replica k's variables in the .var command language as
outvar writes them.

The reference writes the whole energy array in each replica's energy record
(``write(15) eol``) and reads back only its first element
(``read(15) eol(k)``), so every replica restarts with replica 1's energy;
read_par_r keeps that behaviour.  Host code only (no GPU needed)."""
import os
import struct

import numpy as np


def _record(data):
    n = len(data)
    return struct.pack("<i", n) + data + struct.pack("<i", n)


def _records(blob):
    off = 0
    while off < len(blob):
        (n,) = struct.unpack_from("<i", blob, off)
        data = blob[off + 4:off + 4 + n]
        (m,) = struct.unpack_from("<i", blob, off + 4 + n)
        if m != n:
            raise ValueError("par_R.in: record markers differ")
        yield data
        off += 8 + n


def conf_name(k):
    """fileNameMP('conf_0000.var', 6, 9, k): '' if k needs more than 4 digits."""
    return "conf_%04d.var" % k if 0 <= k <= 9999 else ""


def write_par_r(directory, nswp, eol, vlvr, molecule):
    """partem_s.f:237-255: par_R.in and conf_NNNN.var for the replicas' final
    energies eol[num_rep] and variables vlvr[num_rep, nvar] (radians)."""
    eol = np.ascontiguousarray(eol, dtype="<f8")
    vlvr = np.atleast_2d(np.asarray(vlvr, dtype=np.float64))
    with open(os.path.join(directory, "par_R.in"), "wb") as f:
        for k in range(len(eol)):
            f.write(_record(struct.pack("<i", int(nswp))))
            f.write(_record(eol.tobytes()))
            name = conf_name(k + 1)
            with open(os.path.join(directory, name), "w") as g:
                g.write(molecule.outvar(vlvr[k]))


def read_par_r(directory, num_rep, seqfile, **molecule_args):
    """partem_s.f:100-110: (nstart, eol[num_rep], vlvr[num_rep, nvar]); each
    replica's variables come from its conf_NNNN.var through the .var reader."""
    from .ensemble import Molecule
    with open(os.path.join(directory, "par_R.in"), "rb") as f:
        recs = list(_records(f.read()))
    if len(recs) < 2 * num_rep:
        raise ValueError("par_R.in holds fewer replicas than asked for")
    nstart, eol, rows = 0, np.zeros(num_rep), []
    for k in range(num_rep):
        (nstart,) = struct.unpack_from("<i", recs[2 * k])
        (eol[k],) = struct.unpack_from("<d", recs[2 * k + 1])   # read(15) eol(k): first value
        m = Molecule(seqfile, os.path.join(directory, conf_name(k + 1)), **molecule_args)
        rows.append(m.vlvr0)
    return nstart, eol, np.array(rows)
