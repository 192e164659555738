"""Generate the input fixtures and published golden values used by the tests.

Run once in a container that has the SMMP reference mounted (the GPU box does
not): it copies the ECEPP residue libraries, the SASA sphere points and the
Met-enkephalin input decks into tests/golden/smmp_data/, and records the
reference's published numbers (README and EXAMPLES/annealing.out) with their
sources in tests/golden/golden.json.

    python tests/golden/make_fixtures.py <SMMP trunk directory>

The argument is the reference's trunk/ directory (the one holding README,
EXAMPLES/ and SMMP/).
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

DATA = [
    ("SMMP/lib.sh3", "lib.sh3"),        # ECEPP/3 residue library
    ("SMMP/lib.sh2", "lib.sh2"),        # ECEPP/2 residue library
    ("SMMP/tes.dat", "tes.dat"),        # 122 unit-sphere points (enysol)
    ("EXAMPLES/enkefa.seq", "enkefa.seq"),
    ("EXAMPLES/enkefa.var", "enkefa.var"),
    ("EXAMPLES/enkefa.ann", "enkefa.ann"),
    ("EXAMPLES/temperatures", "temperatures"),
]


def read_lines(path):
    with open(path) as f:
        return f.read().split("\n")


def main(ref):
    out = os.path.join(HERE, "smmp_data")
    os.makedirs(out, exist_ok=True)
    for src, dst in DATA:
        shutil.copyfile(os.path.join(ref, src), os.path.join(out, dst))

    readme = read_lines(os.path.join(ref, "README"))
    ann = read_lines(os.path.join(ref, "EXAMPLES/annealing.out"))

    def fnum(s):
        return float(s.replace("D", "E"))

    # README:391-393  "Total:  0.10354E+04" / "Coulomb: ... HB: ..." / "Variables: ..."
    l391, l392, l393 = readme[390].split(), readme[391].split(), readme[392].split()
    golden = {
        "enkefa_ecepp3": {
            "source": "README:389-393",
            "setup": "enkefa.seq + enkefa.var, nh2/cooh, ECEPP/3, epsd=.false., itysol=0",
            "total": fnum(l391[1]),
            "coulomb": fnum(l392[1]),
            "lennard_jones": fnum(l392[3]),
            "hbond": fnum(l392[5]),
            "torsion": fnum(l393[1]),
            "digits": 4,
        },
        "anneal_ecepp2": {
            "source": "EXAMPLES/annealing.out:14-45; EXAMPLES/annealing.f:37-72",
            "setup": "enkefa.seq + enkefa.ann, nh2/cooh, ECEPP/2, seed 81236, "
                     "nequi=100, nswp=100000, tmax=1000, tmin=100, lrand",
            "start": fnum(ann[13].split(":")[1]),
            "after_equilibration": fnum(ann[15].split(":")[1]),
            "acceptance": fnum(ann[16].split(":")[1]),
            "last": fnum(ann[18].split()[-1]),
            "lowest": fnum(ann[44].split()[-1]),
            "lowest_sweep": int(ann[44].split()[-2]),
        },
        # README:389-514: EXAMPLES/minimization.f (enkefa.seq + enkefa.var,
        # ECEPP/3, quasi-Newton, maxit 10000, eps 1e-9): one line per
        # function call (energy, squared gradient; E13.6), the final energy
        # terms and the final free variables (degrees, one decimal)
        "minim_enkefa": {
            "source": "README:395-480 (steps), README:484-486 (energies), "
                      "README:490-513 (variables); EXAMPLES/minimization.f",
            "steps": [[ln.split(":")[1].split()[1], ln.split("(")[1].split(")")[0].strip()]
                      for ln in readme[394:480] if ln.strip().startswith("Step")],
            "total": fnum(readme[483].split()[1]),
            "coulomb": fnum(readme[484].split()[1]),
            "lennard_jones": fnum(readme[484].split()[3]),
            "hbond": fnum(readme[484].split()[5]),
            "torsion": fnum(readme[485].split()[1]),
            "variables": [[ln.split()[0], int(ln.split()[1]), float(ln.split()[2])]
                          for ln in readme[489:513] if ln.strip()],
        },
        # annealing.f:139 calls outvar(0, ' '): the final conformation in the
        # .var command language, as outvar.f:50-121 formats it
        "anneal_outvar": {
            "source": "EXAMPLES/annealing.out:20-43; EXAMPLES/annealing.f:139",
            "setup": "enkefa.seq + enkefa.ann, ECEPP/2",
            "lines": ann[19:43],
        },
    }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print(json.dumps(golden, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <SMMP trunk directory>")
    main(sys.argv[1])
