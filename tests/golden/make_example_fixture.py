"""Builds tests/golden/example_si_p.npz from the reference's own example inputs.

Source: example/X.3d and example/e1.dat of Coulombo-Lattice (Rozanski & Zielinski,
Comput. Phys. Commun. 287 (2023) 108693; CC BY 4.0).  The run in example/run.sh:3-9
(--atoms=X.3d --dielectric=11.4 --orbitals=10 --skip-lines=1 e1.dat) must print
" 1  1  1  1    0.090340071977" as the first 29 characters of eeee.txt.

Both files are fixed-point decimal text (14 decimals for positions, 15 for coefficients),
so they are stored exactly as scaled integers; write_example() regenerates text with the
same values.  Usage: python tests/golden/make_example_fixture.py [reference_root]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "example_si_p.npz")
GOLDEN = " 1  1  1  1    0.090340071977"


def _fixed(s, decimals):
    s = s.strip()
    neg = s.startswith("-")
    s = s.lstrip("+-")
    ip, _, fp = s.partition(".")
    fp = (fp + "0" * decimals)[:decimals]
    v = int(ip) * 10 ** decimals + int(fp or "0")
    return -v if neg else v


def build(ref_root):
    pos = []
    with open(os.path.join(ref_root, "example", "X.3d")) as fh:
        for line in fh:
            parts = line.split()
            pos.append([_fixed(p, 14) for p in parts[:3]])
    coef = []
    with open(os.path.join(ref_root, "example", "e1.dat")) as fh:
        header = fh.readline()
        for line in fh:
            parts = line.split()
            coef.append([_fixed(p, 15) for p in parts[:2]])
    np.savez_compressed(OUT, pos_e14=np.array(pos, dtype=np.int64), coef_e15=np.array(coef, dtype=np.int64),
                        header=np.array(header.rstrip("\n")), golden=np.array(GOLDEN))


def _fmt(v, decimals):
    sign = "-" if v < 0 else ""
    v = abs(int(v))
    return "%s%d.%0*d" % (sign, v // 10 ** decimals, decimals, v % 10 ** decimals)


def load():
    """-> dict(pos [A,3] float64, coeff [A,10] complex128, golden str)."""
    z = np.load(OUT)
    pos = z["pos_e14"].astype(np.float64) / 1e14
    # exact decimal -> nearest double, the way the text parsers read it
    pos = np.array([[float(_fmt(v, 14)) for v in row] for row in z["pos_e14"]])
    c = np.array([float(_fmt(v, 15)) for v in z["coef_e15"][:, 0]]) + 1j * np.array(
        [float(_fmt(v, 15)) for v in z["coef_e15"][:, 1]])
    return dict(pos=pos, coeff=c.reshape(-1, 10), golden=str(z["golden"]), header=str(z["header"]))


def write_example(directory):
    """Writes X.3d and e1.dat (reference text layout) into directory."""
    z = np.load(OUT)
    with open(os.path.join(directory, "X.3d"), "w") as fh:
        for row in z["pos_e14"]:
            fh.write(" ".join(_fmt(v, 14) for v in row) + "\n")
    with open(os.path.join(directory, "e1.dat"), "w") as fh:
        fh.write(str(z["header"]) + "\n")
        for row in z["coef_e15"]:
            fh.write("%s %s\n" % (_fmt(row[0], 15), _fmt(row[1], 15)))


if __name__ == "__main__":
    build(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CL_REFERENCE_ROOT", os.path.join(os.sep, "root", "reference")))
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
