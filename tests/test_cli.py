"""The drop-in binaries' command line and failure behaviour (coulombo.cpp:265-315,
Parser.cpp:35-99, coulombo.cpp:38-117): everything here fails before any GPU work."""
import os
import subprocess

import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from conftest import has_gpu

COULOMBO = os.path.join(cl.BIN_DIR, "coulombo")
POTENTIALS = os.path.join(cl.BIN_DIR, "potentials")


def run(binary, args, cwd):
    p = subprocess.run([binary] + args, cwd=cwd, capture_output=True, text=True, timeout=120)
    return p.returncode, p.stdout, p.stderr


@pytest.fixture()
def inputs(tmp_path):
    from coulombo_lattice_b200 import synth
    d = synth.build("c1", cells=(2, 2, 2))
    d["states"] = d["states"][:, :, :10]
    synth.write_inputs(str(tmp_path), d)
    return tmp_path


def test_usage(tmp_path):
    for b in (COULOMBO, POTENTIALS):
        rc, out, err = run(b, [], tmp_path)
        assert rc == 1 and "USAGE" in err


@pytest.mark.parametrize("args,msg", [
    (["--bogus=1", "e1.dat"], "unknown value 'bogus'"),
    (["--atoms", "e1.dat"], "missing value for parameter 'atoms'"),
    (["--verbose", "e1.dat"], "unknown flag 'verbose'"),
    (["-x", "e1.dat"], "unknown flag 'x'"),
    (["e1.dat"], "parameter 'atoms' not specified"),
    (["--atoms=missing.3d", "e1.dat"], "could not open file: missing.3d"),
    (["--atoms=X.3d", "--orbitals=0", "e1.dat"], "invalid value for orbitals"),
    (["--atoms=X.3d", "--skip-lines=0", "e1.dat"], "invalid value for skip-lines"),
    (["--atoms=X.3d", "--threads-per-node=0", "e1.dat"], "invalid value for threads-per-node"),
    (["--atoms=X.3d", "--method=fast", "e1.dat"], "invalid value for method: fast"),
    (["--atoms=X.3d", "--orbitals=10", "--skip-lines=1", "e1.dat", "h1.dat"],
     "hole states must appear before electron states"),
    (["--atoms=X.3d", "--orbitals=10", "--skip-lines=1", "x1.dat"], "invalid state file name: x1.dat"),
    (["--atoms=X.3d", "--orbitals=11", "--skip-lines=1", "h1.dat"], "file is truncated: h1.dat"),
    (["--atoms=X.3d", "--orbitals=10", "--skip-lines=1", "--integrals=e0ee", "h1.dat"],
     "invalid character '0' in pattern"),
    (["--atoms=X.3d", "--orbitals=10", "--skip-lines=1", "--integrals=ee,", "h1.dat"], "invalid empty pattern"),
    (["--atoms=X.3d", "--orbitals=10", "--skip-lines=1", "--tf-lattice=-1", "h1.dat"],
     "--tf-lattice parameter must be positive"),
    (["--atoms=X.3d", "--orbitals=10", "--skip-lines=1", "--tf-lattice=5.65", "--dielectric=1", "h1.dat"],
     "dielectric constant must be >1 to use Thomas-Fermi model"),
])
def test_errors(inputs, args, msg):
    rc, out, err = run(COULOMBO, args, inputs)
    assert rc == 1
    assert "ERROR: " + msg in err


def test_phase_lines_and_no_gpu_error(inputs):
    if has_gpu():
        pytest.skip("no-GPU path")
    rc, out, err = run(COULOMBO, ["--atoms=X.3d", "--orbitals=10", "--skip-lines=1", "h1.dat", "e1.dat"], inputs)
    assert rc == 1
    for phase in ("Reading atom positions... (", "Reading wavefunctions... (", "Preparing plan... (",
                  "Initializing calculator... ("):
        assert phase in err
    assert "ERROR: no CUDA device is available" in err


def test_non_lattice_atoms(tmp_path):
    np.savetxt(tmp_path / "X.3d", np.array([[0, 0, 0], [1.0, 0, 0], [1.503, 0, 0]]))
    (tmp_path / "e1.dat").write_text("0 0\n" * 3)
    rc, out, err = run(COULOMBO, ["--atoms=X.3d", "--orbitals=1", "e1.dat"], tmp_path)
    assert rc == 1 and "ERROR: could not find common grid step" in err
