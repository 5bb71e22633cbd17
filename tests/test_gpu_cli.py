"""The drop-in binaries end to end on the GPU: the reference's example integration test
(example/run.sh:3-9) and a synthetic run checked line by line against the oracle."""
import os
import subprocess

import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import coulomb as C
from oracle import host as H

pytestmark = pytest.mark.gpu

COULOMBO = os.path.join(cl.BIN_DIR, "coulombo")
POTENTIALS = os.path.join(cl.BIN_DIR, "potentials")


def run(binary, args, cwd):
    p = subprocess.run([binary] + args, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    return p.stderr


def test_example_run_sh(tmp_path):
    import make_example_fixture as fx
    fx.write_example(str(tmp_path))
    err = run(COULOMBO, ["--atoms=X.3d", "--dielectric=11.4", "--orbitals=10", "--skip-lines=1", "e1.dat"], tmp_path)
    assert "Computing requested integrals... (" in err
    assert (tmp_path / "eeee.txt").read_text()[:29] == " 1  1  1  1    0.090340071977"
    assert sorted(os.listdir(tmp_path)) == ["X.3d", "e1.dat", "eeee.txt"]


def test_example_potentials(tmp_path):
    import make_example_fixture as fx
    fx.write_example(str(tmp_path))
    run(POTENTIALS, ["--atoms=X.3d", "--dielectric=11.4", "--orbitals=10", "--skip-lines=1", "e1.dat"], tmp_path)
    got = np.loadtxt(tmp_path / "potential-e1.dat")
    d = fx.load()
    g = H.detect_grid(d["pos"])
    ghat = C.kernel_spectrum(C.kernel_octant(g["pad"], g["step"], 11.4), g["pad"])
    rho = C.pair_density_atoms(d["coeff"], d["coeff"])
    V = C.prepare(C.scatter_density(rho, g["cells"], g["pad"]), ghat).ravel()[g["cells"]].real
    assert np.abs(got - V).max() <= 1e-10 * np.abs(V).max()


@pytest.mark.parametrize("method", ["rounds", "sublattice"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_synthetic_outputs(tmp_path, precision, method):
    d = synth.build("c1", cells=(4, 4, 4))
    names = synth.write_inputs(str(tmp_path), d)
    out = tmp_path / "out"
    out.mkdir()
    run(COULOMBO, ["--atoms=X.3d", "--dielectric=10.89", "--orbitals=10", "--skip-lines=1",
                   "--integrals=eeee,hhhh,ehhe,eheh", "--output-dir=out", "--precision=" + precision, "--method=" + method] + names, tmp_path)
    specs = H.enumerate_integrals(H.Pattern("eeee,hhhh,ehhe,eheh", 2), 4)
    g = H.detect_grid(np.loadtxt(tmp_path / "X.3d"))
    states = [H.load_state(str(tmp_path / n), len(g["cells"]), 10, 1) for n in names]
    vals = H.compute_integrals(states, g["cells"], g["pad"], g["step"], specs, dielectric=10.89)
    want = H.format_outputs(specs, vals, 2, 2)
    assert sorted(os.listdir(out)) == sorted(k + ".txt" for k in want)
    for core, text in want.items():
        got_lines = (out / (core + ".txt")).read_text().splitlines()
        want_lines = text.splitlines()
        assert len(got_lines) == len(want_lines)
        for a, b in zip(got_lines, want_lines):
            assert a[:14] == b[:14]
            ga = np.array(a[14:].split(), float)
            gb = np.array(b[14:].split(), float)
            tol = 2e-14 if precision == "fp64" else max(1e-6 * np.abs(gb).max(), 1e-9)
            assert np.abs(ga - gb).max() <= tol
