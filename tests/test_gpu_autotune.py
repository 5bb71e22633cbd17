"""The autotuner of the register passes: every compiled variant (radix split balanced or
swapped, default or half lines per block) computes the same transforms, and the tuned choice
is reported and agrees with the default variants."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import coulomb as C
from oracle import host as H

pytestmark = pytest.mark.gpu

MODES = [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS]
TOL = {cl.MODE_FP64_PLAIN: 1e-10, cl.MODE_FP32_ROUNDS: 1e-6}
# every axis has a non-square split, so the swapped variant differs from the balanced one
SHAPES = [(96, 128, 40), (160, 72, 48), (48, 80, 96)]


@pytest.mark.parametrize("force", ["0,1", "1,0", "1,1", "0,0,1", "1,1,1"])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dims", SHAPES)
def test_every_variant_matches_oracle(dims, mode, force, monkeypatch):
    monkeypatch.setenv("CL_TUNE_FORCE", force)
    nx, ny, nz = dims
    rng = np.random.default_rng(nx + 3 * ny + 5 * nz)
    F = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    F2 = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    step = (1.1, 0.9, 1.3)
    ghat = C.kernel_spectrum(C.kernel_octant(dims, step, dielectric=5.0), dims)
    V = C.prepare(F, ghat)
    want = C.calculate(V, F2)
    with cl.CoulombCalculator(dims, step, mode) as cc:
        cc.initialize(dielectric=5.0)
        cc.prepare(F)
        Vg = cc.potential()
        got = cc.calculate(F2)
    assert np.abs(Vg - V).max() <= TOL[mode] * 10 * np.abs(V).max()
    assert abs(got - want) <= TOL[mode] * 10 * np.sqrt(np.sum(np.abs(V) ** 2) * np.sum(np.abs(F2) ** 2))


@pytest.mark.parametrize("force", ["0,0", "1,1", "0,1,1"])
@pytest.mark.parametrize("mode", MODES)
def test_variants_on_atoms_with_skipped_rows(mode, force, monkeypatch):
    """The integral path (atom scatter/gather, rows without atoms skipped) under a forced
    variant, against the oracle."""
    monkeypatch.setenv("CL_TUNE_FORCE", force)
    d = synth.build("c1", cells=(12, 10, 8))  # 48 x 40 x 32 grid
    step = (synth.A_ZB / 4,) * 3
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("eeee,hhhh,ehhe,eheh", 4, 2)]
    want = np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], step, specs,
                                        dielectric=10.89))
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 2)
        got = cc.compute(specs)
    err = np.abs(got - want)
    if mode == cl.MODE_FP64_PLAIN:
        assert np.all(err <= 1e-10 * np.abs(want) + 1e-16)
    else:
        assert np.all(err <= np.maximum(1e-6 * np.abs(want), 1e-9))


@pytest.mark.parametrize("mode", MODES)
def test_tuned_choice_is_reported_and_agrees(mode, monkeypatch):
    d = synth.build("c1", cells=(16, 12, 10))  # 64 x 48 x 40 grid
    step = (synth.A_ZB / 4,) * 3
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]

    def run():
        with cl.CoulombCalculator(d["dims"], step, mode) as cc:
            cc.initialize(dielectric=10.89)
            cc.set_states(d["states"], d["cells_idx"], 2)
            return cc.compute(specs)

    tuned = run()
    report = cl.autotune_report()
    prec = "fp64" if mode == cl.MODE_FP64_PLAIN else "fp32"
    lines = [ln for ln in report.splitlines() if "64x48x40" in ln and prec in ln]
    assert {ln.split()[0] for ln in lines} == {"x_forward", "y_forward", "z_pass", "y_inverse", "x_inverse"}
    for ln in lines:
        assert "candidates" in ln and "default" in ln
    monkeypatch.setenv("CL_TUNE_FORCE", "0,0")
    default = run()
    tol = 1e-12 if mode == cl.MODE_FP64_PLAIN else 1e-6
    assert np.abs(tuned - default).max() <= tol * np.abs(default).max()


def test_tune_file_persists_choices(tmp_path):
    """CL_TUNE_FILE: a first process appends its choices; a second one loads them instead of
    timing, and computes the same values."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = (
        "import sys, numpy as np\n"
        "sys.path.insert(0, %r)\n"
        "import coulombo_lattice_b200 as cl\n"
        "from coulombo_lattice_b200 import synth\n"
        "d = synth.build('c1', cells=(10, 12, 8))\n"
        "specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals('****', 4, 2)]\n"
        "with cl.CoulombCalculator(d['dims'], (synth.A_ZB / 4,) * 3, cl.MODE_FP32_ROUNDS) as cc:\n"
        "    cc.initialize(dielectric=10.89)\n"
        "    cc.set_states(d['states'], d['cells_idx'], 2)\n"
        "    v = cc.compute(specs)\n"
        "np.save(sys.argv[1], v)\n"
        "print(cl.autotune_report())\n" % root)
    env = dict(os.environ, CL_TUNE_FILE=str(tmp_path / "tune.txt"))
    env.pop("CL_TUNE_FORCE", None)
    env.pop("CL_AUTOTUNE", None)
    r1 = subprocess.run([sys.executable, "-c", script, str(tmp_path / "a.npy")], env=env, capture_output=True,
                        text=True, timeout=300)
    assert r1.returncode == 0, r1.stderr
    saved = (tmp_path / "tune.txt").read_text().split("\n")
    assert len([ln for ln in saved if ln.strip()]) == 5  # one line per pass of the 40x48x32 shape
    r2 = subprocess.run([sys.executable, "-c", script, str(tmp_path / "b.npy")], env=env, capture_output=True,
                        text=True, timeout=300)
    assert r2.returncode == 0, r2.stderr
    assert r2.stdout.count("from CL_TUNE_FILE") == 5
    a, b = np.load(tmp_path / "a.npy"), np.load(tmp_path / "b.npy")
    np.testing.assert_allclose(b, a, rtol=1e-12, atol=0)
