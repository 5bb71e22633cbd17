"""The fused xy plane passes (a whole xy-plane in shared memory per block: 64^2 and 96^2 in
FP32 and FP64, 128^2 in FP32) against the oracle and against the separate x and y passes, on
zinc-blende atoms, on scattered atoms (rows of every parity, a plane with more atoms than a
block keeps in registers) and on the grid API (every cell an atom)."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import coulomb as C
from oracle import host as H

pytestmark = pytest.mark.gpu

STEP = (synth.A_ZB / 4,) * 3
FP32, FP64 = cl.MODE_FP32_ROUNDS, cl.MODE_FP64_PLAIN


def _gate(mode, want):
    if mode == FP64:
        return 1e-10 * np.abs(want) + 1e-16
    return np.maximum(1e-6 * np.abs(want), 1e-9)


def _integrals(d, mode, specs, plane, monkeypatch):
    monkeypatch.setenv("CL_XY_PLANE", plane)
    try:
        with cl.CoulombCalculator(d["dims"], STEP, mode) as cc:
            cc.initialize(dielectric=10.89)
            cc.set_states(d["states"], d["cells_idx"], d["holes"])
            return cc.compute(specs)
    finally:
        monkeypatch.delenv("CL_XY_PLANE", raising=False)


def _oracle(d, specs):
    return np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], STEP, specs,
                                        dielectric=10.89))


def _check(d, mode, monkeypatch):
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("eeee,hhhh,ehhe,eheh", 4, 2)]
    want = _oracle(d, specs)
    got = _integrals(d, mode, specs, "1", monkeypatch)
    assert np.all(np.abs(got - want) <= _gate(mode, want)), (np.abs(got - want) / _gate(mode, want)).max()
    sep = _integrals(d, mode, specs, "0", monkeypatch)
    tol = 1e-12 if mode == FP64 else 1e-6
    assert np.abs(got - sep).max() <= tol * np.abs(sep).max()


@pytest.mark.parametrize("mode,cells", [(FP32, (24, 24, 3)), (FP64, (24, 24, 3)), (FP32, (32, 32, 2)),
                                        (FP32, (16, 16, 3)), (FP64, (16, 16, 3))],
                         ids=["fp32-96", "fp64-96", "fp32-128", "fp32-64", "fp64-64"])
def test_plane_passes_on_zincblende_atoms(mode, cells, monkeypatch):
    _check(synth.build("c1", cells=cells), mode, monkeypatch)


@pytest.mark.parametrize("mode,n", [(FP32, 96), (FP64, 96), (FP32, 128), (FP32, 64), (FP64, 64)],
                         ids=["fp32-96", "fp64-96", "fp32-128", "fp32-64", "fp64-64"])
def test_plane_passes_on_scattered_atoms(mode, n, monkeypatch):
    """Atoms on random distinct cells: live rows of both classes in every plane, unpaired rows,
    and a first plane holding more atoms (2,100) than a block keeps in registers (copied ahead
    through shared memory where the plane kernel has room, read directly otherwise); the grid
    API below has planes with more atoms than that room."""
    d = synth.build("c1", cells=(n // 4, n // 4, 2))
    n_atoms = d["states"].shape[1]
    rng = np.random.default_rng(n)
    plane = n * n
    first = rng.choice(plane, size=2100, replace=False)
    rest = plane + rng.choice(plane * 7, size=n_atoms - 2100, replace=False)
    d["cells_idx"] = np.sort(np.concatenate([first, rest])).astype(np.int64)
    _check(d, mode, monkeypatch)


@pytest.mark.parametrize("mode,dims", [(FP32, (96, 96, 10)), (FP64, (96, 96, 10)), (FP32, (128, 128, 6)),
                                       (FP32, (64, 64, 12)), (FP64, (64, 64, 12))],
                         ids=["fp32-96", "fp64-96", "fp32-128", "fp32-64", "fp64-64"])
def test_plane_passes_on_grid_api(mode, dims, monkeypatch):
    rng = np.random.default_rng(dims[0] + dims[2])
    nx, ny, nz = dims
    F = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    F2 = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    step = (1.0, 1.2, 0.9)
    V = C.prepare(F, C.kernel_spectrum(C.kernel_octant(dims, step, dielectric=3.0), dims))
    want = C.calculate(V, F2)
    monkeypatch.setenv("CL_XY_PLANE", "1")
    with cl.CoulombCalculator(dims, step, mode) as cc:
        cc.initialize(dielectric=3.0)
        cc.prepare(F)
        Vg = cc.potential()
        got = cc.calculate(F2)
    tol = 1e-10 if mode == FP64 else 1e-6
    assert np.abs(Vg - V).max() <= tol * 10 * np.abs(V).max()
    assert abs(got - want) <= tol * 10 * np.sqrt(np.sum(np.abs(V) ** 2) * np.sum(np.abs(F2) ** 2))


def test_tuner_reports_the_plane_choice():
    """With the autotuner on, the fused passes are timed against the separate ones they
    replace and the choice is reported for both directions."""
    d = synth.build("c1", cells=(24, 24, 1))  # 96 x 96 x 4 grid
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    with cl.CoulombCalculator(d["dims"], STEP, FP32) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 2)
        got = cc.compute(specs)
    want = _oracle(d, specs)
    assert np.all(np.abs(got - want) <= _gate(FP32, want))
    lines = [ln for ln in cl.autotune_report().splitlines() if "96x96x4" in ln and "fp32" in ln]
    names = {ln.split()[0] for ln in lines}
    assert {"xy_forward", "xy_inverse"} <= names
    for ln in lines:
        if ln.startswith("xy_"):
            assert ("fused plane pass" in ln or "separate passes" in ln) and "candidates" in ln
