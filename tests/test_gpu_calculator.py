"""The grid-level calculator (prepare/calculate/potential) against the oracle."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from oracle import coulomb as C

pytestmark = pytest.mark.gpu

MODES = [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS]
# plain FP64 path: 1e-10 relative; FP32 transforms with FP64 sums: 1e-6 relative
TOL = {cl.MODE_FP64_PLAIN: 1e-10, cl.MODE_FP32_ROUNDS: 1e-6}


def _exp_kernel(dims):
    nx, ny, nz = dims
    return np.fromfunction(lambda z, y, x: np.exp(-x - y - z), (nz + 1, ny + 1, nx + 1))


@pytest.mark.parametrize("mode", MODES)
def test_two_point_charges(mode):
    """run-tests.cpp:28-48 through the C ABI: 1 and exp(-5) (1e-12 for FP64)."""
    tol = 1e-12 if mode == cl.MODE_FP64_PLAIN else 1e-6
    with cl.CoulombCalculator((5, 5, 10), mode=mode) as cc:
        cc.initialize_grid(_exp_kernel((5, 5, 10)))
        F = np.zeros((10, 5, 5), complex)
        F[2, 2, 2] = 1.0
        cc.prepare(F)
        r = cc.calculate(F)
        assert abs(r.real - 1.0) < tol and abs(r.imag) < tol
        F2 = np.zeros_like(F)
        F2[7, 2, 2] = 1.0
        r = cc.calculate(F2)   # reuses the last prepare
        assert abs(r.real - np.exp(-5)) < tol and abs(r.imag) < tol


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dims", [(5, 5, 10), (12, 16, 20), (45, 45, 45), (6, 1, 9)])
def test_random_grid_matches_oracle(mode, dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(sum(dims))
    F = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    F2 = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    step = (1.3, 0.9, 1.1)
    G = C.kernel_octant(dims, step, dielectric=10.89, onsite=0.3)
    ghat = C.kernel_spectrum(G, dims)
    V = C.prepare(F, ghat)
    want = C.calculate(V, F2)
    with cl.CoulombCalculator(dims, step, mode) as cc:
        cc.initialize(dielectric=10.89, onsite=0.3)
        cc.prepare(F)
        got = cc.calculate(F2)
        Vg = cc.potential()
    assert abs(got - want) <= TOL[mode] * abs(want)
    assert np.abs(Vg - V).max() <= TOL[mode] * 10 * np.abs(V).max()


@pytest.mark.parametrize("mode", MODES)
def test_thomas_fermi_kernel(mode):
    dims = (16, 12, 10)
    step = (1.4125, 1.4125, 1.4125)
    rng = np.random.default_rng(2)
    F = rng.normal(size=(10, 12, 16)) + 1j * rng.normal(size=(10, 12, 16))
    ghat = C.kernel_spectrum(C.kernel_octant(dims, step, 10.89, 0.0, tf_lattice=5.65), dims)
    want = C.calculate(C.prepare(F, ghat), np.conj(F))
    with cl.CoulombCalculator(dims, step, mode) as cc:
        cc.initialize(dielectric=10.89, tf_lattice=5.65)
        cc.prepare(F)
        got = cc.calculate(np.conj(F))
    assert abs(got - want) <= TOL[mode] * abs(want)


def test_state_errors():
    with cl.CoulombCalculator((4, 4, 4)) as cc:
        with pytest.raises(cl.CoulomboError) as e:
            cc.prepare(np.zeros((4, 4, 4), complex))
        assert e.value.kind == "state"
        cc.initialize(2.0)
        with pytest.raises(cl.CoulomboError) as e:
            cc.calculate(np.zeros((4, 4, 4), complex))
        assert e.value.kind == "state"
        with pytest.raises(cl.CoulomboError, match="Thomas-Fermi"):
            cc.initialize(1.0, tf_lattice=5.0)


# y and z lengths covering the compiled two-factor splits of the register column passes
# (x kept small); the generic passes handle the rest.
SPLIT_SHAPES = [(8, 256, 8), (8, 8, 256), (6, 96, 128), (4, 160, 144), (4, 240, 180), (2, 225, 135),
                (4, 192, 150), (4, 120, 108), (4, 100, 90), (8, 81, 75), (8, 72, 64), (8, 60, 54),
                (8, 50, 48), (8, 45, 40), (8, 36, 32), (8, 30, 27), (8, 25, 24), (8, 20, 16)]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dims", SPLIT_SHAPES)
def test_register_column_passes_match_oracle(mode, dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(nx + 7 * ny + 13 * nz)
    F = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    step = (1.4, 1.1, 0.8)
    ghat = C.kernel_spectrum(C.kernel_octant(dims, step, dielectric=3.0), dims)
    V = C.prepare(F, ghat)
    with cl.CoulombCalculator(dims, step, mode) as cc:
        cc.initialize(dielectric=3.0)
        cc.prepare(F)
        Vg = cc.potential()
    assert np.abs(Vg - V).max() <= TOL[mode] * 10 * np.abs(V).max()


# long x axes with y outside the whole-plane sizes: the register row passes (scatter + FFT
# along x, FFT along x + gather) are exercised
ROW_SHAPES = [(256, 8, 6), (96, 12, 10), (160, 6, 5), (45, 12, 6), (128, 6, 8), (240, 4, 6), (225, 4, 4),
              (20, 6, 6), (192, 10, 4), (100, 12, 3)]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dims", ROW_SHAPES)
def test_register_row_passes_match_oracle(mode, dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(3 * nx + ny + 11 * nz)
    F = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    F2 = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    step = (0.9, 1.3, 1.2)
    ghat = C.kernel_spectrum(C.kernel_octant(dims, step, dielectric=4.0, onsite=0.2), dims)
    V = C.prepare(F, ghat)
    want = C.calculate(V, F2)
    with cl.CoulombCalculator(dims, step, mode) as cc:
        cc.initialize(dielectric=4.0, onsite=0.2)
        cc.prepare(F)
        Vg = cc.potential()
        got = cc.calculate(F2)
    assert np.abs(Vg - V).max() <= TOL[mode] * 10 * np.abs(V).max()
    assert abs(got - want) <= TOL[mode] * 10 * np.sqrt(np.sum(np.abs(V) ** 2) * np.sum(np.abs(F2) ** 2))


# lengths beyond the compiled two-factor splits (> 256) take the generic shared-memory passes,
# mixed with register passes on the other axes
GENERIC_SHAPES = [(288, 6, 5), (6, 270, 5), (5, 6, 300), (320, 4, 270)]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dims", GENERIC_SHAPES)
def test_generic_passes_beyond_register_splits(mode, dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(nx + 5 * ny + 9 * nz)
    F = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    F2 = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    step = (0.7, 1.2, 1.0)
    ghat = C.kernel_spectrum(C.kernel_octant(dims, step, dielectric=2.0), dims)
    V = C.prepare(F, ghat)
    want = C.calculate(V, F2)
    with cl.CoulombCalculator(dims, step, mode) as cc:
        cc.initialize(dielectric=2.0)
        cc.prepare(F)
        Vg = cc.potential()
        got = cc.calculate(F2)
    assert np.abs(Vg - V).max() <= TOL[mode] * 10 * np.abs(V).max()
    assert abs(got - want) <= TOL[mode] * 10 * np.sqrt(np.sum(np.abs(V) ** 2) * np.sum(np.abs(F2) ** 2))
