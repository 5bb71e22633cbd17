"""Pins the CPU oracle to the reference's own known answers (no GPU)."""
import numpy as np
import pytest

from oracle import coulomb as C
from oracle import host as H


def _exp_kernel(dims):
    nx, ny, nz = dims
    return np.fromfunction(lambda z, y, x: np.exp(-x - y - z), (nz + 1, ny + 1, nx + 1))


def test_two_point_charges():
    """run-tests.cpp:28-48: 5x5x10 grid, G = exp(-ix-iy-iz); charge at (2,2,2) -> 1;
    the right charge moved to (2,2,7) without re-preparing -> exp(-5), both to 1e-12."""
    dims = (5, 5, 10)
    ghat = C.kernel_spectrum(_exp_kernel(dims), dims)
    F = np.zeros((10, 5, 5), complex)
    F[2, 2, 2] = 1.0
    V = C.prepare(F, ghat)
    r = C.calculate(V, F)
    assert abs(r.real - 1.0) < 1e-12 and abs(r.imag) < 1e-12
    F2 = np.zeros_like(F)
    F2[7, 2, 2] = 1.0
    r = C.calculate(V, F2)
    assert abs(r.real - np.exp(-5)) < 1e-12 and abs(r.imag) < 1e-12


def test_fft_single_bin():
    """run-tests.cpp:189-214: 1024-point transform of cos(2 pi 16 n/1024 + pi/4) has one bin
    of magnitude 512 and phase pi/4 (FFTW sign -1, unnormalised)."""
    n = np.arange(1024)
    x = np.cos(2 * np.pi * 16 * n / 1024 + np.pi / 4)
    X = np.fft.fft(x)[:513]
    mask = np.ones(513, bool)
    mask[16] = False
    assert np.abs(X[mask]).max() < 1e-12
    assert abs(abs(X[16]) - 512) < 1e-12
    assert abs(np.angle(X[16]) - np.pi / 4) < 1e-12


@pytest.mark.parametrize("dims", [(5, 5, 10), (4, 6, 3), (3, 1, 5), (1, 1, 2)])
def test_rounds_equal_direct_convolution(dims):
    """The 8-round no-padding method reproduces the O(M^2) aperiodic convolution."""
    rng = np.random.default_rng(7)
    nx, ny, nz = dims
    F = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    G = rng.random((nz + 1, ny + 1, nx + 1))
    V = C.prepare(F, C.kernel_spectrum(G, dims))
    Vd = C.direct_convolution(F, G)
    assert np.abs(V - Vd).max() <= 1e-12 * np.abs(Vd).max()


def test_fourier_form_equals_real_space():
    rng = np.random.default_rng(3)
    dims = (6, 5, 4)
    nx, ny, nz = dims
    F = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    F2 = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    ghat = C.kernel_spectrum(rng.random((nz + 1, ny + 1, nx + 1)), dims)
    a = C.calculate(C.prepare(F, ghat), F2)
    b = C.fourier_integral(F, F2, ghat)
    assert abs(a - b) <= 1e-12 * abs(a)


def test_round_known_answers():
    """run-tests.cpp:295-323."""
    assert [H.round_up(n, (2,), 1) for n in (0, 13, 16, 17, 34, 101)] == [1, 16, 16, 32, 64, 128]
    assert [H.round_up(n) for n in (0, 13, 16, 17, 34, 101)] == [1, 15, 16, 18, 36, 108]
    assert [H.round_up(n, c=4) for n in (0, 13, 16, 17, 34, 101)] == [4, 16, 16, 20, 36, 108]


def test_graph_known_answers():
    """run-tests.cpp:230-281."""
    assert len(H.vertex_cover(4, [(i, j) for j in range(4) for i in range(j)])) == 3
    assert H.vertex_cover(3, []) == set()
    assert H.vertex_cover(3, [(0, 0), (1, 1), (2, 2)]) == {0, 1, 2}
    assert H.vertex_cover(3, [(0, 1), (1, 2)]) == {1}
    assert H.vertex_cover(3, [(0, 0), (0, 1), (1, 1), (1, 2), (2, 0)]) == {0, 1}


def test_example_golden():
    """example/run.sh:3-9: J_ee of the Si:P donor = 0.090340071977 eV (first 29 chars)."""
    import make_example_fixture as fx
    d = fx.load()
    g = H.detect_grid(d["pos"])
    assert g["raw"] == (41, 41, 41) and g["pad"] == (45, 45, 45)
    specs = H.enumerate_integrals(H.Pattern("****", 0), 1)
    vals = H.compute_integrals([d["coeff"]], g["cells"], g["pad"], g["step"], specs, dielectric=11.4)
    text = H.format_outputs(specs, vals, 0, 1)["eeee"]
    assert text[:29] == d["golden"]


def test_thomas_fermi_kernel_limits():
    """eps(r) -> dielectric beyond r_TF and -> 1 at r -> 0 (Interaction.cpp:34-39)."""
    r_tf, q_tf = H.C.thomas_fermi_params(10.89, 5.65) if hasattr(H, "C") else C.thomas_fermi_params(10.89, 5.65)
    eps0 = 10.89 * (q_tf * r_tf / (np.sinh(q_tf * r_tf)))
    assert abs(eps0 - 1.0) < 1e-9
