"""The hand-written FFT engine against NumPy and the reference's FFT known answer."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl

pytestmark = pytest.mark.gpu

SIZES = [(5, 5, 10), (1, 1, 2), (2, 3, 5), (32, 32, 32), (45, 45, 45), (16, 24, 40), (64, 64, 96),
         (96, 8, 6), (8, 256, 4), (4, 4, 256), (160, 6, 5), (27, 25, 9), (1024, 1, 1), (3, 1, 1)]


@pytest.mark.parametrize("dims", SIZES)
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft_fp64_matches_numpy(dims, sign):
    nx, ny, nz = dims
    rng = np.random.default_rng(nx * 100 + ny * 10 + nz)
    x = rng.normal(size=(2, nz, ny, nx)) + 1j * rng.normal(size=(2, nz, ny, nx))
    got = cl.fft3d(x, sign=sign)
    want = np.fft.fftn(x, axes=(1, 2, 3)) if sign < 0 else np.fft.ifftn(x, axes=(1, 2, 3), norm="forward")
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("dims", [(32, 32, 32), (45, 45, 45), (96, 96, 96), (256, 16, 8)])
def test_fft_fp32_matches_numpy(dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(1)
    x = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    got = cl.fft3d(x, sign=-1, fp32=True)
    want = np.fft.fftn(x)
    rms = np.sqrt(np.mean(np.abs(got - want) ** 2) / np.mean(np.abs(want) ** 2))
    assert rms < 3e-7


def test_fft_single_bin_known_answer():
    """run-tests.cpp:189-214 (FFTW r2c of 1024 points; here the c2c transform of the same
    real signal): one bin of magnitude 512 and phase pi/4, every other bin zero, to 1e-12."""
    n = np.arange(1024)
    x = np.cos(2 * np.pi * 16 * n / 1024 + np.pi / 4).reshape(1, 1, 1024)
    X = cl.fft3d(x, sign=-1).ravel()[:513]
    mask = np.ones(513, bool)
    mask[16] = False
    assert np.abs(X[mask]).max() < 1e-12
    assert abs(abs(X[16]) - 512) < 1e-12
    assert abs(np.angle(X[16]) - np.pi / 4) < 1e-12
