"""CPU oracle for the Coulomb-integral hot path (TEST INFRASTRUCTURE ONLY).

This module is the FP64 restatement of Coulombo-Lattice's numerics, written with NumPy and
SciPy's pocketfft.  It exists to check the CUDA library: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it.  The product path (``libcoulombo_lattice.so`` and the
``coulombo`` / ``potentials`` binaries) never calls into it.

Parity pins (checked by ``tests/test_oracle_golden.py``):
  * run-tests.cpp:28-48   two point charges on a 5x5x10 grid -> 1 and exp(-5) to 1e-12
  * run-tests.cpp:189-214 FFT sign/scale/phase convention (single bin of magnitude 512)
  * example/run.sh:3-9    Si:P donor J_ee = 0.090340071977 eV (12 decimals, truncated)
plus an O(M^2) direct aperiodic convolution on tiny grids that pins the 8-round
no-padding decomposition independently of any FFT library.

FFTW is the reference's third-party FFT (unpinned "version 3", Makefile:3).  Its
published conventions are restated here: c2c forward = exp(-2 pi i jk/n), backward =
exp(+2 pi i jk/n), both unnormalised; REDFT00 of length n is
Y_k = X_0 + (-1)^k X_{n-1} + 2 sum_{j=1}^{n-2} X_j cos(pi jk/(n-1)), which is
scipy.fft.dct(type=1, norm=None).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.fft as sfft

# e^2 / (4 pi eps0) in eV*Angstrom -- base.hpp:28
E2_4PE0 = 14.39963737103201


# --------------------------------------------------------------------------------------
# Coulomb kernel on the (N+1)^3 octant -- Interaction.hpp:32-51, Interaction.cpp:8-39
# --------------------------------------------------------------------------------------

def thomas_fermi_params(dielectric: float, lattice_constant: float):
    """Newton solve of sinh(x) = eps*x for the Thomas-Fermi-Resta radius.

    Follows Interaction.cpp:18-32 step for step (same start, same stopping rule)."""
    eps = 1.0e-12
    q_tf = 2.0 / math.sqrt(math.pi) * (96.0 * math.pi * math.pi) ** (1.0 / 3.0) / lattice_constant
    x = math.sqrt(6.0 * (dielectric - 1.0))
    while True:
        f = math.sinh(x) - dielectric * x
        df = math.cosh(x) - dielectric
        dx = 0.0 if abs(f) < eps else f / df
        x -= dx
        if not (dx / q_tf > eps):
            break
    return x / q_tf, q_tf


def kernel_octant(dims, step, dielectric=1.0, onsite=0.0, tf_lattice=None):
    """G(ix,iy,iz) = E2_4PE0 / (eps(r) r) on an (Nx+1)x(Ny+1)x(Nz+1) grid, G(0)=onsite.

    Returned as a C-order array indexed [iz, iy, ix] (x fastest in memory), matching the
    reference's column-major x-fastest Domain (run-tests.cpp:169-175)."""
    nx, ny, nz = dims
    ix = np.arange(nx + 1) * step[0]
    iy = np.arange(ny + 1) * step[1]
    iz = np.arange(nz + 1) * step[2]
    z2 = (iz * iz)[:, None, None]
    y2 = (iy * iy)[None, :, None]
    x2 = (ix * ix)[None, None, :]
    r = np.sqrt((z2 + y2) + x2)  # same association as Interaction.hpp:37-41
    with np.errstate(divide="ignore", invalid="ignore"):
        if tf_lattice is None:
            g = E2_4PE0 / (dielectric * r)
        else:
            r_tf, q_tf = thomas_fermi_params(dielectric, tf_lattice)
            eps_r = np.where(
                r < r_tf,
                dielectric * (q_tf * r_tf / (np.sinh(q_tf * (r_tf - r)) + q_tf * r)),
                dielectric,
            )
            g = E2_4PE0 / (eps_r * r)
    g[0, 0, 0] = onsite
    return g


def kernel_spectrum(g_octant, dims):
    """Ghat = REDFT00 (3D DCT-I) of the octant, divided by 8*M -- CoulombCalculator.cpp:57-103.

    The DCT-I of the (N+1)-point octant is the 2N-point DFT of its even extension."""
    nx, ny, nz = dims
    ghat = sfft.dctn(g_octant, type=1, norm=None, workers=-1)
    return ghat / (8.0 * nx * ny * nz)


# --------------------------------------------------------------------------------------
# 8-round zero-padding-free convolution -- CoulombCalculator.cpp:45-54, 105-172
# --------------------------------------------------------------------------------------

def phase_factors(n):
    """phi(i) = exp(i pi i / n) -- CoulombCalculator.cpp:45-54."""
    return np.exp(1j * np.pi * np.arange(n) / n)


def round_phase(dims, round_index):
    """phi_kappa(x,y,z) as a broadcastable [z,y,x] array; bit 0 = x, 1 = y, 2 = z
    (CoulombCalculator.cpp:108-111)."""
    nx, ny, nz = dims
    kx, ky, kz = round_index & 1, (round_index >> 1) & 1, (round_index >> 2) & 1
    px = phase_factors(nx) if kx else np.ones(nx)
    py = phase_factors(ny) if ky else np.ones(ny)
    pz = phase_factors(nz) if kz else np.ones(nz)
    return pz[:, None, None] * py[None, :, None] * px[None, None, :]


def folded_kernel(ghat, dims, round_index):
    """Khat_kappa(k) = Ghat(f(2kx+kx0), f(2ky+ky0), f(2kz+kz0)), f(q) = min(q, 2N-q)
    -- CoulombCalculator.cpp:130-144 (with its y/z transposition undone)."""
    nx, ny, nz = dims
    kx, ky, kz = round_index & 1, (round_index >> 1) & 1, (round_index >> 2) & 1

    def fold(n, kappa):
        q = 2 * np.arange(n) + kappa
        return np.minimum(q, 2 * n - q)

    fx, fy, fz = fold(nx, kx), fold(ny, ky), fold(nz, kz)
    return ghat[np.ix_(fz, fy, fx)]


def prepare(F, ghat, rounds=range(8)):
    """V = aperiodic (G * F) on the N^3 grid by 8 phase-shifted rounds of N-point FFTs
    -- CoulombCalculator.cpp:105-163.  F is a complex [z,y,x] array.  `rounds` restricts the
    sum to some rounds kappa (the partial potentials of a multi-GPU split add up)."""
    nz, ny, nx = F.shape
    dims = (nx, ny, nz)
    V = np.zeros_like(F, dtype=np.complex128)
    for rnd in rounds:
        ph = round_phase(dims, rnd)
        T = F * np.conj(ph)
        T = sfft.fftn(T, workers=-1)
        T *= folded_kernel(ghat, dims, rnd)
        T = sfft.ifftn(T, norm="forward", workers=-1)  # unnormalised backward (FFTW_BACKWARD)
        V += T * ph
    return V


def calculate(V, F):
    """sum_r V(r) F(r), no conjugation -- CoulombCalculator.cpp:165-172."""
    return complex(np.sum(V * F))


def direct_convolution(F, g_octant):
    """O(M^2) aperiodic convolution V(r) = sum_r' G(|r-r'|) F(r') (tiny grids only).

    This is the mathematical definition the 8-round method reproduces; it pins that
    method without any FFT."""
    nz, ny, nx = F.shape
    V = np.zeros_like(F, dtype=np.complex128)
    src = np.argwhere(F != 0)
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    for (sz, sy, sx) in src:
        V += F[sz, sy, sx] * g_octant[np.abs(zz - sz), np.abs(yy - sy), np.abs(xx - sx)]
    return V


# --------------------------------------------------------------------------------------
# Pair densities -- Product.cpp:16-30
# --------------------------------------------------------------------------------------

def pair_density_atoms(c_left, c_right, conjugate=False):
    """Per-atom orbital sum: conj(L).R (or L.conj(R) if conjugate).  c_*: [atom, orb]."""
    if conjugate:
        return np.sum(c_left * np.conj(c_right), axis=1)
    return np.sum(np.conj(c_left) * c_right, axis=1)


def scatter_density(values, cells, dims):
    """F.zeros(); F[cell(a)] = value(a) -- Product.cpp:16-30.  Returns a [z,y,x] array."""
    nx, ny, nz = dims
    F = np.zeros(nx * ny * nz, dtype=np.complex128)
    F[cells] = values
    return F.reshape(nz, ny, nx)


# --------------------------------------------------------------------------------------
# Fourier-space form (equivalent by Parseval on the virtual 2N grid)
# --------------------------------------------------------------------------------------

def round_spectrum(F, rnd):
    nz, ny, nx = F.shape
    return sfft.fftn(F * np.conj(round_phase((nx, ny, nz), rnd)), workers=-1)


def reversed_index(spec, rnd):
    """A(k') where 2k'+kappa = -(2k+kappa) mod 2N, per axis: k' = (-k) mod N for kappa=0,
    N-1-k for kappa=1.  Used with A_ba(k) = conj(A_ab(k'))."""
    out = spec
    for axis, bit in ((2, 0), (1, 1), (0, 2)):
        n = spec.shape[axis]
        if (rnd >> bit) & 1:
            idx = n - 1 - np.arange(n)
        else:
            idx = (-np.arange(n)) % n
        out = np.take(out, idx, axis=axis)
    return out


def fourier_integral(F_left, F_right, ghat):
    """sum_r V_left(r) F_right(r) evaluated in Fourier space:
    sum_kappa sum_k Khat_kappa(k) A_L(k) conj(FFT(conj(F_R) conj(phi_kappa))(k))."""
    nz, ny, nx = F_left.shape
    dims = (nx, ny, nz)
    total = 0.0 + 0.0j
    for rnd in range(8):
        a = round_spectrum(F_left, rnd)
        b = round_spectrum(np.conj(F_right), rnd)
        total += np.sum(folded_kernel(ghat, dims, rnd) * a * np.conj(b))
    return complex(total)
