"""Seeded synthetic zinc-blende structures and LCAO states.

The workloads are synthetic crystal boxes in the reference's own input formats:
  * positions: zinc-blende, lattice constant a = 5.65 A, cation fcc sites
    (0,0,0), (0,1/2,1/2), (1/2,0,1/2), (1/2,1/2,0) and anions at +(1/4,1/4,1/4), on
    Lx x Ly x Lz conventional cells.  Every coordinate is an integer multiple of a/4,
    so the reference's float-GCD grid detection (Broadcaster.cpp:8-43) finds the a/4
    step exactly and the raw grid is 4L per axis with A = M/8 atoms.  Atoms are listed
    sorted by z, then y, then x.
  * states: c[s][atom][orb] = envelope_s(r_atom) * z, z complex normal (or a unit phase)
    from numpy.random.default_rng(1000*config + s), normalised to sum |c|^2 = 1.

The five named workloads:
  c1  8^3 cells (32^3 grid, 4096 atoms), 10 orbitals, 2 e + 2 h, Gaussian sigma = 2 nm.
  c2  24^3 cells (96^3 grid, 110,592 atoms), 20 orbitals, 6 e + 6 h, s/p/d-like envelopes
      inside a lens dot (radius 8 nm, height 3 nm, 1-cell wetting layer) with a random
      phase per orbital.
  c3  64^3 cells (256^3 grid, 2,097,152 atoms), 20 orbitals, 4 e + 4 h, Gaussian x
      hydrogen-like (1s/2p) envelopes, sigma 3-6 nm.
  c4  32^3 cells (128^3 grid, 262,144 atoms), 20 orbitals, 20 e + 20 h, Hermite-Gaussian
      family inside a lens dot, all-pairs integral list.
  c5  16 independent boxes from 48^3 to 96x128x160 grids, 20 orbitals, 4 e + 4 h each.
"""
from __future__ import annotations

import numpy as np

A_ZB = 5.65  # Angstrom

# (cells per axis, orbitals, electrons, holes, integrals)
CONFIGS = {
    "c1": dict(cells=(8, 8, 8), orbitals=10, electrons=2, holes=2, integrals="eeee,hhhh,ehhe,eheh"),
    "c2": dict(cells=(24, 24, 24), orbitals=20, electrons=6, holes=6, integrals="eeee,hhhh,ehhe,eheh"),
    "c3": dict(cells=(64, 64, 64), orbitals=20, electrons=4, holes=4, integrals="eeee,hhhh,ehhe,eheh"),
    "c4": dict(cells=(32, 32, 32), orbitals=20, electrons=20, holes=20, integrals="ijkl"),
}

# c5: sixteen boxes whose grids 4L are 2*3*5-smooth (48^3 ... 96x128x160)
C5_CELLS = [
    (12, 12, 12), (15, 15, 15), (16, 16, 16), (18, 18, 18), (20, 20, 20), (16, 16, 24),
    (24, 24, 24), (25, 25, 25), (27, 27, 27), (30, 30, 30), (20, 24, 30), (32, 32, 32),
    (24, 32, 36), (36, 36, 36), (30, 36, 40), (24, 32, 40),
]


def zincblende_lattice(cells):
    """Integer lattice indices (in units of a/4) of a zinc-blende box, sorted z, y, x.

    Returns int64 [A, 3] (x, y, z)."""
    lx, ly, lz = cells
    basis = np.array([(0, 0, 0), (0, 2, 2), (2, 0, 2), (2, 2, 0),
                      (1, 1, 1), (1, 3, 3), (3, 1, 3), (3, 3, 1)], dtype=np.int64)
    cx, cy, cz = np.meshgrid(np.arange(lx), np.arange(ly), np.arange(lz), indexing="ij")
    corner = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1) * 4
    idx = (corner[:, None, :] + basis[None, :, :]).reshape(-1, 3)
    order = np.lexsort((idx[:, 0], idx[:, 1], idx[:, 2]))
    return idx[order]


def positions_angstrom(lattice_idx):
    return lattice_idx.astype(np.float64) * (A_ZB / 4.0)


def grid_of(cells):
    return tuple(4 * c for c in cells)


def cell_indices(lattice_idx, dims):
    nx, ny, _ = dims
    return (lattice_idx[:, 2] * ny + lattice_idx[:, 1]) * nx + lattice_idx[:, 0]


def _envelopes(kind, pos, centre, n_states, rng_for):
    """Real envelope per state; pos [A,3] in Angstrom."""
    d = pos - centre[None, :]
    r2 = np.sum(d * d, axis=1)
    envs = []
    for s in range(n_states):
        if kind == "gauss":
            sigma = 20.0
            envs.append(np.exp(-r2 / (2 * sigma * sigma)))
        elif kind == "lens":
            # s, px, py, pz, dxy, dx2-y2 ... inside a lens of radius 80 A, height 30 A
            sx, sz = 45.0, 18.0
            g = np.exp(-(d[:, 0] ** 2 + d[:, 1] ** 2) / (2 * sx * sx) - d[:, 2] ** 2 / (2 * sz * sz))
            shapes = [np.ones_like(r2), d[:, 0], d[:, 1], d[:, 0] * d[:, 1],
                      d[:, 0] ** 2 - d[:, 1] ** 2, d[:, 2]]
            envs.append(g * shapes[s % len(shapes)] * (1.0 + 0.1 * (s // len(shapes))))
        elif kind == "hydrogen":
            sigma = 30.0 + 30.0 * (s % 4) / 3.0
            g = np.exp(-r2 / (2 * sigma * sigma))
            shapes = [np.ones_like(r2), d[:, 0], d[:, 1], d[:, 2]]
            envs.append(g * shapes[s % 4] * np.exp(-np.sqrt(r2) / (2 * sigma)))
        elif kind == "hermite":
            sx, sz = 40.0, 16.0
            g = np.exp(-(d[:, 0] ** 2 + d[:, 1] ** 2) / (2 * sx * sx) - d[:, 2] ** 2 / (2 * sz * sz))
            nx_, ny_, nz_ = s % 4, (s // 4) % 3, (s // 12) % 2
            hx = np.polynomial.hermite.hermval(d[:, 0] / sx, [0] * nx_ + [1])
            hy = np.polynomial.hermite.hermval(d[:, 1] / sx, [0] * ny_ + [1])
            hz = np.polynomial.hermite.hermval(d[:, 2] / sz, [0] * nz_ + [1])
            envs.append(g * hx * hy * hz)
        else:
            raise ValueError(kind)
    return envs


def make_states(pos, n_orb, n_states, seed_base, kind, unit_phase=False):
    """Seeded complex LCAO states [n_states][A][n_orb] (complex128), each normalised."""
    centre = 0.5 * (pos.min(axis=0) + pos.max(axis=0))
    envs = _envelopes(kind, pos, centre, n_states, None)
    out = np.empty((n_states, pos.shape[0], n_orb), dtype=np.complex128)
    for s in range(n_states):
        rng = np.random.default_rng(seed_base + s)
        if unit_phase:
            z = np.exp(1j * rng.uniform(0, 2 * np.pi, size=(pos.shape[0], n_orb)))
        else:
            z = rng.standard_normal((pos.shape[0], n_orb)) + 1j * rng.standard_normal((pos.shape[0], n_orb))
        c = envs[s][:, None] * z
        c /= np.sqrt(np.sum(np.abs(c) ** 2))
        out[s] = c
    return out


def build(config, cells=None, seed_index=None):
    """Returns dict(lattice, pos, dims, cells_idx, states, holes, electrons, orbitals,
    integrals).  States are listed holes first, as the reference requires."""
    if config == "c5":
        raise ValueError("c5 is a list; use build_c5")
    cfg = dict(CONFIGS[config])
    if cells is not None:
        cfg["cells"] = cells
    lat = zincblende_lattice(cfg["cells"])
    pos = positions_angstrom(lat)
    dims = grid_of(cfg["cells"])
    n = cfg["electrons"] + cfg["holes"]
    num = int(config[1:]) if seed_index is None else seed_index
    kind = {"c1": "gauss", "c2": "lens", "c3": "hydrogen", "c4": "hermite"}[config]
    states = make_states(pos, cfg["orbitals"], n, 1000 * num, kind, unit_phase=(config == "c2"))
    return dict(lattice=lat, pos=pos, dims=dims, cells_idx=cell_indices(lat, dims), states=states,
                holes=cfg["holes"], electrons=cfg["electrons"], orbitals=cfg["orbitals"],
                integrals=cfg["integrals"])


def build_c5(index, orbitals=20):
    cells = C5_CELLS[index]
    lat = zincblende_lattice(cells)
    pos = positions_angstrom(lat)
    dims = grid_of(cells)
    states = make_states(pos, orbitals, 8, 1000 * 5 + 100 * index, "gauss")
    return dict(lattice=lat, pos=pos, dims=dims, cells_idx=cell_indices(lat, dims), states=states,
                holes=4, electrons=4, orbitals=orbitals, integrals="eeee,hhhh,ehhe,eheh")


def write_inputs(directory, data, header=True):
    """Writes X.3d and h*/e* files in the reference's text formats (one header line)."""
    import os
    os.makedirs(directory, exist_ok=True)
    np.savetxt(os.path.join(directory, "X.3d"), data["pos"], fmt="%.10f")
    names = []
    for s in range(data["states"].shape[0]):
        name = ("h%d.dat" % (s + 1)) if s < data["holes"] else ("e%d.dat" % (s + 1 - data["holes"]))
        c = data["states"][s].reshape(-1)
        arr = np.stack([c.real, c.imag], axis=1)
        np.savetxt(os.path.join(directory, name), arr, fmt="%.17g", header="synthetic state" if header else "",
                   comments="")
        names.append(name)
    return names
