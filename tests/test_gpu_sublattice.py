"""The sub-lattice forms (CL_MODE_FP64_SUBLATTICE, CL_MODE_FP32_SUBLATTICE) against the oracle.

The decomposition is exact, so the FP64 sub-lattice form must meet the plain path's 1e-10 gate
and the FP32 one the FP32 gate, on: zinc-blende boxes of several shapes (the compiled mixing
table), a box whose grid origin falls on another class (the table shifted), a partial class set
and an fcc lattice on an a/2 grid (the generic table, m = 4 and m = 2), and atoms that occupy too
many classes (the 8-round fallback).  Also: the request, batch, overlapped-upload and
potentials paths, and the refusal of round splits.
"""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import coulomb as C
from oracle import host as H

pytestmark = pytest.mark.gpu

SL_MODES = [cl.MODE_FP64_SUBLATTICE, cl.MODE_FP32_SUBLATTICE]
EPS = 10.89


def gate(got, want, mode):
    err = np.abs(np.asarray(got) - np.asarray(want))
    if cl.mode_is_fp64(mode):
        lim = 1e-10 * np.abs(want) + 1e-16
    else:
        lim = np.maximum(1e-6 * np.abs(want), 1e-9)
    return err, lim


def _structure(lat, dims, n_states=4, n_orb=4, seed=11):
    rng = np.random.default_rng(seed)
    a = lat.shape[0]
    st = rng.standard_normal((n_states, a, n_orb)) + 1j * rng.standard_normal((n_states, a, n_orb))
    st /= np.sqrt(np.sum(np.abs(st) ** 2, axis=(1, 2), keepdims=True))
    cells = (lat[:, 2] * dims[1] + lat[:, 1]) * dims[0] + lat[:, 0]
    return st, cells


def _compare(st, cells, dims, step, mode, n_holes=2, pattern="****"):
    n = st.shape[0]
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals(pattern, n, n_holes)]
    want = np.array(H.compute_integrals(list(st), cells, dims, step, specs, dielectric=EPS))
    with cl.CoulombCalculator(dims, step, mode) as cc:
        cc.initialize(dielectric=EPS)
        cc.set_states(st, cells, n_holes)
        info = cc.form_info()
        got = cc.compute(specs)
    err, lim = gate(got, want, mode)
    assert np.all(err <= lim), "worst error/gate %.3g" % (err / lim).max()
    return info


@pytest.mark.parametrize("mode", SL_MODES)
@pytest.mark.parametrize("cells", [(2, 2, 2), (3, 2, 4), (5, 6, 4), (4, 4, 4)])
def test_zincblende_boxes(mode, cells):
    lat = synth.zincblende_lattice(cells)
    dims = synth.grid_of(cells)
    st, cc_ = _structure(lat, dims)
    info = _compare(st, cc_, dims, (synth.A_ZB / 4,) * 3, mode)
    assert info["sublattice"] and info["m"] == 4 and info["classes"] == 8 and info["zincblende"]
    assert info["lengths"] == tuple(d // 2 for d in dims)


@pytest.mark.parametrize("mode", SL_MODES)
def test_c1_default_classes(mode):
    d = synth.build("c1")
    info = _compare(d["states"], d["cells_idx"], d["dims"], (synth.A_ZB / 4,) * 3, mode, n_holes=d["holes"],
                    pattern="eeee,hhhh,ehhe,eheh")
    assert info["zincblende"]


@pytest.mark.parametrize("mode", SL_MODES)
def test_shifted_origin_uses_the_compiled_table(mode):
    """Dropping the first x layer of a zinc-blende box moves the grid origin onto another class."""
    cells = (3, 3, 2)
    lat = synth.zincblende_lattice(cells)
    lat = lat[lat[:, 0] >= 1] - np.array([1, 0, 0])
    dims = synth.grid_of(cells)
    st, cc_ = _structure(lat, dims, seed=3)
    info = _compare(st, cc_, dims, (synth.A_ZB / 4,) * 3, mode)
    assert info["sublattice"] and info["zincblende"]


@pytest.mark.parametrize("mode", SL_MODES)
def test_partial_class_set_generic_table(mode):
    cells = (3, 2, 3)
    lat = synth.zincblende_lattice(cells)
    keep = np.isin((lat[:, 0] % 4) + 4 * (lat[:, 1] % 4) + 16 * (lat[:, 2] % 4), [0, 10, 21, 40, 61])
    lat = lat[keep]
    dims = synth.grid_of(cells)
    st, cc_ = _structure(lat, dims, seed=5)
    info = _compare(st, cc_, dims, (synth.A_ZB / 4,) * 3, mode)
    assert info["sublattice"] and not info["zincblende"] and info["classes"] == 5


@pytest.mark.parametrize("mode", SL_MODES)
def test_fcc_on_half_cell_grid_m2(mode):
    L = (4, 3, 4)
    base = np.array([(0, 0, 0), (0, 1, 1), (1, 0, 1), (1, 1, 0)])
    g = np.stack(np.meshgrid(*[np.arange(v) for v in L], indexing="ij"), -1).reshape(-1, 3) * 2
    lat = (g[:, None, :] + base[None]).reshape(-1, 3)
    lat = lat[np.lexsort((lat[:, 0], lat[:, 1], lat[:, 2]))]
    dims = tuple(2 * v for v in L)
    st, cc_ = _structure(lat, dims, seed=9)
    info = _compare(st, cc_, dims, (2.0, 2.0, 2.0), mode)
    assert info["sublattice"] and info["m"] == 2 and info["classes"] == 4


@pytest.mark.parametrize("mode", SL_MODES)
def test_too_many_classes_fall_back_to_rounds(mode):
    rng = np.random.default_rng(21)
    dims = (12, 8, 10)
    lat = np.unique(np.stack([rng.integers(0, n, 300) for n in dims], 1), axis=0)
    st, cc_ = _structure(lat, dims, seed=2)
    info = _compare(st, cc_, dims, (1.3, 1.1, 1.7), mode)
    assert not info["sublattice"]


@pytest.mark.parametrize("mode", SL_MODES)
def test_medium_box_matches_rounds_and_oracle(mode):
    d = synth.build("c3", cells=(16, 16, 16))
    d["states"] = d["states"][:, :, :6]
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals(d["integrals"], 8, 4)]
    step = (synth.A_ZB / 4,) * 3
    want, covered = H.compute_integrals_sampled(list(d["states"]), d["cells_idx"], d["dims"], step, specs,
                                                dielectric=EPS)
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=EPS)
        cc.set_states(d["states"], d["cells_idx"], 4)
        got = cc.compute(specs)
        assert cc.form_info()["zincblende"]
    err, lim = gate(got, want, mode)
    assert np.all(err <= lim), (err / lim).max()


@pytest.mark.parametrize("mode", SL_MODES)
def test_requests_batches_states_and_potentials(mode):
    step = (synth.A_ZB / 4,) * 3
    ds = [synth.build("c1", cells=c) for c in [(4, 4, 4), (3, 4, 5)]]
    calcs, reqs, wants = [], [], []
    for d in ds:
        n = d["states"].shape[0]
        specs = np.ascontiguousarray(cl.enumerate_integrals("****", n, d["holes"]))
        wants.append(np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], step,
                                                  [tuple(int(v) for v in s) for s in specs], dielectric=EPS)))
        cc = cl.CoulombCalculator(d["dims"], step, mode)
        cc.initialize(dielectric=EPS)
        cc.set_states(d["states"], d["cells_idx"], d["holes"])
        calcs.append(cc)
        reqs.append(cc.request(specs))
        # the overlapped-upload call on the same context
        got = cc.compute_states(d["states"], d["cells_idx"], d["holes"], specs)
        err, lim = gate(got, wants[-1], mode)
        assert np.all(err <= lim)
    batch = cl.Batch(reqs)
    try:
        batch.run()
        outs = batch.run()
    finally:
        batch.close()
    for got, want in zip(outs, wants):
        err, lim = gate(got, want, mode)
        assert np.all(err <= lim)
    # potentials of every state's own density at every atom (potentials.cpp:137-158)
    d, cc = ds[0], calcs[0]
    pot = cc.potentials()
    ghat = C.kernel_spectrum(C.kernel_octant(d["dims"], step, EPS), d["dims"])
    for s in range(d["states"].shape[0]):
        rho = C.pair_density_atoms(d["states"][s], d["states"][s])
        V = C.prepare(C.scatter_density(rho, d["cells_idx"], d["dims"]), ghat).reshape(-1)[d["cells_idx"]].real
        tol = 1e-10 if cl.mode_is_fp64(mode) else 1e-6
        assert np.abs(pot[s] - V).max() <= tol * np.abs(V).max()
    for r in reqs:
        r.close()
    for cc in calcs:
        cc.close()


def test_round_split_is_refused():
    d = synth.build("c1", cells=(4, 4, 4))
    with cl.CoulombCalculator(d["dims"], (synth.A_ZB / 4,) * 3, cl.MODE_FP32_SUBLATTICE) as cc:
        cc.initialize(dielectric=EPS)
        cc.set_states(d["states"], d["cells_idx"], d["holes"])
        specs = cl.enumerate_integrals("****", 4, 2)
        with pytest.raises(cl.CoulomboError, match="no rounds to split"):
            cc.compute_rounds(specs, 0x0F)
        full = cc.compute_rounds(specs, 0xFF)
        assert np.allclose(full, cc.compute(specs), rtol=1e-12, atol=0)


@pytest.mark.parametrize("drop", [0.0, 0.1])
def test_quadrant_plane_passes(drop, monkeypatch):
    """128 x 128 class planes (a 64 x 64 x 2-cell box): the FP32 quadrant forward plane pass
    against the general one (CL_NO_QPLANE=1) and the oracle; with every quadrant point an atom,
    and with a tenth of the atoms removed (planes that must be cleared between densities)."""
    cells = (64, 64, 2)
    lat = synth.zincblende_lattice(cells)
    if drop:
        rng = np.random.default_rng(77)
        lat = lat[rng.random(lat.shape[0]) >= drop]
    dims = synth.grid_of(cells)
    st, cc_ = _structure(lat, dims, n_states=4, n_orb=2, seed=13)
    step = (synth.A_ZB / 4,) * 3
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]

    def run(no_q):
        if no_q:
            monkeypatch.setenv("CL_NO_QPLANE", "1")
        try:
            with cl.CoulombCalculator(dims, step, cl.MODE_FP32_SUBLATTICE) as cc:
                cc.initialize(dielectric=EPS)
                cc.set_states(st, cc_, 2)
                info = cc.form_info()
                return np.asarray(cc.compute(specs)), info
        finally:
            monkeypatch.delenv("CL_NO_QPLANE", raising=False)

    got, info = run(False)
    assert info["sublattice"] and info["lengths"][:2] == (128, 128)
    ref, _ = run(True)
    want = np.array(H.compute_integrals(list(st), cc_, dims, step, specs, dielectric=EPS))
    err, lim = gate(got, want, cl.MODE_FP32_SUBLATTICE)
    assert np.all(err <= lim), (err / lim).max()
    assert np.all(np.abs(got - ref) <= 0.25 * lim)
