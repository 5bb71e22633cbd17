"""Pair densities over more than 8 states (Product::map, Product.cpp:16-30): the register kernel
with 8 product parts (9 to 12 states) and the 4 x 4-state tile kernel (more than 12 states, or
from 9 with CL_NO_PAIR_REG12=1) against the segment kernel (CL_NO_PAIR_TILE=1 with
CL_NO_PAIR_REG12=1) and the FP64 oracle, in every form; dense and sparse product sets (tiles
without a requested product are skipped), state counts that are not multiples of 4 (zero
padding states), and atom counts that are not multiples of the atoms a block stages."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import host as H

pytestmark = pytest.mark.gpu

EPS = 10.89
STEP = (synth.A_ZB / 4,) * 3


def _lim(want, mode):
    if cl.mode_is_fp64(mode):
        return 1e-10 * np.abs(want) + 1e-16
    return np.maximum(1e-6 * np.abs(want), 1e-9)


def _compute(d, specs, holes, mode, monkeypatch, segment, tile=False):
    env = {}
    if segment:
        env = {"CL_NO_PAIR_TILE": "1", "CL_NO_PAIR_REG12": "1"}
    elif tile:
        env = {"CL_NO_PAIR_REG12": "1"}
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    try:
        with cl.CoulombCalculator(d["dims"], STEP, mode) as cc:
            cc.initialize(dielectric=EPS)
            cc.set_states(d["states"], d["cells_idx"], holes)
            return np.asarray(cc.compute(specs))
    finally:
        for k in env:
            monkeypatch.delenv(k, raising=False)


@pytest.mark.parametrize("mode", cl.ALL_MODES)
@pytest.mark.parametrize("n_states,pattern,n_orb,cells,tile",
                         [(12, "****", 6, (3, 4, 5), False), (12, "****", 6, (3, 4, 5), True),
                          (10, "eeee,hhhh,ehhe,eheh", 20, (2, 3, 3), False),
                          (10, "eeee,hhhh,ehhe,eheh", 20, (2, 3, 3), True), (9, "ehhe", 5, (2, 2, 3), False),
                          (22, "eheh", 4, (3, 3, 2), False)])
def test_pair_kernels_match_segment_kernel_and_oracle(mode, n_states, pattern, n_orb, cells, tile, monkeypatch):
    d = synth.build("c2", cells=cells)
    d["states"] = synth.make_states(d["pos"], n_orb, n_states, 7000 + n_states, "gauss")
    holes = n_states // 2
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals(pattern, n_states, holes)]
    if len(specs) > 1500:
        specs = specs[::len(specs) // 1500 + 1]
    got = _compute(d, specs, holes, mode, monkeypatch, segment=False, tile=tile)
    seg = _compute(d, specs, holes, mode, monkeypatch, segment=True)
    want = np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], STEP, specs,
                                        dielectric=EPS))
    lim = _lim(want, mode)
    assert np.all(np.abs(got - want) <= lim), (np.abs(got - want) / lim).max()
    if cl.mode_is_fp64(mode):
        # the same FP64 sums in another order
        assert np.abs(got - seg).max() <= 1e-12 * np.abs(seg).max()
    else:
        # FP64 sums rounded once to FP32 in both kernels
        assert np.all(np.abs(got - seg) <= 0.25 * lim)


def test_forty_states_twenty_orbitals(monkeypatch):
    """40 states x 20 orbitals (the all-pairs workload's state count): 55 tiles, 8 atoms a block."""
    d = synth.build("c2", cells=(2, 2, 3))
    d["states"] = synth.make_states(d["pos"], 20, 40, 9100, "gauss")
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 40, 20)][::4099]
    for mode in (cl.MODE_FP64_PLAIN, cl.MODE_FP32_SUBLATTICE):
        got = _compute(d, specs, 20, mode, monkeypatch, segment=False)
        seg = _compute(d, specs, 20, mode, monkeypatch, segment=True)
        want = np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], STEP, specs,
                                            dielectric=EPS))
        lim = _lim(want, mode)
        assert np.all(np.abs(got - want) <= lim), (np.abs(got - want) / lim).max()
        assert np.all(np.abs(got - seg) <= 0.25 * lim)
