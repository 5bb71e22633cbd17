"""The split-precision tensor-core Gram of the FP32 forms (TF32 hi/lo operands, tcgen05 MMAs,
FP64 accumulation across 32-atom k-tiles) against the FP64 Gram on the same potentials and
against the oracle; and the fused Gram of the FP32 sub-lattice form (split inside the kernel)
against the separate split pass."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import host as H

pytestmark = pytest.mark.gpu

STEP = (synth.A_ZB / 4,) * 3


@pytest.fixture(autouse=True)
def _tf32_gram_at_any_size(monkeypatch):
    """The FP32 forms sum the reductions of boxes under 65,536 atoms in FP64; these small test
    boxes take the TF32x3 Gram unless a test removes this."""
    monkeypatch.setenv("CL_TC_MIN_ATOMS", "0")


def _run(d, specs, holes, env=None, monkeypatch=None, profile=False, mode=cl.MODE_FP32_ROUNDS):
    if env:
        for k, v in env.items():
            monkeypatch.setenv(k, v)
    try:
        with cl.CoulombCalculator(d["dims"], STEP, mode) as cc:
            cc.initialize(dielectric=10.89)
            cc.set_states(d["states"], d["cells_idx"], holes)
            if profile:
                cc.set_profiling(True)
            got = cc.compute(specs)
            prof = cc.kernel_profile() if profile else None
    finally:
        if env:
            for k in env:
                monkeypatch.delenv(k, raising=False)
    return got, prof


def _oracle(d, specs):
    return np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], STEP, specs,
                                        dielectric=10.89))


def _check(got, ref, want, frac):
    """got (tensor-core Gram) vs ref (FP64 Gram, same potentials): within `frac` of the FP32
    gate; got vs the FP64 oracle: within the gate max(1e-6 |I|, 1e-9 eV)."""
    lim = np.maximum(1e-6 * np.abs(want), 1e-9)
    assert np.all(np.abs(got - ref) <= frac * lim), (np.abs(got - ref) / lim).max()
    assert np.all(np.abs(got - want) <= lim), (np.abs(got - want) / lim).max()


def test_tensor_core_gram_is_used_and_accurate(monkeypatch):
    d = synth.build("c1")
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    got, prof = _run(d, specs, 2, profile=True)
    assert "gram_split" in prof and prof["gram"][1] >= 1
    ref, prof64 = _run(d, specs, 2, env={"CL_NO_TC_GRAM": "1"}, monkeypatch=monkeypatch, profile=True)
    assert "gram_split" not in prof64
    _check(got, ref, _oracle(d, specs), 0.25)


def test_several_tiles_of_densities(monkeypatch):
    """12 states -> 78 pair densities on both sides: 2 x 2 tiles of 64 densities, with padding."""
    d = synth.build("c2", cells=(5, 5, 4))
    d["states"] = d["states"][:, :, :8]
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 12, 6)][::7]
    got, _ = _run(d, specs, 6)
    ref, _ = _run(d, specs, 6, env={"CL_NO_TC_GRAM": "1"}, monkeypatch=monkeypatch)
    _check(got, ref, _oracle(d, specs), 0.25)


def test_chunked_atom_range(monkeypatch):
    """Operands staged in 1,024-atom chunks (and a ragged last chunk) give the same sums."""
    d = synth.build("c1", cells=(8, 8, 5))
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("eeee,hhhh,ehhe,eheh", 4, 2)]
    whole, _ = _run(d, specs, 2)
    chunked, _ = _run(d, specs, 2, env={"CL_TC_MAX_ATOMS": "1000"}, monkeypatch=monkeypatch)
    assert np.abs(chunked - whole).max() <= 1e-9 * np.abs(whole).max()


def test_grid_calculate_uses_tensor_core_gram():
    """calculate() on the grid API (one left, one right density, every cell) in the FP32 form."""
    from oracle import coulomb as C
    rng = np.random.default_rng(11)
    dims = (24, 20, 18)
    F = rng.normal(size=dims[::-1]) + 1j * rng.normal(size=dims[::-1])
    F2 = rng.normal(size=dims[::-1]) + 1j * rng.normal(size=dims[::-1])
    g = C.kernel_octant(dims, (1.0, 1.0, 1.0), 1.0, 0.0)
    V = C.prepare(F, C.kernel_spectrum(g, dims))
    want = C.calculate(V, F2)
    with cl.CoulombCalculator(dims, (1.0, 1.0, 1.0), cl.MODE_FP32_ROUNDS) as cc:
        cc.initialize(dielectric=1.0)
        cc.prepare(F)
        got = cc.calculate(F2)
    assert abs(got - want) <= 1e-6 * np.abs(V).max() * np.abs(F2).sum()


def test_profile_recorded_inside_graph():
    """A batch captured while its context profiles records an event pair around every launch in
    the graph; each replay adds one request's launches, the same classes as an eager request."""
    d = synth.build("c1", cells=(4, 4, 4))
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    with cl.CoulombCalculator(d["dims"], STEP, cl.MODE_FP32_ROUNDS) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 2)
        req = cc.request(specs)
        want = req.run()
        cc.set_profiling(True)
        req.run()
        eager = cc.kernel_profile()
        b = cl.Batch([req])
        b.run()
        cc.set_profiling(False)
        cc.set_profiling(True)
        for _ in range(3):
            got = b.run()[0]
        prof = cc.kernel_profile()
        cc.set_profiling(False)
        b.close()
        req.close()
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    assert set(prof) == set(eager)
    for k, (ms, n, nbytes) in prof.items():
        assert n == 3 * eager[k][1] and ms > 0
        assert nbytes == pytest.approx(3 * eager[k][2])


SL32 = cl.MODE_FP32_SUBLATTICE


def _fused_vs_split(d, specs, holes, monkeypatch):
    # CL_TC_FUSED: the fused Gram also where the operands span several tiles
    got, prof = _run(d, specs, holes, env={"CL_TC_FUSED": "1"}, monkeypatch=monkeypatch, profile=True, mode=SL32)
    assert "gram_split" not in prof and prof["gram"][1] >= 1
    ref, prof_s = _run(d, specs, holes, env={"CL_TC_SPLIT": "1"}, monkeypatch=monkeypatch, profile=True, mode=SL32)
    assert "gram_split" in prof_s
    # CL_TC_NO_WS=1: the fused kernel whose warps take every role -- the same TF32 parts
    # (cvt.rna.tf32) and the same MMAs as the split pass, each k-tile drained into FP64: only the
    # order of the FP64 additions differs
    one, _ = _run(d, specs, holes, env={"CL_TC_FUSED": "1", "CL_TC_NO_WS": "1"}, monkeypatch=monkeypatch, mode=SL32)
    assert np.abs(one - ref).max() <= 1e-12 * np.abs(ref).max()
    # up to 40 right densities the warp-specialised kernel runs: TF32 rounding on the integer
    # pipe, k-tiles drained in pairs summed once in FP32 (round to nearest: at most 2^-24 of the
    # pair's magnitude, a quarter of the TF32x3 parts' 2^-22 of each product), and bit-for-bit
    # the same parts (equal sums) where a block holds a single k-tile
    lim = np.maximum(1e-6 * np.abs(ref), 1e-9)
    assert np.all(np.abs(got - ref) <= 0.25 * lim), (np.abs(got - ref) / lim).max()
    if d["pos"].shape[0] <= 32:
        assert np.abs(got - one).max() <= 1e-12 * np.abs(one).max()
    # CL_TC_COPY8=1: the 8-byte copies of rows that do not start on a 16-byte boundary
    c8, _ = _run(d, specs, holes, env={"CL_TC_FUSED": "1", "CL_TC_COPY8": "1"}, monkeypatch=monkeypatch, mode=SL32)
    assert np.abs(got - c8).max() <= 1e-12 * np.abs(one).max()
    return got


def test_fused_gram_matches_split_pass_and_oracle(monkeypatch):
    d = synth.build("c1")
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    got = _fused_vs_split(d, specs, 2, monkeypatch)
    want = _oracle(d, specs)
    lim = np.maximum(1e-6 * np.abs(want), 1e-9)
    assert np.all(np.abs(got - want) <= lim), (np.abs(got - want) / lim).max()


@pytest.mark.parametrize("cells", [(2, 2, 2), (3, 2, 5), (1, 1, 1)])
def test_fused_gram_ragged_and_tiny_atom_ranges(cells, monkeypatch):
    """64, 240 and 8 atoms: a partial last k-tile, and a block of one k-tile."""
    d = synth.build("c1", cells=cells)
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    got = _fused_vs_split(d, specs, 2, monkeypatch)
    want = _oracle(d, specs)
    lim = np.maximum(1e-6 * np.abs(want), 1e-9)
    assert np.all(np.abs(got - want) <= lim), (np.abs(got - want) / lim).max()


@pytest.mark.parametrize("n_states", [5, 8, 9, 12])
def test_fused_gram_right_tile_widths_and_several_tiles(n_states, monkeypatch):
    """15, 36, 45 and 78 right densities: MMA widths 32, 80 (the widest of the warp-specialised
    kernel), 96, and 128 + 32 over two right tiles (and two left tiles at 12 states), each block
    converting its own tiles' densities."""
    d = synth.build("c2", cells=(4, 5, 4))
    d["states"] = d["states"][:n_states, :, :8]
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", n_states, n_states // 2)][::5]
    _fused_vs_split(d, specs, n_states // 2, monkeypatch)


def _dmma_vs_tf32(d, specs, holes, monkeypatch):
    """The FP64 tensor-core Gram (the FP32 sub-lattice form's Gram under 65,536 atoms) against
    the TF32x3 Gram on the same potentials and against the oracle."""
    monkeypatch.delenv("CL_TC_MIN_ATOMS", raising=False)
    got, prof = _run(d, specs, holes, profile=True, mode=SL32)
    assert "gram_split" not in prof and prof["gram"][1] >= 1
    tf32, _ = _run(d, specs, holes, env={"CL_TC_FUSED": "1"}, monkeypatch=monkeypatch, mode=SL32)
    want = _oracle(d, specs)
    lim = np.maximum(1e-6 * np.abs(want), 1e-9)
    assert np.all(np.abs(got - want) <= lim), (np.abs(got - want) / lim).max()
    # TF32x3 sums carry ~2^-22 per product; FP64 sums carry none of it
    assert np.all(np.abs(got - tf32) <= lim)
    return got


@pytest.mark.parametrize("cells", [(4, 4, 4), (3, 2, 5), (1, 1, 1)])
def test_fp64_tensor_core_gram(cells, monkeypatch):
    """1,024, 240 and 8 atoms: several chunks, a partial last chunk, one chunk of one block."""
    d = synth.build("c1", cells=cells)
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    _dmma_vs_tf32(d, specs, 2, monkeypatch)


def test_fp64_tensor_core_gram_two_tiles_each_side(monkeypatch):
    """12 states: 78 densities a side, 156 Gram rows: 2 x 2 blocks of 128 x 128, the second
    of each side partial (14 densities, zero rows beyond)."""
    d = synth.build("c2", cells=(4, 5, 4))
    d["states"] = d["states"][:, :, :8]
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 12, 6)][::5]
    _dmma_vs_tf32(d, specs, 6, monkeypatch)
