"""The integral pipeline (cl_set_states + cl_compute, cl_potentials) against the oracle
and the reference's example golden."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import coulomb as C
from oracle import host as H

pytestmark = pytest.mark.gpu


def gate(got, want, mode):
    """FP64 plain path: 1e-10 relative.  FP32 form: max(1e-6 |I|, 1e-9 eV)."""
    got = np.asarray(got)
    want = np.asarray(want)
    err = np.abs(got - want)
    if mode == cl.MODE_FP64_PLAIN:
        lim = 1e-10 * np.maximum(np.abs(want), 1e-300) + 1e-16
    else:
        lim = np.maximum(1e-6 * np.abs(want), 1e-9)
    return err, lim


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_example_golden(mode):
    import make_example_fixture as fx
    d = fx.load()
    g = cl.detect_grid(d["pos"])
    with cl.CoulombCalculator(g["pad"], g["step"], mode) as cc:
        cc.initialize(dielectric=11.4)
        cc.set_states(d["coeff"][None], g["cells"], 0)
        v = cc.compute([(1, 1, 1, 1)])[0]
    text = H.format_outputs([(1, 1, 1, 1)], [v], 0, 1)["eeee"]
    if mode == cl.MODE_FP64_PLAIN:
        assert text[:29] == d["golden"]
    assert abs(v - 0.09034007197751963) <= 1e-6 * 0.0903


def _oracle_values(d, specs, dielectric=10.89, onsite=0.0, tf=None):
    step = (synth.A_ZB / 4,) * 3
    return np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], step, specs,
                                        dielectric=dielectric, onsite=onsite, tf_lattice=tf))


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
@pytest.mark.parametrize("pattern", ["****", "eeee,hhhh,ehhe,eheh", "ijji,1*2*"])
def test_c1_all_patterns(mode, pattern):
    d = synth.build("c1")
    n = d["states"].shape[0]
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals(pattern, n, d["holes"])]
    want = _oracle_values(d, specs)
    step = (synth.A_ZB / 4,) * 3
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], d["holes"])
        got = cc.compute(specs)
    err, lim = gate(got, want, mode)
    assert np.all(err <= lim), (err / lim).max()


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_medium_structure_eight_states(mode):
    """64^3 grid, 8 states (36 densities), the default four classes."""
    d = synth.build("c3", cells=(16, 16, 16))
    d["states"] = d["states"][:, :, :6]
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals(d["integrals"], 8, 4)]
    want = _oracle_values(d, specs)
    step = (synth.A_ZB / 4,) * 3
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 4)
        got = cc.compute(specs)
    err, lim = gate(got, want, mode)
    assert np.all(err <= lim), (err / lim).max()


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_unsorted_atoms_duplicates_onsite_tf(mode):
    """Atom order does not matter; a later atom in the same cell replaces an earlier one
    (F[cell] = value in atom order, Product.cpp:16-30); onsite and Thomas-Fermi kernel."""
    d = synth.build("c1", cells=(3, 2, 2))
    rng = np.random.default_rng(4)
    perm = rng.permutation(d["states"].shape[1])
    states = d["states"][:, perm]
    cells = d["cells_idx"][perm]
    # duplicate a few atoms into already occupied cells
    dup = rng.choice(len(cells), 5, replace=False)
    cells = np.concatenate([cells, cells[dup]])
    extra = rng.normal(size=(states.shape[0], 5, states.shape[2])) * 0.05
    states = np.concatenate([states, extra + 0j], axis=1)
    d2 = dict(d, states=states, cells_idx=cells)
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    want = _oracle_values(d2, specs, onsite=1.7, tf=5.65)
    step = (synth.A_ZB / 4,) * 3
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89, onsite=1.7, tf_lattice=5.65)
        cc.set_states(states, cells, 2)
        got = cc.compute(specs)
    err, lim = gate(got, want, mode)
    assert np.all(err <= lim), (err / lim).max()


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_potentials_match_oracle(mode):
    d = synth.build("c1", cells=(3, 3, 2))
    step = (synth.A_ZB / 4,) * 3
    ghat = C.kernel_spectrum(C.kernel_octant(d["dims"], step, 10.89), d["dims"])
    want = []
    for s in range(d["states"].shape[0]):
        rho = C.pair_density_atoms(d["states"][s], d["states"][s])
        V = C.prepare(C.scatter_density(rho, d["cells_idx"], d["dims"]), ghat).ravel()
        want.append(V[d["cells_idx"]].real)
    want = np.array(want)
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 0)
        got = cc.potentials()
    tol = 1e-10 if mode == cl.MODE_FP64_PLAIN else 1e-6
    assert np.abs(got - want).max() <= tol * np.abs(want).max()


def test_compute_requires_states_and_kernel():
    with cl.CoulombCalculator((8, 8, 8)) as cc:
        with pytest.raises(cl.CoulomboError) as e:
            cc.compute([(1, 1, 1, 1)])
        assert e.value.kind == "state"
        cc.initialize(1.0)
        with pytest.raises(cl.CoulomboError) as e:
            cc.compute([(1, 1, 1, 1)])
        assert e.value.kind == "state"
        with pytest.raises(cl.CoulomboError, match="outside the grid"):
            cc.set_states(np.ones((1, 2, 1), complex), np.array([0, 512]), 0)


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
@pytest.mark.parametrize("env", [{"CL_XY_PLANE": "0"}, {"CL_NO_REGISTER_FFT": "1"}, {"CL_L2_CHUNK_MB": "4"}])
def test_pass_variants_agree(mode, env, monkeypatch):
    """The register row/column passes (with the fused plane passes off), the generic passes and
    every chunking of the densities compute the same integrals as the default passes (a 64^2
    plane, so the default is the fused plane pass)."""
    d = synth.build("c1", cells=(16, 16, 3))
    step = (synth.A_ZB / 4,) * 3
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]

    def run():
        with cl.CoulombCalculator(d["dims"], step, mode) as cc:
            cc.initialize(dielectric=10.89)
            cc.set_states(d["states"], d["cells_idx"], 2)
            return cc.compute(specs)

    base = run()
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    other = run()
    tol = 1e-12 if mode == cl.MODE_FP64_PLAIN else 1e-6
    assert np.abs(other - base).max() <= tol * np.abs(base).max()


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_round_split_adds_up(mode):
    """cl_compute_rounds over disjoint round masks (the multi-GPU split) sums to cl_compute,
    and matches the oracle's partial sums over the same rounds."""
    from coulombo_lattice_b200 import multi
    d = synth.build("c1", cells=(4, 4, 4))
    step = (synth.A_ZB / 4,) * 3
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("eeee,hhhh,ehhe,eheh", 4, 2)]
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 2)
        full = cc.compute(specs)
        parts = [cc.compute_rounds(specs, multi.round_mask(r, 3)) for r in range(3)]
    tol = 1e-12 if mode == cl.MODE_FP64_PLAIN else 1e-6
    assert np.abs(sum(parts) - full).max() <= tol * np.abs(full).max()
    want0 = np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], step, specs,
                                         dielectric=10.89, rounds=[0, 3, 6]))
    err, lim = gate(parts[0], want0, mode)
    assert np.all(err <= np.maximum(lim, 1e-9 * np.abs(full).max()))


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_prepared_requests_and_graph_batch(mode):
    """cl_request runs equal cl_compute; a batch of uneven structures captured as one CUDA
    graph gives every structure's values, on the first (capturing) run and on replays."""
    step = (synth.A_ZB / 4,) * 3
    structs = []
    for cells in [(3, 3, 3), (4, 3, 5), (2, 4, 4)]:
        d = synth.build("c1", cells=cells)
        specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
        structs.append((d, specs))
    calcs, reqs, wants = [], [], []
    for d, specs in structs:
        cc = cl.CoulombCalculator(d["dims"], step, mode)
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 2)
        wants.append(cc.compute(specs))
        r = cc.request(specs)
        np.testing.assert_allclose(r.run(), wants[-1], rtol=1e-12, atol=0)
        calcs.append(cc)
        reqs.append(r)
    batch = cl.Batch(reqs)
    for _ in range(3):
        outs = batch.run()
        for got, want in zip(outs, wants):
            np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    assert batch.last_ms() > 0
    batch.close()
    for r in reqs:
        r.close()
    for cc in calcs:
        cc.close()


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_round_split_over_more_ranks_than_rounds(mode):
    """With 10 shares of the 8 rounds, the two shares without a round give exact zeros and all
    shares still add up to the full request."""
    from coulombo_lattice_b200 import multi
    d = synth.build("c1", cells=(3, 4, 3))
    step = (synth.A_ZB / 4,) * 3
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 2)
        full = cc.compute(specs)
        parts = [cc.compute_rounds(specs, multi.round_mask(r, 10)) for r in range(10)]
    assert multi.round_mask(8, 10) == 0 and multi.round_mask(9, 10) == 0
    assert np.all(parts[8] == 0) and np.all(parts[9] == 0)
    tol = 1e-12 if mode == cl.MODE_FP64_PLAIN else 1e-6
    assert np.abs(sum(parts) - full).max() <= tol * np.abs(full).max()


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_prepared_request_follows_new_coefficients(mode):
    """New coefficients on the same atoms (cl_set_states) are picked up by an existing prepared
    request and by its graph batch."""
    d = synth.build("c1", cells=(4, 4, 4))
    step = (synth.A_ZB / 4,) * 3
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", 4, 2)]
    other = synth.make_states(d["pos"], d["orbitals"], 4, 777, "gauss")
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 2)
        req = cc.request(specs)
        first = req.run()
        batch = cl.Batch([req])
        np.testing.assert_allclose(batch.run()[0], first, rtol=1e-12, atol=0)
        cc.set_states(other, d["cells_idx"], 2)
        want = cc.compute(specs)
        np.testing.assert_allclose(req.run(), want, rtol=1e-12, atol=0)
        np.testing.assert_allclose(batch.run()[0], want, rtol=1e-12, atol=0)
        assert np.abs(want - first).max() > 1e-6 * np.abs(first).max()
        batch.close()
        req.close()


@pytest.mark.parametrize("mode", [cl.MODE_FP64_PLAIN, cl.MODE_FP32_ROUNDS])
def test_compute_states_overlapped_matches(mode):
    """cl_compute_states (upload overlapped with the transforms, densities grouped by state)
    gives the values of cl_set_states + cl_compute, on a first call and on a repeat with the same
    cells and new coefficients; the oracle agrees."""
    d = synth.build("c2", cells=(5, 6, 4))
    d["states"] = d["states"][:, :, :6]
    step = (synth.A_ZB / 4,) * 3
    specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("eeee,hhhh,ehhe,eheh", 12, 6)]
    other = synth.make_states(d["pos"], 6, 12, 4242, "gauss")
    with cl.CoulombCalculator(d["dims"], step, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 6)
        want = cc.compute(specs)
        got = cc.compute_states(d["states"], d["cells_idx"], 6, specs)
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-15)
        got2 = cc.compute_states(other, d["cells_idx"], 6, specs)
        cc.set_states(other, d["cells_idx"], 6)
        np.testing.assert_allclose(got2, cc.compute(specs), rtol=1e-9, atol=1e-15)
    err, lim = gate(got, _oracle_values(d, specs), mode)
    assert np.all(err <= lim), (err / lim).max()


def test_graph_batch_of_requests_with_different_state_counts():
    """A batch whose requests stage different numbers of states per atom chunk (different
    shared-memory sizes of the pair-density kernel) runs each request as prepared."""
    step = (synth.A_ZB / 4,) * 3
    calcs, reqs, wants = [], [], []
    for n_states, cells in [(8, (4, 4, 3)), (4, (3, 4, 4)), (6, (4, 3, 4))]:
        d = synth.build("c3", cells=cells)
        d["states"] = d["states"][:n_states, :, :5]
        holes = n_states // 2
        specs = [tuple(int(v) for v in s) for s in cl.enumerate_integrals("****", n_states, holes)]
        cc = cl.CoulombCalculator(d["dims"], step, cl.MODE_FP32_ROUNDS)
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], holes)
        wants.append(cc.compute(specs))
        reqs.append(cc.request(specs))
        calcs.append(cc)
    batch = cl.Batch(reqs)
    for _ in range(2):
        for got, want in zip(batch.run(), wants):
            np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-15)
    batch.close()
    for r in reqs:
        r.close()
    for cc in calcs:
        cc.close()
