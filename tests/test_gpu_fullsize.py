"""The bench workloads at their full sizes against the FP64 oracle.

Every integral of the medium lens dot (96^3 grid, 110,592 atoms, 20 orbitals, 6 e + 6 h,
5,184 integrals); every integral of a seeded sample of left densities of the 2.1M-atom box
(256^3 grid, 20 orbitals, 4 e + 4 h); a seeded sample of more than 2,000 integrals of the
all-pairs workload (128^3 grid, 20 e + 20 h, 2,560,000 integrals); and one left density of
each of the 16 uneven-size structures.  The library computes the whole request; the oracle
(CoulombCalculator.cpp:105-172 restated in FP64, ``oracle.host.compute_integrals_sampled``)
computes the integrals of the sampled left densities.

Gates: the all-FP64 forms within 1e-10 relative; the FP32 forms within max(1e-6 |I|, 1e-9 eV).
"""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import host as H

pytestmark = pytest.mark.gpu

STEP = (synth.A_ZB / 4,) * 3
EPS = 10.89
MODES = cl.ALL_MODES


def gate(got, want, mode):
    err = np.abs(np.asarray(got) - np.asarray(want))
    if cl.mode_is_fp64(mode):
        lim = 1e-10 * np.abs(want) + 1e-16
    else:
        lim = np.maximum(1e-6 * np.abs(want), 1e-9)
    return err, lim


def _specs(d):
    n = d["states"].shape[0]
    return np.ascontiguousarray(cl.enumerate_integrals(d["integrals"], n, d["holes"]))


def _gpu_values(d, specs, mode):
    with cl.CoulombCalculator(d["dims"], STEP, mode) as cc:
        cc.initialize(dielectric=EPS)
        cc.set_states(d["states"], d["cells_idx"], d["holes"])
        return cc.compute(specs)


def _seeded_lefts(specs, n, count, seed):
    lefts = H.plan_lefts([tuple(int(v) for v in s) for s in specs], n)
    rng = np.random.default_rng(seed)
    return sorted(int(v) for v in rng.choice(lefts, size=min(count, len(lefts)), replace=False))


_cache = {}


def _workload(name):
    """(data, specs, oracle values, covered mask), computed once per module."""
    if name in _cache:
        return _cache[name]
    if name == "c2":
        d = synth.build("c2")
        specs = _specs(d)
        lefts = None
    elif name == "c3":
        d = synth.build("c3")
        specs = _specs(d)
        lefts = _seeded_lefts(specs, 8, 3, 3003)
    else:
        raise KeyError(name)
    spec_list = [tuple(int(v) for v in s) for s in specs]
    want, covered = H.compute_integrals_sampled(list(d["states"]), d["cells_idx"], d["dims"], STEP, spec_list,
                                                lefts=lefts, dielectric=EPS)
    _cache[name] = (d, specs, want, covered)
    return _cache[name]


@pytest.mark.parametrize("mode", MODES)
def test_c2_every_integral(mode):
    d, specs, want, covered = _workload("c2")
    assert covered.all() and len(specs) == 5184
    got = _gpu_values(d, specs, mode)
    err, lim = gate(got, want, mode)
    assert np.all(err <= lim), "worst error/gate %.3g" % (err / lim).max()


@pytest.mark.parametrize("mode", MODES)
def test_c3_sampled_left_densities(mode):
    d, specs, want, covered = _workload("c3")
    assert len(specs) == 1024 and covered.sum() >= 3 * 8
    got = _gpu_values(d, specs, mode)
    err, lim = gate(got[covered], want[covered], mode)
    assert np.all(err <= lim), "worst error/gate %.3g over %d integrals" % ((err / lim).max(), covered.sum())


def test_c4_sampled_integrals():
    """All-pairs (ijkl) on the 128^3 lens dot: the FP32 form (tensor-core Gram) and the
    plain FP64 form against the oracle on every integral of one seeded left density pair
    (3,200 integrals)."""
    d = synth.build("c4")
    specs = _specs(d)
    assert len(specs) == 2560000
    rng = np.random.default_rng(4004)
    a, b = (int(v) for v in rng.choice(np.arange(1, 41), size=2, replace=False))
    mask = ((specs[:, 0] == a) & (specs[:, 3] == b)) | ((specs[:, 0] == b) & (specs[:, 3] == a))
    sample = [tuple(int(v) for v in s) for s in specs[mask]]
    assert len(sample) >= 2000
    want, covered = H.compute_integrals_sampled(list(d["states"]), d["cells_idx"], d["dims"], STEP, sample,
                                                dielectric=EPS)
    assert covered.all()
    for mode in MODES:
        got = _gpu_values(d, specs, mode)[mask]
        err, lim = gate(got, want, mode)
        assert np.all(err <= lim), "mode %d: worst error/gate %.3g" % (mode, (err / lim).max())


def test_c5_one_left_density_each():
    """Each of the 16 uneven-size structures: every integral of one seeded left density,
    through prepared requests replayed as one graph-captured batch, in every form."""
    structs = []
    for i in range(len(synth.C5_CELLS)):
        d = synth.build_c5(i)
        specs = _specs(d)
        lefts = _seeded_lefts(specs, 8, 1, 5005 + i)
        want, covered = H.compute_integrals_sampled(list(d["states"]), d["cells_idx"], d["dims"], STEP,
                                                    [tuple(int(v) for v in s) for s in specs], lefts=lefts,
                                                    dielectric=EPS)
        assert covered.sum() > 0
        structs.append((d, specs, want, covered))
    for mode in MODES:
        calcs, reqs = [], []
        for d, specs, _, _ in structs:
            cc = cl.CoulombCalculator(d["dims"], STEP, mode)
            cc.initialize(dielectric=EPS)
            cc.set_states(d["states"], d["cells_idx"], d["holes"])
            calcs.append(cc)
            reqs.append(cc.request(specs))
        batch = cl.Batch(reqs)
        try:
            batch.run()
            outs = batch.run()  # the replayed graph
        finally:
            batch.close()
        for i, (got, (_, _, want, covered)) in enumerate(zip(outs, structs)):
            err, lim = gate(got[covered], want[covered], mode)
            assert np.all(err <= lim), "mode %d structure %d: worst error/gate %.3g" % (mode, i, (err / lim).max())
        for r in reqs:
            r.close()
        for cc in calcs:
            cc.close()
