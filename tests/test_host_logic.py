"""Host-side logic of libcoulombo_lattice.so (no GPU) against the oracle restatement and,
where the reference's header-only code compiles here, against the reference itself
(oracle/_ref/libref_host.so, built by oracle/Makefile)."""
import ctypes
import os

import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import synth
from oracle import host as H

REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libref_host.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_LIB):
        pytest.skip("reference host library not built (oracle/Makefile needs the reference tree)")
    L = ctypes.CDLL(REF_LIB)
    L.ref_round_up_235.restype = ctypes.c_int
    L.ref_pattern_enumerate.restype = ctypes.c_int
    return L


def test_round_known_answers():
    assert [cl.round_up_235(n) for n in (0, 13, 16, 17, 34, 101)] == [1, 15, 16, 18, 36, 108]
    assert [cl.round_up_235(n, 4) for n in (0, 13, 16, 17, 34, 101)] == [4, 16, 16, 20, 36, 108]


def test_round_matches_reference(ref):
    for n in list(range(0, 700)) + [1021, 4097, 65537]:
        for c in (1, 2, 3, 4, 5, 6):
            assert cl.round_up_235(n, c) == ref.ref_round_up_235(n, c) == H.round_up(n, c=c)


PATTERNS = ["****", "eeee,hhhh,ehhe,eheh", "ijkl", "ijji", "1*1*", "ehhe", "1212", "iijj", "abba,1h*e",
            "aAaA", "hhee", "*e*h", "9999", "ijki,e**h", "zzzz"]


@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("n,holes", [(1, 0), (3, 1), (4, 2), (5, 5)])
def test_pattern_matches_reference_and_oracle(pattern, n, holes, ref):
    got = cl.enumerate_integrals(pattern, n, holes)
    want = H.enumerate_integrals(H.Pattern(pattern, holes), n)
    assert [tuple(int(v) for v in s) for s in got] == want
    match = np.zeros(n ** 4, dtype=np.uint8)
    err = ctypes.create_string_buffer(256)
    assert ref.ref_pattern_enumerate(pattern.encode(), n, holes, match.ctypes.data_as(ctypes.c_void_p), err) == 0
    idx = np.array([((a - 1) * n ** 3 + (b - 1) * n ** 2 + (c - 1) * n + (d - 1)) for a, b, c, d in want], dtype=int)
    assert set(np.nonzero(match)[0].tolist()) == set(idx.tolist())


def test_readme_examples():
    """README.md:130-150 worked examples."""
    def ids(p, n, h):
        return ["".join(str(int(v)) for v in s) for s in cl.enumerate_integrals(p, n, h)]
    assert ids("1212", 2, 1) == ["1212"]
    assert ids("ijji", 2, 1) == ["1111", "1221", "2112", "2222"]
    assert ids("1*1*", 2, 1) == ["1111", "1112", "1211", "1212"]
    assert ids("ehhe", 3, 2) == ["3113", "3123", "3213", "3223"]


@pytest.mark.parametrize("bad,msg", [("", "invalid empty pattern"), ("ee,,hh", "invalid empty pattern"),
                                     ("e0ee", "invalid character '0'"), ("e-ee", "invalid character '-'")])
def test_pattern_errors(bad, msg, ref):
    with pytest.raises(cl.CoulomboError, match=msg):
        cl.enumerate_integrals(bad, 2, 1)
    err = ctypes.create_string_buffer(256)
    match = np.zeros(16, dtype=np.uint8)
    assert ref.ref_pattern_enumerate(bad.encode(), 2, 1, match.ctypes.data_as(ctypes.c_void_p), err) == 1
    assert msg in err.value.decode()


def test_vertex_cover_known_answers():
    assert len(cl.vertex_cover(4, [(i, j) for j in range(4) for i in range(j)])) == 3
    assert cl.vertex_cover(3, []) == set()
    assert cl.vertex_cover(3, [(0, 0), (1, 1), (2, 2)]) == {0, 1, 2}
    assert cl.vertex_cover(3, [(0, 1), (1, 2)]) == {1}
    assert cl.vertex_cover(3, [(0, 0), (0, 1), (1, 1), (1, 2), (2, 0)]) == {0, 1}


def test_vertex_cover_random_graphs(ref):
    rng = np.random.default_rng(11)
    for trial in range(300):
        nv = int(rng.integers(1, 30))
        ne = int(rng.integers(0, 3 * nv))
        edges = rng.integers(0, nv, size=(ne, 2)).astype(np.int32)
        got = cl.vertex_cover(nv, edges)
        out = np.zeros(nv, dtype=np.uint8)
        e = np.ascontiguousarray(edges)
        ref.ref_vertex_cover(nv, ne, e.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
        assert got == {int(v) for v in np.nonzero(out)[0]}
        assert got == H.vertex_cover(nv, [tuple(x) for x in edges.tolist()])
        for a, b in edges:
            assert a in got or b in got


@pytest.mark.parametrize("pattern,n,holes", [("eeee,hhhh,ehhe,eheh", 8, 4), ("ijkl", 5, 2), ("****", 3, 1),
                                             ("ijji,1*2*", 6, 3)])
def test_plan_matches_oracle(pattern, n, holes):
    specs = H.enumerate_integrals(H.Pattern(pattern, holes), n)
    got = cl.plan(n, specs)
    want = H.compute_plan(specs, n * (n + 1) // 2)
    # same orientation of every step; same order up to ties of equal keys
    by_id = {int(s[0]): (int(s[1]), int(s[2]), int(s[3]), int(s[4])) for s in got}
    for sid, left, right in want:
        assert by_id[sid] == (left[0], left[1], right[0], right[1])
    keys_got = [(s[1], s[3], int(s[2] == s[4])) for s in got]
    keys_want = [(l[0], r[0], int(l[1] == r[1])) for _, l, r in want]
    assert keys_got == keys_want


def test_product_indexing():
    for i in range(1, 12):
        for j in range(1, 12):
            p, c = H.product_of(i, j)
            fl, fr = H.product_states(p)
            assert (fl, fr) == (max(i, j), min(i, j)) and c == int(i < j)


def test_detect_grid_example_and_synthetic():
    import make_example_fixture as fx
    d = fx.load()
    got = cl.detect_grid(d["pos"])
    want = H.detect_grid(d["pos"])
    assert got["raw"] == want["raw"] == (41, 41, 41)
    assert got["pad"] == want["pad"] == (45, 45, 45)
    assert np.array_equal(got["cells"], want["cells"])
    assert np.allclose(got["step"], 1.35775, atol=1e-12)
    lat = synth.zincblende_lattice((3, 4, 5))
    pos = synth.positions_angstrom(lat)
    g = cl.detect_grid(pos)
    assert g["raw"] == (12, 16, 20) and g["pad"] == (12, 16, 20)
    assert np.array_equal(g["cells"], synth.cell_indices(lat, (12, 16, 20)))
    assert len(pos) * 8 == 12 * 16 * 20


def test_detect_grid_errors():
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0], [1.5 + 0.003, 0, 0]])
    with pytest.raises(cl.CoulomboError, match="could not find common grid step"):
        cl.detect_grid(pos)
    with pytest.raises(cl.GridError if hasattr(cl, "GridError") else H.GridError):
        H.detect_grid(pos)


def test_detect_grid_padding_and_origin():
    rng = np.random.default_rng(5)
    idx = rng.integers(0, 41, size=(200, 3))
    idx[0] = (0, 0, 0)
    idx[1] = (40, 12, 6)
    pos = idx * np.array([1.25, 2.5, 0.75]) - 3.0
    got = cl.detect_grid(pos)
    want = H.detect_grid(pos)
    assert got["raw"] == want["raw"] and got["pad"] == want["pad"]
    assert np.array_equal(got["cells"], want["cells"])
