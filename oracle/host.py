"""CPU oracle for Coulombo-Lattice's host-side logic (TEST INFRASTRUCTURE ONLY).

Restates, for checking the C++ host library: size rounding, lattice-grid detection,
the ``--integrals`` pattern language, product indexing with conjugation flags, the
greedy vertex cover and step ordering, the step loop with its left/right caches, and
the ``XXXX.txt`` writer.  Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
legs may use it.
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import coulomb as C


# --------------------------------------------------------------------------------------
# Round::up -- Round.hpp:20-49
# --------------------------------------------------------------------------------------

def round_up(n, primes=(2, 3, 5), c=1):
    """Smallest c * p1^i1 * p2^i2 ... >= n (Round.hpp:20-49, same recursion)."""
    first = primes[0]
    if len(primes) == 1:
        while c < n:
            c *= first
        return c
    best = round_up(n, primes[1:], c)
    while c < n:
        c *= first
        best = min(best, round_up(n, primes[1:], c))
    return best


# --------------------------------------------------------------------------------------
# Grid detection -- Broadcaster.cpp:8-43, 47-87, 136-143
# --------------------------------------------------------------------------------------

class GridError(RuntimeError):
    pass


def float_gcd(a, b):
    """Broadcaster.cpp:8-22: fmod-based GCD with 1e-10 exact / 1e-2 failure tolerances."""
    if a < b:
        a, b = b, a
    while True:
        r = math.fmod(a, b)
        if r < 1.0e-10:
            return b
        elif r < 1.0e-2:
            return 0.0
        a, b = b, r


def compute_grid(coords):
    """Broadcaster.cpp:24-43 -> (size, origin, step)."""
    buf = np.sort(np.asarray(coords, dtype=np.float64))
    step = math.nan
    for a in range(1, len(buf)):
        nxt = buf[a] - buf[a - 1]
        if nxt > 1.0e-10:
            step = nxt if math.isnan(step) else float_gcd(step, nxt)
            if step == 0:
                raise GridError("could not find common grid step")
    size = int(np.rint((buf[-1] - buf[0]) / step)) + 1
    return size, float(buf[0]), step


def detect_grid(positions):
    """positions [A,3] -> dict(raw, pad, origin, step, cells) (Broadcaster.cpp:47-87).

    cells = (iz*Ny + iy)*Nx + ix on the padded grid (single rank, zOffset = 0)."""
    raw, origin, step = [], [], []
    for d in range(3):
        s, o, st = compute_grid(positions[:, d])
        raw.append(s)
        origin.append(o)
        step.append(st)
    pad = [round_up(n) for n in raw]
    idx = [np.rint((positions[:, d] - origin[d]) / step[d]).astype(np.int64) for d in range(3)]
    cells = (idx[2] * pad[1] + idx[1]) * pad[0] + idx[0]
    return dict(raw=tuple(raw), pad=tuple(pad), origin=tuple(origin), step=tuple(step), cells=cells)


# --------------------------------------------------------------------------------------
# Pattern -- Pattern.hpp:15-100
# --------------------------------------------------------------------------------------

class PatternError(RuntimeError):
    pass


class Pattern:
    def __init__(self, description: str, hole_count: int):
        self.hole_count = hole_count
        self.patterns = []
        for part in description.split(","):
            if not part:
                raise PatternError("invalid empty pattern")
            for ch in part:
                if not (ch == "*" or (ch.isalnum() and ch.isascii() and ch != "0")):
                    raise PatternError("invalid character '%s' in pattern" % ch)
            self.patterns.append(part)

    def _letter(self, c, i, assign):
        if c == "*":
            return True
        if "1" <= c <= "9":
            return i == ord(c) - ord("0")
        if c == "h":
            return i <= self.hole_count
        if c == "e":
            return i > self.hole_count
        if assign.get(c):
            return i == assign[c]
        assign[c] = i
        return True

    def match(self, i0, i1, i2, i3):
        for p in self.patterns:
            # chars beyond the pattern's end read as '\0', a free letter (Pattern.hpp:90-93)
            chars = [p[j] if j < len(p) else "\0" for j in range(4)]
            assign = {}
            if (self._letter(chars[0], i0, assign) and self._letter(chars[1], i1, assign)
                    and self._letter(chars[2], i2, assign) and self._letter(chars[3], i3, assign)):
                return True
        return False


def enumerate_integrals(pattern: Pattern, n_inputs: int):
    """coulombo.cpp:135-148: all 1-based (i1..i4) in lexicographic order that match."""
    out = []
    rng = range(1, n_inputs + 1)
    for i1 in rng:
        for i2 in rng:
            for i3 in rng:
                for i4 in rng:
                    if pattern.match(i1, i2, i3, i4):
                        out.append((i1, i2, i3, i4))
    return out


# --------------------------------------------------------------------------------------
# Products, vertex cover, plan -- Planner.hpp:71-144, Graph.hpp:49-91
# --------------------------------------------------------------------------------------

def product_of(i_l, i_r):
    """Planner.hpp:134-144 -> (product index, conjugate flag)."""
    conj = 0
    if i_l < i_r:
        conj = 1
        i_l, i_r = i_r, i_l
    return i_l * (i_l - 1) // 2 + i_r - 1, conj


def product_states(p):
    """Inverse of product_of for conj=0: product p -> (fL, fR) 1-based with fL >= fR
    (FunctionCollection.cpp:91-105 creation order)."""
    fl = int((1 + math.isqrt(1 + 8 * p)) // 2)
    while fl * (fl - 1) // 2 > p:
        fl -= 1
    while (fl + 1) * fl // 2 <= p:
        fl += 1
    fr = p - fl * (fl - 1) // 2 + 1
    return fl, fr


def vertex_cover(vertex_count, edges):
    """Graph.hpp:49-91, the same greedy rule (loops forced in; leaves take their neighbour;
    otherwise the highest-degree vertex, ties by larger index)."""
    edges = set(edges)
    cover = {a for (a, b) in edges if a == b}
    nb = [set() for _ in range(vertex_count)]
    for (a, b) in edges:
        if a != b and a not in cover and b not in cover:
            nb[a].add(b)
            nb[b].add(a)
    queue = {v for v in range(vertex_count) if nb[v]}

    def key(v):
        return (len(nb[v]), v)

    while queue:
        first = min(queue, key=key)
        if len(nb[first]) == 1:
            v = next(iter(nb[first]))
        else:
            v = max(queue, key=key)
        queue.discard(v)
        cover.add(v)
        for w in list(nb[v]):
            if w in queue:
                queue.discard(w)
                nb[w].discard(v)
                if nb[w]:
                    queue.add(w)
    return cover


def compute_plan(specs, product_count):
    """MasterPlanner::addIntegral + computePlan (Planner.hpp:71-104).

    Returns steps: list of (id, (left, lconj), (right, rconj)) in execution order."""
    steps = []
    for sid, (i1, i2, i3, i4) in enumerate(specs):
        steps.append((sid, product_of(i1, i4), product_of(i2, i3)))
    cover = vertex_cover(product_count, [(s[1][0], s[2][0]) for s in steps])
    oriented = []
    for (sid, left, right) in steps:
        if left[0] not in cover:
            left, right = right, left
        oriented.append((sid, left, right))

    import functools

    def cmp(a, b):
        if a[1][0] != b[1][0]:
            return -1 if a[1][0] < b[1][0] else 1
        if a[2][0] != b[2][0]:
            return -1 if a[2][0] < b[2][0] else 1
        a_same = a[1][1] == a[2][1]
        b_same = b[1][1] == b[2][1]
        if a_same and not b_same:
            return -1
        if b_same and not a_same:
            return 1
        return 0

    # std::sort is not stable; ties only differ in step id, whose order never changes a value
    oriented.sort(key=functools.cmp_to_key(cmp))
    return oriented


# --------------------------------------------------------------------------------------
# Reading inputs -- FunctionCollection.cpp:38-84
# --------------------------------------------------------------------------------------

def load_atoms(path):
    """First three numbers of each line until the first line without three numbers."""
    coords = []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            try:
                x, y, z = float(parts[0]), float(parts[1]), float(parts[2])
            except (IndexError, ValueError):
                break
            coords.append((x, y, z))
    return np.array(coords, dtype=np.float64).reshape(-1, 3)


def load_state(path, n_atoms, n_orb, skip_lines):
    """[atom, orb] complex coefficients; 'file is truncated' when lines run out."""
    with open(path) as fh:
        for _ in range(skip_lines):
            fh.readline()
        data = np.loadtxt(fh, usecols=(0, 1), max_rows=n_atoms * n_orb, ndmin=2)
    if data.shape[0] < n_atoms * n_orb:
        raise RuntimeError("file is truncated: %s" % path)
    c = data[:, 0] + 1j * data[:, 1]
    return c.reshape(n_atoms, n_orb)


# --------------------------------------------------------------------------------------
# Whole pipeline -- coulombo.cpp:119-209 and output coulombo.cpp:213-262
# --------------------------------------------------------------------------------------

def compute_integrals(states, cells, dims, step, specs, dielectric=1.0, onsite=0.0,
                      tf_lattice=None, rounds=range(8)):
    """Runs the reference's plan loop (coulombo.cpp:186-209) with the FP64 real-space
    convolution.  states: list of [atom, orb] arrays in input order (holes first)."""
    n = len(states)
    product_count = n * (n + 1) // 2
    plan = compute_plan(specs, product_count)
    g = C.kernel_octant(dims, step, dielectric, onsite, tf_lattice)
    ghat = C.kernel_spectrum(g, dims)
    values = [0j] * len(specs)
    last_left = -1
    last_right = -1
    last_rconj = False
    V = None
    value_last = 0j

    def density(prod, conj):
        fl, fr = product_states(prod)
        rho = C.pair_density_atoms(states[fl - 1], states[fr - 1], conj)
        return C.scatter_density(rho, cells, dims)

    for (sid, left, right) in plan:
        if left[0] != last_left:
            V = C.prepare(density(left[0], False), ghat, rounds)
            last_left = left[0]
        rconj = left[1] != right[1]
        if right[0] != last_right or rconj != last_rconj:
            value_last = C.calculate(V, density(right[0], rconj))
            last_right = right[0]
            last_rconj = rconj
        values[sid] = np.conj(value_last) if left[1] else value_last
    return values


def compute_integrals_sampled(states, cells, dims, step, specs, lefts=None, dielectric=1.0, onsite=0.0,
                              tf_lattice=None, ghat=None, timer=None):
    """The same plan loop as ``compute_integrals`` restricted to the steps whose (oriented)
    left product is in ``lefts`` (all of them when None), for workloads too large for the
    dense per-step grids.

    Each prepared left density is convolved on the dense grid exactly as in the reference
    (8 rounds, CoulombCalculator.cpp:105-163).  ``calculate`` (CoulombCalculator.cpp:165-172)
    is the sum of V(r) F(r) over the grid; F is zero except at atom cells (Product.cpp:16-30,
    where a later atom in a shared cell overwrites an earlier one), so the sum is taken over
    the occupied cells only -- the same terms without the zeros.

    Returns (values, covered): complex values per spec (0 where not covered) and the boolean
    mask of covered specs.  ``timer`` (optional) receives the seconds spent per prepared left
    density, for CPU-baseline timing."""
    import time as _time
    n = len(states)
    product_count = n * (n + 1) // 2
    plan = compute_plan(specs, product_count)
    if ghat is None:
        ghat = C.kernel_spectrum(C.kernel_octant(dims, step, dielectric, onsite, tf_lattice), dims)
    cells = np.asarray(cells, dtype=np.int64)
    # occupied cells and the atom that ends up in each (the last one in input order)
    rev = cells[::-1]
    uniq, first_in_rev = np.unique(rev, return_index=True)
    owner = (len(cells) - 1 - first_in_rev).astype(np.int64)
    chosen = None if lefts is None else set(int(v) for v in lefts)
    values = np.zeros(len(specs), dtype=np.complex128)
    covered = np.zeros(len(specs), dtype=bool)
    right_cache = {}
    # keep every right density while they fit in a few GB, else only the current left's
    keep_all = 2 * product_count * len(uniq) * 16 < (4 << 30)
    owned = [None] * n
    identity = len(owner) == len(cells) and bool(np.all(owner == np.arange(len(cells))))

    def rho_at(prod, conj):
        key = (prod, conj)
        if key not in right_cache:
            fl, fr = product_states(prod)
            for f in (fl, fr):
                if owned[f - 1] is None:
                    owned[f - 1] = states[f - 1] if identity else np.ascontiguousarray(states[f - 1][owner])
            right_cache[key] = C.pair_density_atoms(owned[fl - 1], owned[fr - 1], conj)
        return right_cache[key]

    V_at = None
    last_left = -1
    t0 = None
    for (sid, left, right) in plan:
        if chosen is not None and left[0] not in chosen:
            continue
        if left[0] != last_left:
            if timer is not None and t0 is not None:
                timer.append(_time.perf_counter() - t0)
            t0 = _time.perf_counter()
            if not keep_all:
                right_cache.clear()
            F = C.scatter_density(rho_at(left[0], False), uniq, dims)
            V_at = C.prepare(F, ghat).reshape(-1)[uniq]
            last_left = left[0]
        rconj = left[1] != right[1]
        val = complex(np.sum(V_at * rho_at(right[0], rconj)))
        values[sid] = np.conj(val) if left[1] else val
        covered[sid] = True
    if timer is not None and t0 is not None:
        timer.append(_time.perf_counter() - t0)
    return values, covered


def plan_lefts(specs, n_inputs):
    """Oriented left products of the plan, in execution order (Planner.hpp:83-104)."""
    plan = compute_plan(specs, n_inputs * (n_inputs + 1) // 2)
    seen = []
    for (_, left, _) in plan:
        if not seen or seen[-1] != left[0]:
            if left[0] not in seen:
                seen.append(left[0])
    return seen


def format_outputs(specs, values, n_holes, n_electrons):
    """coulombo.cpp:213-262 -> {core: text}.  Hole numbering is reversed."""
    table = {tuple(s): v for s, v in zip(specs, values)}
    out = {}
    for ti in range(2):
        for tj in range(2):
            for tk in range(2):
                for tl in range(2):
                    t = (ti, tj, tk, tl)
                    core = "".join("e" if b else "h" for b in t)
                    counts = [n_electrons if b else n_holes for b in t]
                    lines = []
                    for ni in range(1, counts[0] + 1):
                        for nj in range(1, counts[1] + 1):
                            for nk in range(1, counts[2] + 1):
                                for nl in range(1, counts[3] + 1):
                                    idx = (ni, nj, nk, nl)
                                    spec = tuple(n_holes + v if b else n_holes + 1 - v
                                                 for v, b in zip(idx, t))
                                    if spec in table:
                                        val = table[spec]
                                        lines.append("%2d %2d %2d %2d   %17.14f %17.14f\n" % (
                                            ni, nj, nk, nl, val.real, val.imag))
                    if lines:
                        out[core] = "".join(lines)
    return out


def write_outputs(outdir, specs, values, n_holes, n_electrons):
    for core, text in format_outputs(specs, values, n_holes, n_electrons).items():
        with open(os.path.join(outdir, core + ".txt"), "w") as fh:
            fh.write(text)
