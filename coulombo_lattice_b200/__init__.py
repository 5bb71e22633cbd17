"""B200 implementation of Coulombo-Lattice's Coulomb-integral path.

The product is ``libcoulombo_lattice.so`` (CUDA kernels for sm_100a behind the C ABI of
``include/coulombo_lattice.h``) and the drop-in binaries ``bin/coulombo`` and
``bin/potentials``.  This module is a ctypes mirror of the reference's compute seam,
``CoulombCalculator`` (src/CoulombCalculator.hpp:28-94): ``initialize`` with a Coulomb or a
custom kernel, ``prepare``/``calculate`` on grids, plus the integral pipeline
(``set_states``/``compute``) and the host helpers.  Failures raise ``CoulomboError`` with
the library's message, the way the reference throws ``std::runtime_error``.

There is no fallback: if the shared library is missing, importing the calculator raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcoulombo_lattice.so")
BIN_DIR = os.path.join(_HERE, "bin")

# precision / algorithm forms (include/coulombo_lattice.h CL_MODE_*)
MODE_FP64_PLAIN = 0   # all-FP64, 8 rounds of N-point transforms (the reference's method)
MODE_FP32_ROUNDS = 1  # FP32 transforms, FP64 kernel/twiddles/round sum/reductions, 8 rounds
MODE_FP32_FOURIER = MODE_FP32_ROUNDS  # former name of MODE_FP32_ROUNDS
MODE_FP64_SUBLATTICE = 2  # all-FP64, per residue class of the atoms' grid points (exact decomposition)
MODE_FP32_SUBLATTICE = 3  # the same with FP32 transforms, FP64-built class kernels and reductions
ALL_MODES = [MODE_FP64_PLAIN, MODE_FP32_ROUNDS, MODE_FP64_SUBLATTICE, MODE_FP32_SUBLATTICE]
MODE_NAMES = {MODE_FP64_PLAIN: "fp64 rounds", MODE_FP32_ROUNDS: "fp32 rounds",
              MODE_FP64_SUBLATTICE: "fp64 sub-lattice", MODE_FP32_SUBLATTICE: "fp32 sub-lattice"}


def mode_is_fp64(mode):
    """True for the all-FP64 forms (parity gate 1e-10 relative)."""
    return mode in (MODE_FP64_PLAIN, MODE_FP64_SUBLATTICE)

# kernel classes of cl_kernel_profile (include/coulombo_lattice.h CL_KCLASS_*)
KERNEL_CLASSES = ["pair_density", "x_forward", "y_pass", "z_pass", "x_inverse", "gram", "kernel_build", "gram_split",
                  "round_sum", "spare"]

_ERR_NAMES = {1: "argument", 2: "state", 3: "cuda", 4: "memory", 5: "unsupported", 6: "timeout"}

_lib = None


class CoulomboError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code
        self.kind = _ERR_NAMES.get(code, "unknown")


# (name, restype, argtypes) of every entry point declared in include/coulombo_lattice.h
_P = ctypes.POINTER
_d = ctypes.c_double
_i = ctypes.c_int
_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
SIGNATURES = [
    ("cl_create", _i, [_P(_vp), _i, _i, _i, _d, _d, _d, _i]),
    ("cl_destroy", None, [_vp]),
    ("cl_last_error", ctypes.c_char_p, []),
    ("cl_set_kernel_coulomb", _i, [_vp, _d, _d, _d]),
    ("cl_set_kernel_grid", _i, [_vp, _P(_d)]),
    ("cl_prepare_grid", _i, [_vp, _P(_d)]),
    ("cl_calculate_grid", _i, [_vp, _P(_d), _P(_d)]),
    ("cl_potential_grid", _i, [_vp, _P(_d)]),
    ("cl_set_states", _i, [_vp, _i, _i, _i64, _i, _P(_d), _P(_i64)]),
    ("cl_compute", _i, [_vp, _i64, _P(ctypes.c_int16), _P(_d)]),
    ("cl_compute_states", _i, [_vp, _i, _i, _i64, _i, _P(_d), _P(_i64), _i64, _P(ctypes.c_int16), _P(_d)]),
    ("cl_potentials", _i, [_vp, _P(_d)]),
    ("cl_last_timings", _i, [_vp, _P(_d)]),
    ("cl_form_info", _i, [_vp, _P(_i)]),
    ("cl_autotune_report", _i, [ctypes.c_char_p, _i64, _P(_i64)]),
    ("cl_compute_rounds", _i, [_vp, _i64, _P(ctypes.c_int16), _i, _P(_d)]),
    ("cl_set_profiling", _i, [_vp, _i]),
    ("cl_kernel_profile", _i, [_vp, _P(_d), _P(_i64), _P(_d)]),
    ("cl_request_create", _i, [_vp, _i64, _P(ctypes.c_int16), _P(_vp)]),
    ("cl_request_create_shard", _i, [_vp, _i64, _P(ctypes.c_int16), _i, _i, _P(_vp)]),
    ("cl_compute_shard", _i, [_vp, _i64, _P(ctypes.c_int16), _i, _i, _P(_d)]),
    ("cl_request_run", _i, [_vp, _P(_d)]),
    ("cl_request_destroy", None, [_vp]),
    ("cl_batch_create", _i, [_P(_vp), _i, _P(_vp)]),
    ("cl_batch_run", _i, [_vp, _P(_P(_d))]),
    ("cl_batch_last_ms", _i, [_vp, _P(_d)]),
    ("cl_batch_destroy", None, [_vp]),
    ("cl_fft3d", _i, [_i, _i, _i, _i, _i, _i, _P(_d)]),
    ("cl_fft3d_noalloc", _i, [_i, _i, _i, _i, _i, _vp]),
    ("cl_round_up_235", _i, [_i, _i]),
    ("cl_detect_grid", _i, [_P(_d), _i64, _P(_i), _P(_i), _P(_d), _P(_d), _P(_i64)]),
    ("cl_enumerate_integrals", _i, [ctypes.c_char_p, _i, _i, _P(_i64), _P(ctypes.c_int16), _i64]),
    ("cl_vertex_cover", _i, [_i, _i64, _P(ctypes.c_int32), _P(ctypes.c_uint8)]),
    ("cl_plan", _i, [_i, _i64, _P(ctypes.c_int16), _P(ctypes.c_int32)]),
    ("cl_write_integrals", _i, [ctypes.c_char_p, _i, _i, _i64, _P(ctypes.c_int16), _P(_d), _i]),
]


def lib():
    """Load libcoulombo_lattice.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libcoulombo_lattice.so is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise CoulomboError(status, lib().cl_last_error().decode())


def _ptr(a, ctype=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _cplx(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


# ----------------------------------------------------------------------------------------
# Host helpers
# ----------------------------------------------------------------------------------------

def round_up_235(n, c=1):
    r = lib().cl_round_up_235(int(n), int(c))
    if r < 0:
        _check(1)
    return r


def detect_grid(positions):
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    n = pos.shape[0]
    raw = (ctypes.c_int * 3)()
    pad = (ctypes.c_int * 3)()
    origin = (ctypes.c_double * 3)()
    step = (ctypes.c_double * 3)()
    cells = np.empty(n, dtype=np.int64)
    _check(lib().cl_detect_grid(_ptr(pos), n, raw, pad, origin, step, _ptr(cells, ctypes.c_int64)))
    return dict(raw=tuple(raw), pad=tuple(pad), origin=tuple(origin), step=tuple(step), cells=cells)


def enumerate_integrals(pattern, n_inputs, n_holes):
    count = ctypes.c_int64()
    _check(lib().cl_enumerate_integrals(pattern.encode(), n_inputs, n_holes, ctypes.byref(count), None, 0))
    specs = np.empty((count.value, 4), dtype=np.int16)
    _check(lib().cl_enumerate_integrals(pattern.encode(), n_inputs, n_holes, ctypes.byref(count),
                                        _ptr(specs, ctypes.c_int16), count.value))
    return specs


def vertex_cover(n_vertices, edges):
    e = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1, 2))
    out = np.zeros(n_vertices, dtype=np.uint8)
    _check(lib().cl_vertex_cover(n_vertices, e.shape[0], _ptr(e, ctypes.c_int32), _ptr(out, ctypes.c_uint8)))
    return {int(v) for v in np.nonzero(out)[0]}


def plan(n_inputs, specs):
    s = np.ascontiguousarray(np.asarray(specs, dtype=np.int16).reshape(-1, 4))
    steps = np.empty((s.shape[0], 5), dtype=np.int32)
    _check(lib().cl_plan(n_inputs, s.shape[0], _ptr(s, ctypes.c_int16), _ptr(steps, ctypes.c_int32)))
    return steps


def write_integrals(out_prefix, n_holes, n_electrons, specs, values, threads=0):
    """cl_write_integrals: the XXXX.txt files of coulombo.cpp:213-262 (out_prefix + class + '.txt')."""
    s = np.ascontiguousarray(np.asarray(specs, dtype=np.int16).reshape(-1, 4))
    v = np.ascontiguousarray(np.asarray(values, dtype=np.complex128)).view(np.float64)
    _check(lib().cl_write_integrals(str(out_prefix).encode(), int(n_holes), int(n_electrons), s.shape[0],
                                    _ptr(s, ctypes.c_int16), _ptr(v), int(threads)))


def autotune_report():
    """The autotuner's choices so far (cl_autotune_report), one line per pass/shape/precision."""
    need = ctypes.c_int64()
    _check(lib().cl_autotune_report(None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(int(need.value))
    _check(lib().cl_autotune_report(buf, need.value, None))
    return buf.value.decode()


def fft3d(data, sign=-1, fp32=False):
    """Unnormalised batched 3D FFT on the GPU; data [..., nz, ny, nx] complex."""
    a = _cplx(data).copy()
    nz, ny, nx = a.shape[-3:]
    batch = int(np.prod(a.shape[:-3])) if a.ndim > 3 else 1
    _check(lib().cl_fft3d(nx, ny, nz, batch, int(sign), int(bool(fp32)), _ptr(a.view(np.float64))))
    return a


def fft3d_noalloc_device(ptr, dims, batch=1, sign=-1):
    """cl_fft3d_noalloc on a caller-owned device buffer at address `ptr` (complex128,
    [batch, nz, ny, nx]), in place; the library allocates no device memory for it."""
    nx, ny, nz = dims
    _check(lib().cl_fft3d_noalloc(int(nx), int(ny), int(nz), int(batch), int(sign), ctypes.c_void_p(int(ptr))))


# ----------------------------------------------------------------------------------------
# Calculator
# ----------------------------------------------------------------------------------------

class CoulombCalculator:
    """Mirror of the reference's CoulombCalculator on one GPU.

    dims = (nx, ny, nz); step in Angstrom; grids are numpy arrays indexed [z, y, x]."""

    def __init__(self, dims, step=(1.0, 1.0, 1.0), mode=MODE_FP64_PLAIN):
        self.dims = tuple(int(d) for d in dims)
        self.mode = mode
        h = ctypes.c_void_p()
        _check(lib().cl_create(ctypes.byref(h), *self.dims, *[float(s) for s in step], mode))
        self._h = h
        self.n_atoms = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().cl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def shape(self):
        nx, ny, nz = self.dims
        return (nz, ny, nx)

    def initialize(self, dielectric=1.0, onsite=0.0, tf_lattice=0.0):
        _check(lib().cl_set_kernel_coulomb(self._h, float(dielectric), float(onsite), float(tf_lattice or 0.0)))

    def initialize_grid(self, G):
        g = np.ascontiguousarray(G, dtype=np.float64)
        nx, ny, nz = self.dims
        if g.shape != (nz + 1, ny + 1, nx + 1):
            raise ValueError("kernel grid must be (nz+1, ny+1, nx+1)")
        _check(lib().cl_set_kernel_grid(self._h, _ptr(g)))

    def prepare(self, rho):
        r = _cplx(rho)
        if r.shape != self.shape:
            raise ValueError("density must be indexed [z, y, x]")
        _check(lib().cl_prepare_grid(self._h, _ptr(r.view(np.float64))))

    def calculate(self, rho2):
        r = _cplx(rho2)
        if r.shape != self.shape:
            raise ValueError("density must be indexed [z, y, x]")
        out = np.zeros(2)
        _check(lib().cl_calculate_grid(self._h, _ptr(r.view(np.float64)), _ptr(out)))
        return complex(out[0], out[1])

    def potential(self):
        v = np.empty(self.shape, dtype=np.complex128)
        _check(lib().cl_potential_grid(self._h, _ptr(v.view(np.float64))))
        return v

    def set_states(self, states, cells, n_holes):
        """states: [n_states, n_atoms, n_orb] complex (input order, holes first)."""
        c = _cplx(states)
        cl = np.ascontiguousarray(cells, dtype=np.int64)
        n, a, o = c.shape
        _check(lib().cl_set_states(self._h, n, int(n_holes), a, o, _ptr(c.view(np.float64)),
                                   _ptr(cl, ctypes.c_int64)))
        self.n_states, self.n_atoms = n, a

    def compute(self, specs):
        s = np.ascontiguousarray(np.asarray(specs, dtype=np.int16).reshape(-1, 4))
        out = np.zeros(2 * s.shape[0])
        _check(lib().cl_compute(self._h, s.shape[0], _ptr(s, ctypes.c_int16), _ptr(out)))
        return out[0::2] + 1j * out[1::2]

    def compute_states(self, states, cells, n_holes, specs):
        """cl_compute_states: set_states + compute in one call, the coefficient upload
        overlapped with the transforms."""
        c = _cplx(states)
        cl_ = np.ascontiguousarray(cells, dtype=np.int64)
        n, a, o = c.shape
        s = np.ascontiguousarray(np.asarray(specs, dtype=np.int16).reshape(-1, 4))
        out = np.zeros(2 * s.shape[0])
        _check(lib().cl_compute_states(self._h, n, int(n_holes), a, o, _ptr(c.view(np.float64)),
                                       _ptr(cl_, ctypes.c_int64), s.shape[0], _ptr(s, ctypes.c_int16), _ptr(out)))
        self.n_states, self.n_atoms = n, a
        return out[0::2] + 1j * out[1::2]

    def compute_states_raw(self, n_states, n_holes, n_atoms, n_orb, coeff_ptr, cells_ptr, n_int, spec_ptr,
                           out_ptr):
        """cl_compute_states on raw host addresses (e.g. pinned buffers)."""
        _check(lib().cl_compute_states(self._h, int(n_states), int(n_holes), int(n_atoms), int(n_orb),
                                       ctypes.cast(coeff_ptr, ctypes.POINTER(ctypes.c_double)),
                                       ctypes.cast(cells_ptr, ctypes.POINTER(ctypes.c_int64)), int(n_int),
                                       ctypes.cast(spec_ptr, ctypes.POINTER(ctypes.c_int16)),
                                       ctypes.cast(out_ptr, ctypes.POINTER(ctypes.c_double))))
        self.n_states, self.n_atoms = int(n_states), int(n_atoms)

    def compute_rounds(self, specs, round_mask):
        """Partial integrals over the rounds in round_mask (bit k = round kappa k)."""
        s = np.ascontiguousarray(np.asarray(specs, dtype=np.int16).reshape(-1, 4))
        out = np.zeros(2 * s.shape[0])
        _check(lib().cl_compute_rounds(self._h, s.shape[0], _ptr(s, ctypes.c_int16), int(round_mask), _ptr(out)))
        return out[0::2] + 1j * out[1::2]

    def compute_shard(self, specs, shard, n_shards):
        """cl_compute_shard: the integrals whose left density is dealt to `shard` of `n_shards`
        (zeros elsewhere); the shards' results add up to compute()'s."""
        s = np.ascontiguousarray(np.asarray(specs, dtype=np.int16).reshape(-1, 4))
        out = np.zeros(2 * s.shape[0])
        _check(lib().cl_compute_shard(self._h, s.shape[0], _ptr(s, ctypes.c_int16), int(shard), int(n_shards),
                                      _ptr(out)))
        return out[0::2] + 1j * out[1::2]

    def set_profiling(self, on=True):
        _check(lib().cl_set_profiling(self._h, int(bool(on))))

    def kernel_profile(self):
        """{class: (ms, launches, algorithmic bytes)} since profiling was switched on."""
        k = len(KERNEL_CLASSES)
        ms = np.zeros(k)
        n = np.zeros(k, dtype=np.int64)
        b = np.zeros(k)
        _check(lib().cl_kernel_profile(self._h, _ptr(ms), _ptr(n, ctypes.c_int64), _ptr(b)))
        return {KERNEL_CLASSES[k]: (float(ms[k]), int(n[k]), float(b[k])) for k in range(len(KERNEL_CLASSES)) if n[k]}

    def set_states_raw(self, n_states, n_holes, n_atoms, n_orb, coeff_ptr, cells_ptr):
        """cl_set_states on raw host addresses (e.g. pinned buffers)."""
        _check(lib().cl_set_states(self._h, int(n_states), int(n_holes), int(n_atoms), int(n_orb),
                                   ctypes.cast(coeff_ptr, ctypes.POINTER(ctypes.c_double)),
                                   ctypes.cast(cells_ptr, ctypes.POINTER(ctypes.c_int64))))
        self.n_states, self.n_atoms = n_states, n_atoms

    def compute_raw_shard(self, n_int, spec_ptr, shard, n_shards, out_ptr):
        """cl_compute_shard on raw host addresses (e.g. pinned buffers)."""
        _check(lib().cl_compute_shard(self._h, int(n_int), ctypes.cast(spec_ptr, ctypes.POINTER(ctypes.c_int16)),
                                      int(shard), int(n_shards), ctypes.cast(out_ptr, ctypes.POINTER(ctypes.c_double))))

    def compute_raw(self, n_int, spec_ptr, out_ptr):
        _check(lib().cl_compute(self._h, int(n_int), ctypes.cast(spec_ptr, ctypes.POINTER(ctypes.c_int16)),
                                ctypes.cast(out_ptr, ctypes.POINTER(ctypes.c_double))))

    def request(self, specs, shard=0, n_shards=1):
        """A prepared request (Request) for repeated runs of the same integral list (of one shard
        of it, see compute_shard)."""
        return Request(self, specs, shard, n_shards)

    def potentials(self):
        out = np.zeros((self.n_states, self.n_atoms))
        _check(lib().cl_potentials(self._h, _ptr(out)))
        return out

    def form_info(self):
        """cl_form_info: which decomposition the loaded states run (sub-lattice or 8 rounds)."""
        info = (ctypes.c_int * 8)()
        _check(lib().cl_form_info(self._h, info))
        return dict(sublattice=bool(info[0]), m=info[1], classes=info[2], zincblende=bool(info[3]),
                    lengths=(info[4], info[5], info[6]), class_kernels=info[7])

    def timings(self):
        t = np.zeros(4)
        _check(lib().cl_last_timings(self._h, _ptr(t)))
        return dict(densities_ms=t[0], transforms_ms=t[1], reductions_ms=t[2], total_ms=t[3])


class Request:
    """cl_request: plan, device buffers and pinned results prepared once; run() enqueues only."""

    def __init__(self, calc, specs, shard=0, n_shards=1):
        self.calc = calc
        self.specs = np.ascontiguousarray(np.asarray(specs, dtype=np.int16).reshape(-1, 4))
        h = ctypes.c_void_p()
        _check(lib().cl_request_create_shard(calc._h, self.specs.shape[0], _ptr(self.specs, ctypes.c_int16),
                                             int(shard), int(n_shards), ctypes.byref(h)))
        self._h = h
        self.out = np.zeros(2 * self.specs.shape[0])

    def run(self):
        _check(lib().cl_request_run(self._h, _ptr(self.out)))
        return self.out[0::2] + 1j * self.out[1::2]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().cl_request_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """cl_batch: requests on distinct contexts, captured once as one CUDA graph and replayed."""

    def __init__(self, requests):
        self.requests = list(requests)
        arr = (ctypes.c_void_p * len(self.requests))(*[r._h.value for r in self.requests])
        h = ctypes.c_void_p()
        _check(lib().cl_batch_create(arr, len(self.requests), ctypes.byref(h)))
        self._h = h
        self._outs = (ctypes.POINTER(ctypes.c_double) * len(self.requests))(
            *[_ptr(r.out) for r in self.requests])

    def run(self):
        _check(lib().cl_batch_run(self._h, self._outs))
        return [r.out[0::2] + 1j * r.out[1::2] for r in self.requests]

    def last_ms(self):
        ms = ctypes.c_double()
        _check(lib().cl_batch_last_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().cl_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
