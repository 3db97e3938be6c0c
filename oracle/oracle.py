"""numpy front end of the CPU checkers.  TEST INFRASTRUCTURE.

Two libraries are wrapped:

* ``libloits_oracle.so`` -- the plain-C restatement of the reference algorithm
  (``loits_oracle.c``; every function cites the reference file:line it
  follows).  :class:`Oracle` exposes the reference 2-D tuple path
  (``r_forward`` / ``r_backward``) and the batched 1-D density path
  (``d_forward`` / ``d_backward`` / ``d_fd`` / ``d_quantile``).
* ``_ref/libloits_ref_{cpp,openmp}.so`` -- the reference's own
  ``cpp/loits_core.cpp`` / ``openmp/loits_core.cpp`` compiled from the
  reference tree by ``oracle/Makefile`` behind ``ref_shim.cpp``.
  :class:`Reference` runs the exact stage sequence of ``cpp/bindings.cpp``.

Nothing here touches a GPU or the CUDA product library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "libloits_oracle.so"
REF_DIR = HERE / "_ref"
# The reference project's source tree: LOITS_REFERENCE_TREE, else the
# `reference` directory beside this repository's root.
REFERENCE_TREE = Path(os.environ.get("LOITS_REFERENCE_TREE", str(HERE.parent.parent / "reference")))

_i64 = C.c_int64
_u64 = C.c_uint64
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_lp = C.POINTER(C.c_int64)
_sp = C.POINTER(C.c_int16)
_ip = C.POINTER(C.c_int32)
_bp = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree is present, the
    reference cores) with ``make`` in this directory."""
    targets = ["oracle"]
    if ref and (REFERENCE_TREE / "cpp" / "loits_core.cpp").exists():
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REFERENCE_TREE}", *targets], check=True)


def _ptr(a: np.ndarray | None, ctype):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle buffers must be C-contiguous"
    return a.ctypes.data_as(ctype)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i64a(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


class _Shape(C.Structure):
    _fields_ = [("batch", _i64), ("nx", _i64), ("ny", _i64), ("kx", _i64), ("kq", _i64)]


def shape_of(x_bins: np.ndarray, q_bins: np.ndarray) -> tuple[int, int, int, int, int]:
    """(batch, nx, ny, kx, kq) of a reference theory tuple (cpp/bindings.cpp:36-37)."""
    return (x_bins.shape[0], x_bins.shape[1], q_bins.shape[1], x_bins.shape[2], q_bins.shape[2])


class Oracle:
    """Plain-C restatement of the reference algorithm (fp64, no contraction)."""

    def __init__(self, path: Path = ORACLE_LIB):
        if not Path(path).exists():
            build(ref=False)
        lib = C.CDLL(str(path))
        lib.oracle_philox4x32_10.argtypes = [_u64, _u64, _u64, _u32p]
        lib.oracle_uniform_float.argtypes = [C.c_uint32]
        lib.oracle_uniform_float.restype = C.c_float
        lib.oracle_fill_uniform.argtypes = [_fp, _i64, _u64, _u64]
        lib.oracle_r_allocate.argtypes = [C.POINTER(_Shape), _dp, _i64, _lp, _lp, _lp]
        lib.oracle_r_cdf.argtypes = [C.POINTER(_Shape), C.c_int, _dp, _dp, _bp, _dp, _dp]
        lib.oracle_r_sample.argtypes = [C.POINTER(_Shape), _dp, _dp, _dp, _dp, _lp, _i64, _u64,
                                        _u64, _dp, _lp, _sp, _sp]
        lib.oracle_r_sample.restype = _i64
        lib.oracle_r_backward.argtypes = [C.POINTER(_Shape), _dp, _lp, _i64, _i64, _u64, _u64,
                                          _dp, _dp, _dp, _dp, _bp, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.oracle_d_nmax.argtypes = [_i64, _lp]
        lib.oracle_d_nmax.restype = _i64
        lib.oracle_d_cdf.argtypes = [_i64, _lp, _dp, _dp, _dp, _dp, _bp]
        lib.oracle_d_sample.argtypes = [_i64, _lp, _lp, _dp, _dp, _bp, _dp, _u64, _u64, _i64, _i64,
                                        _dp, _lp, _ip, _fp, _lp]
        lib.oracle_d_sample.restype = _i64
        lib.oracle_d_quantile.argtypes = [_i64, _lp, _dp, _dp, _dp, _i64, _dp, _ip]
        lib.oracle_d_backward.argtypes = [_i64, _lp, _lp, _dp, _dp, _dp, _dp, _bp, _dp, _u64, _u64,
                                          _i64, _i64, _dp, _dp]
        lib.oracle_d_fd.argtypes = [_i64, _i64, _i64, C.c_double, _lp, _lp, _dp, _dp, _dp, _u64,
                                    _u64, _dp, _lp]
        lib.oracle_d_fd.restype = C.c_double
        self.lib = lib

    # -- RNG ---------------------------------------------------------------
    def philox(self, block: int, stream: int, seed: int) -> list[int]:
        out = (C.c_uint32 * 4)()
        self.lib.oracle_philox4x32_10(block, stream, seed, out)
        return list(out)

    def fill_uniform(self, count: int, seed: int, stream: int) -> np.ndarray:
        out = np.empty(count, dtype=np.float32)
        self.lib.oracle_fill_uniform(_ptr(out, _fp), count, seed, stream)
        return out

    # -- reference 2-D tuple ----------------------------------------------
    def r_forward(self, x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events, seed,
                  sequence):
        """Returns dict(events (valid,2), packed, interval_x, interval_q, norm_x, norm_q,
        cdf_x, cdf_q, counts, nmax, active)."""
        x_bins, xsec_x, q_bins, xsec_q, weights = map(_f64, (x_bins, xsec_x, q_bins, xsec_q, weights))
        acc = np.ascontiguousarray(np.asarray(acceptance).astype(np.uint8))
        s = _Shape(*shape_of(x_bins, q_bins))
        B, nx, ny, kx, kq = shape_of(x_bins, q_bins)
        counts = np.empty(B * nx * ny, dtype=np.int64)
        nmax, active = _i64(), _i64()
        self.lib.oracle_r_allocate(C.byref(s), _ptr(weights, _dp), int(n_events), _ptr(counts, _lp),
                                   C.byref(nmax), C.byref(active))
        norm_x = np.empty((B, ny, nx)); norm_q = np.empty((B, nx, ny))
        cdf_x = np.empty_like(xsec_x); cdf_q = np.empty_like(xsec_q)
        self.lib.oracle_r_cdf(C.byref(s), 0, _ptr(x_bins, _dp), _ptr(xsec_x, _dp), _ptr(acc, _bp),
                              _ptr(norm_x, _dp), _ptr(cdf_x, _dp))
        self.lib.oracle_r_cdf(C.byref(s), 1, _ptr(q_bins, _dp), _ptr(xsec_q, _dp), _ptr(acc, _bp),
                              _ptr(norm_q, _dp), _ptr(cdf_q, _dp))
        n_act = max(active.value, 1)
        events = np.empty((n_act, 2)); packed = np.empty(n_act, dtype=np.int64)
        ix = np.empty(n_act, dtype=np.int16); iq = np.empty(n_act, dtype=np.int16)
        valid = self.lib.oracle_r_sample(C.byref(s), _ptr(x_bins, _dp), _ptr(q_bins, _dp),
                                         _ptr(cdf_x, _dp), _ptr(cdf_q, _dp), _ptr(counts, _lp),
                                         nmax.value, seed, sequence, _ptr(events, _dp),
                                         _ptr(packed, _lp), _ptr(ix, _sp), _ptr(iq, _sp))
        return dict(events=events[:valid], packed=packed[:valid], interval_x=ix[:valid],
                    interval_q=iq[:valid], norm_x=norm_x, norm_q=norm_q, cdf_x=cdf_x, cdf_q=cdf_q,
                    counts=counts.reshape(B, nx * ny), nmax=nmax.value, active=active.value)

    def r_backward(self, grad_events, state, x_bins, xsec_x, q_bins, xsec_q, acceptance, seed,
                   sequence):
        x_bins, xsec_x, q_bins, xsec_q = map(_f64, (x_bins, xsec_x, q_bins, xsec_q))
        g = _f64(grad_events).reshape(-1, 2)
        acc = np.ascontiguousarray(np.asarray(acceptance).astype(np.uint8))
        s = _Shape(*shape_of(x_bins, q_bins))
        packed = _i64a(state["packed"])
        gx = np.empty_like(xsec_x); gq = np.empty_like(xsec_q)
        self.lib.oracle_r_backward(C.byref(s), _ptr(g, _dp), _ptr(packed, _lp), len(packed),
                                   state["nmax"], seed, sequence, _ptr(x_bins, _dp),
                                   _ptr(xsec_x, _dp), _ptr(q_bins, _dp), _ptr(xsec_q, _dp),
                                   _ptr(acc, _bp), _ptr(_f64(state["norm_x"]), _dp),
                                   _ptr(_f64(state["norm_q"]), _dp), _ptr(_f64(state["cdf_x"]), _dp),
                                   _ptr(_f64(state["cdf_q"]), _dp), _ptr(gx, _dp), _ptr(gq, _dp))
        return gx, gq

    # -- batched 1-D densities --------------------------------------------
    def d_cdf(self, knot_offsets, grid, values):
        koff = _i64a(knot_offsets); grid = _f64(grid); values = _f64(values)
        nd = len(koff) - 1
        norm = np.empty(nd); cdf = np.empty_like(values); mono = np.empty(nd, dtype=np.uint8)
        self.lib.oracle_d_cdf(nd, _ptr(koff, _lp), _ptr(grid, _dp), _ptr(values, _dp),
                              _ptr(norm, _dp), _ptr(cdf, _dp), _ptr(mono, _bp))
        return norm, cdf, mono

    def d_forward(self, knot_offsets, event_offsets, grid, values, x_cut, seed, sequence,
                  density_base=0, slot_stride=0):
        """Returns dict(events, row_offsets, intervals, u, slots, norm, cdf, monotone).
        Slot s of density b draws counter (density_base + b) * stride + s,
        stride = slot_stride or max n_b."""
        koff = _i64a(knot_offsets); eoff = _i64a(event_offsets)
        grid = _f64(grid); values = _f64(values)
        nd = len(koff) - 1
        norm, cdf, mono = self.d_cdf(koff, grid, values)
        cap = max(int(eoff[-1]), 1)
        events = np.empty(cap); rows = np.empty(nd + 1, dtype=np.int64)
        ints = np.empty(cap, dtype=np.int32); u = np.empty(cap, dtype=np.float32)
        slots = np.empty(cap, dtype=np.int64)
        xc = None if x_cut is None else _f64(x_cut)
        valid = self.lib.oracle_d_sample(nd, _ptr(koff, _lp), _ptr(eoff, _lp), _ptr(grid, _dp),
                                         _ptr(cdf, _dp), _ptr(mono, _bp), _ptr(xc, _dp), seed,
                                         sequence, int(density_base), int(slot_stride),
                                         _ptr(events, _dp), _ptr(rows, _lp),
                                         _ptr(ints, _ip), _ptr(u, _fp), _ptr(slots, _lp))
        return dict(events=events[:valid], row_offsets=rows, intervals=ints[:valid], u=u[:valid],
                    slots=slots[:valid], norm=norm, cdf=cdf, monotone=mono)

    def d_backward(self, knot_offsets, event_offsets, grid, values, x_cut, seed, sequence,
                   grad_events, fwd=None, density_base=0, slot_stride=0):
        koff = _i64a(knot_offsets); eoff = _i64a(event_offsets)
        grid = _f64(grid); values = _f64(values)
        nd = len(koff) - 1
        if fwd is None:
            norm, cdf, mono = self.d_cdf(koff, grid, values)
        else:
            norm, cdf, mono = fwd["norm"], fwd["cdf"], fwd["monotone"]
        g = _f64(grad_events)
        out = np.empty_like(values)
        xc = None if x_cut is None else _f64(x_cut)
        self.lib.oracle_d_backward(nd, _ptr(koff, _lp), _ptr(eoff, _lp), _ptr(grid, _dp),
                                   _ptr(values, _dp), _ptr(_f64(norm), _dp), _ptr(_f64(cdf), _dp),
                                   _ptr(np.ascontiguousarray(mono), _bp), _ptr(xc, _dp), seed,
                                   sequence, int(density_base), int(slot_stride), _ptr(g, _dp),
                                   _ptr(out, _dp))
        return out

    def d_fd(self, density, knot, h, knot_offsets, event_offsets, grid, values, x_cut, seed,
             sequence, g_rows):
        """Branch-frozen central difference; returns (derivative, flips)."""
        koff = _i64a(knot_offsets); eoff = _i64a(event_offsets)
        grid = _f64(grid); values = _f64(values); g = _f64(g_rows)
        xc = None if x_cut is None else _f64(x_cut)
        flips = _i64()
        d = self.lib.oracle_d_fd(len(koff) - 1, density, knot, float(h), _ptr(koff, _lp),
                                 _ptr(eoff, _lp), _ptr(grid, _dp), _ptr(values, _dp), _ptr(xc, _dp),
                                 seed, sequence, _ptr(g, _dp), C.byref(flips))
        return d, flips.value

    def d_quantile(self, density, knot_offsets, grid, cdf, u):
        koff = _i64a(knot_offsets); grid = _f64(grid); cdf = _f64(cdf); u = _f64(u)
        x = np.empty_like(u); ints = np.empty(len(u), dtype=np.int32)
        self.lib.oracle_d_quantile(density, _ptr(koff, _lp), _ptr(grid, _dp), _ptr(cdf, _dp),
                                   _ptr(u, _dp), len(u), _ptr(x, _dp), _ptr(ints, _ip))
        return x, ints


class Reference:
    """The reference's own compiled core (``cpp`` or ``openmp``) behind the
    stage sequence of cpp/bindings.cpp:24-208."""

    def __init__(self, kind: str = "cpp"):
        path = REF_DIR / f"libloits_ref_{kind}.so"
        if not path.exists():
            build(ref=True)
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (reference tree absent)")
        lib = C.CDLL(str(path))
        lib.ref_allocate.argtypes = [_lp, _dp, _i64, _lp, _lp, _lp]
        lib.ref_forward.argtypes = [_lp, _dp, _dp, _dp, _dp, _bp, _lp, _i64, _u64, _u64, _dp, _dp,
                                    _dp, _dp, _fp, _fp, _sp, _sp, _dp, _lp, _lp]
        lib.ref_forward.restype = _i64
        lib.ref_backward.argtypes = [_lp, _dp, _dp, _dp, _dp, _dp, _bp, _dp, _dp, _dp, _dp, _fp,
                                     _fp, _sp, _sp, _lp, _i64, _lp, _i64, _dp, _dp]
        lib.ref_set_threads.argtypes = [C.c_int]
        lib.ref_max_threads.restype = C.c_int
        self.lib = lib
        self.kind = kind

    def set_threads(self, n: int) -> None:
        self.lib.ref_set_threads(int(n))

    def max_threads(self) -> int:
        return int(self.lib.ref_max_threads())

    def forward(self, x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events, seed,
                sequence):
        """Mirror of the pybind ``forward`` (cpp/bindings.cpp:24-130); returns a dict with
        the same state the reference returns."""
        x_bins, xsec_x, q_bins, xsec_q, weights = map(_f64, (x_bins, xsec_x, q_bins, xsec_q, weights))
        acc = np.ascontiguousarray(np.asarray(acceptance).astype(np.uint8))
        B, nx, ny, kx, kq = shape_of(x_bins, q_bins)
        dims = np.array([B, nx, ny, kx, kq], dtype=np.int64)
        counts = np.empty(B * nx * ny, dtype=np.int64)
        nmax, active = _i64(), _i64()
        self.lib.ref_allocate(_ptr(dims, _lp), _ptr(weights, _dp), int(n_events), _ptr(counts, _lp),
                              C.byref(nmax), C.byref(active))
        total = B * nx * ny * nmax.value
        norm_x = np.empty((B, ny, nx)); norm_q = np.empty((B, nx, ny))
        cdf_x = np.empty_like(xsec_x); cdf_q = np.empty_like(xsec_q)
        u_x = np.empty(max(total, 1), dtype=np.float32); u_q = np.empty_like(u_x)
        i_x = np.zeros(max(total, 1), dtype=np.int16); i_q = np.zeros_like(i_x)
        n_act = max(active.value, 1)
        events = np.empty((n_act, 2)); packed = np.empty(n_act, dtype=np.int64)
        row_offsets = np.zeros(B * nx * ny + 1, dtype=np.int64)
        valid = self.lib.ref_forward(_ptr(dims, _lp), _ptr(x_bins, _dp), _ptr(xsec_x, _dp),
                                     _ptr(q_bins, _dp), _ptr(xsec_q, _dp), _ptr(acc, _bp),
                                     _ptr(counts, _lp), nmax.value, seed, sequence,
                                     _ptr(norm_x, _dp), _ptr(norm_q, _dp), _ptr(cdf_x, _dp),
                                     _ptr(cdf_q, _dp), _ptr(u_x, _fp), _ptr(u_q, _fp),
                                     _ptr(i_x, _sp), _ptr(i_q, _sp), _ptr(events, _dp),
                                     _ptr(packed, _lp), _ptr(row_offsets, _lp))
        return dict(events=events[:valid], norm_x=norm_x, norm_q=norm_q, cdf_x=cdf_x, cdf_q=cdf_q,
                    u_x=u_x[:total].reshape(B, nx * ny, nmax.value),
                    u_q=u_q[:total].reshape(B, nx * ny, nmax.value), interval_x=i_x[:total],
                    interval_q=i_q[:total], packed=packed[:valid], row_offsets=row_offsets,
                    counts=counts.reshape(B, nx * ny), nmax=nmax.value, active=active.value)

    def backward(self, grad_events, state, x_bins, xsec_x, q_bins, xsec_q, acceptance):
        x_bins, xsec_x, q_bins, xsec_q = map(_f64, (x_bins, xsec_x, q_bins, xsec_q))
        acc = np.ascontiguousarray(np.asarray(acceptance).astype(np.uint8))
        B, nx, ny, kx, kq = shape_of(x_bins, q_bins)
        dims = np.array([B, nx, ny, kx, kq], dtype=np.int64)
        g = _f64(grad_events).reshape(-1, 2)
        gx = np.empty_like(xsec_x); gq = np.empty_like(xsec_q)
        packed = _i64a(state["packed"])
        self.lib.ref_backward(_ptr(dims, _lp), _ptr(g, _dp), _ptr(x_bins, _dp), _ptr(xsec_x, _dp),
                              _ptr(q_bins, _dp), _ptr(xsec_q, _dp), _ptr(acc, _bp),
                              _ptr(_f64(state["norm_x"]), _dp), _ptr(_f64(state["norm_q"]), _dp),
                              _ptr(_f64(state["cdf_x"]), _dp), _ptr(_f64(state["cdf_q"]), _dp),
                              _ptr(np.ascontiguousarray(state["u_x"]).reshape(-1), _fp),
                              _ptr(np.ascontiguousarray(state["u_q"]).reshape(-1), _fp),
                              _ptr(state["interval_x"], _sp), _ptr(state["interval_q"], _sp),
                              _ptr(packed, _lp), len(packed), _ptr(_i64a(state["row_offsets"]), _lp),
                              state["nmax"], _ptr(gx, _dp), _ptr(gq, _dp))
        return gx, gq


def embed_densities(knot_offsets, grid, values, event_counts):
    """Exact embedding of B 1-D densities into the reference's 2-D tuple.

    Density b becomes batch entry b of a one-cell theory (nx = ny = 1): its
    knots are the x curve (padded to the longest density by repeating the last
    knot, which adds zero trapezoid area and never changes an interval or a
    value), the q curve is the constant 1 on [1e-3, 1] (finite and non-zero, so
    the reference predicate x * q != 0 reduces to x != 0), weight (n_b + 0.5)/N
    with n_events = N = max n_b gives trunc(w * N) = n_b events.  The counter of
    slot s of density b is then b * N + s, as in the batched sampler.
    """
    koff = _i64a(knot_offsets)
    grid = np.asarray(grid, dtype=np.float64); values = np.asarray(values, dtype=np.float64)
    counts = _i64a(event_counts)
    nd = len(koff) - 1
    kmax = int(np.max(np.diff(koff)))
    x_bins = np.empty((nd, 1, kmax)); xsec_x = np.empty((nd, 1, 1, kmax))
    for b in range(nd):
        o, k = koff[b], koff[b + 1] - koff[b]
        x_bins[b, 0, :k] = grid[o:o + k]; x_bins[b, 0, k:] = grid[o + k - 1]
        xsec_x[b, 0, 0, :k] = values[o:o + k]; xsec_x[b, 0, 0, k:] = values[o + k - 1]
    q_bins = np.tile(np.array([1e-3, 1.0]), (nd, 1, 1))
    xsec_q = np.ones((nd, 1, 1, 2))
    n_events = int(counts.max()) if nd else 0
    weights = ((counts + 0.5) / max(n_events, 1)).reshape(nd, 1, 1)
    acceptance = np.ones((nd, 1, 1), dtype=bool)
    return x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events
