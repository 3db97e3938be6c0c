"""``LOITS(backend="cuda")``: the B200 sampler behind the reference's backend API.

``CudaLOITS(device, compile, profile_regions, epsilon)`` has the constructor
contract of the reference's native backends (cpp/backend.py:74-101): the
Philox seed is ``torch.initial_seed()`` at construction, ``sequence`` starts
at 0 and increases by one per call, and any epsilon other than the reference's
1e-5 raises ``ValueError`` (cpp/backend.py:78-79).  Its call
``sampler(theory_outputs, n_events)`` returns a float64 ``(valid, 2)`` tensor of
events on the input device whose gradient flows to ``xsec_x`` and ``xsec_q2``
only (cpp/backend.py:57-71).  Passing a :class:`~quantom_loits_b200.batched.DensityBatch`
instead of the theory tuple samples a ragged batch of 1-D densities.

``native_forward`` / ``native_backward`` mirror the reference's pybind
``forward`` / ``backward`` (cpp/bindings.cpp:24-208) state by state, for
parity harnesses such as compare_backend_torch.py: the returned list is
``[events, norm_x, norm_q, cdf_x, cdf_q, u_x, u_q, interval_x, interval_q,
packed]``.  The sampler itself never materialises ``u_x``/``u_q``: its
backward regenerates them from (seed, sequence).

Region names (``profile_regions=True``): ``loits::autograd::{forward,backward}``,
``loits::binding::{forward,backward}``, ``loits::{forward,backward}`` as in the
reference; inside them the fused launches are ``loits::forward::prepare``
(allocation + rho + cdf, cpp/bindings.cpp:39-77),
``loits::forward::sample`` (random + interpolation + stream_compaction,
:79-124), ``loits::forward::state_pack`` and ``loits::backward::fused``
(:154-202).
"""
from __future__ import annotations

import ctypes as C
import math
from contextlib import contextmanager, nullcontext

import torch
from torch import nn
from torch.profiler import record_function

from . import _native as N


def availability(device):
    """(ok, reason): a CUDA device of compute capability 10.x and the built library."""
    device = torch.device(device)
    if device.type != "cuda":
        return False, "the cuda backend runs on CUDA devices only"
    if not torch.cuda.is_available():
        return False, "PyTorch CUDA is not available"
    index = device.index if device.index is not None else torch.cuda.current_device()
    major, minor = torch.cuda.get_device_capability(index)
    if major != 10:
        return False, f"needs compute capability 10.x (sm_100a); device {index} is {major}.{minor}"
    if not N.LIB_PATH.exists():
        return False, f"{N.LIB_PATH.name} is not built (python -m quantom_loits_b200.build)"
    return True, ""


@contextmanager
def _region(enabled: bool, name: str, device=None):
    if not enabled:
        yield
        return
    with record_function(name):
        yield
        if device is not None:
            torch.cuda.synchronize(device)


def _check_tuple(x_bins, xsec_x, q_bins, xsec_q, weights, acceptance):
    tensors = (x_bins, xsec_x, q_bins, xsec_q, weights)
    dev = x_bins.device
    N.require_device(dev)
    for name, t in zip(("x_bins", "xsec_x", "q2_bins", "xsec_q2", "weights"), tensors):
        if t.dtype != torch.float64:
            raise TypeError(f"{name} must be float64, got {t.dtype}")
        if t.device != dev:
            raise ValueError(f"{name} is on {t.device}, expected {dev}")
        if not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
    if acceptance.dtype != torch.bool or acceptance.device != dev or not acceptance.is_contiguous():
        raise TypeError("acceptance must be a contiguous bool tensor on the same device")
    if x_bins.dim() != 3 or q_bins.dim() != 3:
        raise ValueError("x_bins and q2_bins must be (batch, cells, knots)")
    B, nx, kx = x_bins.shape
    ny, kq = q_bins.shape[1], q_bins.shape[2]
    expect = {"xsec_x": (B, ny, nx, kx), "q2_bins": (B, ny, kq), "xsec_q2": (B, nx, ny, kq),
              "weights": (B, nx, ny), "acceptance": (B, nx, ny)}
    got = {"xsec_x": tuple(xsec_x.shape), "q2_bins": tuple(q_bins.shape),
           "xsec_q2": tuple(xsec_q.shape), "weights": tuple(weights.shape),
           "acceptance": tuple(acceptance.shape)}
    for k, v in expect.items():
        if got[k] != v:
            raise ValueError(f"{k} has shape {got[k]}, expected {v}")
    return N.Shape(B, nx, ny, kx, kq)


def tuple_forward(x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events, seed, sequence,
                  profile_regions=False, want_intervals=False):
    """Sample the reference theory tuple; returns (events, state dict)."""
    shape = _check_tuple(x_bins, xsec_x, q_bins, xsec_q, weights, acceptance)
    n_events = int(n_events)
    if n_events < 0:
        raise ValueError("n_events must be >= 0")
    dev = x_bins.device
    lib = N.lib()
    B, nx, ny, kx, kq = shape.batch, shape.nx, shape.ny, shape.kx, shape.kq
    ncell = B * nx * ny
    f64 = dict(dtype=torch.float64, device=dev)
    i64 = dict(dtype=torch.int64, device=dev)
    with torch.cuda.device(dev), _region(profile_regions, "loits::forward", dev):
        stream = N.stream_of(dev)
        with _region(profile_regions, "loits::forward::prepare", dev):
            counts = torch.empty(ncell, **i64)
            cell_offsets = torch.empty(ncell + 1, **i64)
            norm_x = torch.empty((B, ny, nx), **f64)
            norm_q = torch.empty((B, nx, ny), **f64)
            cdf_x = torch.empty_like(xsec_x)
            cdf_q = torch.empty_like(xsec_q)
            alloc = torch.empty(2, **i64)
            acc_u8 = acceptance.view(torch.uint8)
            N.check(lib.loits_tuple_prepare(C.byref(shape), x_bins.data_ptr(), xsec_x.data_ptr(),
                                            q_bins.data_ptr(), xsec_q.data_ptr(),
                                            weights.data_ptr(), acc_u8.data_ptr(), n_events,
                                            counts.data_ptr(), cell_offsets.data_ptr(),
                                            norm_x.data_ptr(), norm_q.data_ptr(), cdf_x.data_ptr(),
                                            cdf_q.data_ptr(), alloc.data_ptr(), stream),
                    "loits_tuple_prepare")
            nmax, active = (int(v) for v in alloc.tolist())
        with _region(profile_regions, "loits::forward::sample", dev):
            cap = max(active, 1)
            events = torch.empty((cap, 2), **f64)
            packed = torch.empty(cap, **i64)
            ix = torch.empty(cap, dtype=torch.int16, device=dev) if want_intervals else None
            iq = torch.empty(cap, dtype=torch.int16, device=dev) if want_intervals else None
            out = torch.zeros(2, **i64)  # [valid, status (int32 in the low word)]
            ws_bytes = int(lib.loits_tuple_sample_workspace(active))
            ws = torch.empty(max(ws_bytes, 16), dtype=torch.uint8, device=dev)
            N.check(lib.loits_tuple_sample(C.byref(shape), x_bins.data_ptr(), q_bins.data_ptr(),
                                           cdf_x.data_ptr(), cdf_q.data_ptr(),
                                           cell_offsets.data_ptr(), nmax, active, int(seed),
                                           int(sequence), events.data_ptr(), packed.data_ptr(),
                                           N.ptr(ix), N.ptr(iq), out[0:1].data_ptr(),
                                           out[1:2].data_ptr(), ws.data_ptr(), ws.numel(), stream),
                    "loits_tuple_sample")
            valid, status = (int(v) for v in out.tolist())
            N.check(status, "loits_tuple_sample (device)")
        with _region(profile_regions, "loits::forward::state_pack"):
            state = dict(norm_x=norm_x, norm_q=norm_q, cdf_x=cdf_x, cdf_q=cdf_q,
                         packed=packed[:valid], nmax=nmax, active=active, counts=counts,
                         interval_x=None if ix is None else ix[:valid],
                         interval_q=None if iq is None else iq[:valid])
    return events[:valid], state


def tuple_backward(grad_events, x_bins, xsec_x, q_bins, xsec_q, acceptance, state, seed, sequence,
                   profile_regions=False):
    """d(sum grad_events * events)/d(xsec_x, xsec_q2) for a tuple_forward result."""
    shape = _check_tuple(x_bins, xsec_x, q_bins, xsec_q, x_bins.new_empty(
        (x_bins.shape[0], x_bins.shape[1], q_bins.shape[1])), acceptance)
    dev = x_bins.device
    packed = state["packed"]
    g = grad_events.to(dtype=torch.float64).contiguous()
    if g.shape != (packed.numel(), 2):
        raise ValueError(f"grad_events has shape {tuple(g.shape)}, expected ({packed.numel()}, 2)")
    lib = N.lib()
    with torch.cuda.device(dev), _region(profile_regions, "loits::backward", dev):
        gx = torch.empty_like(xsec_x)
        gq = torch.empty_like(xsec_q)
        with _region(profile_regions, "loits::backward::fused", dev):
            ws_bytes = int(lib.loits_tuple_backward_workspace(C.byref(shape), packed.numel()))
            ws = torch.empty(max(ws_bytes, 16), dtype=torch.uint8, device=dev)
            N.check(lib.loits_tuple_backward(C.byref(shape), g.data_ptr(), packed.data_ptr(),
                                             packed.numel(), int(state["nmax"]), int(seed),
                                             int(sequence), x_bins.data_ptr(), xsec_x.data_ptr(),
                                             q_bins.data_ptr(), xsec_q.data_ptr(),
                                             acceptance.view(torch.uint8).data_ptr(),
                                             state["norm_x"].data_ptr(), state["norm_q"].data_ptr(),
                                             state["cdf_x"].data_ptr(), state["cdf_q"].data_ptr(),
                                             gx.data_ptr(), gq.data_ptr(), ws.data_ptr(),
                                             ws.numel(), N.stream_of(dev)),
                    "loits_tuple_backward")
        with _region(profile_regions, "loits::backward::state_pack"):
            pass
    return gx, gq


class TupleStep:
    """Forward + backward of the reference theory tuple on static buffers, so
    that both can be captured in one CUDA graph (``capture()``, then
    ``step()`` replays it).

    The reference's call returns (valid, 2) events: a shape the host learns
    only by waiting for the device (twice per forward in ``tuple_forward``).
    Here every count stays on the device: prepare writes {nmax, active}, the
    sampler covers a host-known bound on active -- each cell draws
    trunc(|w| n_events) slots, so n_events * sum |w| bounds the total; the
    weights are read once, here -- and writes the kept-row count to
    ``valid``, which the backward reads.  ``events`` (capacity x 2) and
    ``packed`` hold ``capacity`` rows, the first ``valid`` of them the sample
    (the same rows, bit for bit, as ``tuple_forward``); put the cotangent of
    those rows into ``grad_events`` before each backward.  The inputs are the
    caller's tensors, read in place at every step; seed and sequence are
    fixed.  ``grad_xsec_x`` / ``grad_xsec_q`` receive the gradients."""

    def __init__(self, x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events, seed,
                 sequence=0):
        shape = _check_tuple(x_bins, xsec_x, q_bins, xsec_q, weights, acceptance)
        n_events = int(n_events)
        if n_events < 0:
            raise ValueError("n_events must be >= 0")
        dev = x_bins.device
        self.device, self.shape = dev, shape
        self.inputs = (x_bins, xsec_x, q_bins, xsec_q, weights, acceptance)
        self.n_events, self.seed, self.sequence = n_events, int(seed), int(sequence)
        B, nx, ny = shape.batch, shape.nx, shape.ny
        ncell = B * nx * ny
        w_sum = float(weights.abs().sum().item())  # the only host read, at set-up
        self.capacity = max(int(math.ceil(n_events * w_sum * (1.0 + 1e-12))) + ncell, 1)
        f64 = dict(dtype=torch.float64, device=dev)
        i64 = dict(dtype=torch.int64, device=dev)
        self.counts = torch.empty(ncell, **i64)
        self.cell_offsets = torch.empty(ncell + 1, **i64)
        self.norm_x = torch.empty((B, ny, nx), **f64)
        self.norm_q = torch.empty((B, nx, ny), **f64)
        self.cdf_x = torch.empty_like(xsec_x)
        self.cdf_q = torch.empty_like(xsec_q)
        self.alloc = torch.zeros(2, **i64)
        self.events = torch.zeros((self.capacity, 2), **f64)
        self.packed = torch.zeros(self.capacity, **i64)
        self.valid = torch.zeros(1, **i64)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        lib = N.lib()
        self.ws_sample = torch.empty(max(int(lib.loits_tuple_sample_workspace(self.capacity)), 16),
                                     dtype=torch.uint8, device=dev)
        self.grad_events = torch.zeros((self.capacity, 2), **f64)
        self.grad_xsec_x = torch.empty_like(xsec_x)
        self.grad_xsec_q = torch.empty_like(xsec_q)
        nb = int(lib.loits_tuple_backward_workspace(C.byref(shape), self.capacity))
        self.ws_backward = torch.empty(max(nb, 16), dtype=torch.uint8, device=dev)
        self.graph = None

    def forward(self):
        x_bins, xsec_x, q_bins, xsec_q, weights, acceptance = self.inputs
        lib = N.lib()
        with torch.cuda.device(self.device):
            stream = N.stream_of(self.device)
            N.check(lib.loits_tuple_prepare(C.byref(self.shape), x_bins.data_ptr(),
                                            xsec_x.data_ptr(), q_bins.data_ptr(),
                                            xsec_q.data_ptr(), weights.data_ptr(),
                                            acceptance.view(torch.uint8).data_ptr(),
                                            self.n_events, self.counts.data_ptr(),
                                            self.cell_offsets.data_ptr(), self.norm_x.data_ptr(),
                                            self.norm_q.data_ptr(), self.cdf_x.data_ptr(),
                                            self.cdf_q.data_ptr(), self.alloc.data_ptr(), stream),
                    "loits_tuple_prepare")
            N.check(lib.loits_tuple_sample_bounded(
                C.byref(self.shape), x_bins.data_ptr(), q_bins.data_ptr(), self.cdf_x.data_ptr(),
                self.cdf_q.data_ptr(), self.cell_offsets.data_ptr(), self.alloc.data_ptr(),
                self.capacity, self.seed, self.sequence, self.events.data_ptr(),
                self.packed.data_ptr(), None, None, self.valid.data_ptr(), self.status.data_ptr(),
                self.ws_sample.data_ptr(), self.ws_sample.numel(), stream),
                "loits_tuple_sample_bounded")

    def backward(self):
        x_bins, xsec_x, q_bins, xsec_q, _, acceptance = self.inputs
        with torch.cuda.device(self.device):
            N.check(N.lib().loits_tuple_backward_bounded(
                C.byref(self.shape), self.grad_events.data_ptr(), self.packed.data_ptr(),
                self.valid.data_ptr(), self.alloc.data_ptr(), self.capacity, self.seed,
                self.sequence, x_bins.data_ptr(), xsec_x.data_ptr(), q_bins.data_ptr(),
                xsec_q.data_ptr(), acceptance.view(torch.uint8).data_ptr(),
                self.norm_x.data_ptr(), self.norm_q.data_ptr(), self.cdf_x.data_ptr(),
                self.cdf_q.data_ptr(), self.grad_xsec_x.data_ptr(), self.grad_xsec_q.data_ptr(),
                self.ws_backward.data_ptr(), self.ws_backward.numel(), N.stream_of(self.device)),
                "loits_tuple_backward_bounded")

    def step(self):
        if self.graph is not None:
            self.graph.replay()
        else:
            self.forward()
            self.backward()

    def capture(self):
        """Capture forward + backward into one CUDA graph (warms up first)."""
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self.forward()
            self.backward()
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.forward()
            self.backward()
        self.graph = g
        return g

    def check_status(self):
        """Synchronising read of the device status word."""
        N.check(int(self.status.item()), "loits_tuple_sample_bounded (device)")

    def result(self):
        """(events, packed) of the last step: the first ``valid`` rows (a sync)."""
        n = int(self.valid.item())
        return self.events[:n], self.packed[:n]


def fill_uniform(count: int, seed: int, stream_id: int, device="cuda") -> torch.Tensor:
    """values[p] = uniform of Philox slot p on (stream_id, seed) (cpp/loits_core.cpp:39-53)."""
    dev = torch.device(device)
    N.require_device(dev)
    out = torch.empty(max(int(count), 0), dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        N.check(N.lib().loits_fill_uniform(out.data_ptr() if out.numel() else None, out.numel(),
                                           int(seed), int(stream_id), N.stream_of(dev)),
                "loits_fill_uniform")
    return out


def native_forward(x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events, seed, sequence,
                   profile_regions=False):
    """State-by-state mirror of the reference pybind ``forward``
    (cpp/bindings.cpp:24-130): [events, norm_x, norm_q, cdf_x, cdf_q, u_x, u_q,
    interval_x, interval_q, packed].  u_x / u_q are generated for every padded
    slot (batch, cells, nmax) like the reference; interval_x / interval_q are
    padded int16 with the kept rows' intervals at their packed slots."""
    with _region(profile_regions, "loits::binding::forward", x_bins.device):
        events, st = tuple_forward(x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events,
                                   seed, sequence, profile_regions, want_intervals=True)
        B, cells, nmax = x_bins.shape[0], x_bins.shape[1] * q_bins.shape[1], st["nmax"]
        total = B * cells * nmax
        u_x = fill_uniform(total, seed, 2 * int(sequence), x_bins.device).view(B, cells, nmax)
        u_q = fill_uniform(total, seed, 2 * int(sequence) + 1, x_bins.device).view(B, cells, nmax)
        ix = torch.zeros(total, dtype=torch.int16, device=x_bins.device)
        iq = torch.zeros(total, dtype=torch.int16, device=x_bins.device)
        ix[st["packed"]] = st["interval_x"]
        iq[st["packed"]] = st["interval_q"]
    return [events, st["norm_x"], st["norm_q"], st["cdf_x"], st["cdf_q"], u_x, u_q, ix, iq,
            st["packed"]]


def native_backward(grad_events, x_bins, xsec_x, q_bins, xsec_q, acceptance, norm_x, norm_q,
                    cdf_x, cdf_q, u_x, u_q, interval_x, interval_q, packed, profile_regions=False,
                    *, seed=None, sequence=None):
    """Mirror of the reference pybind ``backward`` (cpp/bindings.cpp:132-208).

    The reference reads u and the intervals from the saved state; this
    backend regenerates them from (seed, sequence), which must be the
    forward's (keyword arguments)."""
    if seed is None or sequence is None:
        raise ValueError("native_backward needs the forward's seed and sequence")
    state = dict(norm_x=norm_x, norm_q=norm_q, cdf_x=cdf_x, cdf_q=cdf_q, packed=packed,
                 nmax=u_x.shape[2])
    with _region(profile_regions, "loits::binding::backward", x_bins.device):
        return list(tuple_backward(grad_events, x_bins, xsec_x, q_bins, xsec_q, acceptance, state,
                                   seed, sequence, profile_regions))


class _CudaLOITSFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events, seed,
                sequence, profile_regions):
        profile_regions = bool(profile_regions)
        with _region(profile_regions, "loits::binding::forward", x_bins.device):
            events, st = tuple_forward(x_bins, xsec_x, q_bins, xsec_q, weights, acceptance,
                                       n_events, seed, sequence, profile_regions)
        ctx.profile_regions = profile_regions
        ctx.seed, ctx.sequence, ctx.nmax = int(seed), int(sequence), st["nmax"]
        ctx.save_for_backward(x_bins, xsec_x, q_bins, xsec_q, acceptance, st["norm_x"],
                              st["norm_q"], st["cdf_x"], st["cdf_q"], st["packed"])
        return events

    @staticmethod
    def backward(ctx, grad_events):
        with _region(ctx.profile_regions, "loits::autograd::backward"):
            (x_bins, xsec_x, q_bins, xsec_q, acceptance, norm_x, norm_q, cdf_x, cdf_q,
             packed) = ctx.saved_tensors
            state = dict(norm_x=norm_x, norm_q=norm_q, cdf_x=cdf_x, cdf_q=cdf_q, packed=packed,
                         nmax=ctx.nmax)
            with _region(ctx.profile_regions, "loits::binding::backward", x_bins.device):
                gx, gq = tuple_backward(grad_events.contiguous(), x_bins, xsec_x, q_bins, xsec_q,
                                        acceptance, state, ctx.seed, ctx.sequence,
                                        ctx.profile_regions)
        return None, gx, None, gq, None, None, None, None, None, None


class CudaLOITS(nn.Module):
    """The B200 LOITS sampler (registered as ``LOITS(backend="cuda")``)."""

    def __init__(self, device="cuda", compile=False, profile_regions=False, epsilon=1e-5,
                 batch_config=None):
        super().__init__()
        self.device = torch.device(device)
        if epsilon != 1e-5:
            raise ValueError("The CUDA backend uses the LOITS epsilon 1e-5")
        ok, reason = availability(self.device)
        if not ok:
            raise RuntimeError(f"CUDA LOITS backend unavailable: {reason}")
        N.lib()
        self.compile = bool(compile)  # accepted for API parity; kernels are already native
        self.profile_regions = profile_regions
        self.seed = torch.initial_seed()
        self.sequence = 0
        self.batch_config = batch_config
        self._batched = None

    def forward(self, theory_outputs, n_events):
        from .batched import DensityBatch, BatchedLOITS

        sequence = self.sequence
        self.sequence += 1
        if isinstance(theory_outputs, DensityBatch):
            if self._batched is None:
                self._batched = BatchedLOITS(self.device, seed=self.seed, config=self.batch_config)
            with _region(self.profile_regions, "loits::autograd::forward"):
                return self._batched.sample(theory_outputs, n_events, sequence=sequence)
        x_bins, xsec_x, q2_bins, xsec_q2, weights, acceptance = theory_outputs[:6]
        with _region(self.profile_regions, "loits::autograd::forward"):
            return _CudaLOITSFunction.apply(x_bins, xsec_x, q2_bins, xsec_q2, weights, acceptance,
                                            n_events, self.seed, sequence, self.profile_regions)
