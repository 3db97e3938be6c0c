"""Batched ragged 1-D densities: the sampler's batched mode.

A :class:`DensityBatch` is B independent densities tabulated on their own
grids (fp32), described by an offsets table: knots of density b are
``[knot_offsets[b], knot_offsets[b+1])`` (at least 2), it receives
``event_counts[b]`` event slots, and an optional per-density cut keeps only
events with ``x > x_cut[b]``.

Each density is, exactly, the reference's x curve of a one-cell theory
(nx = ny = 1, weight (n_b + 0.5)/nmax, n_events = nmax = max n_b), so slot s of
density b draws Philox counter ``b * nmax + s`` on stream ``2 * sequence``
(cpp/bindings.cpp:79-92) and the kept events come out in (density, slot)
order like the reference's compaction (cpp/loits_core.cpp:239-266).

:class:`BatchPlan` wraps a native plan (tile and chunk tables built once per
batch shape); :class:`BatchedLOITS` is the autograd-facing sampler;
:class:`BatchStep` captures forward + backward in one CUDA graph.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N


def _host_i64(a) -> np.ndarray:
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


@dataclass
class DensityBatch:
    """Ragged batch of densities.  grid / values / x_cut live on the device;
    knot_offsets / event_counts are host tables (they shape the plan)."""

    grid: torch.Tensor
    values: torch.Tensor
    knot_offsets: np.ndarray
    event_counts: np.ndarray
    x_cut: torch.Tensor | None = None

    def __post_init__(self):
        self.knot_offsets = _host_i64(self.knot_offsets)
        self.event_counts = _host_i64(self.event_counts)
        nd = len(self.knot_offsets) - 1
        if nd < 1 or len(self.event_counts) != nd:
            raise ValueError("knot_offsets must have B+1 entries and event_counts B")
        for name in ("grid", "values"):
            t = getattr(self, name)
            if t.dtype != torch.float32 or t.dim() != 1 or t.numel() != self.knot_offsets[-1]:
                raise ValueError(f"{name} must be fp32 with knot_offsets[-1] entries")
        if self.grid.device != self.values.device:
            raise ValueError("grid and values must share a device")
        if self.x_cut is not None and (self.x_cut.dtype != torch.float32 or
                                       self.x_cut.numel() != nd):
            raise ValueError("x_cut must be fp32 with one entry per density")

    @property
    def n_densities(self) -> int:
        return len(self.knot_offsets) - 1

    @property
    def device(self) -> torch.device:
        return self.values.device

    @classmethod
    def from_spec(cls, spec, device="cuda", requires_grad=False) -> "DensityBatch":
        """From a quantom_loits_b200.workloads.DensityBatchSpec (host arrays)."""
        dev = torch.device(device)
        values = torch.as_tensor(spec.values, dtype=torch.float32).to(dev)
        if requires_grad:
            values.requires_grad_(True)
        x_cut = None if spec.x_cut is None else torch.as_tensor(spec.x_cut).to(dev)
        return cls(torch.as_tensor(spec.grid, dtype=torch.float32).to(dev), values,
                   spec.knot_offsets, spec.event_counts, x_cut)


def default_config() -> N.BatchConfig:
    return N.BatchConfig()


def make_config(threads=0, blocks_per_item=0, scan_knots=0, ctas_per_sm=0, plain=0,
                density_base=0, slot_stride=0, guide_ratio=0, wait_limit=0,
                withhold_tile=0) -> N.BatchConfig:
    return N.BatchConfig(threads=int(threads), blocks_per_item=int(blocks_per_item),
                         scan_knots=int(scan_knots), ctas_per_sm=int(ctas_per_sm),
                         plain=int(plain), guide_ratio=int(guide_ratio),
                         wait_limit=int(wait_limit), withhold_tile=int(withhold_tile),
                         density_base=int(density_base), slot_stride=int(slot_stride))


class BatchPlan:
    """Native plan for one batch shape (offsets table + launch geometry).

    ``density_blocks`` / ``density_scan`` (optional, one int per density):
    each density's Philox blocks per thread per sampling tile (at most the
    config's blocks_per_item) and knots per thread in its CDF scan, e.g.
    from :meth:`tuning.Autotuner.density_tables`; the config's values
    otherwise."""

    def __init__(self, knot_offsets, event_counts, config: N.BatchConfig | dict | None = None,
                 device="cuda", density_blocks=None, density_scan=None):
        self.device = torch.device(device)
        N.require_device(self.device)
        self.knot_offsets = _host_i64(knot_offsets)
        self.event_counts = _host_i64(event_counts)
        self.n_densities = len(self.knot_offsets) - 1
        if isinstance(config, dict):
            config = make_config(**config)
        tables = []
        for t in (density_blocks, density_scan):
            if t is None:
                tables.append(None)
                continue
            t = np.ascontiguousarray(np.asarray(t, dtype=np.int32))
            if t.shape != (self.n_densities,):
                raise ValueError("per-density tables need one entry per density")
            tables.append(t)
        self._tables = tables  # kept alive for the call
        lib = N.lib()
        handle = C.c_void_p()
        with torch.cuda.device(self.device):
            N.check(lib.loits_batch_plan_create_ex(
                self.n_densities, self.knot_offsets.ctypes.data, self.event_counts.ctypes.data,
                C.byref(config) if config is not None else None,
                None if tables[0] is None else tables[0].ctypes.data,
                None if tables[1] is None else tables[1].ctypes.data, C.byref(handle)),
                "loits_batch_plan_create_ex")
        self._lib = lib
        self.handle = handle
        self.capacity = int(lib.loits_batch_capacity(handle))
        self.total_knots = int(lib.loits_batch_total_knots(handle))
        self.workspace_bytes = int(lib.loits_batch_workspace_bytes(handle))
        self.status_offset = int(lib.loits_batch_status_offset(handle))
        cfg = N.BatchConfig()
        N.check(lib.loits_batch_plan_config(handle, C.byref(cfg)), "loits_batch_plan_config")
        self.config = cfg.as_dict()

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.loits_batch_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    # -- buffers -----------------------------------------------------------
    def new_workspace(self) -> torch.Tensor:
        return torch.empty(max(self.workspace_bytes, 16), dtype=torch.uint8, device=self.device)

    def new_events(self) -> torch.Tensor:
        return torch.empty(max(self.capacity, 4), dtype=torch.float32, device=self.device)

    def new_row_offsets(self) -> torch.Tensor:
        return torch.empty(self.n_densities + 1, dtype=torch.int64, device=self.device)

    def new_state(self) -> tuple[torch.Tensor, torch.Tensor]:
        """Buffers of a saved state: (intervals int32, offsets fp32), capacity rows."""
        n = max(self.capacity, 4)
        return (torch.empty(n, dtype=torch.int32, device=self.device),
                torch.empty(n, dtype=torch.float32, device=self.device))

    def status_view(self, workspace: torch.Tensor) -> torch.Tensor:
        return workspace[self.status_offset:self.status_offset + 4].view(torch.int32)

    # -- launches (asynchronous, on the current stream) ---------------------
    def forward(self, grid, values, x_cut, seed, sequence, events, row_offsets, workspace,
                intervals=None) -> None:
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_forward(
                self.handle, grid.data_ptr(), values.data_ptr(), N.ptr(x_cut), int(seed),
                int(sequence), events.data_ptr(), row_offsets.data_ptr(), N.ptr(intervals),
                workspace.data_ptr(), N.stream_of(self.device)), "loits_batch_forward")

    def backward(self, grid, values, x_cut, seed, sequence, grad_events, grad_values,
                 workspace) -> None:
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_backward(
                self.handle, grid.data_ptr(), values.data_ptr(), N.ptr(x_cut), int(seed),
                int(sequence), grad_events.data_ptr(), grad_values.data_ptr(),
                workspace.data_ptr(), N.stream_of(self.device)), "loits_batch_backward")

    def forward_state(self, grid, values, x_cut, seed, sequence, events, row_offsets, intervals,
                      offsets, workspace) -> None:
        """Forward that also saves, per kept row, its interval and its offset
        u - c_j (the saved state ``backward_state`` reads)."""
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_forward_state(
                self.handle, grid.data_ptr(), values.data_ptr(), N.ptr(x_cut), int(seed),
                int(sequence), events.data_ptr(), row_offsets.data_ptr(), intervals.data_ptr(),
                offsets.data_ptr(), workspace.data_ptr(), N.stream_of(self.device)),
                "loits_batch_forward_state")

    def backward_state(self, grid, values, x_cut, intervals, offsets, grad_events, grad_values,
                       workspace) -> None:
        """VJP from the saved state of ``forward_state`` (same workspace)."""
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_backward_state(
                self.handle, grid.data_ptr(), values.data_ptr(), N.ptr(x_cut),
                intervals.data_ptr(), offsets.data_ptr(), grad_events.data_ptr(),
                grad_values.data_ptr(), workspace.data_ptr(), N.stream_of(self.device)),
                "loits_batch_backward_state")

    def forward_hist(self, grid, values, x_cut, seed, sequence, bins, lo, hi, hist, kept,
                     workspace) -> None:
        """Histogram mode: bin the kept events (triangular weights, see
        include/loits_b200.h) into hist (B x bins fp32); kept (B int64).
        sequence: an int, or a one-element int64 device tensor read by the
        kernels (so that a captured CUDA graph can advance it)."""
        seq, seq_dev = _sequence_args(sequence)
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_forward_hist(
                self.handle, grid.data_ptr(), values.data_ptr(), N.ptr(x_cut), int(seed), seq,
                int(bins), float(lo), float(hi), hist.data_ptr(), kept.data_ptr(),
                workspace.data_ptr(), seq_dev, N.stream_of(self.device)),
                "loits_batch_forward_hist")

    def backward_hist(self, grid, values, x_cut, seed, sequence, bins, lo, hi, grad_hist,
                      grad_values, workspace) -> None:
        seq, seq_dev = _sequence_args(sequence)
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_backward_hist(
                self.handle, grid.data_ptr(), values.data_ptr(), N.ptr(x_cut), int(seed), seq,
                int(bins), float(lo), float(hi), grad_hist.data_ptr(), grad_values.data_ptr(),
                workspace.data_ptr(), seq_dev, N.stream_of(self.device)),
                "loits_batch_backward_hist")

    def forward_hist_powerlaw(self, grid, params, x_cut, seed, sequence, bins, lo, hi, hist,
                              kept, workspace) -> None:
        """forward_hist with the densities given by power-law theory
        parameters (B x 6, the GAN theory), evaluated in the kernels' CDF
        tile loads instead of read from a values tensor."""
        seq, seq_dev = _sequence_args(sequence)
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_forward_hist_powerlaw(
                self.handle, grid.data_ptr(), params.data_ptr(), N.ptr(x_cut), int(seed), seq,
                int(bins), float(lo), float(hi), hist.data_ptr(), kept.data_ptr(),
                workspace.data_ptr(), seq_dev, N.stream_of(self.device)),
                "loits_batch_forward_hist_powerlaw")

    def backward_hist_powerlaw(self, grid, params, x_cut, seed, sequence, bins, lo, hi,
                               grad_hist, grad_params, workspace) -> None:
        """VJP of forward_hist_powerlaw: grad_hist -> grad_params (B x 6)."""
        seq, seq_dev = _sequence_args(sequence)
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_backward_hist_powerlaw(
                self.handle, grid.data_ptr(), params.data_ptr(), N.ptr(x_cut), int(seed), seq,
                int(bins), float(lo), float(hi), grad_hist.data_ptr(), grad_params.data_ptr(),
                workspace.data_ptr(), seq_dev, N.stream_of(self.device)),
                "loits_batch_backward_hist_powerlaw")

    def check_status(self, workspace) -> None:
        """Synchronising read of the device status word."""
        N.check(int(self.status_view(workspace).item()), "batched sampler (device)")

    def cdf(self, workspace) -> tuple[torch.Tensor, torch.Tensor]:
        """The forward's CDF per knot (fp64 hi + lo) and the fp64 normalisers."""
        out = torch.empty(self.total_knots, dtype=torch.float64, device=self.device)
        norm = torch.empty(self.n_densities, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_cdf(self.handle, workspace.data_ptr(), out.data_ptr(),
                                              norm.data_ptr(), N.stream_of(self.device)),
                    "loits_batch_cdf")
        return out, norm

    def quantile(self, workspace, density: int, u: torch.Tensor):
        """Inverse CDF of one density at given fp32 uniforms: (x, intervals)."""
        u = u.to(device=self.device, dtype=torch.float32).contiguous()
        x = torch.empty_like(u)
        j = torch.empty(u.numel(), dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            N.check(self._lib.loits_batch_quantile(self.handle, workspace.data_ptr(), int(density),
                                                   u.data_ptr(), u.numel(), x.data_ptr(),
                                                   j.data_ptr(), N.stream_of(self.device)),
                    "loits_batch_quantile")
        return x, j


def _sequence_args(sequence):
    """(host sequence, device address or None) of an int or a device tensor."""
    if isinstance(sequence, torch.Tensor):
        if sequence.dtype != torch.int64 or sequence.numel() != 1 or not sequence.is_cuda:
            raise ValueError("a device sequence is a one-element int64 CUDA tensor")
        return 0, sequence.data_ptr()
    return int(sequence), None


def _aligned(t: torch.Tensor) -> torch.Tensor:
    t = t.contiguous()
    if t.data_ptr() % 16:
        t = t.clone()
    return t


class _BatchFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, grid, x_cut, plan: BatchPlan, seed, sequence):
        events = plan.new_events()
        rows = plan.new_row_offsets()
        ws = plan.new_workspace()
        plan.forward(grid, values, x_cut, seed, sequence, events, rows, ws)
        status = plan.status_view(ws)
        head = torch.cat([rows[-1:], status.to(torch.int64)]).tolist()  # one sync
        valid, st = int(head[0]), int(head[1])
        N.check(st, "loits_batch_forward (device)")
        ctx.plan, ctx.seed, ctx.sequence = plan, int(seed), int(sequence)
        ctx.x_cut = x_cut
        ctx.valid = valid
        ctx.save_for_backward(values, grid, ws)
        ctx.mark_non_differentiable(rows)
        return events[:valid], rows

    @staticmethod
    def backward(ctx, grad_events, grad_rows):
        values, grid, ws = ctx.saved_tensors
        plan: BatchPlan = ctx.plan
        g = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=values.device)
        if grad_events is not None and ctx.valid:
            g[:ctx.valid] = grad_events.to(torch.float32)
        grad_values = torch.empty_like(values)
        plan.backward(grid, values, ctx.x_cut, ctx.seed, ctx.sequence, _aligned(g), grad_values, ws)
        return grad_values, None, None, None, None, None


class _StateFunction(torch.autograd.Function):
    """Saved-state form of _BatchFunction: the forward keeps each kept row's
    interval and offset (8 bytes per row) and the backward reads them."""

    @staticmethod
    def forward(ctx, values, grid, x_cut, plan: BatchPlan, seed, sequence):
        events = plan.new_events()
        rows = plan.new_row_offsets()
        ws = plan.new_workspace()
        ints, offs = plan.new_state()
        plan.forward_state(grid, values, x_cut, seed, sequence, events, rows, ints, offs, ws)
        status = plan.status_view(ws)
        head = torch.cat([rows[-1:], status.to(torch.int64)]).tolist()  # one sync
        valid, st = int(head[0]), int(head[1])
        N.check(st, "loits_batch_forward_state (device)")
        ctx.plan, ctx.x_cut, ctx.valid = plan, x_cut, valid
        ctx.save_for_backward(values, grid, ws, ints, offs)
        ctx.mark_non_differentiable(rows)
        return events[:valid], rows

    @staticmethod
    def backward(ctx, grad_events, grad_rows):
        values, grid, ws, ints, offs = ctx.saved_tensors
        plan: BatchPlan = ctx.plan
        g = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=values.device)
        if grad_events is not None and ctx.valid:
            g[:ctx.valid] = grad_events.to(torch.float32)
        grad_values = torch.empty_like(values)
        plan.backward_state(grid, values, ctx.x_cut, ints, offs, g, grad_values, ws)
        return grad_values, None, None, None, None, None


class _HistFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, grid, x_cut, plan: BatchPlan, seed, sequence, bins, lo, hi):
        hist = torch.empty((plan.n_densities, bins), dtype=torch.float32, device=values.device)
        kept = torch.empty(plan.n_densities, dtype=torch.int64, device=values.device)
        ws = plan.new_workspace()
        plan.forward_hist(grid, values, x_cut, seed, sequence, bins, lo, hi, hist, kept, ws)
        ctx.plan, ctx.seed, ctx.sequence = plan, int(seed), sequence
        ctx.bins, ctx.lo, ctx.hi, ctx.x_cut = int(bins), float(lo), float(hi), x_cut
        ctx.save_for_backward(values, grid, ws)
        ctx.mark_non_differentiable(kept)
        return hist, kept

    @staticmethod
    def backward(ctx, grad_hist, grad_kept):
        values, grid, ws = ctx.saved_tensors
        grad_values = torch.empty_like(values)
        if grad_hist is None:
            grad_values.zero_()
        else:
            ctx.plan.backward_hist(grid, values, ctx.x_cut, ctx.seed, ctx.sequence, ctx.bins,
                                   ctx.lo, ctx.hi, grad_hist.to(torch.float32).contiguous(),
                                   grad_values, ws)
        return grad_values, None, None, None, None, None, None, None, None


class _PowerLawHistFunction(torch.autograd.Function):
    """Theory parameters -> per-density histograms, the theory evaluated inside
    the sampler (forward_hist_powerlaw) and its VJP reduced there too."""

    @staticmethod
    def forward(ctx, params, grid, x_cut, plan: BatchPlan, seed, sequence, bins, lo, hi):
        hist = torch.empty((plan.n_densities, bins), dtype=torch.float32, device=params.device)
        kept = torch.empty(plan.n_densities, dtype=torch.int64, device=params.device)
        ws = plan.new_workspace()
        plan.forward_hist_powerlaw(grid, params, x_cut, seed, sequence, bins, lo, hi, hist, kept,
                                   ws)
        ctx.plan, ctx.seed, ctx.sequence = plan, int(seed), sequence
        ctx.bins, ctx.lo, ctx.hi, ctx.x_cut = int(bins), float(lo), float(hi), x_cut
        ctx.save_for_backward(params, grid, ws)
        ctx.mark_non_differentiable(kept)
        return hist, kept

    @staticmethod
    def backward(ctx, grad_hist, grad_kept):
        params, grid, ws = ctx.saved_tensors
        grad_params = torch.empty_like(params)
        if grad_hist is None:
            grad_params.zero_()
        else:
            ctx.plan.backward_hist_powerlaw(grid, params, ctx.x_cut, ctx.seed, ctx.sequence,
                                            ctx.bins, ctx.lo, ctx.hi,
                                            grad_hist.to(torch.float32).contiguous(),
                                            grad_params, ws)
        return grad_params, None, None, None, None, None, None, None, None


class BatchedLOITS:
    """Autograd-facing batched sampler: ``sample(batch) -> (events, row_offsets)``.

    events: fp32 (valid,) in (density, slot) order; row_offsets: int64 (B+1),
    kept rows of density b are [row_offsets[b], row_offsets[b+1]).  Gradients
    flow to ``batch.values``.  Plans are cached per batch shape.

    ``config``: None (the plan's defaults: CTA size by occupancy), a
    ``loits_batch_config`` / dict (a tuned dict may carry per-bucket tables,
    :func:`quantom_loits_b200.tuning.density_tables`), or ``"auto"``: the
    launch geometry is timed on the first batch of each shape bucket
    (:mod:`quantom_loits_b200.tuning`).

    ``saved_state`` (default True): keep each kept row's interval and offset
    between forward and backward (8 bytes per row, as the reference keeps its
    uniforms and intervals for its backward) so that the backward reads them;
    False: keep nothing per row, the backward regenerates the uniforms and
    searches the intervals again (slower, for callers short of memory)."""

    def __init__(self, device="cuda", seed=None, config=None, device_sequence=False,
                 saved_state=True):
        self.device = torch.device(device)
        N.require_device(self.device)
        self.seed = torch.initial_seed() if seed is None else int(seed)
        self.config = config
        self.sequence = 0
        # histogram calls may keep the sequence counter on the device: each
        # call takes a device snapshot and advances the counter there, so a
        # captured CUDA graph draws fresh uniforms on every replay
        self.sequence_dev = (torch.zeros(1, dtype=torch.int64, device=self.device)
                             if device_sequence else None)
        self.saved_state = bool(saved_state)
        self._plans: dict = {}

    def plan_for(self, knot_offsets, event_counts, batch=None, hist=None) -> BatchPlan:
        key = (knot_offsets.tobytes(), event_counts.tobytes())
        plan = self._plans.get(key)
        if plan is None:
            config = self.config
            if isinstance(config, str):
                if config != "auto" or batch is None:
                    raise ValueError(f"unknown config {config!r} (expected 'auto')")
                from .tuning import default_tuner

                tuner = default_tuner(self.device, self.saved_state and hist is None)
                config = tuner.config_for(batch, event_counts, self.seed, self.sequence, hist)
            blocks = scan = None
            if isinstance(config, dict):
                # a tuned geometry, possibly with per-bucket tables
                from .tuning import density_tables, plain_config

                blocks, scan = density_tables(knot_offsets, config)
                config = make_config(**plain_config(config))
            plan = BatchPlan(knot_offsets, event_counts, config, self.device,
                             density_blocks=blocks, density_scan=scan)
            self._plans[key] = plan
        return plan

    def sample(self, batch: DensityBatch, n_events=None, sequence=None):
        counts = batch.event_counts
        if n_events is not None:
            if isinstance(n_events, (int, np.integer)):
                counts = np.full(batch.n_densities, int(n_events), dtype=np.int64)
            else:
                counts = _host_i64(n_events)
        if sequence is None:
            sequence = self.sequence
            self.sequence += 1
        plan = self.plan_for(batch.knot_offsets, counts, batch)
        grid = batch.grid.detach().contiguous()
        x_cut = None if batch.x_cut is None else batch.x_cut.detach().contiguous()
        fn = _StateFunction if self.saved_state else _BatchFunction
        return fn.apply(batch.values, grid, x_cut, plan, self.seed, sequence)

    __call__ = sample

    def histogram(self, batch: DensityBatch, bins: int = 64, lo: float = 0.0, hi: float = 1.0,
                  n_events=None, sequence=None):
        """Per-density histograms of the events ``sample`` would return, binned
        in the kernels without writing the events: ``(hist, kept)``, hist
        (B, bins) fp32 of triangular weights on bins centred at
        lo + (k + 1/2)(hi - lo)/bins, differentiable w.r.t. ``batch.values``;
        kept (B,) int64 kept events per density."""
        counts = batch.event_counts
        if n_events is not None:
            if isinstance(n_events, (int, np.integer)):
                counts = np.full(batch.n_densities, int(n_events), dtype=np.int64)
            else:
                counts = _host_i64(n_events)
        if sequence is None:
            if self.sequence_dev is not None:
                sequence = self.sequence_dev.clone()
                self.sequence_dev.add_(1)
            else:
                sequence = self.sequence
                self.sequence += 1
        plan = self.plan_for(batch.knot_offsets, counts, batch, (bins, lo, hi))
        grid = batch.grid.detach().contiguous()
        x_cut = None if batch.x_cut is None else batch.x_cut.detach().contiguous()
        return _HistFunction.apply(batch.values.contiguous(), grid, x_cut, plan, self.seed,
                                   sequence, int(bins), float(lo), float(hi))

    def histogram_powerlaw(self, params: torch.Tensor, batch: DensityBatch, bins: int = 64,
                           lo: float = 0.0, hi: float = 1.0, sequence=None):
        """``histogram`` of the densities the two-component power-law theory
        gives for ``params`` (B x 6 raw parameters, see
        ``gan.PowerLawTheory``) on ``batch.grid``, the theory evaluated inside
        the sampler's kernels (its values never stored) and its VJP reduced
        there: ``(hist, kept)``, hist differentiable w.r.t. ``params``.
        ``batch.values`` is not read (only its shape)."""
        counts = batch.event_counts
        if sequence is None:
            if self.sequence_dev is not None:
                sequence = self.sequence_dev.clone()
                self.sequence_dev.add_(1)
            else:
                sequence = self.sequence
                self.sequence += 1
        plan = self.plan_for(batch.knot_offsets, counts, batch, (bins, lo, hi))
        grid = batch.grid.detach().contiguous()
        x_cut = None if batch.x_cut is None else batch.x_cut.detach().contiguous()
        return _PowerLawHistFunction.apply(params.to(torch.float32).contiguous(), grid, x_cut, plan,
                                           self.seed, sequence, int(bins), float(lo), float(hi))


class BatchStep:
    """Forward + backward of one batch shape on static buffers, optionally
    captured in a CUDA graph (``capture()`` then ``replay()``).

    Inputs are written into ``values`` / ``grid`` / ``x_cut`` / ``grad_events``
    in place; outputs appear in ``events`` / ``row_offsets`` / ``grad_values``
    after each step (the kept-row count is ``row_offsets[-1]``, on the device).
    """

    def __init__(self, plan: BatchPlan, seed: int, sequence: int = 0, with_cut=False,
                 saved_state=False):
        self.plan = plan
        dev = plan.device
        self.seed, self.sequence = int(seed), int(sequence)
        self.grid = torch.zeros(plan.total_knots, dtype=torch.float32, device=dev)
        self.values = torch.zeros(plan.total_knots, dtype=torch.float32, device=dev)
        self.x_cut = (torch.zeros(plan.n_densities, dtype=torch.float32, device=dev)
                      if with_cut else None)
        self.events = plan.new_events()
        self.row_offsets = plan.new_row_offsets()
        self.grad_events = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=dev)
        self.grad_values = torch.empty(plan.total_knots, dtype=torch.float32, device=dev)
        self.workspace = plan.new_workspace()
        self.state = plan.new_state() if saved_state else None
        self.graph = None

    def forward(self):
        if self.state is not None:
            self.plan.forward_state(self.grid, self.values, self.x_cut, self.seed, self.sequence,
                                    self.events, self.row_offsets, *self.state, self.workspace)
        else:
            self.plan.forward(self.grid, self.values, self.x_cut, self.seed, self.sequence,
                              self.events, self.row_offsets, self.workspace)

    def backward(self):
        if self.state is not None:
            self.plan.backward_state(self.grid, self.values, self.x_cut, *self.state,
                                     self.grad_events, self.grad_values, self.workspace)
        else:
            self.plan.backward(self.grid, self.values, self.x_cut, self.seed, self.sequence,
                               self.grad_events, self.grad_values, self.workspace)

    def step(self):
        if self.graph is not None:
            self.graph.replay()
        else:
            self.forward()
            self.backward()

    def capture(self):
        """Capture forward + backward into one CUDA graph (warms up first)."""
        s = torch.cuda.Stream(self.plan.device)
        s.wait_stream(torch.cuda.current_stream(self.plan.device))
        with torch.cuda.stream(s):
            self.forward()
            self.backward()
        torch.cuda.current_stream(self.plan.device).wait_stream(s)
        torch.cuda.synchronize(self.plan.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.forward()
            self.backward()
        self.graph = g
        return g

    def check_status(self):
        self.plan.check_status(self.workspace)
