"""Launch-geometry autotuner for the batched sampler.

The batched kernels take three launch parameters (``loits_batch_config``):
threads per CTA (256, 512, 1024), Philox blocks per thread per sampling tile
(2, 4, 8, 16) and knots per thread in the CDF scan.  ``base`` fixes other
fields for every candidate (``plain=1`` tunes the one-launch-per-density
form, with ``PLAIN_CANDIDATES``).  Which is fastest depends on the batch: the largest density decides
how much shared memory a CTA holds (hence how many CTAs fit on an SM), the
event counts decide how many tiles there are to balance, and the cut decides
whether the identity compaction applies.  Without tuning, the plan picks the
CTA size with the most resident threads per SM.

:class:`Autotuner` times forward + backward of each candidate on the caller's
own batch (values, grid, cut; a fixed cotangent) with CUDA events and keeps
the fastest, per shape bucket: (log2 densities, log2 largest knot count,
log2 total events, cut or not).  Every candidate samples the same events (the
configuration changes only the launch geometry), so tuning never changes
results beyond the backward's fp32 accumulation order.  Results can be kept
in a JSON file (``cache_path`` or the ``LOITS_TUNE_CACHE`` environment
variable) so later processes skip the timing.
"""
from __future__ import annotations

import json
import math
import os
import threading
from pathlib import Path

import numpy as np
import torch

from . import _native as N

# (threads, blocks_per_item, scan_knots) of the persistent form
CANDIDATES = (
    (256, 16, 8), (256, 8, 8), (256, 4, 8),
    (512, 16, 8), (512, 8, 8), (512, 16, 16), (512, 4, 8),
    (1024, 16, 8), (1024, 8, 8), (1024, 4, 8), (1024, 16, 16), (1024, 8, 16), (1024, 16, 4),
)

# Per grid-size bucket: candidate tile lengths (Philox blocks per thread, at
# most the launch's) and CDF scan widths.
BUCKET_BLOCKS = (2, 4, 8)
BUCKET_SCAN = (4, 16)


def density_buckets(knot_offsets) -> np.ndarray:
    """Grid-size bucket of each density: ceil(log2 of its knot count)."""
    g = np.diff(np.asarray(knot_offsets, dtype=np.int64))
    return np.ceil(np.log2(np.maximum(g, 1))).astype(np.int64)


def density_tables(knot_offsets, config: dict):
    """Per-density (blocks, scan) arrays of a tuned config's bucket tables,
    or (None, None) when it has none."""
    bb, bs = config.get("bucket_blocks") or {}, config.get("bucket_scan") or {}
    if not bb and not bs:
        return None, None
    buckets = density_buckets(knot_offsets)
    r = int(config.get("blocks_per_item") or 0)
    sk = int(config.get("scan_knots") or 8)
    blocks = np.array([int(bb.get(str(k), r)) for k in buckets], np.int32) if bb and r else None
    scan = np.array([int(bs.get(str(k), sk)) for k in buckets], np.int32) if bs else None
    return blocks, scan


def plain_config(config: dict) -> dict:
    """The fields of a tuned config that ``make_config`` takes."""
    return {k: v for k, v in config.items() if k not in ("bucket_blocks", "bucket_scan")}


# The one-launch-per-density form runs each density on its own: smaller tiles
# give a density of 1e4 - 1e6 events more CTAs to fill the GPU with.
PLAIN_CANDIDATES = (
    (256, 2, 8), (256, 4, 8), (256, 8, 8), (256, 16, 8),
    (512, 2, 8), (512, 4, 8), (512, 8, 8),
    (1024, 2, 8), (1024, 4, 8), (1024, 8, 8), (1024, 16, 8),
)


def shape_key(knot_offsets, event_counts, has_cut: bool) -> str:
    """Shape bucket of a batch: densities, largest knot count and total
    events rounded up to powers of two, and whether a cut is applied."""
    koff = np.asarray(knot_offsets, dtype=np.int64)
    counts = np.asarray(event_counts, dtype=np.int64)
    g = int(np.diff(koff).max())
    n = int(counts.sum())
    lg = lambda v: int(math.ceil(math.log2(max(int(v), 1))))  # noqa: E731
    return f"d{lg(len(counts))}-g{lg(g)}-n{lg(n)}-{'cut' if has_cut else 'all'}"


class Autotuner:
    """Chooses (threads, blocks_per_item, scan_knots) per shape bucket by
    timing forward + backward on the batch being sampled."""

    def __init__(self, device="cuda", candidates=CANDIDATES, reps: int = 3,
                 cache_path: str | os.PathLike | None = None, base: dict | None = None,
                 saved_state: bool = True, buckets: bool = True):
        self.device = torch.device(device)
        self.candidates = tuple(candidates)
        # fields every candidate shares (e.g. plain=1, guide_ratio)
        self.base = dict(base or {})
        # time the saved-state form (the sampler's default) or the replay form
        self.saved_state = bool(saved_state)
        # refine the best geometry per grid-size bucket (tune_buckets)
        self.buckets = bool(buckets)
        self.reps = max(1, int(reps))
        path = cache_path if cache_path is not None else os.environ.get("LOITS_TUNE_CACHE")
        self.cache_path = Path(path) if path else None
        self._lock = threading.Lock()
        self.table: dict[str, dict] = {}
        self.timings: dict[str, dict] = {}
        if self.cache_path is not None and self.cache_path.exists():
            try:
                self.table.update(json.loads(self.cache_path.read_text()))
            except (OSError, ValueError):
                pass

    def key_for(self, batch, event_counts=None, hist=None) -> str:
        """This tuner's table key of a batch: its shape bucket, the fields
        every candidate shares, the timed form and the histogram mode."""
        counts = batch.event_counts if event_counts is None else np.asarray(event_counts, np.int64)
        key = shape_key(batch.knot_offsets, counts, batch.x_cut is not None)
        for k in sorted(self.base):
            key += f"-{k}{self.base[k]}"
        key += "-state" if self.saved_state else "-replay"
        if hist is not None:
            key += f"-hist{int(hist[0])}"
        return key

    def config_for(self, batch, event_counts=None, seed: int = 0, sequence: int = 0,
                   hist=None) -> dict:
        """The tuned configuration (a dict for ``make_config``) for this
        batch's shape bucket, timing the candidates on first use.  hist:
        (bins, lo, hi) to time the histogram mode instead of event writing."""
        counts = batch.event_counts if event_counts is None else np.asarray(event_counts, np.int64)
        key = self.key_for(batch, counts, hist)
        with self._lock:
            hit = self.table.get(key)
        if hit is not None:
            return dict(hit)
        best, times = self.tune(batch, counts, seed, sequence, hist)
        with self._lock:
            self.table[key] = best
            self.timings[key] = times
            self._save()
        return dict(best)

    def _timer(self, batch, event_counts, seed, sequence, hist):
        """A function plan -> median ms of one forward + backward of this
        batch (the form this tuner times) with the plan's geometry."""
        grid = batch.grid.detach().contiguous()
        values = batch.values.detach().contiguous()
        x_cut = None if batch.x_cut is None else batch.x_cut.detach().contiguous()
        counts = np.asarray(event_counts, dtype=np.int64)
        capacity = int(counts.sum())
        gen = torch.Generator(device=self.device).manual_seed(0)
        cot = torch.randn(max(capacity, 4), generator=gen, device=self.device, dtype=torch.float32)
        grad_values = torch.empty_like(values)
        stream = torch.cuda.current_stream(self.device)

        def time_plan(plan) -> float:
            events, rows, ws = plan.new_events(), plan.new_row_offsets(), plan.new_workspace()
            ints, offs = plan.new_state() if self.saved_state else (None, None)
            if hist is not None:
                bins, lo, hi = int(hist[0]), float(hist[1]), float(hist[2])
                hbuf = torch.empty((plan.n_densities, bins), dtype=torch.float32,
                                   device=self.device)
                kept = torch.empty(plan.n_densities, dtype=torch.int64, device=self.device)
                ghist = torch.randn((plan.n_densities, bins), generator=gen, device=self.device)

                def step():
                    plan.forward_hist(grid, values, x_cut, seed, sequence, bins, lo, hi, hbuf,
                                      kept, ws)
                    plan.backward_hist(grid, values, x_cut, seed, sequence, bins, lo, hi, ghist,
                                       grad_values, ws)
            elif self.saved_state:
                def step():
                    plan.forward_state(grid, values, x_cut, seed, sequence, events, rows, ints,
                                       offs, ws)
                    plan.backward_state(grid, values, x_cut, ints, offs, cot, grad_values, ws)
            else:
                def step():
                    plan.forward(grid, values, x_cut, seed, sequence, events, rows, ws)
                    plan.backward(grid, values, x_cut, seed, sequence, cot, grad_values, ws)

            step()
            torch.cuda.synchronize(self.device)
            plan.check_status(ws)
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            samples = []
            for _ in range(self.reps):
                t0.record(stream)
                step()
                t1.record(stream)
                t1.synchronize()
                samples.append(t0.elapsed_time(t1))
            plan.check_status(ws)
            return float(np.median(samples))

        return time_plan

    def tune(self, batch, event_counts, seed: int = 0, sequence: int = 0, hist=None):
        """Time every candidate; returns (best config dict, {label: ms}).  The
        best launch geometry is then refined per grid-size bucket
        (:meth:`tune_buckets`): the dict's ``bucket_blocks`` /
        ``bucket_scan`` map ceil(log2 G) to a tile length and scan width."""
        from .batched import BatchPlan, make_config

        counts = np.asarray(event_counts, dtype=np.int64)
        time_plan = self._timer(batch, counts, seed, sequence, hist)
        times: dict[str, float] = {}
        best, best_ms = None, math.inf
        for threads, blocks, scan in self.candidates:
            label = f"{threads}x{blocks}/{scan}"
            try:
                plan = BatchPlan(batch.knot_offsets, counts,
                                 make_config(**{**self.base, "threads": threads,
                                                "blocks_per_item": blocks, "scan_knots": scan}),
                                 self.device)
            except RuntimeError:
                continue  # geometry not supported for this shape (shared memory)
            ms = time_plan(plan)
            times[label] = ms
            if ms < best_ms:
                best_ms = ms
                best = dict(self.base, threads=threads, blocks_per_item=blocks, scan_knots=scan)
            del plan
        if best is None:
            raise RuntimeError("no launch geometry of the batched sampler fits this batch")
        if self.buckets:
            bb, bs, btimes = self.tune_buckets(batch, counts, best, time_plan, best_ms)
            if bb or bs:
                best = dict(best, bucket_blocks=bb, bucket_scan=bs)
            times.update(btimes)
        return best, times

    def tune_buckets(self, batch, event_counts, config: dict, time_plan, base_ms: float):
        """Per grid-size bucket (densities with the same ceil(log2 G)), the
        sampling tile length (Philox blocks per thread, at most the config's)
        and the CDF scan width: one bucket at a time, every other bucket held,
        the whole batch timed; a change is kept when the step gets at least
        1 % faster.  Returns ({bucket: blocks}, {bucket: scan}, {label: ms})
        with the changed buckets only."""
        from .batched import BatchPlan, make_config

        counts = np.asarray(event_counts, dtype=np.int64)
        buckets = density_buckets(batch.knot_offsets)
        # buckets holding the most events first
        order = sorted(set(buckets.tolist()), key=lambda k: -int(counts[buckets == k].sum()))
        rmax = int(config["blocks_per_item"])
        sk0 = int(config.get("scan_knots") or 8)
        blocks = {k: rmax for k in order}
        scan = {k: sk0 for k in order}
        cfg = make_config(**{k: v for k, v in config.items()
                             if k not in ("bucket_blocks", "bucket_scan")})
        times: dict[str, float] = {}
        best_ms = base_ms

        def trial(bl, sc) -> float:
            plan = BatchPlan(batch.knot_offsets, counts, cfg, self.device,
                             density_blocks=np.array([bl[k] for k in buckets], np.int32),
                             density_scan=np.array([sc[k] for k in buckets], np.int32))
            try:
                return time_plan(plan)
            finally:
                del plan

        for k in order:
            for r in BUCKET_BLOCKS:
                if r >= rmax or r == blocks[k]:
                    continue
                ms = trial({**blocks, k: r}, scan)
                times[f"g{k}:blocks{r}"] = ms
                if ms < 0.99 * best_ms:
                    best_ms, blocks[k] = ms, r
            for sk in BUCKET_SCAN:
                if sk == scan[k]:
                    continue
                ms = trial(blocks, {**scan, k: sk})
                times[f"g{k}:scan{sk}"] = ms
                if ms < 0.99 * best_ms:
                    best_ms, scan[k] = ms, sk
        return ({str(k): v for k, v in blocks.items() if v != rmax},
                {str(k): v for k, v in scan.items() if v != sk0}, times)

    def _save(self) -> None:
        if self.cache_path is None:
            return
        try:
            self.cache_path.parent.mkdir(parents=True, exist_ok=True)
            tmp = self.cache_path.with_suffix(".tmp")
            tmp.write_text(json.dumps(self.table, indent=1, sort_keys=True))
            tmp.replace(self.cache_path)
        except OSError:
            pass


_DEFAULT: dict[str, Autotuner] = {}


def default_tuner(device, saved_state: bool = True) -> Autotuner:
    """Process-wide tuner of a device and sampler form (shared by every
    ``BatchedLOITS`` created with ``config="auto"``)."""
    dev = torch.device(device)
    key = f"{dev}-{'state' if saved_state else 'replay'}"
    if key not in _DEFAULT:
        N.require_device(dev)
        _DEFAULT[key] = Autotuner(dev, saved_state=saved_state)
    return _DEFAULT[key]
