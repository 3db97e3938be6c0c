"""Data-parallel sharding of a density batch across ranks (one GPU each).

Densities are independent and Philox is counter based, so a batch splits into
contiguous density ranges with no exchange on the data path: rank r plans its
range with ``density_base`` = the global index of its first density and
``slot_stride`` = the whole batch's max n_b, and then draws exactly the
counters the unsplit batch would (slot s of global density g uses counter
g * slot_stride + s).  Concatenating the ranks' kept rows in rank order gives
the unsplit batch's rows.

Ranges are balanced by cumulative event count (the work measure).
"""
from __future__ import annotations

import numpy as np


def shard_range(event_counts, world_size: int, rank: int) -> tuple[int, int]:
    """[lo, hi) densities of `rank`: the densities whose first event falls in
    the rank's equal share of the total event count."""
    counts = np.asarray(event_counts, dtype=np.int64)
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("bad world_size / rank")
    nd = len(counts)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    total = int(counts.sum())
    if total == 0:
        per = -(-nd // world_size)
        return min(rank * per, nd), min((rank + 1) * per, nd)
    # density d belongs to the rank whose share contains its first event
    owner = np.minimum((starts * world_size) // max(total, 1), world_size - 1)
    idx = np.flatnonzero(owner == rank)
    if idx.size == 0:
        # empty share: an empty range positioned after the previous rank's
        before = np.flatnonzero(owner < rank)
        lo = int(before[-1]) + 1 if before.size else 0
        return lo, lo
    return int(idx[0]), int(idx[-1]) + 1


def sub_case(case: dict, lo: int, hi: int) -> dict:
    """Densities [lo, hi) of a batch given as a dict of host arrays
    (knot_offsets, event_counts, grid, values, optional x_cut, scalars)."""
    koff = np.asarray(case["knot_offsets"], dtype=np.int64)
    k0, k1 = int(koff[lo]), int(koff[hi])
    out = dict(case)
    out["knot_offsets"] = koff[lo:hi + 1] - k0
    out["event_counts"] = np.asarray(case["event_counts"])[lo:hi]
    out["grid"] = np.asarray(case["grid"])[k0:k1]
    out["values"] = np.asarray(case["values"])[k0:k1]
    if case.get("x_cut") is not None:
        out["x_cut"] = np.asarray(case["x_cut"])[lo:hi]
    for k in ("cotangent", "events", "intervals", "row_offsets", "grad_values", "slots"):
        out.pop(k, None)
    return out


def shard_spec(spec, world_size: int, rank: int):
    """(sub-spec, density_base, slot_stride) of a workloads.DensityBatchSpec."""
    from dataclasses import replace

    lo, hi = shard_range(spec.event_counts, world_size, rank)
    koff = spec.knot_offsets
    k0, k1 = int(koff[lo]), int(koff[hi])
    sub = replace(spec, knot_offsets=koff[lo:hi + 1] - k0, grid=spec.grid[k0:k1],
                  values=spec.values[k0:k1], event_counts=spec.event_counts[lo:hi],
                  x_cut=None if spec.x_cut is None else spec.x_cut[lo:hi])
    return sub, lo, int(np.max(spec.event_counts)) if len(spec.event_counts) else 0


def _collective_device():
    """Tensors for collectives live where the process group's backend wants
    them: the current CUDA device for NCCL, the host for gloo."""
    import torch
    import torch.distributed as dist

    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float, group=None) -> float:
    """Max of a per-rank float (step times are reported as the slowest rank's)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=_collective_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def global_rows(local_rows: int, group=None) -> tuple[int, int]:
    """(first global row of this rank's kept events, total kept rows): the
    ranks' rows concatenate in rank order, so a consumer that needs the whole
    batch's row numbering exchanges one count per rank and nothing else."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = _collective_device()
    mine = torch.tensor([int(local_rows)], dtype=torch.int64, device=dev)
    counts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(counts, mine, group=group)
    c = [int(x.item()) for x in counts]
    r = dist.get_rank(group)
    return sum(c[:r]), sum(c)


def gather_batch(events, row_offsets, group=None):
    """The unsplit batch on every rank, for a consumer that needs all of it:
    (events, row_offsets) of the whole batch from each rank's kept rows and
    its densities' row offsets (ranks hold contiguous density ranges in rank
    order).  ``events`` may be longer than the rank's kept rows (the plan's
    capacity-sized buffer): its first ``row_offsets[-1]`` entries are the
    rows.  One all_gather of the row counts, one of the events (padded to
    the largest rank's count) and one of the row offsets (padded to the most
    densities); over NCCL on GPU tensors, gloo on host tensors."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = _collective_device()
    ro = row_offsets.to(device=dev, dtype=torch.int64).contiguous()
    kept = int(ro[-1].item()) if ro.numel() else 0
    if kept > events.numel():
        raise ValueError(f"row_offsets end at row {kept} but events holds {events.numel()} rows")
    ev = events.reshape(-1)[:kept].to(dev).contiguous()
    sizes = torch.tensor([ev.numel(), ro.numel()], dtype=torch.int64, device=dev)
    all_sizes = [torch.zeros(2, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(all_sizes, sizes, group=group)
    n_ev = [int(s[0].item()) for s in all_sizes]
    n_ro = [int(s[1].item()) for s in all_sizes]
    pad_ev = torch.zeros(max(max(n_ev), 1), dtype=ev.dtype, device=dev)
    pad_ev[:ev.numel()] = ev
    pad_ro = torch.zeros(max(n_ro), dtype=torch.int64, device=dev)
    pad_ro[:ro.numel()] = ro
    evs = [torch.empty_like(pad_ev) for _ in range(world)]
    ros = [torch.empty_like(pad_ro) for _ in range(world)]
    dist.all_gather(evs, pad_ev, group=group)
    dist.all_gather(ros, pad_ro, group=group)
    out_ev = torch.cat([evs[r][:n_ev[r]] for r in range(world)])
    offs, base = [torch.zeros(1, dtype=torch.int64, device=dev)], 0
    for r in range(world):
        if n_ro[r] > 1:
            offs.append(ros[r][1:n_ro[r]] + base)
        base += n_ev[r]
    return out_ev, torch.cat(offs)
