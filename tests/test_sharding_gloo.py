"""Two ranks over gloo (CPU) reproduce the unsplit batch.

The multi-GPU path shards densities into contiguous ranges with no data-path
collective: each rank plans its range with density_base = its first global
density and slot_stride = the batch's largest event count, so it draws the
unsplit batch's Philox counters.  Here each rank runs the CPU oracle on its
shard (standing in for its GPU), the ranks exchange one kept-row count each
(``sharding.global_rows``) to place their rows, and rank 0 checks that the
gathered events, row offsets and gradients equal the unsplit batch's.  Step
times are reduced with ``sharding.max_over_ranks``; ``sharding.gather_batch``
gives every rank the unsplit batch's events and row offsets.
"""
from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import torch.multiprocessing as mp

WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    from conftest import GOLDEN, golden_case
    from oracle.oracle import Oracle
    from quantom_loits_b200 import sharding

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ora = Oracle()
        case = golden_case(np.load(GOLDEN), "ragged_workload_small")
        seed, seq = (int(v) for v in case["scalars"][:2])
        counts = np.asarray(case["event_counts"], np.int64)
        nmax = int(counts.max())
        lo, hi = sharding.shard_range(counts, world, rank)
        sub = sharding.sub_case(case, lo, hi)
        eoff = np.concatenate([[0], np.cumsum(sub["event_counts"])])
        fwd = ora.d_forward(sub["knot_offsets"], eoff, sub["grid"], sub["values"],
                            sub.get("x_cut"), seed, seq, lo, nmax)
        first, total = sharding.global_rows(len(fwd["events"]))
        # the whole batch's cotangent, of which this rank reads its own rows
        cot = np.random.default_rng(9).standard_normal(total)
        grad = ora.d_backward(sub["knot_offsets"], eoff, sub["grid"], sub["values"],
                              sub.get("x_cut"), seed, seq, cot[first:first + len(fwd["events"])],
                              fwd=fwd, density_base=lo, slot_stride=nmax)
        parts = [None] * world
        dist.all_gather_object(parts, dict(lo=lo, hi=hi, first=first, events=fwd["events"],
                                           rows=fwd["row_offsets"], grad=grad))
        # the whole batch on every rank (a consumer that needs all of it)
        import torch

        # the rank's events as a sampler returns them in its capacity-sized
        # buffer: kept rows first, then unused tail rows
        ev_buf = np.full(sub["event_counts"].sum() + 7, -123.0)
        ev_buf[:len(fwd["events"])] = fwd["events"]
        ev_all, rows_all = sharding.gather_batch(torch.from_numpy(ev_buf),
                                                 torch.from_numpy(fwd["row_offsets"]))
        step_ms = sharding.max_over_ranks(1.5 + rank)
        if rank == 0:
            out.put(dict(parts=parts, total=total, step_ms=step_ms, seed=seed, seq=seq,
                         ev_all=ev_all.numpy(), rows_all=rows_all.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_unsplit_batch(oracle_lib, golden):
    from conftest import golden_case

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, WORLD, port, out)) for r in range(WORLD)]
    for p in procs:
        p.start()
    try:
        res = out.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    case = golden_case(golden, "ragged_workload_small")
    counts = np.asarray(case["event_counts"], np.int64)
    eoff = np.concatenate([[0], np.cumsum(counts)])
    ref = oracle_lib.d_forward(case["knot_offsets"], eoff, case["grid"], case["values"],
                               case.get("x_cut"), res["seed"], res["seq"])
    parts = sorted(res["parts"], key=lambda p: p["lo"])
    # contiguous, covering shards
    assert parts[0]["lo"] == 0 and parts[-1]["hi"] == len(counts)
    assert all(a["hi"] == b["lo"] for a, b in zip(parts, parts[1:]))
    assert np.array_equal(np.concatenate([p["events"] for p in parts]), ref["events"])
    # row offsets: each shard's local offsets shifted by its first global row
    rows = np.concatenate([parts[0]["rows"][:1]] +
                          [p["rows"][1:] + p["first"] for p in parts])
    assert np.array_equal(rows, ref["row_offsets"]) and res["total"] == len(ref["events"])
    cot = np.random.default_rng(9).standard_normal(res["total"])
    gref = oracle_lib.d_backward(case["knot_offsets"], eoff, case["grid"], case["values"],
                                 case.get("x_cut"), res["seed"], res["seq"], cot, fwd=ref)
    np.testing.assert_allclose(np.concatenate([p["grad"] for p in parts]), gref,
                               rtol=1e-12, atol=1e-15)
    assert res["step_ms"] == 2.5  # max over the ranks' 1.5 and 2.5
    # gather_batch: every rank can hold the unsplit batch's events and rows
    assert np.array_equal(res["ev_all"], ref["events"])
    assert np.array_equal(res["rows_all"], ref["row_offsets"])
