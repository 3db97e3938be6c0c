"""Bounded device-side waits (the sampler's failure detection).

Every wait of the batched kernels -- a compaction tile's look-back on its
predecessors, the CDF readiness and chunk-completion counters -- gives up
after a limited number of polls, records LOITS_ERR_TIMEOUT in the launch's
device status word and lets the launch run to its end, so that a stalled
dependency costs an error, not a hung GPU.  These tests make one wait run
out on purpose without faulting anything: a plan built with the test-only
``withhold_tile`` field has one sampling tile that never publishes its
compaction state (every other tile still does), and a short ``wait_limit``
(a few thousand polls, about a millisecond) bounds its successor's wait.
The launch must end promptly with LOITS_ERR_TIMEOUT, every row it wrote must
stay inside the output buffer, and the GPU context must stay usable: the same
batch sampled again without the injection matches the oracle exactly.
"""
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")


def _spec():
    from quantom_loits_b200 import workloads

    # 4 densities x 256 knots, 50 000 events each: with 256-thread CTAs and 2
    # Philox blocks per thread a tile covers 2048 slots, ~25 tiles per density
    return workloads.uniform(scale=0.05, n_densities=4, knots=256)


def _buffers(B, spec, plan):
    grid = torch.from_numpy(spec.grid).to(DEV)
    values = torch.from_numpy(spec.values).to(DEV)
    events = torch.full((max(plan.capacity, 4),), float("nan"), dtype=torch.float32, device=DEV)
    return grid, values, events, plan.new_row_offsets(), plan.new_workspace()


@pytest.mark.parametrize("withhold", [1, 4])
def test_unpublished_lookback_state_ends_in_a_timeout(withhold):
    from quantom_loits_b200 import _native as N
    from quantom_loits_b200 import batched as B

    spec = _spec()
    cfg = B.make_config(threads=256, blocks_per_item=2, wait_limit=4096, withhold_tile=withhold)
    plan = B.BatchPlan(spec.knot_offsets, spec.event_counts, cfg, DEV)
    grid, values, events, rows, ws = _buffers(B, spec, plan)
    torch.cuda.synchronize(DEV)
    t0 = time.perf_counter()
    plan.forward(grid, values, None, spec.seed, 0, events, rows, ws)
    torch.cuda.synchronize(DEV)
    elapsed = time.perf_counter() - t0
    with pytest.raises(N.LoitsError) as err:
        plan.check_status(ws)
    assert err.value.code == N.LOITS_ERR_TIMEOUT
    assert elapsed < 10.0, elapsed
    # rows written after a timed-out wait still lie inside the output
    r = rows.cpu().numpy()
    assert r[0] == 0 and np.all(np.diff(r) >= 0) and r[-1] <= plan.capacity


def test_context_stays_usable_after_a_timeout(oracle_lib):
    from quantom_loits_b200 import batched as B

    spec = _spec()
    bad = B.BatchPlan(spec.knot_offsets, spec.event_counts,
                      B.make_config(threads=256, blocks_per_item=2, wait_limit=4096,
                                    withhold_tile=2), DEV)
    grid, values, events, rows, ws = _buffers(B, spec, bad)
    bad.forward(grid, values, None, spec.seed, 0, events, rows, ws)
    torch.cuda.synchronize(DEV)
    assert int(bad.status_view(ws).item()) != 0
    good = B.BatchPlan(spec.knot_offsets, spec.event_counts,
                       B.make_config(threads=256, blocks_per_item=2), DEV)
    grid, values, events, rows, ws = _buffers(B, spec, good)
    good.forward(grid, values, None, spec.seed, 0, events, rows, ws)
    good.check_status(ws)
    eoff = np.concatenate([[0], np.cumsum(spec.event_counts)])
    ref = oracle_lib.d_forward(spec.knot_offsets, eoff, spec.grid, spec.values, None, spec.seed, 0)
    assert np.array_equal(rows.cpu().numpy(), ref["row_offsets"])
    n = int(ref["row_offsets"][-1])
    np.testing.assert_allclose(events[:n].cpu().numpy(), ref["events"], rtol=1e-5, atol=0)


def test_wait_fields_are_validated_on_host():
    from quantom_loits_b200 import _native as N
    from quantom_loits_b200 import batched as B

    spec = _spec()
    for kw in (dict(wait_limit=-1), dict(withhold_tile=-3)):
        with pytest.raises(N.LoitsError) as err:
            B.BatchPlan(spec.knot_offsets, spec.event_counts, B.make_config(**kw), DEV)
        assert err.value.code == N.LOITS_ERR_INVALID
