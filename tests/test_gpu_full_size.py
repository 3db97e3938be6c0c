"""Parity at the full sizes of the batched workloads (ragged, uniform,
precision), the forms the bench times: the persistent saved-state forward and
backward of the WHOLE batch on the GPU, then densities sampled across the
batch checked one by one against the fp64 oracle, which draws exactly the
same Philox counters for a single density (density_base = b, slot_stride =
the batch's largest event count).  Kept-row counts exact; events within 1e-5
relative; intervals equal except where the uniform lies within 2 ulp of a
CDF knot; the density's gradient within 1e-4 of its scale.  The whole batch
is also checked for size-independent properties: row offsets non-decreasing
and ending at the kept count, every event finite, inside its density's grid
and not below its cut (the stored fp32 event of an fp64 x just above the cut
may round onto it).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")
EVENT_RTOL = 1e-5
GRAD_TOL = 1e-4

# densities checked against the oracle, per workload (spread over the batch)
CHECKED = {"ragged": [0, 97, 255, 386, 511], "uniform": [0, 31, 63], "precision": [0, 15]}


def near_knot(u, cdf_row, ulps=2):
    u = np.asarray(u, np.float32)
    spacing = np.spacing(u).astype(np.float64) * ulps
    idx = np.searchsorted(cdf_row, u.astype(np.float64))
    lo = np.abs(u - cdf_row[np.clip(idx - 1, 0, len(cdf_row) - 1)])
    hi = np.abs(u - cdf_row[np.clip(idx, 0, len(cdf_row) - 1)])
    return np.minimum(lo, hi) <= np.maximum(spacing, 2.0**-24 * ulps)


@pytest.mark.parametrize("name", ["ragged", "uniform", "precision"])
def test_full_size_workload_matches_oracle_on_sampled_densities(name, oracle_lib):
    from quantom_loits_b200 import batched as B
    from quantom_loits_b200 import workloads

    spec = getattr(workloads, name)()
    nmax = int(spec.event_counts.max())
    plan = B.BatchPlan(spec.knot_offsets, spec.event_counts, B.make_config(slot_stride=nmax), DEV)
    step = B.BatchStep(plan, seed=spec.seed, sequence=3, with_cut=spec.x_cut is not None,
                       saved_state=True)
    step.grid.copy_(torch.from_numpy(np.ascontiguousarray(spec.grid)))
    step.values.copy_(torch.from_numpy(np.ascontiguousarray(spec.values)))
    if spec.x_cut is not None:
        step.x_cut.copy_(torch.from_numpy(np.asarray(spec.x_cut, np.float32)))
    step.forward()
    step.check_status()
    rows = step.row_offsets.cpu().numpy()
    kept = int(rows[-1])
    step.grad_events[:kept].normal_(generator=torch.Generator(device=DEV).manual_seed(1))
    step.backward()
    step.check_status()

    # size-independent properties over the whole batch
    assert np.all(np.diff(rows) >= 0) and rows[0] == 0
    assert np.all(np.diff(rows) <= spec.event_counts)
    ev = step.events[:kept]
    assert bool(torch.isfinite(ev).all())
    koff = spec.knot_offsets
    lo = torch.from_numpy(spec.grid[koff[:-1]].astype(np.float32)).to(DEV)
    hi = torch.from_numpy(spec.grid[koff[1:] - 1].astype(np.float32)).to(DEV)
    dens = torch.repeat_interleave(torch.arange(spec.n_densities, device=DEV),
                                   torch.from_numpy(np.diff(rows)).to(DEV))
    assert bool((ev >= lo[dens]).all()) and bool((ev <= hi[dens] * (1 + 1e-6)).all())
    if spec.x_cut is not None:
        # kept where the reference's fp64 x is above the cut; the stored fp32
        # event is that x rounded, so it may sit on the cut (or an ulp below)
        cut_t = step.x_cut[dens]
        assert bool((ev >= cut_t - cut_t.abs() * 2.0**-22).all())

    ints_all, offs_all = step.state
    gvals = step.grad_values.cpu().numpy()
    cot = step.grad_events[:kept].cpu().numpy()
    for b in CHECKED[name]:
        k0, k1 = int(koff[b]), int(koff[b + 1])
        n = int(spec.event_counts[b])
        cut = None if spec.x_cut is None else np.asarray([spec.x_cut[b]], np.float32)
        sub_koff = np.array([0, k1 - k0])
        sub_eoff = np.array([0, n])
        ref = oracle_lib.d_forward(sub_koff, sub_eoff, spec.grid[k0:k1], spec.values[k0:k1], cut,
                                   spec.seed, 3, b, nmax)
        r0, r1 = int(rows[b]), int(rows[b + 1])
        assert r1 - r0 == int(ref["row_offsets"][-1]), (name, b)
        np.testing.assert_allclose(ev[r0:r1].cpu().numpy(), ref["events"], rtol=EVENT_RTOL)
        mine = ints_all[r0:r1].cpu().numpy()
        diff = np.flatnonzero(mine != ref["intervals"])
        if len(diff):
            assert near_knot(ref["u"][diff], ref["cdf"]).all(), (name, b, len(diff))
        gref = oracle_lib.d_backward(sub_koff, sub_eoff, spec.grid[k0:k1], spec.values[k0:k1], cut,
                                     spec.seed, 3, cot[r0:r1], fwd=ref, density_base=b,
                                     slot_stride=nmax)
        scale = max(np.abs(gref).max(), 1e-30)
        assert np.abs(gvals[k0:k1] - gref).max() <= GRAD_TOL * scale, (name, b)


def test_reference_tuple_at_benchmark_scale_matches_oracle(oracle_lib):
    """The reference's 2-D tuple at its GPU-benchmark scale (grid 100: 99 x 99
    cells, K = 10, 1e7 events): packed slots and events bit-exact with the
    oracle's restatement of the reference core, gradients within the tuple
    tolerance (rtol 1e-9)."""
    from quantom_loits_b200 import backend
    from quantom_loits_b200 import workloads

    spec = workloads.theory_tuple(grid=100, knots=10, n_events=10_000_000)
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(DEV) for a in spec.arrays]
    ev, st = backend.tuple_forward(*t, spec.n_events, spec.seed, spec.sequence)
    ref = oracle_lib.r_forward(*spec.arrays, spec.n_events, spec.seed, spec.sequence)
    assert np.array_equal(st["packed"].cpu().numpy(), ref["packed"])
    assert np.array_equal(ev.cpu().numpy(), ref["events"])
    g = np.random.default_rng(5).standard_normal(ref["events"].shape)
    gx, gq = backend.tuple_backward(torch.from_numpy(g).to(DEV), t[0], t[1], t[2], t[3], t[5], st,
                                    spec.seed, spec.sequence)
    rgx, rgq = oracle_lib.r_backward(g, ref, spec.x_bins, spec.xsec_x, spec.q_bins, spec.xsec_q,
                                     spec.acceptance, spec.seed, spec.sequence)
    np.testing.assert_allclose(gx.cpu().numpy(), rgx, rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(gq.cpu().numpy(), rgq, rtol=1e-9, atol=1e-10)
