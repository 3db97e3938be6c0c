"""GPU parity of the batched ragged-density sampler (fp32 storage) through the C ABI.

References:
* golden vectors of the reference's own compiled core on the exact embedding
  of a batch into the reference tuple (tests/golden/make_golden.py);
* the CPU oracle (fp64) for larger shapes, the CDF, quantiles and the
  branch-frozen central finite differences;
* a plain PyTorch fp64 restatement of the reference's torch stages
  (pytorch/loits.py:16-63) differentiated by autograd with the same uniforms.

Tolerances (stated by the sampler's contract): events within 1e-5 relative of
the reference; intervals bit-exact except where u lies within 2 ulp of a CDF
knot (counted); row offsets / compaction order exact; gradients within 1e-4
of the gradient scale; CDF within 1e-6 of the fp64 oracle.
"""
import numpy as np
import pytest
import torch

from conftest import DENSITY_CASES, golden_case

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")
EVENT_RTOL = 1e-5
GRAD_TOL = 1e-4
CDF_TOL = 1e-6


@pytest.fixture(scope="module")
def B():
    from quantom_loits_b200 import batched

    return batched


def run_batch(B, case, config=None, with_intervals=True, seed=None, sequence=None):
    """Forward (+ backward when a cotangent is given) on static buffers."""
    koff, counts = case["knot_offsets"], case["event_counts"]
    plan = B.BatchPlan(koff, counts, config, DEV)
    grid = torch.from_numpy(np.ascontiguousarray(case["grid"], dtype=np.float32)).to(DEV)
    values = torch.from_numpy(np.ascontiguousarray(case["values"], dtype=np.float32)).to(DEV)
    x_cut = case.get("x_cut")
    x_cut = None if x_cut is None else torch.from_numpy(np.asarray(x_cut, np.float32)).to(DEV)
    seed = int(case["scalars"][0]) if seed is None else seed
    seq = int(case["scalars"][1]) if sequence is None else sequence
    events, rows, ws = plan.new_events(), plan.new_row_offsets(), plan.new_workspace()
    ints = torch.full((max(plan.capacity, 1),), -1, dtype=torch.int32, device=DEV) if with_intervals else None
    plan.forward(grid, values, x_cut, seed, seq, events, rows, ws, ints)
    plan.check_status(ws)
    valid = int(rows[-1].item())
    out = dict(plan=plan, events=events[:valid].cpu().numpy(), rows=rows.cpu().numpy(), ws=ws,
               valid=valid, grid=grid, values=values, x_cut=x_cut, seed=seed, seq=seq)
    if with_intervals:
        out["intervals"] = ints[:valid].cpu().numpy()
    if "cotangent" in case:
        g = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=DEV)
        g[:valid] = torch.from_numpy(np.asarray(case["cotangent"], dtype=np.float32)).to(DEV)
        gv = torch.empty_like(values)
        plan.backward(grid, values, x_cut, seed, seq, g, gv, ws)
        plan.check_status(ws)
        out["grad_values"] = gv.cpu().numpy()
    return out


def near_knot(u, cdf_row, ulps=2):
    """True where fp32 u lies within `ulps` fp32 ulps of some CDF knot."""
    u = np.asarray(u, np.float32)
    spacing = np.spacing(u.astype(np.float32)).astype(np.float64) * ulps
    idx = np.searchsorted(cdf_row, u.astype(np.float64))
    lo = np.abs(u - cdf_row[np.clip(idx - 1, 0, len(cdf_row) - 1)])
    hi = np.abs(u - cdf_row[np.clip(idx, 0, len(cdf_row) - 1)])
    return np.minimum(lo, hi) <= np.maximum(spacing, 2.0**-24 * ulps)


def check_against_oracle(out, case, ora, x_cut=None, density_base=0, slot_stride=0):
    eoff = np.concatenate([[0], np.cumsum(case["event_counts"])])
    ref = ora.d_forward(case["knot_offsets"], eoff, case["grid"], case["values"], x_cut,
                        out["seed"], out["seq"], density_base, slot_stride)
    return ref


@pytest.mark.parametrize("name", DENSITY_CASES)
def test_forward_backward_match_reference(B, golden, oracle_lib, name):
    c = golden_case(golden, name)
    out = run_batch(B, c)
    # compaction order and per-density row offsets: exact
    assert np.array_equal(out["rows"], c["row_offsets"])
    np.testing.assert_allclose(out["events"], c["events"], rtol=EVENT_RTOL, atol=0)
    # intervals: exact except u within 2 ulp of a knot
    diff = out["intervals"] != c["intervals"]
    if diff.any():
        eoff = np.concatenate([[0], np.cumsum(c["event_counts"])])
        ref = oracle_lib.d_forward(c["knot_offsets"], eoff, c["grid"], c["values"], c.get("x_cut"),
                                   out["seed"], out["seq"])
        for r in np.flatnonzero(diff):
            b = np.searchsorted(c["row_offsets"], r, side="right") - 1
            o, e = c["knot_offsets"][b], c["knot_offsets"][b + 1]
            assert near_knot(ref["u"][r:r + 1], ref["cdf"][o:e])[0], f"row {r} flipped far from a knot"
    scale = np.abs(c["grad_values"]).max()
    assert np.abs(out["grad_values"] - c["grad_values"]).max() <= GRAD_TOL * scale


def test_single_density_workload_matches_reference_digest(B, golden):
    """The 256-knot, 1e5-event workload: every kept event within 1e-5 of the
    reference (strided sample) and the same number of rows."""
    c = golden_case(golden, "single")
    c = dict(c)
    out = run_batch(B, c)
    assert out["valid"] == 100_000
    np.testing.assert_allclose(out["events"][c["sample_index"]], c["events_sample"],
                               rtol=EVENT_RTOL, atol=0)


def test_cdf_matches_fp64_oracle(B, golden, oracle_lib):
    for name in DENSITY_CASES:
        c = golden_case(golden, name)
        out = run_batch(B, c, with_intervals=False)
        cdf, norm = out["plan"].cdf(out["ws"])
        onorm, ocdf, _ = oracle_lib.d_cdf(c["knot_offsets"], c["grid"], c["values"])
        err = np.abs(cdf.cpu().numpy() - ocdf).max()
        assert err <= CDF_TOL, (name, err)
        np.testing.assert_allclose(norm.cpu().numpy(), onorm, rtol=1e-12)


# The backward accumulates each chunk's grad-CDF with fp32 atomics, whose
# order varies from run to run, or with order-independent fixed-point sums:
# gradients are reproducible to fp32 accumulation rounding, events and row
# offsets bit for bit.
GRAD_REPRO = 1e-6


def test_plain_and_persistent_forms_agree(B, golden):
    c = golden_case(golden, "ragged_workload_small")
    a = run_batch(B, c)
    b = run_batch(B, c, B.make_config(plain=1))
    assert np.array_equal(a["rows"], b["rows"])
    assert np.array_equal(a["events"], b["events"])
    scale = np.abs(a["grad_values"]).max()
    assert np.abs(a["grad_values"] - b["grad_values"]).max() <= GRAD_REPRO * scale


@pytest.mark.parametrize("threads,blocks,scan", [(256, 2, 1), (256, 2, 3), (512, 4, 8),
                                                 (512, 8, 16), (256, 16, 64), (1024, 2, 1),
                                                 (1024, 8, 4), (1024, 16, 8)])
def test_launch_geometries_agree(B, golden, threads, blocks, scan):
    c = golden_case(golden, "ragged_small")
    a = run_batch(B, c)
    b = run_batch(B, c, B.make_config(threads=threads, blocks_per_item=blocks, scan_knots=scan))
    assert np.array_equal(a["rows"], b["rows"])
    assert np.array_equal(a["events"], b["events"])
    assert np.array_equal(a["intervals"], b["intervals"])
    scale = np.abs(a["grad_values"]).max()
    assert np.abs(a["grad_values"] - b["grad_values"]).max() <= GRAD_REPRO * scale


def test_graph_replay_matches_eager(B):
    from quantom_loits_b200 import workloads

    spec = workloads.uniform(scale=5e-3, n_densities=8)
    plan = B.BatchPlan(spec.knot_offsets, spec.event_counts, None, DEV)
    step = B.BatchStep(plan, seed=spec.seed)
    step.grid.copy_(torch.from_numpy(spec.grid))
    step.values.copy_(torch.from_numpy(spec.values))
    step.grad_events.normal_()
    step.step()
    step.check_status()
    ev0, gv0 = step.events.clone(), step.grad_values.clone()
    step.capture()
    step.events.zero_()
    step.grad_values.zero_()
    for _ in range(3):
        step.step()
    torch.cuda.synchronize()
    step.check_status()
    assert torch.equal(step.events, ev0)
    scale = gv0.abs().max()
    assert (step.grad_values - gv0).abs().max() <= GRAD_REPRO * scale


def test_shards_reproduce_the_whole_batch(B, golden):
    """Densities split across plans with (density_base, slot_stride) sample the
    same events as the unsplit batch (the multi-GPU sharding contract)."""
    c = golden_case(golden, "ragged_workload_small")
    full = run_batch(B, c)
    from quantom_loits_b200 import sharding

    nmax = int(np.max(c["event_counts"]))
    parts = []
    for rank in range(3):
        lo, hi = sharding.shard_range(c["event_counts"], 3, rank)
        if lo == hi:
            continue
        sub = sharding.sub_case(c, lo, hi)
        cfg = B.make_config(density_base=lo, slot_stride=nmax)
        parts.append(run_batch(B, sub, cfg, seed=full["seed"], sequence=full["seq"]))
    assert np.array_equal(np.concatenate([p["events"] for p in parts]), full["events"])


def test_quantiles_match_oracle(B, oracle_lib):
    from quantom_loits_b200 import workloads

    spec = workloads.uniform(scale=1e-3, n_densities=4)
    case = dict(knot_offsets=spec.knot_offsets, event_counts=spec.event_counts, grid=spec.grid,
                values=spec.values, scalars=np.array([1234, 0]))
    out = run_batch(B, case, with_intervals=False)
    _, ocdf, _ = oracle_lib.d_cdf(spec.knot_offsets, spec.grid, spec.values)
    p = np.array([1e-6, 0.5, 1 - 1e-6], dtype=np.float32)
    for b in range(4):
        x, j = out["plan"].quantile(out["ws"], b, torch.from_numpy(p))
        xo, jo = oracle_lib.d_quantile(b, spec.knot_offsets, spec.grid, ocdf, p.astype(np.float64))
        np.testing.assert_allclose(x.cpu().numpy(), xo, rtol=EVENT_RTOL)
        assert np.array_equal(j.cpu().numpy(), jo)


def torch_reference_events(grid, values, koff, u_rows, rows_density, x_cut):
    """fp64 restatement of the reference torch stages (pytorch/loits.py:16-63)
    on 1-D densities with given uniforms; differentiable w.r.t. values."""
    xs = []
    for b in range(len(koff) - 1):
        o, e = int(koff[b]), int(koff[b + 1])
        g, f = grid[o:e], values[o:e]
        norm = torch.trapezoid(f, g)
        rho = f / norm
        cdf = torch.nn.functional.pad(torch.cumulative_trapezoid(rho, g), (1, 0))
        m = (g[1:] - g[:-1]) / (cdf[1:] - cdf[:-1] + 1e-5)
        c0 = g[:-1] - m * cdf[:-1]
        u = u_rows[rows_density == b]
        j = ((u[:, None] >= cdf[None, :]).sum(-1) - 1).clamp(0, len(m) - 1)
        xs.append(torch.gather(m, 0, j) * u + torch.gather(c0, 0, j))
    return torch.cat(xs)


def test_gradient_matches_torch_autograd(B, golden, oracle_lib):
    c = golden_case(golden, "ragged_small")
    out = run_batch(B, c)
    eoff = np.concatenate([[0], np.cumsum(c["event_counts"])])
    ref = oracle_lib.d_forward(c["knot_offsets"], eoff, c["grid"], c["values"], c["x_cut"],
                               out["seed"], out["seq"])
    rows_d = np.repeat(np.arange(len(c["event_counts"])), np.diff(ref["row_offsets"]))
    values = torch.tensor(c["values"], dtype=torch.float64, requires_grad=True)
    x = torch_reference_events(torch.tensor(c["grid"], dtype=torch.float64), values,
                               c["knot_offsets"], torch.tensor(ref["u"], dtype=torch.float64),
                               torch.tensor(rows_d), c["x_cut"])
    np.testing.assert_allclose(x.detach().numpy(), out["events"], rtol=EVENT_RTOL)
    (x * torch.tensor(c["cotangent"], dtype=torch.float64)).sum().backward()
    tg = values.grad.numpy()
    scale = np.abs(tg).max()
    assert np.abs(out["grad_values"] - tg).max() <= GRAD_TOL * scale


def test_finite_difference_gradient_uniform_workload(B, oracle_lib):
    """The 64 x 1024-knot workload (event count scaled to 2e4 per density):
    analytic VJP vs branch-frozen FP64 central differences, step 1e-6
    relative, at 32 random grid entries."""
    from quantom_loits_b200 import workloads

    spec = workloads.uniform(scale=0.02)
    rng = np.random.default_rng(0)
    case = dict(knot_offsets=spec.knot_offsets, event_counts=spec.event_counts, grid=spec.grid,
                values=spec.values, scalars=np.array([spec.seed, 0]))
    case["cotangent"] = rng.standard_normal(spec.total_events).astype(np.float32)
    out = run_batch(B, case, with_intervals=False)
    assert out["valid"] == spec.total_events
    eoff = spec.event_offsets
    rows = out["rows"]
    flips_total = 0
    for _ in range(32):
        b = int(rng.integers(0, spec.n_densities))
        o, k = int(spec.knot_offsets[b]), int(spec.knot_offsets[b + 1] - spec.knot_offsets[b])
        t = int(rng.integers(0, k))
        fmean = float(np.abs(spec.values[o:o + k]).mean())
        h = 1e-6 * max(abs(float(spec.values[o + t])), fmean)
        d, flips = oracle_lib.d_fd(b, t, h, spec.knot_offsets, eoff, spec.grid, spec.values, None,
                                   spec.seed, 0, case["cotangent"][rows[b]:rows[b + 1]])
        flips_total += flips
        scale = max(np.abs(out["grad_values"][o:o + k]).max(), 1e-12)
        assert abs(out["grad_values"][o + t] - d) <= GRAD_TOL * scale, (b, t, d)


def test_non_monotone_density_uses_count_semantics(B, oracle_lib):
    """Negative density values make the CDF non-monotone; the reference then
    counts every knot (cpp/loits_core.cpp:12-18) and so must the sampler."""
    grid = np.linspace(0.0, 1.0, 9, dtype=np.float32)
    values = np.array([1.0, 2.0, -1.5, -0.5, 1.0, 3.0, 0.5, -0.2, 1.0], dtype=np.float32)
    case = dict(knot_offsets=np.array([0, 9]), event_counts=np.array([5000]), grid=grid,
                values=values, scalars=np.array([7, 3]))
    out = run_batch(B, case)
    ref = oracle_lib.d_forward(case["knot_offsets"], np.array([0, 5000]), grid, values, None, 7, 3)
    assert ref["monotone"][0] == 0
    assert out["valid"] == len(ref["events"])
    np.testing.assert_allclose(out["events"], ref["events"], rtol=EVENT_RTOL, atol=1e-6)
    assert np.mean(out["intervals"] == ref["intervals"]) > 0.999


def test_empty_and_tiny_densities(B, oracle_lib):
    grid = np.concatenate([np.array([0.2, 0.4], np.float32), np.linspace(0.1, 1, 5, dtype=np.float32),
                           np.array([0.5, 0.6], np.float32)])
    values = np.concatenate([np.array([1.0, 1.0], np.float32), np.ones(5, np.float32),
                             np.array([0.0, 2.0], np.float32)])
    koff = np.array([0, 2, 7, 9])
    for counts in ([0, 0, 0], [0, 13, 0], [3, 0, 1], [1, 1, 1]):
        case = dict(knot_offsets=koff, event_counts=np.array(counts), grid=grid, values=values,
                    scalars=np.array([3, 1]))
        out = run_batch(B, case)
        ref = oracle_lib.d_forward(koff, np.concatenate([[0], np.cumsum(counts)]), grid, values,
                                   None, 3, 1)
        assert np.array_equal(out["rows"], ref["row_offsets"]), counts
        np.testing.assert_allclose(out["events"], ref["events"], rtol=EVENT_RTOL)


def test_identity_compaction_path_matches_general_path(B):
    """Densities whose every event is kept (grid > 0, no effective cut) take
    the identity-compaction path; putting the cut exactly at the first knot
    forces the general compaction path, which may only additionally drop
    events with x == g_0.  Both must give the same surviving rows, and the
    same gradient for the same cotangent."""
    from quantom_loits_b200 import workloads

    spec = workloads.uniform(scale=4e-3, n_densities=5)
    base = dict(knot_offsets=spec.knot_offsets, event_counts=spec.event_counts, grid=spec.grid,
                values=spec.values, scalars=np.array([spec.seed, 3]))
    fast = run_batch(B, base)
    g0 = spec.grid[spec.knot_offsets[:-1]]
    slow = run_batch(B, dict(base, x_cut=g0.astype(np.float32)))
    keep = np.concatenate([fast["events"][fast["rows"][b]:fast["rows"][b + 1]] > g0[b]
                           for b in range(spec.n_densities)])
    assert np.array_equal(fast["events"][keep], slow["events"])
    assert np.array_equal(fast["intervals"][keep], slow["intervals"])
    rng = np.random.default_rng(3)
    cot = rng.standard_normal(fast["valid"]).astype(np.float32)
    gf = run_batch(B, dict(base, cotangent=cot))["grad_values"]
    gs = run_batch(B, dict(base, x_cut=g0.astype(np.float32), cotangent=cot[keep]))["grad_values"]
    scale = np.abs(gf).max()
    assert np.abs(gf - gs).max() <= GRAD_REPRO * scale


@pytest.mark.parametrize("threads", [256, 1024])
def test_large_knot_densities_match_oracle(B, oracle_lib, threads):
    """Densities of up to 8192 knots (the most a sampling CTA holds), where
    shared memory caps the guide table below 2G buckets so buckets hold several
    knots, with a cut: rows exact, events and gradients against the fp64
    oracle, intervals exact except next to a knot."""
    rng = np.random.default_rng(21)
    sizes = [8192, 5001, 8191, 64]
    grids, vals = [], []
    for g in sizes:
        x = np.linspace(1e-3, 1.0, g, dtype=np.float32)
        a, b = rng.uniform(-0.5, 1.0), rng.uniform(1.0, 5.0)
        grids.append(x)
        vals.append((np.power(x.astype(np.float64), a) * np.power(1.0 - x, b)).astype(np.float32))
    koff = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    counts = np.array([60_000, 25_000, 40_000, 3_000], dtype=np.int64)
    x_cut = rng.uniform(0.01, 0.1, len(sizes)).astype(np.float32)
    grid, values = np.concatenate(grids), np.concatenate(vals)
    eoff = np.concatenate([[0], np.cumsum(counts)])
    ref = oracle_lib.d_forward(koff, eoff, grid, values, x_cut, 99, 2)
    cot = rng.standard_normal(len(ref["events"])).astype(np.float32)
    case = dict(knot_offsets=koff, event_counts=counts, grid=grid, values=values, x_cut=x_cut,
                scalars=np.array([99, 2]), cotangent=cot)
    out = run_batch(B, case, B.make_config(threads=threads))
    assert np.array_equal(out["rows"], ref["row_offsets"])
    np.testing.assert_allclose(out["events"], ref["events"], rtol=EVENT_RTOL)
    for r in np.flatnonzero(out["intervals"] != ref["intervals"]):
        b = np.searchsorted(ref["row_offsets"], r, side="right") - 1
        assert near_knot(ref["u"][r:r + 1], ref["cdf"][koff[b]:koff[b + 1]])[0], r
    gref = oracle_lib.d_backward(koff, eoff, grid, values, x_cut, 99, 2, cot, fwd=ref)
    for b in range(len(sizes)):
        o, e = koff[b], koff[b + 1]
        scale = np.abs(gref[o:e]).max()
        assert np.abs(out["grad_values"][o:e] - gref[o:e]).max() <= GRAD_TOL * scale, b


def test_default_cta_size_follows_occupancy(B):
    """Without a configuration the plan takes the CTA size with the most
    resident threads: 256 for 1024-knot densities (five CTAs per SM), 1024
    when 8192-knot records leave room for one CTA per SM."""
    small = B.BatchPlan(np.array([0, 1024, 2048]), np.array([10, 10]), None, DEV)
    large = B.BatchPlan(np.array([0, 8192, 8256]), np.array([10, 10]), None, DEV)
    assert small.config["threads"] == 256 and small.config["blocks_per_item"] == 16
    assert large.config["threads"] == 1024 and large.config["blocks_per_item"] == 8


def test_plans_of_different_sizes_coexist(B, oracle_lib):
    """A plan for small densities built after one for large densities must not
    lower the shared memory the large plan launches with."""
    rng = np.random.default_rng(4)
    big = dict(knot_offsets=np.array([0, 8000]), event_counts=np.array([5000]),
               grid=np.linspace(0.01, 1.0, 8000, dtype=np.float32),
               values=rng.uniform(0.5, 1.5, 8000).astype(np.float32), scalars=np.array([5, 1]))
    cfg = B.make_config(threads=256)
    keep = B.BatchPlan(big["knot_offsets"], big["event_counts"], cfg, DEV)
    small = B.BatchPlan(np.array([0, 16]), np.array([100]), cfg, DEV)
    out = run_batch(B, big, cfg)
    ref = oracle_lib.d_forward(big["knot_offsets"], np.array([0, 5000]), big["grid"],
                               big["values"], None, 5, 1)
    np.testing.assert_allclose(out["events"], ref["events"], rtol=EVENT_RTOL)
    del keep, small


def test_autotuner_picks_a_geometry_that_samples_identically(B, tmp_path):
    from quantom_loits_b200 import tuning, workloads

    spec = workloads.ragged(scale=0.01, n_densities=24)
    batch = B.DensityBatch.from_spec(spec, DEV)
    tuner = tuning.Autotuner(DEV, reps=2, cache_path=tmp_path / "tune.json")
    cfg = tuner.config_for(batch, seed=spec.seed)
    key = tuner.key_for(batch)
    assert key.startswith(tuning.shape_key(spec.knot_offsets, spec.event_counts, True))
    assert tuner.table[key] == cfg and len(tuner.timings[key]) >= 4
    # the cache file serves a new tuner without timing
    again = tuning.Autotuner(DEV, cache_path=tmp_path / "tune.json")
    assert again.config_for(batch) == cfg and not again.timings
    case = dict(knot_offsets=spec.knot_offsets, event_counts=spec.event_counts, grid=spec.grid,
                values=spec.values, x_cut=spec.x_cut, scalars=np.array([spec.seed, 0]))
    a = run_batch(B, case)
    b = run_batch(B, case, B.make_config(**tuning.plain_config(cfg)))
    assert np.array_equal(a["rows"], b["rows"]) and np.array_equal(a["events"], b["events"])
    # BatchedLOITS(config="auto") goes through the same tuner
    sampler = B.BatchedLOITS(DEV, seed=spec.seed, config="auto")
    ev, rows = sampler.sample(batch, sequence=0)
    assert torch.equal(ev.cpu(), torch.from_numpy(a["events"]))


def _large_case(rng, sizes, counts, cut=True, seed=77, seq=5):
    grids, vals = [], []
    for g in sizes:
        x = np.linspace(1e-3, 1.0, g, dtype=np.float32)
        mu, sig = rng.uniform(0.2, 0.8), 10 ** rng.uniform(-3, -1.5)
        f = np.exp(-0.5 * ((x.astype(np.float64) - mu) / sig) ** 2) + 1e-3 * np.power(x, -0.5)
        grids.append(x)
        vals.append(f.astype(np.float32))
    koff = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    case = dict(knot_offsets=koff, event_counts=np.asarray(counts, np.int64),
                grid=np.concatenate(grids), values=np.concatenate(vals),
                scalars=np.array([seed, seq]))
    if cut:
        case["x_cut"] = rng.uniform(0.01, 0.1, len(sizes)).astype(np.float32)
    return case


@pytest.mark.parametrize("threads", [256, 1024])
def test_large_densities_sampled_from_global_memory(B, oracle_lib, threads):
    """Densities above 8192 knots (here up to 70001, past 16-bit guide counts)
    are sampled from records and guide in global memory, beside small ones in
    the same batch; events, rows and intervals against the fp64 oracle, the
    VJP (fp64 global atomics + multi-tile reverse scan) against the oracle's."""
    rng = np.random.default_rng(31)
    case = _large_case(rng, [20000, 300, 70001, 9000], [150_000, 20_000, 200_000, 50_000])
    koff, counts = case["knot_offsets"], case["event_counts"]
    eoff = np.concatenate([[0], np.cumsum(counts)])
    ref = oracle_lib.d_forward(koff, eoff, case["grid"], case["values"], case["x_cut"], 77, 5)
    case["cotangent"] = rng.standard_normal(len(ref["events"])).astype(np.float32)
    out = run_batch(B, case, B.make_config(threads=threads))
    assert np.array_equal(out["rows"], ref["row_offsets"])
    np.testing.assert_allclose(out["events"], ref["events"], rtol=EVENT_RTOL)
    for r in np.flatnonzero(out["intervals"] != ref["intervals"]):
        b = np.searchsorted(ref["row_offsets"], r, side="right") - 1
        assert near_knot(ref["u"][r:r + 1], ref["cdf"][koff[b]:koff[b + 1]])[0], r
    gref = oracle_lib.d_backward(koff, eoff, case["grid"], case["values"], case["x_cut"], 77, 5,
                                 case["cotangent"], fwd=ref)
    for b in range(len(counts)):
        o, e = koff[b], koff[b + 1]
        scale = np.abs(gref[o:e]).max()
        assert np.abs(out["grad_values"][o:e] - gref[o:e]).max() <= GRAD_TOL * scale, b
    cdf, _ = out["plan"].cdf(out["ws"])
    assert np.abs(cdf.cpu().numpy() - ref["cdf"]).max() <= CDF_TOL


@pytest.mark.parametrize("threads,cut", [(256, True), (512, True), (1024, True), (1024, False)])
def test_large_densities_across_many_chunks(B, oracle_lib, threads, cut):
    """Large densities with millions of events beside small ones: each CTA
    takes several forward tiles and backward chunks in turn, on different
    densities (the backward's coarse shared guide is reloaded when the
    density changes).  Events, rows and the VJP against the fp64 oracle."""
    rng = np.random.default_rng(33)
    case = _large_case(rng, [20000, 300, 70001, 9000, 15000],
                       [2_000_000, 200_000, 2_500_000, 800_000, 1_500_000], cut=cut)
    koff, counts = case["knot_offsets"], case["event_counts"]
    eoff = np.concatenate([[0], np.cumsum(counts)])
    ref = oracle_lib.d_forward(koff, eoff, case["grid"], case["values"], case.get("x_cut"), 77, 5)
    case["cotangent"] = rng.standard_normal(len(ref["events"])).astype(np.float32)
    out = run_batch(B, case, B.make_config(threads=threads), with_intervals=False)
    assert np.array_equal(out["rows"], ref["row_offsets"])
    np.testing.assert_allclose(out["events"], ref["events"], rtol=EVENT_RTOL)
    gref = oracle_lib.d_backward(koff, eoff, case["grid"], case["values"], case.get("x_cut"), 77,
                                 5, case["cotangent"], fwd=ref)
    for b in range(len(counts)):
        o, e = koff[b], koff[b + 1]
        scale = np.abs(gref[o:e]).max()
        assert np.abs(out["grad_values"][o:e] - gref[o:e]).max() <= GRAD_TOL * scale, b


def test_large_densities_plain_and_persistent_agree(B):
    rng = np.random.default_rng(32)
    case = _large_case(rng, [12000, 40000], [80_000, 120_000])
    a = run_batch(B, case)
    b = run_batch(B, case, B.make_config(plain=1))
    assert np.array_equal(a["rows"], b["rows"]) and np.array_equal(a["events"], b["events"])


def test_large_non_monotone_density_is_reported_unsupported(B):
    """Count semantics over every knot would cost O(G) per event for a large
    density: the sampler reports LOITS_ERR_UNSUPPORTED instead of sampling."""
    g = 10000
    grid = np.linspace(0.0, 1.0, g, dtype=np.float32)
    values = np.ones(g, np.float32)
    values[5000] = -100.0
    plan = B.BatchPlan(np.array([0, g]), np.array([1000]), None, DEV)
    ws, ev, rows = plan.new_workspace(), plan.new_events(), plan.new_row_offsets()
    plan.forward(torch.from_numpy(grid).to(DEV), torch.from_numpy(values).to(DEV), None, 1, 0,
                 ev, rows, ws)
    with pytest.raises(RuntimeError, match="supported|UNSUPPORTED|unsupported"):
        plan.check_status(ws)
    assert int(rows[-1].item()) == 0


def test_precision_workload_shape_matches_oracle(B, oracle_lib):
    """Two densities of the precision workload (2^20 knots over [1e-6, 1],
    narrow Gaussian plus x^-0.5 tail) with 2e5 events each: CDF within 1e-6
    of fp64, events within 1e-5, quantiles at p = 1e-6, 0.5, 1 - 1e-6."""
    from quantom_loits_b200 import workloads

    spec = workloads.precision(scale=0.02, n_densities=2)
    case = dict(knot_offsets=spec.knot_offsets, event_counts=spec.event_counts, grid=spec.grid,
                values=spec.values, scalars=np.array([spec.seed, 0]))
    out = run_batch(B, case)
    eoff = spec.event_offsets
    ref = oracle_lib.d_forward(spec.knot_offsets, eoff, spec.grid, spec.values, None, spec.seed, 0)
    assert np.array_equal(out["rows"], ref["row_offsets"])
    np.testing.assert_allclose(out["events"], ref["events"], rtol=EVENT_RTOL)
    cdf, _ = out["plan"].cdf(out["ws"])
    assert np.abs(cdf.cpu().numpy() - ref["cdf"]).max() <= CDF_TOL
    p = np.array([1e-6, 0.5, 1 - 1e-6], dtype=np.float32)
    for b in range(2):
        x, j = out["plan"].quantile(out["ws"], b, torch.from_numpy(p))
        xo, jo = oracle_lib.d_quantile(b, spec.knot_offsets, spec.grid, ref["cdf"],
                                       p.astype(np.float64))
        np.testing.assert_allclose(x.cpu().numpy(), xo, rtol=EVENT_RTOL)


def _fixed_point_case(n_dens=6, knots=1024, events=60_000):
    """Densities whose backward sums run in fixed point on 512/1024-thread
    CTAs (one fp32 copy of the sums would fill the slot: G = gcap <= 4096)."""
    from quantom_loits_b200 import workloads

    spec = workloads.uniform(scale=events / 1e6, n_densities=n_dens, knots=knots)
    return dict(knot_offsets=spec.knot_offsets, event_counts=spec.event_counts, grid=spec.grid,
                values=spec.values, scalars=np.array([spec.seed, 2]))


@pytest.mark.parametrize("threads", [512, 1024])
def test_fixed_point_backward_is_bit_reproducible(B, oracle_lib, threads):
    """Integer sums do not depend on the order of the atomics: two backward
    runs give bit-identical gradients, within 1e-4 of the oracle's."""
    case = _fixed_point_case()
    koff, counts = case["knot_offsets"], case["event_counts"]
    eoff = np.concatenate([[0], np.cumsum(counts)])
    seed, seq = int(case["scalars"][0]), int(case["scalars"][1])
    ref = oracle_lib.d_forward(koff, eoff, case["grid"], case["values"], None, seed, seq)
    case["cotangent"] = np.random.default_rng(3).standard_normal(len(ref["events"])).astype(np.float32)
    out = run_batch(B, case, B.make_config(threads=threads), with_intervals=False)
    plan, ws = out["plan"], out["ws"]
    g = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=DEV)
    g[:out["valid"]] = torch.from_numpy(case["cotangent"]).to(DEV)
    again = torch.empty_like(out["values"])
    plan.backward(out["grid"], out["values"], None, out["seed"], out["seq"], g, again, ws)
    plan.check_status(ws)
    assert np.array_equal(again.cpu().numpy(), out["grad_values"])
    gref = oracle_lib.d_backward(koff, eoff, case["grid"], case["values"], None, seed, seq,
                                 case["cotangent"], fwd=ref)
    for b in range(len(counts)):
        o, e = koff[b], koff[b + 1]
        scale = np.abs(gref[o:e]).max()
        assert np.abs(out["grad_values"][o:e] - gref[o:e]).max() <= GRAD_TOL * scale, b


@pytest.mark.parametrize("threads", [256, 512])
def test_non_finite_cotangent_poisons_only_its_density(B, threads):
    """A NaN cotangent makes its density's gradient non-finite (the
    normaliser VJP sums over every knot, as in the reference); the other
    densities' gradients are unchanged."""
    case = _fixed_point_case(n_dens=4, events=20_000)
    out = run_batch(B, case, B.make_config(threads=threads), with_intervals=False)
    plan, ws = out["plan"], out["ws"]
    rows = out["rows"]
    g = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=DEV)
    g[:out["valid"]] = torch.randn(out["valid"], generator=torch.Generator(device=DEV).manual_seed(9),
                                   device=DEV)
    clean = torch.empty_like(out["values"])
    plan.backward(out["grid"], out["values"], None, out["seed"], out["seq"], g, clean, ws)
    g[int(rows[1]) + 17] = float("nan")
    dirty = torch.empty_like(out["values"])
    plan.backward(out["grid"], out["values"], None, out["seed"], out["seq"], g, dirty, ws)
    plan.check_status(ws)
    koff = case["knot_offsets"]
    c, d = clean.cpu().numpy(), dirty.cpu().numpy()
    assert not np.isfinite(d[koff[1]:koff[2]]).any()
    for b in (0, 2, 3):
        o, e = koff[b], koff[b + 1]
        assert np.isfinite(d[o:e]).all()
        np.testing.assert_allclose(d[o:e], c[o:e], rtol=1e-5, atol=1e-6 * np.abs(c[o:e]).max())


@pytest.mark.parametrize("threads", [512, 1024])
def test_fixed_point_backward_takes_outlier_cotangents_in_fp32(B, oracle_lib, threads):
    """Three cotangents ~4e12 times the typical one, in the same interval and
    far past the rows a chunk's fixed-point scale is taken from: each term is
    below the old 2^63 limit, but their sum is not.  Terms above the chunk's
    cap (2^62 / its kept rows) go through fp32 reductions instead, so the
    gradient still matches the fp64 oracle within 1e-4 of its scale."""
    case = _fixed_point_case(n_dens=3, events=60_000)
    koff, counts = case["knot_offsets"], case["event_counts"]
    eoff = np.concatenate([[0], np.cumsum(counts)])
    seed, seq = int(case["scalars"][0]), int(case["scalars"][1])
    ref = oracle_lib.d_forward(koff, eoff, case["grid"], case["values"], None, seed, seq)
    cot = np.random.default_rng(11).standard_normal(len(ref["events"])).astype(np.float32)
    # density 1's rows past its first 20000, three of them in one interval
    lo, hi = int(ref["row_offsets"][1]) + 20_000, int(ref["row_offsets"][2])
    ints = ref["intervals"][lo:hi]
    vals, first, cnt = np.unique(ints, return_index=True, return_counts=True)
    pick = lo + np.flatnonzero(ints == vals[np.argmax(cnt)])[:3]
    assert len(pick) == 3
    cot[pick] = 3.0e12
    case["cotangent"] = cot
    out = run_batch(B, case, B.make_config(threads=threads), with_intervals=False)
    gref = oracle_lib.d_backward(koff, eoff, case["grid"], case["values"], None, seed, seq, cot,
                                 fwd=ref)
    for b in range(len(counts)):
        o, e = koff[b], koff[b + 1]
        assert np.isfinite(out["grad_values"][o:e]).all(), b
        scale = np.abs(gref[o:e]).max()
        assert np.abs(out["grad_values"][o:e] - gref[o:e]).max() <= GRAD_TOL * scale, b


def test_per_density_tile_lengths_and_scan_widths_change_no_result(B):
    """A plan whose densities each have their own sampling tile length and
    CDF scan width (loits_batch_plan_create_ex, the autotuner's per-bucket
    tables) samples the same events and rows as the uniform geometry, and its
    gradient agrees to fp32 accumulation order; out-of-range tables are
    rejected on the host."""
    from quantom_loits_b200 import _native as N
    from quantom_loits_b200 import workloads

    spec = workloads.ragged(scale=0.02, n_densities=20)
    case = dict(knot_offsets=spec.knot_offsets, event_counts=spec.event_counts, grid=spec.grid,
                values=spec.values, x_cut=spec.x_cut, scalars=np.array([spec.seed, 3]))
    cfg = B.make_config(threads=512, blocks_per_item=16, scan_knots=8)
    kept = run_batch(B, case, cfg, with_intervals=False)["valid"]
    case["cotangent"] = np.random.default_rng(2).standard_normal(kept).astype(np.float32)
    ref = run_batch(B, case, cfg)
    rng = np.random.default_rng(5)
    blocks = rng.choice([1, 2, 4, 7, 16], size=spec.n_densities).astype(np.int32)
    scan = rng.choice([1, 3, 8, 16, 64], size=spec.n_densities).astype(np.int32)
    koff, counts = spec.knot_offsets, spec.event_counts
    plan = B.BatchPlan(koff, counts, cfg, DEV, density_blocks=blocks, density_scan=scan)
    grid = torch.from_numpy(spec.grid).to(DEV)
    values = torch.from_numpy(spec.values).to(DEV)
    x_cut = torch.from_numpy(spec.x_cut).to(DEV)
    events, rows, ws = plan.new_events(), plan.new_row_offsets(), plan.new_workspace()
    ints = torch.full((max(plan.capacity, 1),), -1, dtype=torch.int32, device=DEV)
    plan.forward(grid, values, x_cut, spec.seed, 3, events, rows, ws, ints)
    plan.check_status(ws)
    n = int(rows[-1].item())
    assert np.array_equal(rows.cpu().numpy(), ref["rows"])
    assert np.array_equal(events[:n].cpu().numpy(), ref["events"])
    assert np.array_equal(ints[:n].cpu().numpy(), ref["intervals"])
    g = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=DEV)
    g[:n] = torch.from_numpy(case["cotangent"][:n]).to(DEV)
    gv = torch.empty_like(values)
    plan.backward(grid, values, x_cut, spec.seed, 3, g, gv, ws)
    plan.check_status(ws)
    scale = np.abs(ref["grad_values"]).max()
    assert np.abs(gv.cpu().numpy() - ref["grad_values"]).max() <= GRAD_REPRO * scale
    for bad in (dict(density_blocks=np.full(spec.n_densities, 17, np.int32)),
                dict(density_blocks=np.zeros(spec.n_densities, np.int32)),
                dict(density_scan=np.full(spec.n_densities, 65, np.int32))):
        with pytest.raises(N.LoitsError) as err:
            B.BatchPlan(koff, counts, cfg, DEV, **bad)
        assert err.value.code == N.LOITS_ERR_INVALID


def test_kept_threshold_edges_match_oracle(B, oracle_lib):
    """Threshold compaction (monotone densities, cut >= 0) at its edges: a cut
    below every value (everything kept), above every value (nothing kept),
    exactly at a knot, and inside a stretch of zero density (a flat CDF);
    densities from 2 to 8000 knots.  Row offsets exact, events within
    tolerance of the oracle."""
    rng = np.random.default_rng(31)
    sizes = [2, 3, 64, 500, 4096, 8000]
    grids, vals, cuts = [], [], []
    for i, g in enumerate(sizes):
        x = np.linspace(0.05, 1.0, g, dtype=np.float32)
        f = (1.0 + rng.uniform(0, 1, g)).astype(np.float32)
        if g >= 64:
            f[g // 3: g // 2] = 0.0  # a flat stretch of the CDF
        grids.append(x)
        vals.append(f)
    koff = np.concatenate([[0], np.cumsum(sizes)])
    grid, values = np.concatenate(grids), np.concatenate(vals)
    counts = np.array([3000, 2000, 50_000, 20_000, 120_000, 70_000])
    for mode in ("below", "above", "at_knot", "flat"):
        for i, g in enumerate(sizes):
            x = grids[i]
            cuts.append({"below": 0.0, "above": 2.0, "at_knot": float(x[g // 4]),
                         "flat": float(0.5 * (x[g // 3] + x[g // 2 - 1])) if g >= 64 else float(x[0])}[mode])
        cut = np.array(cuts[-len(sizes):], np.float32)
        case = dict(knot_offsets=koff, event_counts=counts, grid=grid, values=values, x_cut=cut,
                    scalars=np.array([17, 4]))
        out = run_batch(B, case)
        ref = oracle_lib.d_forward(koff, np.concatenate([[0], np.cumsum(counts)]), grid, values,
                                   cut, 17, 4)
        assert np.array_equal(out["rows"], ref["row_offsets"]), mode
        np.testing.assert_allclose(out["events"], ref["events"], rtol=EVENT_RTOL)
        if mode == "above":
            assert out["valid"] == 0
        if mode == "below":
            assert out["valid"] == counts.sum()
