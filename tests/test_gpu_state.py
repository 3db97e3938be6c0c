"""GPU parity of the batched sampler's saved-state form through the C ABI.

``loits_batch_forward_state`` writes, per kept row, the interval j and the
offset t = u - c_j; ``loits_batch_backward_state`` takes the VJP from them
instead of regenerating the uniforms.  Checks, on seeded batches that take
every compaction path (identity, threshold, general with a cut, non-monotone
count semantics, densities in global memory):

* events and row offsets equal the plain forward's, bit for bit;
* intervals equal the forward's interval output; offsets equal u - c_j of the
  fp64 oracle within 2^-22 (fp32 rounding of u - c_j);
* the state VJP equals the replaying VJP within 1e-5 of the gradient scale
  (only the fp32 accumulation order differs) and the oracle's within 1e-4.
"""
import numpy as np
import pytest
import torch

from conftest import golden_case

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")
GRAD_TOL = 1e-4
SAME_TOL = 1e-5
OFFSET_TOL = 2.0 ** -22


@pytest.fixture(scope="module")
def B():
    from quantom_loits_b200 import batched

    return batched


def _tensors(case):
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(DEV)  # noqa: E731
    x_cut = case.get("x_cut")
    return f32(case["grid"]), f32(case["values"]), None if x_cut is None else f32(x_cut)


def _run_both(B, case, config=None):
    """Replay form and saved-state form on the same inputs and cotangent."""
    koff, counts = case["knot_offsets"], case["event_counts"]
    seed, seq = int(case["scalars"][0]), int(case["scalars"][1])
    grid, values, x_cut = _tensors(case)
    plan = B.BatchPlan(koff, counts, config, DEV)
    out = {}
    for mode in ("replay", "state"):
        ev, rows, ws = plan.new_events(), plan.new_row_offsets(), plan.new_workspace()
        ints, offs = plan.new_state()
        if mode == "replay":
            plan.forward(grid, values, x_cut, seed, seq, ev, rows, ws, ints)
        else:
            plan.forward_state(grid, values, x_cut, seed, seq, ev, rows, ints, offs, ws)
        plan.check_status(ws)
        valid = int(rows[-1].item())
        gen = torch.Generator(device=DEV).manual_seed(5)
        g = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=DEV)
        g[:valid] = torch.randn(valid, generator=gen, device=DEV)
        gv = torch.empty_like(values)
        if mode == "replay":
            plan.backward(grid, values, x_cut, seed, seq, g, gv, ws)
        else:
            plan.backward_state(grid, values, x_cut, ints, offs, g, gv, ws)
        plan.check_status(ws)
        out[mode] = dict(events=ev[:valid].cpu().numpy(), rows=rows.cpu().numpy(),
                         ints=ints[:valid].cpu().numpy(), offs=offs[:valid].cpu().numpy(),
                         grad=gv.cpu().numpy(), cot=g[:valid].cpu().numpy())
    return out


def _large_case(rng, sizes, counts, cut=True):
    grids, vals = [], []
    for g in sizes:
        x = np.linspace(1e-3, 1.0, g, dtype=np.float32)
        mu, sig = rng.uniform(0.2, 0.8), 10 ** rng.uniform(-3, -1.5)
        f = np.exp(-0.5 * ((x.astype(np.float64) - mu) / sig) ** 2) + 1e-3 * np.power(x, -0.5)
        grids.append(x)
        vals.append(f.astype(np.float32))
    case = dict(knot_offsets=np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64),
                event_counts=np.asarray(counts, np.int64), grid=np.concatenate(grids),
                values=np.concatenate(vals), scalars=np.array([77, 5]))
    if cut:
        case["x_cut"] = rng.uniform(0.01, 0.1, len(sizes)).astype(np.float32)
    return case


def _cases():
    from quantom_loits_b200 import workloads

    rng = np.random.default_rng(41)
    out = {}
    rag = workloads.ragged(scale=0.01, n_densities=40)  # general path (cut above g_0)
    out["ragged_cut"] = dict(knot_offsets=rag.knot_offsets, event_counts=rag.event_counts,
                             grid=rag.grid, values=rag.values, x_cut=rag.x_cut,
                             scalars=np.array([rag.seed, 3]))
    uni = workloads.uniform(scale=0.02, n_densities=12)  # identity compaction
    out["uniform_all"] = dict(knot_offsets=uni.knot_offsets, event_counts=uni.event_counts,
                              grid=uni.grid, values=uni.values, scalars=np.array([uni.seed, 1]))
    thr = dict(out["uniform_all"])  # threshold compaction: monotone, cut >= g_0
    thr["x_cut"] = np.full(len(uni.event_counts), 0.3, np.float32)
    thr["scalars"] = np.array([uni.seed, 2])
    out["uniform_threshold"] = thr
    nm = _large_case(rng, [300, 700], [40_000, 60_000], cut=False)  # count semantics
    nm["values"] = nm["values"].copy()
    nm["values"][120] = -5.0
    out["non_monotone"] = nm
    out["large_mixed"] = _large_case(rng, [20000, 300, 70001], [150_000, 20_000, 200_000])
    return out


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("threads", [256, 1024])
def test_saved_state_matches_replay_and_oracle(B, oracle_lib, name, threads):
    case = CASES[name]
    out = _run_both(B, case, B.make_config(threads=threads))
    rp, sv = out["replay"], out["state"]
    assert np.array_equal(rp["rows"], sv["rows"])
    assert np.array_equal(rp["events"], sv["events"])
    assert np.array_equal(rp["ints"], sv["ints"])
    # offsets against the fp64 oracle's u - c_j
    koff = case["knot_offsets"]
    eoff = np.concatenate([[0], np.cumsum(case["event_counts"])])
    seed, seq = int(case["scalars"][0]), int(case["scalars"][1])
    ref = oracle_lib.d_forward(koff, eoff, case["grid"], case["values"], case.get("x_cut"),
                               seed, seq)
    assert np.array_equal(sv["rows"], ref["row_offsets"])
    dens = np.searchsorted(ref["row_offsets"], np.arange(len(sv["ints"])), side="right") - 1
    t_ref = ref["u"] - ref["cdf"][koff[dens] + sv["ints"]]
    assert np.abs(sv["offs"] - t_ref).max() <= OFFSET_TOL
    # the state VJP: replay's gradient up to accumulation order, and the oracle's
    gref = oracle_lib.d_backward(koff, eoff, case["grid"], case["values"], case.get("x_cut"),
                                 seed, seq, sv["cot"], fwd=ref)
    for b in range(len(case["event_counts"])):
        o, e = koff[b], koff[b + 1]
        scale = max(np.abs(gref[o:e]).max(), 1e-30)
        assert np.abs(sv["grad"][o:e] - rp["grad"][o:e]).max() <= SAME_TOL * scale, b
        assert np.abs(sv["grad"][o:e] - gref[o:e]).max() <= GRAD_TOL * scale, b


def test_saved_state_golden_ragged(B, golden):
    """The committed golden batch (reference core on the exact embedding):
    the state VJP reproduces its gradient."""
    c = golden_case(golden, "ragged_small")
    case = dict(knot_offsets=c["knot_offsets"], event_counts=c["event_counts"], grid=c["grid"],
                values=c["values"], x_cut=c["x_cut"], scalars=c["scalars"])
    koff, counts = case["knot_offsets"], case["event_counts"]
    grid, values, x_cut = _tensors(case)
    plan = B.BatchPlan(koff, counts, None, DEV)
    ev, rows, ws = plan.new_events(), plan.new_row_offsets(), plan.new_workspace()
    ints, offs = plan.new_state()
    seed, seq = int(c["scalars"][0]), int(c["scalars"][1])
    plan.forward_state(grid, values, x_cut, seed, seq, ev, rows, ints, offs, ws)
    plan.check_status(ws)
    assert np.array_equal(rows.cpu().numpy(), c["row_offsets"])
    # intervals bit-exact except where u lies within fp32 rounding of a knot
    assert np.mean(ints[:len(c["intervals"])].cpu().numpy() == c["intervals"]) > 0.999
    g = torch.zeros(max(plan.capacity, 4), dtype=torch.float32, device=DEV)
    g[:len(c["cotangent"])] = torch.from_numpy(c["cotangent"].astype(np.float32)).to(DEV)
    gv = torch.empty_like(values)
    plan.backward_state(grid, values, x_cut, ints, offs, g, gv, ws)
    plan.check_status(ws)
    scale = np.abs(c["grad_values"]).max()
    assert np.abs(gv.cpu().numpy() - c["grad_values"]).max() <= GRAD_TOL * scale


def test_saved_state_autograd_matches_replay(B):
    from quantom_loits_b200 import workloads

    spec = workloads.ragged(scale=0.005, n_densities=16)
    grads = []
    for saved in (False, True):
        batch = B.DensityBatch.from_spec(spec, DEV)
        batch.values.requires_grad_(True)
        sampler = B.BatchedLOITS(DEV, seed=spec.seed, saved_state=saved)
        ev, rows = sampler.sample(batch, sequence=4)
        w = torch.linspace(-1.0, 1.0, ev.numel(), device=DEV)
        (ev * w).sum().backward()
        grads.append((ev.detach().cpu().numpy(), batch.values.grad.cpu().numpy()))
    assert np.array_equal(grads[0][0], grads[1][0])
    scale = np.abs(grads[0][1]).max()
    assert np.abs(grads[0][1] - grads[1][1]).max() <= SAME_TOL * scale


def test_saved_state_out_of_range_intervals_stay_in_bounds(B):
    """Saved intervals outside [0, G - 2] are clamped: the VJP reads and
    writes only inside each density and stays finite."""
    case = CASES["uniform_all"]
    grid, values, x_cut = _tensors(case)
    plan = B.BatchPlan(case["knot_offsets"], case["event_counts"], None, DEV)
    ev, rows, ws = plan.new_events(), plan.new_row_offsets(), plan.new_workspace()
    ints, offs = plan.new_state()
    plan.forward_state(grid, values, x_cut, int(case["scalars"][0]), 1, ev, rows, ints, offs, ws)
    plan.check_status(ws)
    valid = int(rows[-1].item())
    ints[:valid:3] = -7
    ints[1:valid:3] = 1 << 30
    g = torch.ones(max(plan.capacity, 4), dtype=torch.float32, device=DEV)
    gv = torch.empty_like(values)
    plan.backward_state(grid, values, x_cut, ints, offs, g, gv, ws)
    plan.check_status(ws)
    assert torch.isfinite(gv).all()


def test_saved_state_empty_batch(B):
    koff = np.array([0, 64, 128], np.int64)
    grid = torch.linspace(1e-3, 1.0, 64, device=DEV).repeat(2)
    values = torch.ones(128, device=DEV)
    plan = B.BatchPlan(koff, np.array([0, 0]), None, DEV)
    ev, rows, ws = plan.new_events(), plan.new_row_offsets(), plan.new_workspace()
    ints, offs = plan.new_state()
    plan.forward_state(grid, values, None, 1, 0, ev, rows, ints, offs, ws)
    g = torch.zeros(4, device=DEV)
    gv = torch.full_like(values, float("nan"))
    plan.backward_state(grid, values, None, ints, offs, g, gv, ws)
    plan.check_status(ws)
    assert rows.cpu().tolist() == [0, 0, 0]
    assert torch.equal(gv, torch.zeros_like(gv))
