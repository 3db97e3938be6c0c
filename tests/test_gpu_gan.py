"""GPU checks of the batched GAN pieces: the theory kernels, the sampler's
histogram mode and the training step.

* theory: values against a float64 numpy restatement of the same formula
  (rtol 2e-5: fp32 exp/log), VJP against torch float64 autograd of it (1e-4 of
  the gradient scale);
* histogram mode: histograms against the events of the event-writing forward
  (same plan, seed, sequence) binned in float64 numpy (rtol 1e-4 per bin; fp32
  atomics), kept counts exact; its VJP against the event-mode VJP driven by
  the per-event cotangents (gh[k+1] - gh[k]) / h (1e-5 of the scale);
* the trainer: steps run, losses are finite, both networks move.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")


def np_theory(params, grid):
    sig = lambda z: 1.0 / (1.0 + np.exp(-z))  # noqa: E731
    out = np.zeros((len(params), len(grid)))
    x = grid.astype(np.float64)
    for d, p in enumerate(params.astype(np.float64)):
        for i in range(2):
            a, b = -0.5 + 1.5 * sig(p[2 * i]), 1.0 + 4.0 * sig(p[2 * i + 1])
            w = np.log1p(np.exp(p[4 + i]))
            out[d] += w * np.power(x, a) * np.power(1.0 - x, b)
    return out


def torch_theory(params, grid):
    a = -0.5 + 1.5 * torch.sigmoid(params[:, 0::2][:, :2])
    b = 1.0 + 4.0 * torch.sigmoid(params[:, 1::2][:, :2])
    w = torch.nn.functional.softplus(params[:, 4:6])
    x = grid[None, None, :]
    return (w[:, :, None] * x ** a[:, :, None] * (1.0 - x) ** b[:, :, None]).sum(1)


def np_bin(x, lo, hi, bins):
    """The kernel's fp32 bin position: s = fma(x - lo, bins / (hi - lo), -1/2)
    (the fp32 product is exact in fp64; one rounding to fp32 after the add)."""
    lo32 = np.float32(lo)
    inv_h = np.float32(bins / (np.float64(hi) - np.float64(lo)))
    d = (x.astype(np.float32) - lo32).astype(np.float64)
    s = (d * np.float64(inv_h) - 0.5).astype(np.float32)
    s = np.clip(s, np.float32(-2.0), np.float32(bins + 1.0))
    k = np.floor(s).astype(np.int64)
    f = (s - k.astype(np.float32)).astype(np.float32)
    return k, f, inv_h


def np_hist(x, lo, hi, bins):
    k, f, _ = np_bin(x, lo, hi, bins)
    f = f.astype(np.float64)
    out = np.zeros(bins)
    m0 = (k >= 0) & (k < bins)
    m1 = (k + 1 >= 0) & (k + 1 < bins)
    np.add.at(out, k[m0], 1.0 - f[m0])
    np.add.at(out, k[m1] + 1, f[m1])
    return out


def np_hist_cotangent(x, gh, lo, hi):
    bins = len(gh)
    k, _, inv_h = np_bin(x, lo, hi, bins)
    pad = np.concatenate([[0.0], gh, [0.0]]).astype(np.float32)
    g0 = pad[np.clip(k + 1, 0, bins + 1)]
    g1 = pad[np.clip(k + 2, 0, bins + 1)]
    return ((g1 - g0) * inv_h).astype(np.float32)


def test_theory_kernels_match_float64():
    from quantom_loits_b200.gan import PowerLawTheory

    rng = np.random.default_rng(0)
    grid = np.linspace(1e-3, 1.0, 777).astype(np.float32)
    params = rng.normal(0, 1.5, (9, 6)).astype(np.float32)
    th = PowerLawTheory(torch.from_numpy(grid)).to(DEV)
    p = torch.from_numpy(params).to(DEV).requires_grad_(True)
    v = th(p)
    np.testing.assert_allclose(v.detach().cpu().numpy(), np_theory(params, grid), rtol=2e-5,
                               atol=1e-30)
    gv = torch.from_numpy(rng.standard_normal((9, 777)).astype(np.float32)).to(DEV)
    (v * gv).sum().backward()
    p64 = torch.from_numpy(params.astype(np.float64)).requires_grad_(True)
    (torch_theory(p64, torch.from_numpy(grid.astype(np.float64))) *
     gv.cpu().double()).sum().backward()
    ref = p64.grad.numpy()
    assert np.abs(p.grad.cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()


@pytest.mark.parametrize("cut", [False, True])
def test_histogram_mode_matches_binned_events(cut):
    from quantom_loits_b200 import batched as B
    from quantom_loits_b200 import workloads

    spec = workloads.ragged(scale=0.05, n_densities=12)
    case = dict(knot_offsets=spec.knot_offsets, event_counts=spec.event_counts)
    plan = B.BatchPlan(spec.knot_offsets, spec.event_counts, None, DEV)
    grid = torch.from_numpy(spec.grid).to(DEV)
    values = torch.from_numpy(spec.values).to(DEV)
    x_cut = torch.from_numpy(spec.x_cut).to(DEV) if cut else None
    ws = plan.new_workspace()
    ev, rows = plan.new_events(), plan.new_row_offsets()
    plan.forward(grid, values, x_cut, 77, 3, ev, rows, ws)
    plan.check_status(ws)
    rows_h = rows.cpu().numpy()
    events = ev[:rows_h[-1]].cpu().numpy()
    bins, lo, hi = 64, 1e-3, 1.0
    hist = torch.empty((plan.n_densities, bins), device=DEV)
    kept = torch.empty(plan.n_densities, dtype=torch.int64, device=DEV)
    ws2 = plan.new_workspace()
    plan.forward_hist(grid, values, x_cut, 77, 3, bins, lo, hi, hist, kept, ws2)
    plan.check_status(ws2)
    assert np.array_equal(kept.cpu().numpy(), np.diff(rows_h))
    h = hist.cpu().numpy()
    for b in range(plan.n_densities):
        ref = np_hist(events[rows_h[b]:rows_h[b + 1]], lo, hi, bins)
        np.testing.assert_allclose(h[b], ref, rtol=1e-4, atol=1e-2)
    # VJP: histogram cotangent -> per-event cotangents -> event-mode backward
    rng = np.random.default_rng(5)
    gh = rng.standard_normal((plan.n_densities, bins)).astype(np.float32)
    gv_hist = torch.empty_like(values)
    plan.backward_hist(grid, values, x_cut, 77, 3, bins, lo, hi, torch.from_numpy(gh).to(DEV),
                       gv_hist, ws2)
    plan.check_status(ws2)
    cot = np.concatenate([np_hist_cotangent(events[rows_h[b]:rows_h[b + 1]], gh[b], lo, hi)
                          for b in range(plan.n_densities)])
    g = torch.zeros(max(plan.capacity, 4), device=DEV)
    g[:len(cot)] = torch.from_numpy(cot).to(DEV)
    gv_ev = torch.empty_like(values)
    plan.backward(grid, values, x_cut, 77, 3, g, gv_ev, ws)
    plan.check_status(ws)
    a, b_ = gv_hist.cpu().numpy(), gv_ev.cpu().numpy()
    assert np.abs(a - b_).max() <= 1e-5 * np.abs(b_).max(), case


def test_histogram_autograd_path():
    from quantom_loits_b200 import batched as B
    from quantom_loits_b200 import workloads

    spec = workloads.uniform(scale=2e-3, n_densities=6)
    batch = B.DensityBatch.from_spec(spec, DEV, requires_grad=True)
    sampler = B.BatchedLOITS(DEV, seed=11)
    hist, kept = sampler.histogram(batch, bins=32, lo=1e-3, hi=1.0)
    assert hist.shape == (6, 32) and int(kept.sum()) == spec.total_events
    # weights of an event sum to 1 except within half a bin of lo or hi
    tot = hist.sum(1).detach().cpu().numpy()
    assert np.all(tot <= spec.event_counts * (1 + 1e-5)) and np.all(tot > 0.5 * spec.event_counts)
    (hist * torch.linspace(0, 1, 32, device=DEV)).sum().backward()
    assert torch.isfinite(batch.values.grad).all() and batch.values.grad.abs().max() > 0


@pytest.mark.parametrize("knots,threads", [(512, 256), (2048, 1024)])
def test_powerlaw_theory_fused_into_the_sampler(knots, threads):
    """histogram_powerlaw (the theory evaluated in the sampler's CDF tile
    loads, its VJP reduced in the backward's finalize) against the theory's
    own kernels followed by the tabulated-value histogram: the same values
    bit for bit, hence the same kept counts and events; histograms and the
    parameter gradient to fp32 summation order."""
    from quantom_loits_b200 import batched as B
    from quantom_loits_b200.gan import PowerLawTheory

    nd = 12
    grid1 = torch.linspace(1e-3, 1.0, knots, dtype=torch.float64).to(torch.float32)
    th = PowerLawTheory(grid1).to(DEV)
    gen = torch.Generator().manual_seed(7)
    params = (torch.randn((nd, 6), generator=gen) * 0.8).to(DEV)
    koff = np.arange(nd + 1, dtype=np.int64) * knots
    counts = np.full(nd, 30_000, dtype=np.int64)
    grid = th.grid.repeat(nd)
    cfg = B.make_config(threads=threads, blocks_per_item=4)
    sampler = B.BatchedLOITS(DEV, seed=5, config=cfg)
    cot = torch.randn((nd, 32), generator=gen).to(DEV)

    p_a = params.clone().requires_grad_(True)
    batch = B.DensityBatch(grid, th(p_a).reshape(-1), koff, counts)
    h_a, k_a = sampler.histogram(batch, 32, 1e-3, 1.0, sequence=9)
    (g_a,) = torch.autograd.grad((h_a * cot).sum(), p_a)

    p_b = params.clone().requires_grad_(True)
    shape = B.DensityBatch(grid, torch.zeros(nd * knots, device=DEV), koff, counts)
    h_b, k_b = sampler.histogram_powerlaw(p_b, shape, 32, 1e-3, 1.0, sequence=9)
    (g_b,) = torch.autograd.grad((h_b * cot).sum(), p_b)

    assert torch.equal(k_a, k_b)
    # the same events; the per-tile merges into the global histogram are fp32
    # additions in arrival order, so the bins agree to fp32 accumulation order
    torch.testing.assert_close(h_b.detach(), h_a.detach(), rtol=1e-5, atol=1e-3)
    scale = g_a.abs().max().item()
    assert scale > 0 and (g_a - g_b).abs().max().item() <= 1e-4 * scale


def test_powerlaw_theory_fused_rejects_densities_it_cannot_stage():
    from quantom_loits_b200 import _native as N
    from quantom_loits_b200 import batched as B

    knots = 70_001  # above the shared-memory knot count: sampled from global memory
    koff = np.array([0, knots], dtype=np.int64)
    plan = B.BatchPlan(koff, np.array([1000]), B.make_config(threads=1024), DEV)
    grid = torch.linspace(1e-3, 1.0, knots, device=DEV)
    params = torch.zeros((1, 6), device=DEV)
    hist = torch.empty((1, 8), device=DEV)
    kept = torch.empty(1, dtype=torch.int64, device=DEV)
    ws = plan.new_workspace()
    with pytest.raises(N.LoitsError) as e:
        plan.forward_hist_powerlaw(grid, params, None, 1, 0, 8, 0.0, 1.0, hist, kept, ws)
    assert e.value.code == N.LOITS_ERR_UNSUPPORTED


def test_gan_trainer_steps():
    from quantom_loits_b200.gan import BatchedGANTrainer

    tr = BatchedGANTrainer(DEV, batch=8, n_events=20_000, grid_size=512, seed=3)
    g0 = [p.detach().clone() for p in tr.generator.parameters()]
    d0 = [p.detach().clone() for p in tr.discriminator.parameters()]
    for _ in range(3):
        d_loss, g_loss = tr.step()
        assert torch.isfinite(d_loss) and torch.isfinite(g_loss)
    assert any(not torch.equal(a, b) for a, b in zip(g0, tr.generator.parameters()))
    assert any(not torch.equal(a, b) for a, b in zip(d0, tr.discriminator.parameters()))
    assert tr.real_hist.shape == (8, 64)


def test_gan_step_captured_in_one_graph():
    """The captured step replays with finite losses, advances the sampler's
    device-side sequence by two histogram calls per step, and later calls
    draw fresh uniforms."""
    from quantom_loits_b200.gan import BatchedGANTrainer

    tr = BatchedGANTrainer(DEV, batch=8, n_events=20_000, grid_size=512, seed=5)
    tr.capture()
    seq0 = int(tr.sampler.sequence_dev.item())
    zs = [torch.randn((2, 8, 64), device=DEV) for _ in range(3)]
    out = [tr.replay(z[0], z[1]) for z in zs]
    torch.cuda.synchronize()
    # two histogram calls per step advance the device sequence
    assert int(tr.sampler.sequence_dev.item()) == seq0 + 2 * len(zs)
    losses = [(float(d), float(g)) for d, g in out]
    assert all(np.isfinite(v).all() for v in losses)
    # fresh uniforms each replay: the same latents give different fake histograms
    with torch.no_grad():
        h1 = tr.generate(zs[0][0])
        h2 = tr.generate(zs[0][0])
    assert not torch.equal(h1, h2)
