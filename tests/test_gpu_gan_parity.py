"""One batched GAN step against its fp64 oracle.

The reference trains one 2-D theory on raw events (pytorch/gan.py:107-122:
a discriminator step on real vs. generated events with the generator frozen,
then the generator's gradients through the sampler by autograd).  Its batched
counterpart, ``BatchedGANTrainer.step()``, is re-run here in float64 on the
CPU with the same weights, latents, seed and sequences:

* the sampler's events come from the oracle's restatement of the reference
  core (oracle/loits_oracle.c) on the same fp32 densities, seed, sequence and
  Philox slots, binned in float64 with the kernel's triangular weights;
* the discriminator and the binary cross-entropy run in float64 autograd;
* the generator step's histogram cotangent becomes per-event cotangents
  (gh[k + 1] - gh[k]) / h, which drive the oracle's fp64 VJP of the sampler
  (so the histogram-mode VJP is pinned to the oracle, not only to the
  event-mode VJP); the theory's VJP is float64 autograd of its formula.

Tolerances: losses 1e-4 relative; histograms 1e-4 relative per bin;
discriminator gradients 1e-4 of their scale; the gradient at the theory's
parameters 1e-3 of its scale (an event within an ulp of a bin edge can bin
differently in fp32 and fp64); generator weight gradients, back-propagated
through the same bf16 generator from either parameter gradient, 2e-2 of
their scale (bf16 rounding of the generator's own backward).
"""
import copy

import numpy as np
import pytest
import torch

from test_gpu_gan import np_hist, np_hist_cotangent, torch_theory

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")
B_DENS, N_EV, G_KNOTS, SEED = 8, 20_000, 512, 7


def _rel(a, b):
    return abs(float(a) - float(b)) / max(abs(float(b)), 1e-30)


def test_gan_step_matches_fp64_oracle(oracle_lib):
    from quantom_loits_b200 import batched as B
    from quantom_loits_b200.gan import BatchedGANTrainer

    cfg = B.make_config(threads=512, blocks_per_item=4)
    tr = BatchedGANTrainer(DEV, batch=B_DENS, n_events=N_EV, grid_size=G_KNOTS, seed=SEED,
                           config=cfg)
    seq0 = int(tr.sampler.sequence_dev.item())  # the real histogram took sequence 0
    assert seq0 == 1
    gen0 = copy.deepcopy(tr.generator)
    d0 = copy.deepcopy(tr.discriminator).double().cpu()
    g = torch.Generator(device=DEV).manual_seed(123)
    z_d = torch.randn((B_DENS, tr.latent), generator=g, device=DEV)
    z_g = torch.randn((B_DENS, tr.latent), generator=g, device=DEV)

    d_loss, g_loss = tr.step(z_d, z_g)
    torch.cuda.synchronize()
    d_grads = [p.grad.detach().double().cpu() for p in tr.discriminator.parameters()]
    g_grads = [p.grad.detach().float().cpu() for p in tr.generator.parameters()]
    d1 = copy.deepcopy(tr.discriminator).double().cpu()  # after the discriminator's update

    grid32 = tr.theory.grid.detach().cpu().numpy()
    grid_all = np.tile(grid32, B_DENS)
    koff = tr.knot_offsets
    eoff = np.concatenate([[0], np.cumsum(tr.event_counts)])
    bins, lo, hi = tr.bins, tr.lo, tr.hi

    def oracle_hist(values32, seq):
        fwd = oracle_lib.d_forward(koff, eoff, grid_all, values32.reshape(-1), None, SEED, seq)
        rows = fwd["row_offsets"]
        raw = np.stack([np_hist(fwd["events"][rows[b]:rows[b + 1]], lo, hi, bins)
                        for b in range(B_DENS)])
        return fwd, raw

    with torch.no_grad():
        target = torch.tensor([[0.4, -0.3, -1.2, 0.8, 0.5, -0.2]], dtype=torch.float32,
                              device=DEV).repeat(B_DENS, 1)
        v_real = tr.theory(target).cpu().numpy()
        params_d = gen0(z_d)
        v_d = tr.theory(params_d).cpu().numpy()
        params_g = gen0(z_g)
        v_g = tr.theory(params_g).cpu().numpy()
    _, real_raw = oracle_hist(v_real, 0)
    np.testing.assert_allclose(tr.real_hist.cpu().numpy() * N_EV, real_raw, rtol=1e-4, atol=1e-2)
    _, fake_d_raw = oracle_hist(v_d, seq0)
    fwd_g, fake_g_raw = oracle_hist(v_g, seq0 + 1)

    # the sampler's own histogram of the discriminator step (same sequence)
    batch_d = B.DensityBatch(tr.grid, torch.from_numpy(v_d.reshape(-1)).to(DEV), koff,
                             tr.event_counts)
    with torch.no_grad():
        h_d, _ = tr.sampler.histogram(batch_d, bins, lo, hi, sequence=seq0)
    np.testing.assert_allclose(h_d.cpu().numpy(), fake_d_raw, rtol=1e-4, atol=1e-2)

    # discriminator step in float64
    bce = torch.nn.BCEWithLogitsLoss()
    real = torch.from_numpy(real_raw / N_EV)
    fake_d = torch.from_numpy(fake_d_raw / N_EV)
    rl, fl = d0(real), d0(fake_d)
    d_ref = bce(rl, torch.ones_like(rl)) + bce(fl, torch.zeros_like(fl))
    d_ref.backward()
    assert _rel(d_loss, d_ref) <= 1e-4, (float(d_loss), float(d_ref))
    for mine, p in zip(d_grads, d0.parameters()):
        scale = p.grad.abs().max().item()
        assert (mine - p.grad).abs().max().item() <= 1e-4 * scale

    # generator step in float64: loss, histogram cotangent, sampler VJP, theory VJP
    fake_g = torch.from_numpy(fake_g_raw / N_EV).requires_grad_(True)
    lg = d1(fake_g)
    g_ref = bce(lg, torch.ones_like(lg))
    (gh,) = torch.autograd.grad(g_ref, fake_g)
    assert _rel(g_loss, g_ref) <= 1e-4, (float(g_loss), float(g_ref))
    gh_raw = (gh.numpy() / N_EV).astype(np.float32)  # d loss / d (raw histogram)
    rows = fwd_g["row_offsets"]
    cot = np.concatenate([np_hist_cotangent(fwd_g["events"][rows[b]:rows[b + 1]], gh_raw[b], lo,
                                            hi) for b in range(B_DENS)])
    gv_ref = oracle_lib.d_backward(koff, eoff, grid_all, v_g.reshape(-1), None, SEED, seq0 + 1,
                                   cot.astype(np.float64), fwd=fwd_g)
    p64 = params_g.detach().double().cpu().requires_grad_(True)
    vals64 = torch_theory(p64, torch.from_numpy(grid32.astype(np.float64)))
    (gp_ref,) = torch.autograd.grad(vals64, p64, torch.from_numpy(gv_ref.reshape(B_DENS, -1)))

    # the same chain on the GPU: theory -> sampler histogram -> discriminator
    p_gpu = params_g.detach().clone().requires_grad_(True)
    batch_g = B.DensityBatch(tr.grid, tr.theory(p_gpu).reshape(-1), koff, tr.event_counts)
    h_g, _ = tr.sampler.histogram(batch_g, bins, lo, hi, sequence=seq0 + 1)
    logits = tr.discriminator(h_g * (1.0 / N_EV))
    (gp,) = torch.autograd.grad(bce(logits, torch.ones_like(logits)), p_gpu)
    scale = gp_ref.abs().max().item()
    assert (gp.double().cpu() - gp_ref).abs().max().item() <= 1e-3 * scale
    # ... and with the theory evaluated inside the sampler (the step's own path)
    p_f = params_g.detach().clone().requires_grad_(True)
    h_f, _ = tr.sampler.histogram_powerlaw(p_f, batch_g, bins, lo, hi, sequence=seq0 + 1)
    torch.testing.assert_close(h_f.detach(), h_g.detach(), rtol=1e-5, atol=1e-3)
    logits_f = tr.discriminator(h_f * (1.0 / N_EV))
    (gpf,) = torch.autograd.grad(bce(logits_f, torch.ones_like(logits_f)), p_f)
    assert (gpf.double().cpu() - gp_ref).abs().max().item() <= 1e-3 * scale

    # generator weights: the bf16 generator's backward from either gradient
    z = z_g.clone()
    out = gen0(z)
    ref_w = torch.autograd.grad(out, list(gen0.parameters()), gp_ref.float().to(DEV))
    for mine, ref in zip(g_grads, ref_w):
        ref = ref.float().cpu()
        scale = ref.abs().max().item()
        assert (mine - ref).abs().max().item() <= 2e-2 * scale
