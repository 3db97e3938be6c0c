"""Batched GAN training step on the B200 sampler.

The reference's ``GANTrainer`` (pytorch/gan.py:26-122) fits the parameters of
one theory by an adversarial game on raw 2-D events.  ``BatchedGANTrainer``
is its batched counterpart: a generator MLP maps latent noise to the
parameters of a batch of densities, the theory tabulates them on a shared
grid, the sampler draws the events of every density and bins them in its own
kernels (no event is written), and a discriminator MLP scores the per-density
histograms.  The step keeps the reference's structure: a discriminator step
on real vs. generated histograms with the generator frozen, then a generator
step whose gradient runs back through the sampler's VJP, the theory's VJP and
the generator.

Shapes (defaults): latent 64 ~ N(0, 1) -> 256 -> 256 -> 6 parameters (SiLU,
bf16 weights, fp32 accumulation), batch 256, grid 2048 points on [1e-3, 1],
200 000 events per density, 64 bins, discriminator 64 -> 256 -> 1, Adam with
learning rate 1e-4, binary cross-entropy on logits as in the reference.
"""
from __future__ import annotations

from contextlib import nullcontext

import numpy as np
import torch
from torch import nn
from torch.profiler import record_function

from . import _native as N
from .batched import BatchedLOITS, DensityBatch


class _TheoryFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, grid):
        params = params.to(torch.float32).contiguous()
        nd, G = params.shape[0], grid.numel()
        values = torch.empty((nd, G), dtype=torch.float32, device=params.device)
        with torch.cuda.device(params.device):
            N.check(N.lib().loits_theory_powerlaw(nd, G, params.data_ptr(), grid.data_ptr(),
                                                  values.data_ptr(), N.stream_of(params.device)),
                    "loits_theory_powerlaw")
        ctx.save_for_backward(params, grid)
        return values

    @staticmethod
    def backward(ctx, grad_values):
        params, grid = ctx.saved_tensors
        gv = grad_values.to(torch.float32).contiguous()
        gp = torch.empty_like(params)
        with torch.cuda.device(params.device):
            N.check(N.lib().loits_theory_powerlaw_vjp(params.shape[0], grid.numel(),
                                                      params.data_ptr(), grid.data_ptr(),
                                                      gv.data_ptr(), gp.data_ptr(),
                                                      N.stream_of(params.device)),
                    "loits_theory_powerlaw_vjp")
        return gp, None


class PowerLawTheory(nn.Module):
    """Raw parameters (B, 6) -> two-component power-law densities (B, G) on a
    shared grid, in CUDA (include/loits_b200.h: loits_theory_powerlaw):
    a_i = -1/2 + 3/2 sigmoid(p[2i]), b_i = 1 + 4 sigmoid(p[2i+1]),
    w_i = softplus(p[4+i]), f = sum_i w_i x^a_i (1-x)^b_i."""

    n_params = 6

    def __init__(self, grid: torch.Tensor):
        super().__init__()
        self.register_buffer("grid", grid.to(torch.float32).contiguous())

    def forward(self, params: torch.Tensor) -> torch.Tensor:
        return _TheoryFunction.apply(params, self.grid)


class Generator(nn.Module):
    """latent -> 256 -> 256 -> 6 with SiLU; bf16 weights, fp32 accumulation
    (cuBLAS bf16 GEMMs), fp32 output."""

    def __init__(self, latent: int = 64, width: int = 256, n_params: int = 6):
        super().__init__()
        self.net = nn.Sequential(nn.Linear(latent, width), nn.SiLU(), nn.Linear(width, width),
                                 nn.SiLU(), nn.Linear(width, n_params))
        self.net.to(torch.bfloat16)

    def forward(self, z: torch.Tensor) -> torch.Tensor:
        return self.net(z.to(torch.bfloat16)).to(torch.float32)


class Discriminator(nn.Module):
    """Per-density histogram (bins) -> 256 -> 1 logit."""

    def __init__(self, bins: int = 64, width: int = 256):
        super().__init__()
        self.net = nn.Sequential(nn.Linear(bins, width), nn.SiLU(), nn.Linear(width, 1))

    def forward(self, hist: torch.Tensor) -> torch.Tensor:
        return self.net(hist)


class BatchedGANTrainer:
    """Adversarial fit of a batch of generated theories to a target theory
    (step() -> (d_loss, g_loss) like the reference's GANTrainer.step)."""

    def __init__(self, device="cuda", batch: int = 256, n_events: int = 200_000,
                 grid_size: int = 2048, bins: int = 64, latent: int = 64, lr: float = 1e-4,
                 seed: int = 0, config="auto", profile_regions: bool = False,
                 fused_theory: bool = True):
        self.device = torch.device(device)
        N.require_device(self.device)
        torch.manual_seed(int(seed))
        self.batch, self.n_events, self.bins, self.latent = batch, int(n_events), bins, latent
        self.profile_regions = profile_regions
        # the theory evaluated inside the sampler's CDF tiles and its VJP
        # reduced there (BatchedLOITS.histogram_powerlaw), or as its own
        # kernels (PowerLawTheory, then BatchedLOITS.histogram)
        self.fused_theory = bool(fused_theory)
        grid1 = torch.linspace(1e-3, 1.0, grid_size, dtype=torch.float64).to(torch.float32)
        self.theory = PowerLawTheory(grid1).to(self.device)
        self.generator = Generator(latent).to(self.device)
        self.discriminator = Discriminator(bins).to(self.device)
        self.sampler = BatchedLOITS(self.device, seed=int(seed), config=config,
                                    device_sequence=True)
        self.lo, self.hi = 1e-3, 1.0
        # the batch's knots: every density on the same grid
        self.grid = self.theory.grid.repeat(batch)
        self.knot_offsets = np.arange(batch + 1, dtype=np.int64) * grid_size
        self.event_counts = np.full(batch, self.n_events, dtype=np.int64)
        self._shape_values = torch.zeros(batch * grid_size, dtype=torch.float32,
                                         device=self.device)  # shape only: never read
        self.loss = nn.BCEWithLogitsLoss()
        # one fused multi-tensor kernel per optimizer step instead of one per
        # tensor; step counts on the device so that the step can be captured
        self.d_optimizer = torch.optim.Adam(self.discriminator.parameters(), lr=lr, fused=True,
                                            capturable=True)
        self.g_optimizer = torch.optim.Adam(self.generator.parameters(), lr=lr, fused=True,
                                            capturable=True)
        self.graph = None
        self.gen = torch.Generator(device=self.device).manual_seed(int(seed) + 1)
        # target theory: fixed raw parameters, the same for every density
        target = torch.tensor([[0.4, -0.3, -1.2, 0.8, 0.5, -0.2]], dtype=torch.float32,
                              device=self.device).repeat(batch, 1)
        with torch.no_grad():
            self.real_hist = self.histogram(self.theory(target)).detach()

    def _region(self, name):
        return record_function(name) if self.profile_regions else nullcontext()

    def histogram(self, values: torch.Tensor) -> torch.Tensor:
        """Normalised per-density event histograms of densities (B, G)."""
        batch = DensityBatch(self.grid, values.reshape(-1), self.knot_offsets, self.event_counts)
        hist, _ = self.sampler.histogram(batch, self.bins, self.lo, self.hi)
        return hist * (1.0 / self.n_events)

    def latent_noise(self) -> torch.Tensor:
        return torch.randn((self.batch, self.latent), generator=self.gen, device=self.device)

    def histogram_of_params(self, params: torch.Tensor) -> torch.Tensor:
        """histogram(theory(params)) with the theory fused into the sampler."""
        batch = DensityBatch(self.grid, self._shape_values, self.knot_offsets, self.event_counts)
        hist, _ = self.sampler.histogram_powerlaw(params, batch, self.bins, self.lo, self.hi)
        return hist * (1.0 / self.n_events)

    def generate_from(self, params: torch.Tensor) -> torch.Tensor:
        """Normalised histograms of the densities the theory gives for
        params (B x 6)."""
        if self.fused_theory:
            return self.histogram_of_params(params)
        return self.histogram(self.theory(params))

    def generate(self, z: torch.Tensor) -> torch.Tensor:
        return self.generate_from(self.generator(z))

    def _step_body(self, z_d: torch.Tensor, z_g: torch.Tensor):
        with self._region("gan::discriminator_step"):
            self.d_optimizer.zero_grad(set_to_none=True)
            with torch.no_grad():
                fake = self.generate(z_d)
            real_logits = self.discriminator(self.real_hist)
            fake_logits = self.discriminator(fake)
            d_loss = (self.loss(real_logits, torch.ones_like(real_logits)) +
                      self.loss(fake_logits, torch.zeros_like(fake_logits)))
            d_loss.backward()
            self.d_optimizer.step()
        with self._region("gan::generator_step"):
            # gradients of the generator only (pytorch/gan.py:117-121)
            logits = self.discriminator(self.generate(z_g))
            g_loss = self.loss(logits, torch.ones_like(logits))
            params = list(self.generator.parameters())
            for p, g in zip(params, torch.autograd.grad(g_loss, params)):
                p.grad = g
            self.g_optimizer.step()
        return d_loss.detach(), g_loss.detach()

    def step(self, z_d: torch.Tensor | None = None, z_g: torch.Tensor | None = None):
        """One discriminator step and one generator step; (d_loss, g_loss)."""
        if self.graph is not None:
            return self.replay(z_d, z_g)
        z_d = self.latent_noise() if z_d is None else z_d
        z_g = self.latent_noise() if z_g is None else z_g
        return self._step_body(z_d, z_g)

    def capture(self, warmup: int = 3):
        """Capture the whole training step (both networks' forward and
        backward, the theory, the sampler's histogram forwards and VJP, both
        optimizer steps) as one CUDA graph; later steps replay it.  The
        sampler reads its sequence from device memory, so every replay draws
        fresh events; latents are inputs filled before each replay."""
        self.static_zd = self.latent_noise()
        self.static_zg = self.latent_noise()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            for _ in range(warmup):
                self._step_body(self.static_zd, self.static_zg)
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.static_losses = self._step_body(self.static_zd, self.static_zg)
        self.graph = graph
        return graph

    def replay(self, z_d: torch.Tensor | None = None, z_g: torch.Tensor | None = None):
        if z_d is None:
            torch.randn(self.static_zd.shape, generator=self.gen, device=self.device,
                        out=self.static_zd)
        else:
            self.static_zd.copy_(z_d, non_blocking=True)
        if z_g is None:
            torch.randn(self.static_zg.shape, generator=self.gen, device=self.device,
                        out=self.static_zg)
        else:
            self.static_zg.copy_(z_g, non_blocking=True)
        self.graph.replay()
        return self.static_losses
