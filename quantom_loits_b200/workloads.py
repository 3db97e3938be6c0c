"""Seeded synthetic density batches for the sampler's benchmark shapes.

No dataset is involved anywhere in this project: every workload is a batch of
analytic 1-D densities tabulated on a grid, drawn from a fixed torch
``Generator`` seed, stored as fp32 like the sampler's batched inputs.

* ``single``    1 density  x^a (1-x)^b on 256 uniform knots over [1e-3, 1],
                a ~ U(-0.5, 1), b ~ U(1, 5); 100 000 events; Philox seed 1234.
* ``uniform``   64 densities, each a Dirichlet(1)-weighted sum of 1-3 such
                components on 1024 uniform knots; 1 000 000 events each.
* ``ragged``    512 densities as ``uniform`` but with knot counts log-uniform
                integers in [64, 8192], event counts log-uniform in [1e4, 1e6]
                and a per-density acceptance cut x > x_cut, x_cut ~ U(0.01, 0.1).
* ``precision`` 16 densities on 2^20 uniform knots over [1e-6, 1]: a narrow
                Gaussian (mean ~ U(0.1, 0.9), sigma log-uniform in [1e-4, 1e-2])
                plus a tail 1e-8 x^-0.5; 10 000 000 events each.

Each factory returns a :class:`DensityBatchSpec` of host arrays; ``scale``
shrinks event counts (and, for ``ragged``, the number of densities) for the
quick cases used by tests.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class DensityBatchSpec:
    """Host description of a batch of 1-D densities (offsets-table layout)."""

    name: str
    knot_offsets: np.ndarray  # int64 [B+1]
    grid: np.ndarray  # float32 [total_knots]
    values: np.ndarray  # float32 [total_knots]
    event_counts: np.ndarray  # int64 [B]
    x_cut: np.ndarray | None  # float32 [B] or None
    seed: int = 1234
    sequence: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def n_densities(self) -> int:
        return len(self.knot_offsets) - 1

    @property
    def event_offsets(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.event_counts)]).astype(np.int64)

    @property
    def total_events(self) -> int:
        return int(self.event_counts.sum())

    @property
    def total_knots(self) -> int:
        return int(self.knot_offsets[-1])


def _uniform(gen, lo, hi, n=1):
    return (lo + (hi - lo) * torch.rand(n, generator=gen, dtype=torch.float64)).numpy()


def _powerlaw_mixture(gen, x: np.ndarray, components: int) -> np.ndarray:
    # Dirichlet(1) weights are normalised i.i.d. unit exponentials
    e = -torch.log(torch.rand(components, generator=gen, dtype=torch.float64)).numpy()
    w = e / e.sum()
    f = np.zeros_like(x)
    for c in range(components):
        a = _uniform(gen, -0.5, 1.0)[0]
        b = _uniform(gen, 1.0, 5.0)[0]
        f += w[c] * np.power(x, a) * np.power(1.0 - x, b)
    return f


def _pack(name, grids, values, counts, x_cut, seed, meta) -> DensityBatchSpec:
    koff = np.concatenate([[0], np.cumsum([len(g) for g in grids])]).astype(np.int64)
    return DensityBatchSpec(
        name=name,
        knot_offsets=koff,
        grid=np.concatenate(grids).astype(np.float32),
        values=np.concatenate(values).astype(np.float32),
        event_counts=np.asarray(counts, dtype=np.int64),
        x_cut=None if x_cut is None else np.asarray(x_cut, dtype=np.float32),
        seed=seed,
        meta=meta,
    )


def single(scale: float = 1.0) -> DensityBatchSpec:
    gen = torch.Generator().manual_seed(0)
    x = np.linspace(1e-3, 1.0, 256, dtype=np.float64).astype(np.float32).astype(np.float64)
    a = _uniform(gen, -0.5, 1.0)[0]
    b = _uniform(gen, 1.0, 5.0)[0]
    f = np.power(x, a) * np.power(1.0 - x, b)
    n = max(1, int(round(100_000 * scale)))
    return _pack("single", [x], [f], [n], None, 1234, {"a": a, "b": b, "knots": 256})


def uniform(scale: float = 1.0, n_densities: int = 64, knots: int = 1024,
            events: int = 1_000_000) -> DensityBatchSpec:
    gen = torch.Generator().manual_seed(1)
    x = np.linspace(1e-3, 1.0, knots, dtype=np.float64).astype(np.float32).astype(np.float64)
    grids, vals = [], []
    for _ in range(n_densities):
        comps = int(torch.randint(1, 4, (1,), generator=gen))
        grids.append(x)
        vals.append(_powerlaw_mixture(gen, x, comps))
    n = max(1, int(round(events * scale)))
    return _pack("uniform", grids, vals, [n] * n_densities, None, 1234,
                 {"knots": knots, "events_per_density": n})


def ragged(scale: float = 1.0, n_densities: int = 512) -> DensityBatchSpec:
    gen = torch.Generator().manual_seed(2)
    grids, vals, counts, cuts = [], [], [], []
    for _ in range(n_densities):
        g = int(round(math.exp(_uniform(gen, math.log(64), math.log(8192))[0])))
        n = int(round(math.exp(_uniform(gen, math.log(1e4), math.log(1e6))[0]) * scale))
        comps = int(torch.randint(1, 4, (1,), generator=gen))
        x = np.linspace(1e-3, 1.0, g, dtype=np.float64).astype(np.float32).astype(np.float64)
        grids.append(x)
        vals.append(_powerlaw_mixture(gen, x, comps))
        counts.append(max(n, 0))
        cuts.append(_uniform(gen, 0.01, 0.1)[0])
    return _pack("ragged", grids, vals, counts, cuts, 1234, {})


def precision(scale: float = 1.0, n_densities: int = 16, knots: int = 1 << 20) -> DensityBatchSpec:
    gen = torch.Generator().manual_seed(3)
    x = np.linspace(1e-6, 1.0, knots, dtype=np.float64).astype(np.float32).astype(np.float64)
    grids, vals = [], []
    for _ in range(n_densities):
        mu = _uniform(gen, 0.1, 0.9)[0]
        sigma = math.exp(_uniform(gen, math.log(1e-4), math.log(1e-2))[0])
        f = np.exp(-0.5 * ((x - mu) / sigma) ** 2) / (sigma * math.sqrt(2 * math.pi))
        f = f + 1e-8 * np.power(x, -0.5)
        grids.append(x)
        vals.append(f)
    n = max(1, int(round(10_000_000 * scale)))
    return _pack("precision", grids, vals, [n] * n_densities, None, 1234, {"knots": knots})


WORKLOADS = {"single": single, "uniform": uniform, "ragged": ragged, "precision": precision}


@dataclass
class TupleSpec:
    """The reference's 2-D theory tuple (pytorch/theory.py:118-126 layout):
    x_bins (B,nx,kx), xsec_x (B,ny,nx,kx), q_bins (B,ny,kq), xsec_q (B,nx,ny,kq),
    weights (B,nx,ny), acceptance (B,nx,ny), all fp64 but acceptance (bool)."""

    name: str
    x_bins: np.ndarray
    xsec_x: np.ndarray
    q_bins: np.ndarray
    xsec_q: np.ndarray
    weights: np.ndarray
    acceptance: np.ndarray
    n_events: int
    seed: int = 1234
    sequence: int = 0

    @property
    def arrays(self):
        return (self.x_bins, self.xsec_x, self.q_bins, self.xsec_q, self.weights, self.acceptance)

    @property
    def cells(self) -> int:
        return int(np.prod(self.weights.shape))

    @property
    def total_events(self) -> int:
        return int(self.n_events)


def theory_tuple(grid: int = 100, knots: int = 10, n_events: int = 1_000_000,
                 batch: int = 1) -> TupleSpec:
    """Seeded synthetic theory tuple with the shapes of the reference's GPU
    benchmark (grid 100: 99 x 99 cells, K = 10 knots per curve): cell ix of
    the x axis spans the ix-th of 99 log-spaced ranges of (1e-3, 1) with K
    uniform knots, likewise q; cross sections are positive power laws
    x^a (1-x)^b (a ~ U(-0.5, 1), b ~ U(1, 5) per curve) scaled by a smooth
    factor of the other axis; weights are Dirichlet(1) over the cells;
    acceptance is True with probability 0.95."""
    gen = torch.Generator().manual_seed(4)
    n = grid - 1
    edges = np.geomspace(1e-3, 1.0, n + 1)

    def bins():
        out = np.empty((batch, n, knots))
        for i in range(n):
            out[:, i, :] = np.linspace(edges[i], edges[i + 1], knots)
        return out

    x_bins, q_bins = bins(), bins()

    def curves(b_of, other):
        shape = (batch, n, n, knots)
        a = _uniform(gen, -0.5, 1.0, batch * n * n).reshape(batch, n, n, 1)
        b = _uniform(gen, 1.0, 5.0, batch * n * n).reshape(batch, n, n, 1)
        x = np.broadcast_to(b_of[:, None, :, :], shape)  # (B, other, cell, K)
        scale = 1.0 + 0.3 * np.cos(np.arange(n) * 0.37)[None, :, None, None] * other
        return np.ascontiguousarray(np.power(x, a) * np.power(1.0 - x + 1e-12, b) * scale)

    xsec_x = curves(x_bins, 1.0)   # (B, ny, nx, kx)
    xsec_q = curves(q_bins, -1.0)  # (B, nx, ny, kq)
    e = -torch.log(torch.rand(batch * n * n, generator=gen, dtype=torch.float64)).numpy()
    weights = (e.reshape(batch, n * n) / e.reshape(batch, n * n).sum(1, keepdims=True)).reshape(
        batch, n, n)
    acceptance = torch.rand(batch * n * n, generator=gen, dtype=torch.float64).numpy().reshape(
        batch, n, n) < 0.95
    return TupleSpec("tuple", x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events)


def cotangent(n: int, seed: int = 0) -> np.ndarray:
    """Upstream cotangent ~ N(0, 1) of n events (fp32), from a fixed seed."""
    gen = torch.Generator().manual_seed(seed)
    return torch.randn(n, generator=gen, dtype=torch.float32).numpy()
