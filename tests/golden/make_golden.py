"""Generate the golden vectors in this directory from the REFERENCE itself.

Run in a container that has the reference tree (by default the `reference`
directory beside this repository's root; override with
LOITS_REFERENCE_TREE):

    python tests/golden/make_golden.py

What it does:
* builds the reference's own ``cpp/loits_core.cpp`` and
  ``openmp/loits_core.cpp`` (oracle/Makefile, outputs in oracle/_ref/);
* builds theory tuples with the reference's own ``TorchProxyTheoryLite``
  (pytorch/theory.py) and the fixed inputs of the reference tests
  (tests/test_cpp_loits.py:11-29, tests/test_sycl_loits.py:40-71,
  tests/test_triton_loits.py:94 K sweep);
* runs the reference forward/backward stage sequence (cpp/bindings.cpp) on
  them, checks cpp == openmp bit for bit, and replays the reference's torch
  stages (pytorch/loits.py TorchLOITSCore, as compare_backend_torch.py:54-67
  does) with the cpp core's own uniforms to get torch-autograd gradients;
* embeds batched 1-D densities exactly into the reference tuple
  (oracle.oracle.embed_densities) and records the reference's answer for them.

Everything is written to ``golden.npz`` (small arrays in full; the large
"single" workload as SHA-256 digests plus a strided sample).
"""
from __future__ import annotations

import hashlib
import os
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
# the reference project's source tree: LOITS_REFERENCE_TREE, else the
# `reference` directory beside this repository's root
REF = Path(os.environ.get("LOITS_REFERENCE_TREE", str(ROOT.parent / "reference")))
sys.path.insert(0, str(REF))

from oracle import oracle as O  # noqa: E402
from quantom_loits_b200 import workloads  # noqa: E402

from pytorch.loits import TorchLOITSCore  # noqa: E402  (reference)
from pytorch.theory import TorchProxyTheoryLite  # noqa: E402  (reference)

OUT = Path(__file__).resolve().parent / "golden.npz"
PARAMS = [[0.67, 0.20, 0.23, 0.67, 0.50]]  # tests/test_cpp_loits.py:24-29


def theory_outputs(grid, k, params=PARAMS):
    th = TorchProxyTheoryLite({"n_points_x": grid, "n_points_y": grid, "n_cdf_points_x": k,
                               "n_cdf_points_y": k, "average": False}, "cpu")
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    return th(p)[:6]


def manual_outputs(acceptance=None):
    """tests/test_sycl_loits.py:40-71 (the reference's hand-written fixture)."""
    x_bins = torch.tensor([[[0.10, 0.20, 0.30, 0.40, 0.50], [0.20, 0.30, 0.40, 0.50, 0.60]]],
                          dtype=torch.float64)
    q_bins = torch.tensor([[[1.0, 1.5, 2.0, 2.5, 3.0], [2.0, 2.5, 3.0, 3.5, 4.0]]],
                          dtype=torch.float64)
    xsec_x = torch.tensor([[[[1.0, 1.1, 1.2, 1.3, 1.4], [1.1, 1.2, 1.3, 1.4, 1.5]],
                            [[1.2, 1.3, 1.4, 1.5, 1.6], [1.3, 1.4, 1.5, 1.6, 1.7]]]],
                          dtype=torch.float64, requires_grad=True)
    xsec_q = torch.tensor([[[[1.0, 1.2, 1.4, 1.6, 1.8], [1.1, 1.3, 1.5, 1.7, 1.9]],
                            [[1.2, 1.4, 1.6, 1.8, 2.0], [1.3, 1.5, 1.7, 1.9, 2.1]]]],
                          dtype=torch.float64, requires_grad=True)
    weights = torch.tensor([[[0.20, 0.30], [0.40, 0.10]]], dtype=torch.float64)
    if acceptance is None:
        acceptance = torch.ones((1, 2, 2), dtype=torch.bool)
    return x_bins, xsec_x, q_bins, xsec_q, weights, acceptance


def torch_with_samples(outputs, n_events, u_x, u_q):
    """Replay of the reference torch stages with given uniforms
    (compare_backend_torch.py:54-67)."""
    x_bins, xsec_x, q2_bins, xsec_q2, weights, acceptance = outputs[:6]
    core = TorchLOITSCore()
    grid0, grid1 = weights.shape[1:]
    mask = core.allocation(weights, n_events)
    rho_x = core.rho_x(x_bins, xsec_x)
    rho_q2 = core.rho_q2(q2_bins, xsec_q2)
    cdf_x = core.cdf_x(x_bins, rho_x, acceptance, True)
    cdf_q2 = core.cdf_q2(q2_bins, rho_q2, acceptance, False)
    cdf_x, bins_x = core.flatten_x(x_bins, cdf_x, grid0, grid1, True)
    cdf_q2, bins_q2 = core.flatten_q2(q2_bins, cdf_q2, grid0, grid1, False)
    x = core.interpolation_x(u_x, cdf_x, bins_x, mask)
    q2 = core.interpolation_q2(u_q, cdf_q2, bins_q2, mask)
    return core.stream_compaction(x, q2, mask)


def np_of(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def tuple_case(store, name, outputs, n_events, seed, sequence, torch_grads=True):
    cpp, omp = O.Reference("cpp"), O.Reference("openmp")
    arrs = [np_of(t) for t in outputs]
    st = cpp.forward(*arrs, n_events, seed, sequence)
    so = omp.forward(*arrs, n_events, seed, sequence)
    for key in ("events", "packed", "u_x", "u_q", "cdf_x", "cdf_q", "norm_x", "norm_q"):
        assert np.array_equal(st[key], so[key]), f"{name}: cpp and openmp disagree on {key}"
    gen = torch.Generator().manual_seed(seed + 1)
    g = torch.randn(st["events"].shape, generator=gen, dtype=torch.float64).numpy()
    gx, gq = cpp.backward(g, st, arrs[0], arrs[1], arrs[2], arrs[3], arrs[5])
    ox, oq = omp.backward(g, so, arrs[0], arrs[1], arrs[2], arrs[3], arrs[5])
    np.testing.assert_allclose(gx, ox, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(gq, oq, rtol=1e-12, atol=1e-14)
    pre = f"{name}/"
    for i, key in enumerate(("x_bins", "xsec_x", "q_bins", "xsec_q", "weights", "acceptance")):
        store[pre + key] = arrs[i]
    store[pre + "scalars"] = np.array([n_events, seed, sequence], dtype=np.int64)
    store[pre + "events"] = st["events"]
    store[pre + "packed"] = st["packed"]
    store[pre + "u_x_rows"] = st["u_x"].reshape(-1)[st["packed"]]
    store[pre + "u_q_rows"] = st["u_q"].reshape(-1)[st["packed"]]
    store[pre + "interval_x_rows"] = st["interval_x"][st["packed"]]
    store[pre + "interval_q_rows"] = st["interval_q"][st["packed"]]
    store[pre + "u_x_head"] = st["u_x"].reshape(-1)[:64]
    store[pre + "norm_x"], store[pre + "norm_q"] = st["norm_x"], st["norm_q"]
    store[pre + "cdf_x"], store[pre + "cdf_q"] = st["cdf_x"], st["cdf_q"]
    store[pre + "alloc"] = np.array([st["nmax"], st["active"]], dtype=np.int64)
    store[pre + "cotangent"] = g
    store[pre + "grad_x"], store[pre + "grad_q"] = gx, gq
    if torch_grads:
        ref = torch_with_samples(outputs, n_events, torch.from_numpy(st["u_x"]),
                                 torch.from_numpy(st["u_q"]))
        np.testing.assert_allclose(np_of(ref), st["events"], rtol=1e-12, atol=1e-12)
        tgx, tgq = torch.autograd.grad((ref * torch.from_numpy(g)).sum(), (outputs[1], outputs[3]))
        store[pre + "torch_grad_x"], store[pre + "torch_grad_q"] = np_of(tgx), np_of(tgq)
    print(f"{name}: nmax={st['nmax']} active={st['active']} valid={len(st['events'])}")


def density_case(store, name, spec: workloads.DensityBatchSpec, full=True):
    """Reference answer for a batch of 1-D densities through the exact embedding."""
    cpp = O.Reference("openmp")
    tup = O.embed_densities(spec.knot_offsets, spec.grid, spec.values, spec.event_counts)
    *arrs, n_events = tup
    st = cpp.forward(*arrs, n_events, spec.seed, spec.sequence)
    x = st["events"][:, 0]
    b = st["packed"] // max(st["nmax"], 1)
    slot = st["packed"] - b * st["nmax"]
    keep = np.ones(len(x), dtype=bool)
    if spec.x_cut is not None:
        keep = x > spec.x_cut.astype(np.float64)[b]
    nd = spec.n_densities
    rows = np.concatenate([[0], np.cumsum(np.bincount(b[keep], minlength=nd))]).astype(np.int64)
    # fp32 cotangent (the batched sampler's storage type), exact in fp64
    gen = torch.Generator().manual_seed(spec.seed + 7)
    g_kept = torch.randn(int(keep.sum()), generator=gen, dtype=torch.float32).numpy()
    g = np.zeros((len(x), 2))
    g[keep, 0] = g_kept
    gx, _ = cpp.backward(g, st, arrs[0], arrs[1], arrs[2], arrs[3], arrs[5])
    grad_values = np.concatenate([gx[d, 0, 0, : spec.knot_offsets[d + 1] - spec.knot_offsets[d]]
                                  for d in range(nd)])
    pre = f"{name}/"
    store[pre + "knot_offsets"] = spec.knot_offsets
    store[pre + "grid"], store[pre + "values"] = spec.grid, spec.values
    store[pre + "event_counts"] = spec.event_counts
    if spec.x_cut is not None:
        store[pre + "x_cut"] = spec.x_cut
    store[pre + "scalars"] = np.array([spec.seed, spec.sequence], dtype=np.int64)
    store[pre + "row_offsets"] = rows
    ints = st["interval_x"][st["packed"]][keep].astype(np.int32)
    if full:
        store[pre + "grad_values"] = grad_values
        store[pre + "cotangent"] = g_kept
        store[pre + "events"] = x[keep]
        store[pre + "slots"] = slot[keep]
        store[pre + "intervals"] = ints
    else:
        store[pre + "events_sha256"] = np.array(digest(x[keep]))
        store[pre + "slots_sha256"] = np.array(digest(slot[keep].astype(np.int64)))
        store[pre + "intervals_sha256"] = np.array(digest(ints))
        idx = np.arange(0, int(keep.sum()), 97)
        store[pre + "sample_index"] = idx
        store[pre + "events_sample"] = x[keep][idx]
    print(f"{name}: densities={nd} events={spec.total_events} kept={int(keep.sum())}")


def main():
    O.build(ref=True)
    torch.manual_seed(0)
    store: dict[str, np.ndarray] = {}
    # Random123 known answer the reference pins (tests/test_native_rng.py:43-55)
    store["kat/words"] = np.array([0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8], dtype=np.uint32)
    tuple_case(store, "theory3_k5", theory_outputs(3, 5), 80, 23, 0)
    tuple_case(store, "theory3_k5_seed0", theory_outputs(3, 5), 80, 0, 0)
    tuple_case(store, "manual", manual_outputs(), 80, 23, 7)
    acc = torch.tensor([[[True, False], [True, True]]])
    tuple_case(store, "manual_rejected_cell", manual_outputs(acc), 80, 23, 0)
    for k in (4, 5, 7, 8, 10, 16, 32):
        tuple_case(store, f"theory3_k{k}_n257", theory_outputs(3, k), 257, 23, 0)
    tuple_case(store, "theory10_k10", theory_outputs(10, 10, [[0.45, 0.35, 0.35, 0.55, 0.35]]),
               5000, 31, 3)
    tuple_case(store, "theory6_k5_batch2",
               theory_outputs(6, 5, [[0.67, 0.20, 0.23, 0.67, 0.50], [0.3, 0.6, 0.1, 0.9, 0.2]]),
               1000, 5, 2)
    # batched 1-D densities
    density_case(store, "single", workloads.single(), full=False)
    ragged_small = workloads.DensityBatchSpec(
        name="ragged_small",
        knot_offsets=np.array([0, 2, 5, 22, 86, 386], dtype=np.int64),
        grid=np.concatenate([np.linspace(0.1, 0.9, 2), np.linspace(1e-3, 1, 3),
                             np.linspace(0.2, 0.7, 17), np.linspace(1e-3, 1, 64),
                             np.linspace(1e-3, 1, 300)]).astype(np.float32),
        values=np.concatenate([[1.0, 3.0], [0.5, 2.0, 0.0], np.linspace(1, 2, 17),
                               np.linspace(1e-3, 1, 64) ** -0.5 * (1 - np.linspace(1e-3, 1, 64)) ** 4,
                               np.exp(-0.5 * ((np.linspace(1e-3, 1, 300) - 0.4) / 0.05) ** 2)]
                              ).astype(np.float32),
        event_counts=np.array([7, 0, 5, 1000, 333], dtype=np.int64),
        x_cut=np.array([0.3, 0.05, 0.25, 0.02, 0.35], dtype=np.float32), seed=99, sequence=4)
    density_case(store, "ragged_small", ragged_small)
    density_case(store, "uniform_small", workloads.uniform(scale=2e-3, n_densities=6))
    density_case(store, "ragged_workload_small", workloads.ragged(scale=4e-3, n_densities=6))
    np.savez_compressed(OUT, **store)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1024:.0f} KiB, {len(store)} arrays)")


if __name__ == "__main__":
    main()
