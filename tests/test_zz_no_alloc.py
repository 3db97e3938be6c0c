"""The allocation-free sampling call (loits_tuple_sample_noalloc).

Callers that cannot allocate device memory where they sample -- code inside
a framework that owns the whole GPU through its own pool, or a loop that must
not allocate after start-up -- use this form: its only scratch is a fixed
array inside the library.  Here it is called through the C ABI and must give
exactly what the ordinary call (workspace passed by the caller) gives, on two
calls in a row (the shared array keeps the previous call's contents, which
the call must clear).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden_case

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")


def _prepare(lib, N, t, n_events):
    xb, xs, qb, qs, w, acc = t
    B, nx, kx = xb.shape
    ny, kq = qb.shape[1], qb.shape[2]
    shape = N.Shape(B, nx, ny, kx, kq)
    ncell = B * nx * ny
    counts = torch.empty(ncell, dtype=torch.int64, device=DEV)
    cell_off = torch.empty(ncell + 1, dtype=torch.int64, device=DEV)
    norm_x = torch.empty((B, ny, nx), dtype=torch.float64, device=DEV)
    norm_q = torch.empty((B, nx, ny), dtype=torch.float64, device=DEV)
    cdf_x, cdf_q = torch.empty_like(xs), torch.empty_like(qs)
    alloc = torch.empty(2, dtype=torch.int64, device=DEV)
    stream = N.stream_of(DEV)
    assert lib.loits_tuple_prepare(C.byref(shape), xb.data_ptr(), xs.data_ptr(), qb.data_ptr(),
                                   qs.data_ptr(), w.data_ptr(), acc.view(torch.uint8).data_ptr(),
                                   n_events, counts.data_ptr(), cell_off.data_ptr(),
                                   norm_x.data_ptr(), norm_q.data_ptr(), cdf_x.data_ptr(),
                                   cdf_q.data_ptr(), alloc.data_ptr(), stream) == 0
    nmax, active = (int(v) for v in alloc.tolist())
    return shape, cell_off, cdf_x, cdf_q, nmax, active


def _sample(lib, N, t, prep, seed, seq, noalloc):
    xb, _, qb, _, _, _ = t
    shape, cell_off, cdf_x, cdf_q, nmax, active = prep
    cap = max(active, 1)
    events = torch.full((cap, 2), float("nan"), dtype=torch.float64, device=DEV)
    packed = torch.full((cap,), -1, dtype=torch.int64, device=DEV)
    ix = torch.full((cap,), -1, dtype=torch.int16, device=DEV)
    out = torch.zeros(2, dtype=torch.int64, device=DEV)  # [valid, status]
    stream = N.stream_of(DEV)
    args = (C.byref(shape), xb.data_ptr(), qb.data_ptr(), cdf_x.data_ptr(), cdf_q.data_ptr(),
            cell_off.data_ptr(), nmax, active, seed, seq, events.data_ptr(), packed.data_ptr(),
            ix.data_ptr(), None, out[0:1].data_ptr(), out[1:2].data_ptr())
    if noalloc:
        rc = lib.loits_tuple_sample_noalloc(*args, stream)
    else:
        ws = torch.empty(int(lib.loits_tuple_sample_workspace(active)), dtype=torch.uint8,
                         device=DEV)
        rc = lib.loits_tuple_sample(*args, ws.data_ptr(), ws.numel(), stream)
    assert rc == 0
    valid, status = (int(v) for v in out.tolist())
    assert status == 0
    return valid, events[:valid].cpu(), packed[:valid].cpu(), ix[:valid].cpu()


def _tensors(arrays):
    return [torch.from_numpy(np.ascontiguousarray(a)).to(DEV) for a in arrays]


def test_noalloc_matches_the_workspace_call_twice(golden):
    from quantom_loits_b200 import _native as N

    lib = N.lib()
    c = golden_case(golden, "theory10_k10")
    n_events, seed, seq = (int(v) for v in c["scalars"])
    t = _tensors([c[k] for k in ("x_bins", "xsec_x", "q_bins", "xsec_q", "weights",
                                 "acceptance")])
    prep = _prepare(lib, N, t, n_events)
    ref = _sample(lib, N, t, prep, seed, seq, noalloc=False)
    first = _sample(lib, N, t, prep, seed, seq, noalloc=True)
    second = _sample(lib, N, t, prep, seed, seq, noalloc=True)
    for got in (first, second):
        assert got[0] == ref[0]
        for a, b in zip(got[1:], ref[1:]):
            assert torch.equal(a, b)
    # and against the reference's own answer for this fixture
    assert np.array_equal(first[1].numpy(), c["events"])
    assert np.array_equal(first[2].numpy(), c["packed"])


def test_noalloc_large_call_then_small_call():
    """A call with many tiles, then one with few: the second must not see the
    first call's look-back words left in the shared array."""
    from quantom_loits_b200 import _native as N

    lib = N.lib()
    rng = np.random.default_rng(4)
    B, nx, ny, kx, kq = 1, 20, 20, 8, 6
    arrays = [np.sort(rng.uniform(0.01, 0.99, (B, nx, kx)), axis=-1),
              rng.uniform(0.2, 2.0, (B, ny, nx, kx)),
              np.sort(rng.uniform(0.01, 0.99, (B, ny, kq)), axis=-1),
              rng.uniform(0.2, 2.0, (B, nx, ny, kq)),
              rng.dirichlet(np.ones(nx * ny)).reshape(B, nx, ny),
              np.ones((B, nx, ny), dtype=bool)]
    t = _tensors(arrays)
    for n_events in (300_000, 5_000, 300_000):
        prep = _prepare(lib, N, t, n_events)
        ref = _sample(lib, N, t, prep, 9, 2, noalloc=False)
        got = _sample(lib, N, t, prep, 9, 2, noalloc=True)
        assert got[0] == ref[0]
        for a, b in zip(got[1:], ref[1:]):
            assert torch.equal(a, b)


def test_noalloc_rejects_more_slots_than_its_scratch_holds():
    from quantom_loits_b200 import _native as N

    lib = N.lib()
    shape = N.Shape(1, 1, 1, 2, 2)
    over = N.LOITS_TUPLE_NOALLOC_MAX_ACTIVE + 1
    rc = lib.loits_tuple_sample_noalloc(C.byref(shape), 1, 1, 1, 1, 1, over, over, 0, 0, 1, 1,
                                        None, None, 1, 1, None)
    assert rc == N.LOITS_ERR_CAPACITY
