"""GPU parity of the reference-tuple sampler (fp64, 2-D cells) through the C ABI.

The expected values are the reference's own outputs (golden vectors from the
reference's compiled cpp core) and the CPU oracle.  RNG, packed slot indices,
intervals and, with both sides rounding every fp64 operation separately in the
reference's order, the event values are bit-exact.  Gradients are compared with
the reference cpp-vs-torch tolerance (compare_backend_torch.py:16-24):
rtol 1e-10, atol 2e-12.
"""
import numpy as np
import pytest
import torch

from conftest import TUPLE_CASES, golden_case

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")


def tensors(c):
    xb, xs, qb, qs, w = (torch.from_numpy(np.ascontiguousarray(c[k])).to(DEV) for k in
                         ("x_bins", "xsec_x", "q_bins", "xsec_q", "weights"))
    acc = torch.from_numpy(np.ascontiguousarray(c["acceptance"])).to(DEV)
    return xb, xs, qb, qs, w, acc


@pytest.fixture(scope="module")
def backend():
    from quantom_loits_b200 import backend as B

    return B


def test_philox_known_answer_on_device(backend, golden):
    u = backend.fill_uniform(4, seed=0, stream_id=0, device=DEV).cpu().numpy()
    expected = np.array([(int(w) >> 8) * 2.0**-24 for w in golden["kat/words"]], dtype=np.float32)
    assert np.array_equal(u, expected)


@pytest.mark.parametrize("count", [1, 3, 4, 5, 1023, 4099, 1 << 20])
def test_fill_uniform_matches_oracle(backend, oracle_lib, count):
    for seed, stream in ((23, 14), (2**40 + 7, 2**33 + 1)):
        u = backend.fill_uniform(count, seed, stream, DEV).cpu().numpy()
        assert np.array_equal(u, oracle_lib.fill_uniform(count, seed, stream))


@pytest.mark.parametrize("name", TUPLE_CASES)
def test_forward_matches_reference(backend, golden, name):
    c = golden_case(golden, name)
    n_events, seed, seq = (int(v) for v in c["scalars"])
    events, st = backend.tuple_forward(*tensors(c), n_events, seed, seq, want_intervals=True)
    assert [st["nmax"], st["active"]] == list(c["alloc"])
    assert np.array_equal(st["packed"].cpu().numpy(), c["packed"])
    assert np.array_equal(st["interval_x"].cpu().numpy(), c["interval_x_rows"])
    assert np.array_equal(st["interval_q"].cpu().numpy(), c["interval_q_rows"])
    assert np.array_equal(st["norm_x"].cpu().numpy(), c["norm_x"])
    assert np.array_equal(st["cdf_x"].cpu().numpy(), c["cdf_x"])
    assert np.array_equal(st["cdf_q"].cpu().numpy(), c["cdf_q"])
    assert np.array_equal(events.cpu().numpy(), c["events"])


@pytest.mark.parametrize("name", TUPLE_CASES)
def test_backward_matches_reference_and_torch(backend, golden, name):
    c = golden_case(golden, name)
    n_events, seed, seq = (int(v) for v in c["scalars"])
    xb, xs, qb, qs, w, acc = tensors(c)
    events, st = backend.tuple_forward(xb, xs, qb, qs, w, acc, n_events, seed, seq)
    g = torch.from_numpy(c["cotangent"]).to(DEV)
    gx, gq = backend.tuple_backward(g, xb, xs, qb, qs, acc, st, seed, seq)
    np.testing.assert_allclose(gx.cpu().numpy(), c["grad_x"], rtol=1e-10, atol=2e-12)
    np.testing.assert_allclose(gq.cpu().numpy(), c["grad_q"], rtol=1e-10, atol=2e-12)
    np.testing.assert_allclose(gx.cpu().numpy(), c["torch_grad_x"], rtol=1e-10, atol=2e-12)
    np.testing.assert_allclose(gq.cpu().numpy(), c["torch_grad_q"], rtol=1e-10, atol=2e-12)


def test_backward_is_deterministic(backend, golden):
    c = golden_case(golden, "theory10_k10")
    n_events, seed, seq = (int(v) for v in c["scalars"])
    xb, xs, qb, qs, w, acc = tensors(c)
    g = torch.from_numpy(c["cotangent"]).to(DEV)
    outs = []
    for _ in range(2):
        _, st = backend.tuple_forward(xb, xs, qb, qs, w, acc, n_events, seed, seq)
        outs.append(backend.tuple_backward(g, xb, xs, qb, qs, acc, st, seed, seq))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


def test_native_state_mirror_replays_like_reference(backend, golden):
    """native_forward returns the reference pybind state list; its u_x / u_q
    are the reference's padded uniforms (cpp/bindings.cpp:79-92)."""
    c = golden_case(golden, "theory3_k5")
    n_events, seed, seq = (int(v) for v in c["scalars"])
    state = backend.native_forward(*tensors(c), n_events, seed, seq)
    events, norm_x, norm_q, cdf_x, cdf_q, u_x, u_q, ix, iq, packed = state
    assert u_x.shape == (1, 4, int(c["alloc"][0]))
    assert np.array_equal(u_x.reshape(-1)[:64].cpu().numpy(), c["u_x_head"][:u_x.numel()])
    assert np.array_equal(u_x.reshape(-1)[packed].cpu().numpy(), c["u_x_rows"])
    assert np.array_equal(u_q.reshape(-1)[packed].cpu().numpy(), c["u_q_rows"])
    xb, xs, qb, qs, w, acc = tensors(c)
    g = torch.from_numpy(c["cotangent"]).to(DEV)
    gx, gq = backend.native_backward(g, xb, xs, qb, qs, acc, *state[1:], False, seed=seed,
                                     sequence=seq)
    np.testing.assert_allclose(gx.cpu().numpy(), c["grad_x"], rtol=1e-10, atol=2e-12)


def test_public_autograd_path_reaches_leaves(golden):
    """LOITS(backend="cuda") through torch.autograd (tests/test_cpp_loits.py:98-107)."""
    from quantom_loits_b200.loits import LOITS

    c = golden_case(golden, "theory3_k5")
    xb, xs, qb, qs, w, acc = tensors(c)
    xs.requires_grad_(True)
    qs.requires_grad_(True)
    torch.manual_seed(17)
    sampler = LOITS(backend="cuda", device=DEV)
    events = sampler((xb, xs, qb, qs, w, acc), 50)
    assert events.dtype == torch.float64 and events.ndim == 2 and events.shape[1] == 2
    assert events.shape[0] > 0
    events.square().mean().backward()
    assert xs.grad is not None and torch.isfinite(xs.grad).all()
    assert qs.grad is not None and torch.isfinite(qs.grad).all()
    # sequence advances per call, seed is torch.initial_seed() (cpp/backend.py:81-88)
    assert sampler.impl.sequence == 1 and sampler.impl.seed == torch.initial_seed()


def test_sequence_and_seed_change_the_stream(backend, golden):
    c = golden_case(golden, "theory3_k5")
    t = tensors(c)
    a, _ = backend.tuple_forward(*t, 80, 31, 4)
    b, _ = backend.tuple_forward(*t, 80, 31, 4)
    d, _ = backend.tuple_forward(*t, 80, 31, 5)
    e, _ = backend.tuple_forward(*t, 80, 32, 4)
    assert torch.equal(a, b)
    assert not torch.equal(a, d) and not torch.equal(a, e)


def test_zero_events_and_rejected_cells(backend, oracle_lib, golden):
    c = golden_case(golden, "manual_rejected_cell")
    t = tensors(c)
    ev, st = backend.tuple_forward(*t, 0, 23, 0)
    assert ev.shape == (0, 2) and st["packed"].numel() == 0
    # acceptance=False cells give an all-zero CDF whose events are still kept
    # (Appendix semantics of the reference: large but finite x)
    ev, st = backend.tuple_forward(*t, 80, 23, 0)
    ref = oracle_lib.r_forward(c["x_bins"], c["xsec_x"], c["q_bins"], c["xsec_q"], c["weights"],
                               c["acceptance"], 80, 23, 0)
    assert np.array_equal(ev.cpu().numpy(), ref["events"])


def test_large_tuple_matches_oracle(backend, oracle_lib):
    """A 30x30-cell theory tuple with K=10 and 2e5 events against the oracle."""
    rng = np.random.default_rng(11)
    B, nx, ny, kx, kq = 2, 30, 30, 10, 10
    x_bins = np.sort(rng.uniform(0.001, 0.999, (B, nx, kx)), axis=-1)
    q_bins = np.sort(rng.uniform(0.001, 0.999, (B, ny, kq)), axis=-1)
    xsec_x = rng.uniform(0.1, 2.0, (B, ny, nx, kx))
    xsec_q = rng.uniform(0.1, 2.0, (B, nx, ny, kq))
    w = rng.dirichlet(np.ones(nx * ny), B).reshape(B, nx, ny)
    acc = rng.uniform(size=(B, nx, ny)) > 0.05
    n_events, seed, seq = 200_000, 5, 9
    t = [torch.from_numpy(a).to(DEV) for a in (x_bins, xsec_x, q_bins, xsec_q, w, acc)]
    ev, st = backend.tuple_forward(*t, n_events, seed, seq)
    ref = oracle_lib.r_forward(x_bins, xsec_x, q_bins, xsec_q, w, acc, n_events, seed, seq)
    assert np.array_equal(st["packed"].cpu().numpy(), ref["packed"])
    assert np.array_equal(ev.cpu().numpy(), ref["events"])
    g = rng.standard_normal(ref["events"].shape)
    gx, gq = backend.tuple_backward(torch.from_numpy(g).to(DEV), t[0], t[1], t[2], t[3], t[5], st,
                                    seed, seq)
    rgx, rgq = oracle_lib.r_backward(g, ref, x_bins, xsec_x, q_bins, xsec_q, acc, seed, seq)
    np.testing.assert_allclose(gx.cpu().numpy(), rgx, rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(gq.cpu().numpy(), rgq, rtol=1e-9, atol=1e-10)


@pytest.mark.parametrize("name", TUPLE_CASES[:3])
def test_tuple_step_captured_in_one_graph(backend, golden, name):
    """Forward + backward of the reference tuple captured in one CUDA graph
    (counts kept on the device, outputs sized by n_events * sum |w|): every
    replay gives the events, packed rows and gradients of the eager
    tuple_forward / tuple_backward, bit for bit."""
    c = golden_case(golden, name)
    n_events, seed, seq = (int(v) for v in c["scalars"])
    t = tensors(c)
    events, st = backend.tuple_forward(*t, n_events, seed, seq)
    valid = events.shape[0]
    g = torch.randn((valid, 2), generator=torch.Generator(device=DEV).manual_seed(4),
                    device=DEV, dtype=torch.float64)
    gx, gq = backend.tuple_backward(g, t[0], t[1], t[2], t[3], t[5], st, seed, seq)
    step = backend.TupleStep(*t, n_events, seed, seq)
    assert step.capacity >= st["active"]
    step.grad_events.zero_()
    step.grad_events[:valid] = g
    step.capture()
    for _ in range(2):
        step.events.zero_()
        step.grad_xsec_x.zero_()
        step.step()
        torch.cuda.synchronize()
        step.check_status()
        ev, packed = step.result()
        assert torch.equal(ev, events) and torch.equal(packed, st["packed"])
        assert torch.equal(step.grad_xsec_x, gx) and torch.equal(step.grad_xsec_q, gq)


def test_tuple_step_reports_a_capacity_overrun(backend, golden):
    """Weights raised after the step was sized: the sampler writes nothing
    and reports LOITS_ERR_CAPACITY on the device instead of overrunning."""
    from quantom_loits_b200 import _native as N

    c = golden_case(golden, TUPLE_CASES[0])
    n_events, seed, seq = (int(v) for v in c["scalars"])
    t = list(tensors(c))
    step = backend.TupleStep(*t, n_events, seed, seq)
    t[4].mul_(4.0)  # the step reads the caller's weights in place
    step.forward()
    torch.cuda.synchronize()
    with pytest.raises(N.LoitsError) as err:
        step.check_status()
    assert err.value.code == N.LOITS_ERR_CAPACITY
    assert int(step.valid.item()) == 0


def test_sparse_cells_match_oracle(backend, oracle_lib):
    """A tuple whose cells hold 0-3 events each, so that one 1024-slot
    sampling tile spans hundreds of cells (the tile's cells are found by one
    warp-wide search, each event's cell by a search among them) and the
    backward's chunks start in far-apart cells; bit-exact with the oracle."""
    rng = np.random.default_rng(23)
    B, nx, ny, kx, kq = 1, 120, 150, 6, 5
    x_bins = np.sort(rng.uniform(0.001, 0.999, (B, nx, kx)), axis=-1)
    q_bins = np.sort(rng.uniform(0.001, 0.999, (B, ny, kq)), axis=-1)
    xsec_x = rng.uniform(0.1, 2.0, (B, ny, nx, kx))
    xsec_q = rng.uniform(0.1, 2.0, (B, nx, ny, kq))
    # heavy-tailed weights: most cells get trunc(|w| n) = 0, a few get many
    w = rng.pareto(1.2, (B, nx, ny))
    w /= w.sum()
    acc = np.ones((B, nx, ny), bool)
    n_events, seed, seq = 30_000, 7, 2
    t = [torch.from_numpy(a).to(DEV) for a in (x_bins, xsec_x, q_bins, xsec_q, w, acc)]
    ev, st = backend.tuple_forward(*t, n_events, seed, seq)
    ref = oracle_lib.r_forward(x_bins, xsec_x, q_bins, xsec_q, w, acc, n_events, seed, seq)
    counts = np.trunc(np.abs(w.reshape(-1) * n_events))
    assert (counts == 0).mean() > 0.5  # the shape this test is about
    assert np.array_equal(st["packed"].cpu().numpy(), ref["packed"])
    assert np.array_equal(ev.cpu().numpy(), ref["events"])
    g = rng.standard_normal(ref["events"].shape)
    gx, gq = backend.tuple_backward(torch.from_numpy(g).to(DEV), t[0], t[1], t[2], t[3], t[5], st,
                                    seed, seq)
    rgx, rgq = oracle_lib.r_backward(g, ref, x_bins, xsec_x, q_bins, xsec_q, acc, seed, seq)
    np.testing.assert_allclose(gx.cpu().numpy(), rgx, rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(gq.cpu().numpy(), rgq, rtol=1e-9, atol=1e-10)
