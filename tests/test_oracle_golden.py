"""Pin the CPU oracle (oracle/loits_oracle.c) to the reference.

The golden vectors were produced by the reference's own compiled cores
(tests/golden/make_golden.py).  Integer/index/RNG outputs must match bit for
bit; with both sides built without floating-point contraction the values
match bit for bit as well (asserted exactly, not with a tolerance).
"""
import hashlib

import numpy as np
import pytest

from conftest import DENSITY_CASES, TUPLE_CASES, golden_case


def test_philox_known_answer(oracle_lib, golden):
    # Random123 Philox4x32-10, counter 0 / key 0 (tests/test_native_rng.py:43-55)
    assert oracle_lib.philox(0, 0, 0) == [int(w) for w in golden["kat/words"]]
    u = oracle_lib.fill_uniform(4, seed=0, stream=0)
    expected = np.array([(int(w) >> 8) * 2.0**-24 for w in golden["kat/words"]], dtype=np.float32)
    assert np.array_equal(u, expected)


def test_uniform_range_and_streams(oracle_lib):
    ux = oracle_lib.fill_uniform(4096, seed=23, stream=14)
    uq = oracle_lib.fill_uniform(4096, seed=23, stream=15)
    assert ux.min() >= 0.0 and ux.max() < 1.0
    assert not np.array_equal(ux, uq)
    # 24-bit grid: every value is an exact multiple of 2^-24
    assert np.all(np.floor(ux.astype(np.float64) * 2**24) == ux.astype(np.float64) * 2**24)


@pytest.mark.parametrize("name", TUPLE_CASES)
def test_reference_tuple_forward_matches_reference(oracle_lib, golden, name):
    c = golden_case(golden, name)
    n_events, seed, seq = (int(v) for v in c["scalars"])
    out = oracle_lib.r_forward(c["x_bins"], c["xsec_x"], c["q_bins"], c["xsec_q"], c["weights"],
                               c["acceptance"], n_events, seed, seq)
    assert [out["nmax"], out["active"]] == list(c["alloc"])
    assert np.array_equal(out["packed"], c["packed"])
    assert np.array_equal(out["interval_x"], c["interval_x_rows"])
    assert np.array_equal(out["interval_q"], c["interval_q_rows"])
    assert np.array_equal(out["norm_x"], c["norm_x"]) and np.array_equal(out["norm_q"], c["norm_q"])
    assert np.array_equal(out["cdf_x"], c["cdf_x"]) and np.array_equal(out["cdf_q"], c["cdf_q"])
    assert np.array_equal(out["events"], c["events"])


@pytest.mark.parametrize("name", TUPLE_CASES)
def test_reference_tuple_backward_matches_reference(oracle_lib, golden, name):
    c = golden_case(golden, name)
    n_events, seed, seq = (int(v) for v in c["scalars"])
    out = oracle_lib.r_forward(c["x_bins"], c["xsec_x"], c["q_bins"], c["xsec_q"], c["weights"],
                               c["acceptance"], n_events, seed, seq)
    gx, gq = oracle_lib.r_backward(c["cotangent"], out, c["x_bins"], c["xsec_x"], c["q_bins"],
                                   c["xsec_q"], c["acceptance"], seed, seq)
    # the reference sums per row in the same order: identical up to the last bit
    np.testing.assert_allclose(gx, c["grad_x"], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(gq, c["grad_q"], rtol=1e-13, atol=1e-15)
    # and against the reference's torch autograd (tolerance of cpp vs torch,
    # compare_backend_torch.py:16-24)
    np.testing.assert_allclose(gx, c["torch_grad_x"], rtol=1e-10, atol=2e-12)
    np.testing.assert_allclose(gq, c["torch_grad_q"], rtol=1e-10, atol=2e-12)


@pytest.mark.parametrize("name", DENSITY_CASES)
def test_density_batch_matches_reference_embedding(oracle_lib, golden, name):
    c = golden_case(golden, name)
    seed, seq = (int(v) for v in c["scalars"])
    eoff = np.concatenate([[0], np.cumsum(c["event_counts"])])
    x_cut = c.get("x_cut")
    out = oracle_lib.d_forward(c["knot_offsets"], eoff, c["grid"], c["values"], x_cut, seed, seq)
    assert np.array_equal(out["row_offsets"], c["row_offsets"])
    assert np.array_equal(out["slots"], c["slots"])
    assert np.array_equal(out["intervals"], c["intervals"])
    assert np.array_equal(out["events"], c["events"])
    grad = oracle_lib.d_backward(c["knot_offsets"], eoff, c["grid"], c["values"], x_cut, seed, seq,
                                 c["cotangent"], fwd=out)
    np.testing.assert_allclose(grad, c["grad_values"], rtol=1e-12, atol=1e-14)


def test_single_density_workload_digest(oracle_lib, golden):
    c = golden_case(golden, "single")
    seed, seq = (int(v) for v in c["scalars"])
    eoff = np.concatenate([[0], np.cumsum(c["event_counts"])])
    out = oracle_lib.d_forward(c["knot_offsets"], eoff, c["grid"], c["values"], None, seed, seq)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
    assert np.array_equal(out["events"][c["sample_index"]], c["events_sample"])
    assert sha(out["events"]) == str(c["events_sha256"])
    assert sha(out["slots"].astype(np.int64)) == str(c["slots_sha256"])
    assert sha(out["intervals"]) == str(c["intervals_sha256"])


def test_workload_generator_is_pinned(golden):
    """The synthetic workload generators still produce the golden inputs."""
    from quantom_loits_b200 import workloads

    c = golden_case(golden, "single")
    spec = workloads.single()
    assert np.array_equal(spec.grid, c["grid"]) and np.array_equal(spec.values, c["values"])
    c = golden_case(golden, "uniform_small")
    spec = workloads.uniform(scale=2e-3, n_densities=6)
    assert np.array_equal(spec.values, c["values"])
    c = golden_case(golden, "ragged_workload_small")
    spec = workloads.ragged(scale=4e-3, n_densities=6)
    assert np.array_equal(spec.values, c["values"]) and np.array_equal(spec.x_cut, c["x_cut"])


def test_branch_frozen_fd_matches_oracle_vjp(oracle_lib, golden):
    """The FD checker agrees with the oracle's own analytic VJP (fp64)."""
    c = golden_case(golden, "uniform_small")
    seed, seq = (int(v) for v in c["scalars"])
    eoff = np.concatenate([[0], np.cumsum(c["event_counts"])])
    out = oracle_lib.d_forward(c["knot_offsets"], eoff, c["grid"], c["values"], None, seed, seq)
    grad = oracle_lib.d_backward(c["knot_offsets"], eoff, c["grid"], c["values"], None, seed, seq,
                                 c["cotangent"], fwd=out)
    rows = out["row_offsets"]
    rng = np.random.default_rng(5)
    # FD of a sum over events is rounding-limited (error ~ 1/h): a 1e-5
    # relative step resolves 1e-6 of the gradient scale; the 1e-6 step used
    # by the GPU gradient checks resolves 1e-4.
    for rel, tol in ((1e-5, 1e-6), (1e-6, 1e-4)):
        for _ in range(8):
            b = int(rng.integers(0, len(c["event_counts"])))
            o, k = int(c["knot_offsets"][b]), int(c["knot_offsets"][b + 1] - c["knot_offsets"][b])
            t = int(rng.integers(0, k))
            # relative to the knot's value, floored at the density's mean
            # magnitude (a knot where the density vanishes has no scale)
            fmean = float(np.abs(c["values"][o:o + k]).mean())
            h = rel * max(abs(float(c["values"][o + t])), fmean)
            d, flips = oracle_lib.d_fd(b, t, h, c["knot_offsets"], eoff, c["grid"], c["values"],
                                       None, seed, seq, c["cotangent"][rows[b]:rows[b + 1]])
            scale = max(np.abs(grad[o:o + k]).max(), 1e-12)
            assert abs(d - grad[o + t]) <= tol * scale, (b, t, d, grad[o + t], flips)
