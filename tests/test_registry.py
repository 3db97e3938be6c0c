"""The backend registry keeps the reference's contract (loits.py:9-145)."""
import pytest
import torch

from quantom_loits_b200 import loits


def test_cuda_backend_is_registered():
    assert "cuda" in loits.registered_backends()


def test_unknown_backend_raises_value_error():
    with pytest.raises(ValueError, match="is not registered"):
        loits.LOITS(backend="does-not-exist")


def test_status_of_unregistered_backend():
    ok, reason = loits.backend_status("nope")
    assert not ok and "not registered" in reason


def test_register_backend_with_probe_and_factory():
    calls = []

    def factory(**kw):
        calls.append(kw)
        return torch.nn.Identity()

    loits.register_backend("fake", factory, lambda device: (device.type == "cpu", "cpu only"))
    try:
        assert loits.backend_status("fake", "cpu") == (True, "cpu only")
        assert "fake" in loits.available_backends("cpu")
        m = loits.LOITS(backend="fake", device="cpu")
        assert m.backend == "fake" and isinstance(m.impl, torch.nn.Identity)
        assert calls == [{"device": "cpu"}]
        with pytest.raises(loits.BackendUnavailableError):
            loits.LOITS(backend="fake", device="meta")
    finally:
        loits._BACKENDS.pop("fake", None)
        loits._BACKEND_PROBES.pop("fake", None)


def test_probe_exception_becomes_reason():
    def boom(device):
        raise RuntimeError("probe exploded")

    loits.register_backend("boom", lambda **kw: None, boom)
    try:
        assert loits.backend_status("boom", "cpu") == (False, "probe exploded")
    finally:
        loits._BACKENDS.pop("boom", None)
        loits._BACKEND_PROBES.pop("boom", None)


def test_cuda_probe_needs_a_cuda_device():
    ok, reason = loits.backend_status("cuda", "cpu")
    assert not ok and "CUDA" in reason


def test_epsilon_other_than_reference_is_rejected():
    from quantom_loits_b200.backend import CudaLOITS

    with pytest.raises(ValueError, match="1e-5"):
        CudaLOITS(device="cuda", epsilon=1e-4)
