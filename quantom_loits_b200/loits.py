"""Backend registry and public sampler, with the reference's interface.

Mirrors niteya-shah/quantom_loits ``loits.py``: ``register_backend(name,
factory, probe)`` (loits.py:13-15), ``registered_backends`` (:18-19),
``backend_status`` (:34-46), ``available_backends`` (:49-50),
``BackendUnavailableError`` (:9-10) and the ``LOITS`` module (:129-145), whose
constructor raises ``ValueError`` for an unknown backend name and
``BackendUnavailableError`` when the backend's probe fails for the device.

This package registers one backend, ``"cuda"``: the B200 sampler
(``quantom_loits_b200.backend.CudaLOITS``).  Its call is the reference's
``sampler(theory_outputs, n_events)``; ``theory_outputs`` is either the
reference's theory tuple (pytorch/theory.py:118-126) or a
``quantom_loits_b200.batched.DensityBatch`` of ragged 1-D densities.
"""
from __future__ import annotations

import torch
from torch import nn

_BACKENDS: dict = {}
_BACKEND_PROBES: dict = {}


class BackendUnavailableError(RuntimeError):
    pass


def register_backend(name, factory, probe=None):
    _BACKENDS[name] = factory
    _BACKEND_PROBES[name] = probe


def registered_backends():
    return tuple(sorted(_BACKENDS))


def backend_status(name, device="cpu"):
    """(ok, reason) of backend `name` on `device`; probe exceptions become reasons."""
    if name not in _BACKENDS:
        return False, f"backend {name!r} is not registered"
    probe = _BACKEND_PROBES.get(name)
    if probe is None:
        return True, ""
    try:
        result = probe(torch.device(device))
    except Exception as exc:  # the reference reports probe failures as reasons
        return False, str(exc)
    if isinstance(result, tuple):
        return bool(result[0]), str(result[1])
    return bool(result), "" if result else "backend probe returned unavailable"


def available_backends(device="cpu"):
    return tuple(name for name in registered_backends() if backend_status(name, device)[0])


def _load_cuda(**kwargs):
    from .backend import CudaLOITS

    return CudaLOITS(**kwargs)


def _probe_cuda(device):
    from .backend import availability

    return availability(device)


register_backend("cuda", _load_cuda, _probe_cuda)


class LOITS(nn.Module):
    def __init__(self, backend="cuda", **kwargs):
        super().__init__()
        if backend not in _BACKENDS:
            available = ", ".join(registered_backends())
            raise ValueError(f"backend={backend!r} is not registered; registered: {available}")
        device = kwargs.get("device", "cuda")
        ok, reason = backend_status(backend, device)
        if not ok:
            raise BackendUnavailableError(
                f"backend={backend!r} is unavailable for device={device!s}: {reason}")
        self.backend = backend
        self.impl = _BACKENDS[backend](**kwargs)

    def forward(self, theory_outputs, n_events):
        return self.impl(theory_outputs, n_events)
