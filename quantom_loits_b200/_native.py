"""ctypes binding of libloits_b200.so (the C ABI declared in include/loits_b200.h).

The library is the product: there is no Python, PyTorch or CPU fallback for
any of its entry points.  ``lib()`` raises if the library has not been built
or cannot be loaded; callers that launch work additionally require a CUDA
device (``require_device``).
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "libloits_b200.so"

_i32 = C.c_int32
_i64 = C.c_int64
_u64 = C.c_uint64
_vp = C.c_void_p
_sz = C.c_size_t

LOITS_OK = 0
LOITS_ERR_INVALID = 1
LOITS_ERR_UNSUPPORTED = 2
LOITS_ERR_CUDA = 3
LOITS_ERR_TIMEOUT = 4
LOITS_ERR_CAPACITY = 5
LOITS_ERR_EPSILON = 6
LOITS_TUPLE_NOALLOC_MAX_ACTIVE = 67108864


class LoitsError(RuntimeError):
    """A non-zero loits_status from the library (host or device side)."""

    def __init__(self, code: int, where: str):
        self.code = int(code)
        super().__init__(f"{where}: {status_string(code)} (status {code})")


class Shape(C.Structure):
    _fields_ = [("batch", _i64), ("nx", _i64), ("ny", _i64), ("kx", _i64), ("kq", _i64)]


class BatchConfig(C.Structure):
    _fields_ = [("threads", _i32), ("blocks_per_item", _i32), ("scan_knots", _i32),
                ("ctas_per_sm", _i32), ("plain", _i32), ("guide_ratio", _i32),
                ("wait_limit", _i32), ("withhold_tile", _i32),
                ("density_base", _i64), ("slot_stride", _i64)]

    def as_dict(self) -> dict:
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


# name -> (restype, argtypes); every symbol include/loits_b200.h declares
SIGNATURES = {
    "loits_status_string": (C.c_char_p, [C.c_int]),
    "loits_version": (C.c_int, []),
    "loits_fill_uniform": (C.c_int, [_vp, _i64, _u64, _u64, _vp]),
    "loits_tuple_prepare": (C.c_int, [C.POINTER(Shape), _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp,
                                      _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "loits_tuple_sample_workspace": (_sz, [_i64]),
    "loits_tuple_sample": (C.c_int, [C.POINTER(Shape), _vp, _vp, _vp, _vp, _vp, _i64, _i64, _u64,
                                     _u64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "loits_tuple_sample_noalloc": (C.c_int, [C.POINTER(Shape), _vp, _vp, _vp, _vp, _vp, _i64, _i64,
                                             _u64, _u64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "loits_tuple_sample_bounded": (C.c_int, [C.POINTER(Shape), _vp, _vp, _vp, _vp, _vp, _vp,
                                             _i64, _u64, _u64, _vp, _vp, _vp, _vp, _vp, _vp,
                                             _vp, _sz, _vp]),
    "loits_tuple_backward_workspace": (_sz, [C.POINTER(Shape), _i64]),
    "loits_tuple_backward": (C.c_int, [C.POINTER(Shape), _vp, _vp, _i64, _i64, _u64, _u64, _vp,
                                       _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                       _sz, _vp]),
    "loits_tuple_backward_bounded": (C.c_int, [C.POINTER(Shape), _vp, _vp, _vp, _vp, _i64, _u64,
                                               _u64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                               _vp, _vp, _vp, _vp, _sz, _vp]),
    "loits_batch_plan_create": (C.c_int, [_i64, _vp, _vp, C.POINTER(BatchConfig),
                                          C.POINTER(_vp)]),
    "loits_batch_plan_create_ex": (C.c_int, [_i64, _vp, _vp, C.POINTER(BatchConfig), _vp, _vp,
                                             C.POINTER(_vp)]),
    "loits_batch_plan_destroy": (None, [_vp]),
    "loits_batch_capacity": (_i64, [_vp]),
    "loits_batch_total_knots": (_i64, [_vp]),
    "loits_batch_workspace_bytes": (_sz, [_vp]),
    "loits_batch_status_offset": (_sz, [_vp]),
    "loits_batch_plan_config": (C.c_int, [_vp, C.POINTER(BatchConfig)]),
    "loits_batch_forward": (C.c_int, [_vp, _vp, _vp, _vp, _u64, _u64, _vp, _vp, _vp, _vp, _vp]),
    "loits_batch_backward": (C.c_int, [_vp, _vp, _vp, _vp, _u64, _u64, _vp, _vp, _vp, _vp]),
    "loits_batch_forward_state": (C.c_int, [_vp, _vp, _vp, _vp, _u64, _u64, _vp, _vp, _vp, _vp,
                                            _vp, _vp]),
    "loits_batch_backward_state": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "loits_batch_cdf": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "loits_batch_quantile": (C.c_int, [_vp, _vp, _i64, _vp, _i64, _vp, _vp, _vp]),
    "loits_batch_forward_hist": (C.c_int, [_vp, _vp, _vp, _vp, _u64, _u64, _i32, C.c_float,
                                           C.c_float, _vp, _vp, _vp, _vp, _vp]),
    "loits_batch_backward_hist": (C.c_int, [_vp, _vp, _vp, _vp, _u64, _u64, _i32, C.c_float,
                                            C.c_float, _vp, _vp, _vp, _vp, _vp]),
    "loits_batch_forward_hist_powerlaw": (C.c_int, [_vp, _vp, _vp, _vp, _u64, _u64, _i32,
                                                    C.c_float, C.c_float, _vp, _vp, _vp, _vp,
                                                    _vp]),
    "loits_batch_backward_hist_powerlaw": (C.c_int, [_vp, _vp, _vp, _vp, _u64, _u64, _i32,
                                                     C.c_float, C.c_float, _vp, _vp, _vp, _vp,
                                                     _vp]),
    "loits_theory_powerlaw": (C.c_int, [_i64, _i64, _vp, _vp, _vp, _vp]),
    "loits_theory_powerlaw_vjp": (C.c_int, [_i64, _i64, _vp, _vp, _vp, _vp, _vp]),
}

_LIB = None
_LOCK = threading.Lock()


def lib():
    """Load the library once; raise if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    with _LOCK:
        if _LIB is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is not built; run `python -m quantom_loits_b200.build` "
                    "(the CUDA sampler has no fallback implementation)")
            handle = C.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _LIB = handle
    return _LIB


def status_string(code: int) -> str:
    try:
        return lib().loits_status_string(int(code)).decode()
    except Exception:  # pragma: no cover - library missing
        return "unknown status"


def check(code: int, where: str) -> None:
    if code != LOITS_OK:
        raise LoitsError(code, where)


def require_device(device: torch.device) -> None:
    if device.type != "cuda":
        raise RuntimeError(f"the CUDA LOITS sampler needs a CUDA tensor, got device {device}")
    if not torch.cuda.is_available():
        raise RuntimeError("the CUDA LOITS sampler needs a CUDA device; none is available")


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_of(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream
