"""CPU checks of the C ABI boundary: the library loads, exports every symbol
include/loits_b200.h declares, and rejects bad arguments on the host before
touching a device.  No kernel runs here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "loits_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(loits_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def native():
    from quantom_loits_b200 import build, _native

    build.build()
    return _native


def test_header_declares_the_abi():
    names = declared_symbols()
    for required in ("loits_fill_uniform", "loits_tuple_prepare", "loits_tuple_sample",
                     "loits_tuple_backward", "loits_batch_plan_create", "loits_batch_forward",
                     "loits_batch_backward"):
        assert required in names


def test_library_exports_every_declared_symbol(native):
    lib = native.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), f"{name} declared in the header but not exported"
    # and the Python binding covers every declared entry point
    assert set(declared_symbols()) <= set(native.SIGNATURES)


def test_bindings_match_header_arity(native):
    """Every ctypes binding passes as many arguments as the header declares."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    seen = 0
    for m in re.finditer(r"\b(loits_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
        name, args = m.group(1), m.group(2).strip()
        n = 0 if args in ("", "void") else len(args.split(","))
        assert len(native.SIGNATURES[name][1]) == n, name
        seen += 1
    assert seen == len(declared_symbols())


def test_status_strings(native):
    lib = native.lib()
    assert lib.loits_status_string(0) == b"ok"
    assert lib.loits_status_string(4).decode().startswith("a bounded device-side wait")
    assert lib.loits_version() >= 100


def _plan(native, koff, counts, cfg=None):
    koff = np.asarray(koff, dtype=np.int64)
    counts = np.asarray(counts, dtype=np.int64)
    h = C.c_void_p()
    rc = native.lib().loits_batch_plan_create(len(counts), koff.ctypes.data, counts.ctypes.data,
                                              C.byref(cfg) if cfg is not None else None,
                                              C.byref(h))
    return rc, h


def test_batch_plan_rejects_bad_tables_on_host(native):
    # a density with fewer than two knots
    rc, h = _plan(native, [0, 1, 5], [10, 10])
    assert rc == native.LOITS_ERR_INVALID and not h.value
    # negative event count
    rc, _ = _plan(native, [0, 3, 5], [10, -1])
    assert rc == native.LOITS_ERR_INVALID
    # offsets not starting at zero
    rc, _ = _plan(native, [1, 3, 5], [1, 1])
    assert rc == native.LOITS_ERR_INVALID
    # more knots than the sampler indexes (2^28 per density)
    rc, _ = _plan(native, [0, 2**28 + 1], [5])
    assert rc == native.LOITS_ERR_UNSUPPORTED
    # slot stride smaller than the largest event count
    cfg = native.BatchConfig(slot_stride=3)
    rc, _ = _plan(native, [0, 3, 5], [10, 2], cfg)
    assert rc == native.LOITS_ERR_INVALID
    # unsupported launch geometry
    cfg = native.BatchConfig(threads=128)
    rc, _ = _plan(native, [0, 3], [10], cfg)
    assert rc == native.LOITS_ERR_INVALID
    # guide resolution out of range
    cfg = native.BatchConfig(guide_ratio=7)
    rc, _ = _plan(native, [0, 3], [10], cfg)
    assert rc == native.LOITS_ERR_INVALID


def test_entry_points_reject_bad_arguments_on_host(native):
    lib = native.lib()
    assert lib.loits_fill_uniform(None, -1, 0, 0, None) == native.LOITS_ERR_INVALID
    assert lib.loits_fill_uniform(None, 5, 0, 0, None) == native.LOITS_ERR_INVALID
    assert lib.loits_fill_uniform(None, 0, 0, 0, None) == native.LOITS_OK  # nothing to do
    bad = native.Shape(1, 2, 2, 1, 5)  # kx < 2
    assert lib.loits_tuple_prepare(C.byref(bad), *([None] * 6), 10, *([None] * 7), None) == \
        native.LOITS_ERR_INVALID
    big = native.Shape(1, 2, 2, 40000, 5)  # int16 intervals cannot index 40000 knots
    assert lib.loits_tuple_prepare(C.byref(big), *([None] * 6), 10, *([None] * 7), None) == \
        native.LOITS_ERR_UNSUPPORTED
    assert lib.loits_batch_forward(None, None, None, None, 0, 0, None, None, None, None, None) == \
        native.LOITS_ERR_INVALID
    # saved-state entry points: a missing plan or buffer is rejected before any launch
    assert lib.loits_batch_forward_state(None, None, None, None, 0, 0, None, None, None, None,
                                         None, None) == native.LOITS_ERR_INVALID
    assert lib.loits_batch_backward_state(None, None, None, None, None, None, None, None, None,
                                          None) == native.LOITS_ERR_INVALID
    assert lib.loits_tuple_sample_workspace(0) >= 16


def test_product_path_has_no_cpu_fallback(native):
    """Without a CUDA device the sampler refuses to run instead of falling back."""
    import torch

    from quantom_loits_b200 import backend
    from quantom_loits_b200.loits import LOITS, BackendUnavailableError, backend_status

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    ok, reason = backend_status("cuda", "cpu")
    assert not ok and "CUDA" in reason
    with pytest.raises(BackendUnavailableError):
        LOITS(backend="cuda", device="cpu")
    x = torch.zeros((1, 2, 5), dtype=torch.float64)
    with pytest.raises(RuntimeError):
        backend.tuple_forward(x, torch.zeros((1, 2, 2, 5), dtype=torch.float64), x,
                              torch.zeros((1, 2, 2, 5), dtype=torch.float64),
                              torch.zeros((1, 2, 2), dtype=torch.float64),
                              torch.ones((1, 2, 2), dtype=torch.bool), 10, 0, 0)
