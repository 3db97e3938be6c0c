import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O

    O.build(ref=False)
    return O.Oracle()


def golden_case(golden, name):
    """Dict view of one golden case (keys without the ``name/`` prefix)."""
    pre = name + "/"
    return {k[len(pre):]: golden[k] for k in golden.files if k.startswith(pre)}


TUPLE_CASES = ["theory3_k5", "theory3_k5_seed0", "manual", "manual_rejected_cell",
               "theory3_k4_n257", "theory3_k5_n257", "theory3_k7_n257", "theory3_k8_n257",
               "theory3_k10_n257", "theory3_k16_n257", "theory3_k32_n257", "theory10_k10",
               "theory6_k5_batch2"]
DENSITY_CASES = ["ragged_small", "uniform_small", "ragged_workload_small"]


def have_cuda() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False
