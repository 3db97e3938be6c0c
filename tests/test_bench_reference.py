"""The CPU reference legs of bench.py (the reference arm and the
cpu_baseline field): one method for both, a bounded sample of the workload
refined toward the requested seconds, the reference's own openmp core on the
exact embedding.  CPU only (the reference core is compiled from the reference
tree into oracle/_ref/; skipped where that tree was absent at build time)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def _reference_built():
    return (ROOT / "oracle" / "_ref" / "libloits_ref_openmp.so").exists()


@pytest.mark.skipif(not _reference_built(), reason="reference core not built")
def test_reference_timing_takes_a_bounded_sample():
    import bench
    from quantom_loits_b200 import workloads

    spec = workloads.ragged(scale=2e-3, n_densities=24)
    value, n_dens, events, seconds = bench.reference_timing(spec, 0.05, 1, 2)
    assert 1 <= n_dens <= spec.n_densities
    assert events == int(np.asarray(spec.event_counts)[:n_dens].sum())
    assert value > 0 and seconds > 0
    assert abs(value - events / seconds) <= 1e-6 * value


@pytest.mark.skipif(not _reference_built(), reason="reference core not built")
def test_reference_arm_line_keeps_the_contract():
    import argparse

    import bench

    spec = bench.workload_spec("single", 0)
    args = argparse.Namespace(ref_seconds=0.05, steps=2, warmup=3, gpus=1)
    out = bench.run_reference(args, spec)
    assert out["impl"] == "reference" and out["unit"] == "events/s"
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["e2e"]["d2h_bytes_per_step"] == 0
    assert out["cpu_baseline"]["kind"] == "reference" and out["cpu_baseline"]["value"] == out["value"]
    assert out["value"] > 0 and out["higher_is_better"] is True
