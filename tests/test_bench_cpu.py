"""The bench's CPU legs that need no GPU: the reference's own step timed on
the host cores (3+1D and boost-invariant builds) and the ensemble's
events/s extrapolated from it."""
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


@pytest.mark.skipif(not all(os.path.exists(os.path.join(REF, f"libref_{v}.so")) for v in ("milne_3d", "milne_lbi")),
                    reason="the reference's CPU builds are absent (oracle/Makefile)")
def test_reference_rates_and_ensemble_extrapolation(monkeypatch):
    import bench
    monkeypatch.setattr(bench, "reference_procs", lambda: 2)
    rate3, cores = bench.cpu_reference(0.5, 2)
    assert cores == 2 and rate3 > 0
    out = bench.ensemble_cpu_baseline(0.5, 1.0e9, 100)
    assert out["unit"] == "events/s" and out["kind"] == "reference" and out["cores"] == 2
    assert out["value"] == pytest.approx(100 * out["cell_updates_per_s"] / 1.0e9)
    assert bench.ensemble_cpu_baseline(0.0, 1.0e9, 100) is None
