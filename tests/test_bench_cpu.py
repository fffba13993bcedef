"""The bench's CPU legs that need no GPU: the reference's own step timed on
the host cores on windows of the benchmarked states (3+1D and
boost-invariant table-EOS builds), the ensemble's events/s extrapolated from
it, and the error norms of the mixed-precision record."""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


@pytest.mark.skipif(not all(os.path.exists(os.path.join(REF, f"libref_{v}.so")) for v in ("window_3d", "window_lbi")),
                    reason="the reference's CPU builds are absent (oracle/Makefile)")
def test_reference_rates_and_ensemble_extrapolation(monkeypatch):
    import bench
    monkeypatch.setattr(bench, "reference_procs", lambda: 2)
    rates, procs, desc = bench.reference_windows("glauber_161x161x41", 0.5, 2, 2)
    assert procs == 2 and len(rates) == 2 and all(r > 0 for r in rates)
    assert "36 windows of 30x30x41" in desc
    out = bench.ensemble_cpu_baseline(0.3, 1.0e9, 100)
    assert out["unit"] == "events/s" and out["kind"] == "reference" and out["cores"] == 2
    assert out["value"] == pytest.approx(100 * out["cell_updates_per_s"] / 1.0e9)
    assert bench.ensemble_cpu_baseline(0.0, 1.0e9, 100) is None


def test_state_errors_norms():
    import bench
    rng = np.random.default_rng(0)
    b = rng.normal(size=(18, 50))
    a = b.copy()
    a[0] += 1e-3
    m = np.ones(50, bool)
    m[:5] = False
    e = bench.state_errors(a, b, m)
    assert e["e"]["max_rel"] == pytest.approx(1e-3 / np.max(np.abs(b[0, m])))
    assert e["e"]["l2_rel"] == pytest.approx(1e-3 * np.sqrt(45) / np.linalg.norm(b[0, m]))
    assert e["u"]["max_rel"] == 0 and e["pi"]["l2_rel"] == 0


def test_both_arms_print_the_same_config():
    import bench
    assert bench.line_config("glauber_161x161x41", "fp64", 1) == bench.line_config("glauber_161x161x41", "fp64", 1)
    c = bench.line_config("glauber_161x161x41", "fp64", 1)
    assert c["workload"] == "glauber_161x161x41" and c["interior_cells"] == 161 * 161 * 41


def test_every_name_bench_uses_is_defined():
    """bench.py's GPU paths cannot run here; at least every name they load is
    defined somewhere in the module (a function, an import, an assignment, an
    argument) or is a builtin"""
    import ast
    import builtins
    with open(os.path.join(ROOT, "bench.py")) as fh:
        tree = ast.parse(fh.read())
    defined = set(dir(builtins)) | {"__file__"}
    for n in ast.walk(tree):
        if isinstance(n, (ast.FunctionDef, ast.ClassDef)):
            defined.add(n.name)
        elif isinstance(n, ast.Import):
            defined.update(a.asname or a.name.split(".")[0] for a in n.names)
        elif isinstance(n, ast.ImportFrom):
            defined.update(a.asname or a.name for a in n.names)
        elif isinstance(n, ast.Name) and isinstance(n.ctx, (ast.Store, ast.Del)):
            defined.add(n.id)
        elif isinstance(n, ast.arg):
            defined.add(n.arg)
        elif isinstance(n, ast.ExceptHandler) and n.name:
            defined.add(n.name)
    used = {n.id for n in ast.walk(tree) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load)}
    assert not used - defined, sorted(used - defined)
