import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libvh.so")
    config.addinivalue_line("markers", "late: runs after every other test, so that a failure there (under -x) "
                                       "leaves the rest already run; for GPU paths not yet run on hardware")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    src = os.path.join(ROOT, "oracle", "oracle.c")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       capture_output=True)


def _ensure_libvh():
    from viral_b200 import build
    build.build()


@pytest.fixture(scope="session", autouse=True)
def built_libs():
    _ensure_oracle()
    _ensure_libvh()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    # stable: file order otherwise; the allocation-free step's file runs after everything, late tests included
    items.sort(key=lambda it: 2 if os.path.basename(str(it.fspath)).startswith("test_zz_")
               else (1 if "late" in it.keywords else 0))
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def rel_err(a, b):
    """max |a-b| / max |b| (0 when both vanish)."""
    a = np.asarray(a); b = np.asarray(b)
    den = np.max(np.abs(b))
    num = np.max(np.abs(a - b))
    return 0.0 if num == 0 else num / (den if den > 0 else 1.0)
