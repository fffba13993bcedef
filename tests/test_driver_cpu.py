"""The C++ host driver (viral_b200/vh_run) on the CPU: it builds, parses its
options, and without a GPU stops with the library's error (no CPU path)."""
import os
import subprocess

import pytest

from viral_b200 import build


@pytest.fixture(scope="module")
def driver():
    return build.build_driver()


def test_help_and_bad_options(driver):
    r = subprocess.run([driver, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "--scenario" in r.stdout
    r = subprocess.run([driver, "--scenario", "shock"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "unknown scenario" in r.stderr
    r = subprocess.run([driver, "--precision", "fp16"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2


def test_without_a_gpu_the_driver_reports_the_library_error(driver):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    r = subprocess.run([driver, "--scenario", "gubser", "--nx", "9", "--ny", "9", "--steps", "1", "--quiet"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "vh_create" in r.stderr
