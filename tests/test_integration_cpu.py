"""The binding INTEGRATION.md shows a maintainer of the reference (its
`vh_bind.h` code block) compiles against include/vh.h and the reference's own
NEWEST5 types (maindef.h: cell, GRID, the scenario constants).  Runs where
the reference tree is present; syntax and types only, nothing is linked."""
import os
import re
import shutil
import subprocess

import pytest
from refpath import reference_root  # oracle/ is on sys.path via conftest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = reference_root()

PRELUDE = """#include <cstdio>
#include <cstdlib>
#include <vector>
#include <iostream>
#include <math.h>
#define GEVFM 0.1973
#define PIE 3.141592653589793
using namespace std;
#include "s95p.h"
#include "maindef.h"
"""


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "NEWEST5")) or not shutil.which("g++"),
                    reason="needs the reference tree and g++")
def test_documented_binding_compiles(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = re.search(r"```cpp\n(.*?)```", text, flags=re.S).group(1)
    assert "TVDRK2" in block and "vh_step" in block
    src = tmp_path / "bind.cpp"
    src.write_text(PRELUDE + block)
    shim = os.path.join(ROOT, "oracle", "ref_shim")
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-w", "-DKT", "-DZCMA=10", "-DZCM=16", "-I", shim, "-include",
           os.path.join(shim, "mpi.h"), "-iquote", os.path.join(REF, "NEWEST5"), "-I", os.path.join(ROOT, "include"),
           str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
