"""Where the reference's source tree lies, for the recipes and tests that
compile or read it (the checker's side only; nothing on the product path).

$VH_REFERENCE when set, else the default of the `REF ?=` line of
oracle/Makefile, the recipe that compiles the reference's headers."""
from __future__ import annotations

import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root() -> str:
    env = os.environ.get("VH_REFERENCE")
    if env:
        return env
    try:
        with open(os.path.join(_HERE, "Makefile")) as fh:
            for line in fh:
                m = re.match(r"\s*REF\s*\?=\s*(\S+)", line)
                if m:
                    return m.group(1)
    except OSError:
        pass
    return ""
