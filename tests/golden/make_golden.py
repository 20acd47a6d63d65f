"""Regenerates the oracle regression fixtures in this folder.

The reference ships no golden data and cannot be compiled here, so these
fixtures freeze the oracle's own output on two small cases; they detect any
later drift of the oracle (tests/test_oracle_kat.py::test_golden_fixtures).
Run: python tests/golden/make_golden.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

import pyoracle as po  # noqa: E402
from golden_cases import golden_case  # noqa: E402

for name in ("tgv16_step3", "curv4_step2"):
    cs, n = golden_case(name)
    o = po.Oracle(cs)
    o.step(n)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **{f"qa{b}": o.state(b) for b in range(len(cs.blocks))})
    print(name, "written")
