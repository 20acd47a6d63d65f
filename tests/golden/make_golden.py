"""Regenerates the oracle regression fixtures in this folder.

The reference ships no golden data and cannot be compiled here, so these
fixtures freeze the oracle's own output: the states of two small cases, and
SHA-256 digests of the states after 1, 10 and 100 steps of a small TGV, of the
curvilinear and toy layouts, and of two split (sub-domain) layouts. They
detect any later drift of the oracle (tests/test_oracle_kat.py).
Run: python tests/golden/make_golden.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import hashlib  # noqa: E402
import json  # noqa: E402

import numpy as np  # noqa: E402

import pyoracle as po  # noqa: E402
from golden_cases import DIGEST_CASES, golden_case  # noqa: E402


def digests(name):
    """SHA-256 of each block's (rank's) FP64 state after the case's steps."""
    cs, n = golden_case(name)
    o = po.Oracle(cs)
    o.step(n)
    return [hashlib.sha256(np.ascontiguousarray(o.state(b), np.float64).tobytes()).hexdigest()
            for b in range(len(cs.blocks))]


if __name__ == "__main__":
    for name in ("tgv16_step3", "curv4_step2"):
        cs, n = golden_case(name)
        o = po.Oracle(cs)
        o.step(n)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **{f"qa{b}": o.state(b) for b in range(len(cs.blocks))})
        print(name, "written")
    out = {name: digests(name) for name in DIGEST_CASES}
    with open(os.path.join(HERE, "digests.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("digests.json written")
