"""Sub-domains (the reference's nbpc > 1) on the device against the oracle's
split runs: phases bit for bit and 12 steps within 1e-10. The device's
averaging plans for these splits already equal the oracle's on the CPU
(tests/test_subdomains.py); these runs add the interface contractions across
code-40 faces and the GCBC faces of split blocks on the device."""
import numpy as np
import pytest

import pyoracle as po
from canard_b200 import api, cases

pytestmark = pytest.mark.gpu

SPLITS = {
    "tgv_box": (lambda: cases.tgv(nx=48, ny=40, nz=32), [(2, 2, 2)]),
    "validation": (lambda: cases.reference_validation(48, 40, 12), [(2, 2, 1)]),
    "toy": (lambda: cases.reference_toy(52, 26, 12), [(4, 2, 1)] * 6),
}


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.parametrize("name", list(SPLITS))
def test_split_phases_bit_exact(name):
    make, nbpc = SPLITS[name]
    cs = cases.decompose(make(), nbpc)
    o = po.Oracle(cs)
    g = api.Context(cs)
    for r in range(len(cs.blocks)):
        for fo, fg in ((po.A_XIM, api.F_XIM), (po.A_YACO, api.F_YACO)):
            np.testing.assert_array_equal(g.field(fg, r).ravel(), o.get(r, fo))
    o.phase(po.PH_FILTER)
    g.phase(api.PH_FILTER)
    for r in range(len(cs.blocks)):
        np.testing.assert_array_equal(g.field(api.F_QA, r).ravel(), o.get(r, po.A_QA))


@pytest.mark.parametrize("name", list(SPLITS))
def test_split_steps_match_the_oracle(name):
    make, nbpc = SPLITS[name]
    cs = cases.decompose(make(), nbpc)
    o = po.Oracle(cs)
    g = api.Context(cs)
    o.step(12)
    g.step(12)
    for r in range(len(cs.blocks)):
        assert rel_l2(g.state(r), o.state(r)) <= 1e-10, r
