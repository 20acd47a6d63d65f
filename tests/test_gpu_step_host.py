"""canard_step_host: steps through host memory with pipelined copies, against
the same steps as set_state + step + get_state per step, bit for bit (the copies
move the same values; only their scheduling differs)."""
import numpy as np
import pytest
import torch

from canard_b200 import api, cases

pytestmark = pytest.mark.gpu


def pinned_states(cs):
    out = []
    for b, blk in enumerate(cs.blocks):
        t = torch.empty((5,) + blk.shape, dtype=torch.float64, pin_memory=True)
        t.copy_(torch.from_numpy(np.ascontiguousarray(cs.qa[b])))
        out.append(t)
    return out


@pytest.mark.parametrize("prec", [api.FP64, api.FP64_FAST, api.FP32_MIXED])
def test_step_host_equals_set_step_get(prec):
    cs = cases.curvilinear_4block(24, 16, 14)
    a = api.Context(cs, precision=prec)
    b = api.Context(cs, precision=prec)
    ha = [t.numpy() for t in pinned_states(cs)]
    hb_t = pinned_states(cs)
    hb = [t.numpy() for t in hb_t]
    for _ in range(3):
        for k in range(len(cs.blocks)):
            a.set_state(k, ha[k])
        a.step(1)
        for k in range(len(cs.blocks)):
            a.get_state_into(k, ha[k])
    b.step_host(3, hb)
    for k in range(len(cs.blocks)):
        np.testing.assert_array_equal(hb[k], ha[k], err_msg=f"block {k}")
        np.testing.assert_array_equal(b.state(k), a.state(k), err_msg=f"device state of block {k}")


def test_step_host_subset_of_blocks_and_host_edits_between_calls():
    """Two of four blocks through host memory; an edit of a host array between
    two calls reaches the device (the next call reads the array again)."""
    cs = cases.curvilinear_4block(24, 16, 14)
    a = api.Context(cs)
    b = api.Context(cs)
    hb = [t.numpy() for t in pinned_states(cs)][1:3]
    b.step_host(2, hb, [(0, 1), (0, 2)])
    for k in (1, 2):
        a.set_state(k, np.ascontiguousarray(cs.qa[k]))
    a.step(1)
    a.step(1)
    np.testing.assert_array_equal(hb[0], a.state(1))
    np.testing.assert_array_equal(hb[1], a.state(2))
    hb[0][0] *= 1.0 + 1e-3
    a.set_state(1, hb[0])
    b.step_host(1, hb, [(0, 1), (0, 2)])
    a.step(1)
    np.testing.assert_array_equal(hb[0], a.state(1))
    np.testing.assert_array_equal(hb[1], a.state(2))


def test_step_host_rejects_bad_arguments():
    cs = cases.tgv(16)
    g = api.Context(cs)
    h = [np.ascontiguousarray(cs.qa[0])]
    with pytest.raises(api.CanardError):
        g.step_host(1, h + h, [(0, 0), (0, 0)])
    with pytest.raises(api.CanardError):
        g.step_host(1, h, [(0, 1)])
