"""The derivative entry point that allocates no device memory.

Some callers cannot allocate device memory on their step path: solvers that
own every device buffer themselves, code under a memory budget that forbids
allocator calls between steps, host threads that must not block in the
allocator. canard_deriv_noalloc serves them: the caller passes device input
and output, and the scratch lives in a fixed static device array. These tests
call it through the C ABI twice in a row, with different inputs, and check
each result against the context entry points canard_mpigo + canard_deriv and
against the oracle (bit for bit, the tolerance of the other derivative
tests), at small sizes and at the longest lines the FP64 tile holds with the
output written over the input; canard_deriv_noalloc_status reports no failed
wait after each call. They live in their own file so that pytest collects
them last.
"""
import ctypes

import numpy as np
import pytest

import pyoracle as po
from canard_b200 import api, cases

pytestmark = pytest.mark.gpu


def _block(periodic):
    bc = 45 if periodic else 10
    nb = 0 if periodic else -1
    return cases.BlockSpec(24, 20, 16, [[bc, bc]] * 3, [[nb, nb]] * 3)


def _reference(blk, f, nn):
    cs = cases.CaseSpec([blk])
    ctx = api.Context(cs, setup=False, upload_state=False)
    ctx.mpigo([f.copy()], 0, 1, 0, 1, 1)
    out = np.zeros_like(f)
    ctx.deriv(0, f, out, nn, 1)
    ctx.close()
    return out.reshape(blk.shape)


def _oracle(blk, f, nn):
    o = po.Oracle(cases.CaseSpec([blk]), setup=False)
    o.mpigo([f.copy()], 0, 1, 0, 1, 1)
    out = np.zeros_like(f)
    o.deriv(0, f, out, nn, 1)
    return out.reshape(blk.shape)


def _call(d_in, d_out, blk, pitch, nn, bc, stream):
    return api.lib().canard_deriv_noalloc(
        ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()), blk.lxi, blk.let, blk.lze,
        pitch, nn, bc, bc, 0.85, 0.85, ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("nn", [1, 2, 3])
def test_noalloc_derivative_matches_context_path(periodic, nn):
    import torch

    blk = _block(periodic)
    Z, Y, X = blk.shape
    pitch = (X + 3) // 4 * 4
    rng = np.random.default_rng(100 + nn)
    stream = torch.cuda.current_stream()
    bc = 45 if periodic else 10
    for call in range(2):
        f = rng.standard_normal(blk.npts)
        ref = _reference(blk, f, nn)
        d_in = torch.zeros((Z, Y, pitch), dtype=torch.float64, device="cuda")
        d_out = torch.zeros((Z, Y, pitch), dtype=torch.float64, device="cuda")
        d_in[:, :, :X] = torch.from_numpy(f.reshape(blk.shape)).cuda()
        torch.cuda.synchronize()
        rc = api.lib().canard_deriv_noalloc(
            ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()), blk.lxi, blk.let, blk.lze,
            pitch, nn, bc, bc, 0.85, 0.85, ctypes.c_void_p(stream.cuda_stream))
        assert rc == api.OK, f"call {call}: rc {rc}"
        assert api.lib().canard_deriv_noalloc_status(ctypes.c_void_p(stream.cuda_stream)) == api.OK
        got = d_out[:, :, :X].cpu().numpy()
        np.testing.assert_array_equal(got, ref, err_msg=f"call {call}, nn={nn}, periodic={periodic}")
        if call == 0:  # the context path above is itself pinned to the oracle; check once directly
            np.testing.assert_array_equal(got, _oracle(blk, f, nn))


@pytest.mark.parametrize("nn,dims", [(1, (905, 12, 12)), (2, (12, 895, 12)), (3, (12, 12, 895))])
def test_noalloc_longest_lines_in_place(nn, dims):
    """Lines of the longest length the FP64 tile holds (906 points along xi, 896
    along eta or zeta), with the output written over the input, two calls in a
    row, against the oracle."""
    import torch

    blk = cases.BlockSpec(*dims, [[10, 10]] * 3, [[-1, -1]] * 3)
    Z, Y, X = blk.shape
    pitch = (X + 3) // 4 * 4
    rng = np.random.default_rng(7 + nn)
    stream = torch.cuda.current_stream()
    for call in range(2):
        f = rng.standard_normal(blk.npts)
        d = torch.zeros((Z, Y, pitch), dtype=torch.float64, device="cuda")
        d[:, :, :X] = torch.from_numpy(f.reshape(blk.shape)).cuda()
        torch.cuda.synchronize()
        assert _call(d, d, blk, pitch, nn, 10, stream) == api.OK
        assert api.lib().canard_deriv_noalloc_status(ctypes.c_void_p(stream.cuda_stream)) == api.OK
        np.testing.assert_array_equal(d[:, :, :X].cpu().numpy(), _oracle(blk, f, nn), err_msg=f"call {call}")


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(d.data_ptr())
    lib = api.lib()
    # 907 points along xi, 897 along eta: one more than the FP64 tile holds
    assert lib.canard_deriv_noalloc(p, p, 906, 12, 12, 908, 1, 10, 10, 0.85, 0.85, None) == api.ERR_ARG
    assert lib.canard_deriv_noalloc(p, p, 12, 896, 12, 16, 2, 10, 10, 0.85, 0.85, None) == api.ERR_ARG
    # pitch not a multiple of 4
    assert lib.canard_deriv_noalloc(p, p, 24, 20, 16, 26, 1, 10, 10, 0.85, 0.85, None) == api.ERR_ARG
    # periodic at one end only
    assert lib.canard_deriv_noalloc(p, p, 24, 20, 16, 28, 1, 45, 10, 0.85, 0.85, None) == api.ERR_UNSUPPORTED
