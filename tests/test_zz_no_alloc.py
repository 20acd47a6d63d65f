"""The derivative entry point that allocates no device memory.

Some callers cannot allocate device memory on their step path: solvers that
own every device buffer themselves, code under a memory budget that forbids
allocator calls between steps, host threads that must not block in the
allocator. canard_deriv_noalloc serves them: the caller passes device input
and output, and the scratch lives in a fixed static device array. This test
calls it through the C ABI twice in a row, with different inputs, and checks
each result against the context entry points canard_mpigo + canard_deriv
(bit for bit, the tolerance of the other derivative tests). It lives in its
own file so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

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
        stream.synchronize()
        got = d_out[:, :, :X].cpu().numpy()
        np.testing.assert_array_equal(got, ref, err_msg=f"call {call}, nn={nn}, periodic={periodic}")


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(d.data_ptr())
    lib = api.lib()
    # 1025 points per line: beyond the 1024-point limit
    assert lib.canard_deriv_noalloc(p, p, 1024, 12, 12, 1028, 1, 10, 10, 0.85, 0.85, None) == api.ERR_ARG
    # pitch not a multiple of 4
    assert lib.canard_deriv_noalloc(p, p, 24, 20, 16, 26, 1, 10, 10, 0.85, 0.85, None) == api.ERR_ARG
    # periodic at one end only
    assert lib.canard_deriv_noalloc(p, p, 24, 20, 16, 28, 1, 45, 10, 0.85, 0.85, None) == api.ERR_UNSUPPORTED
