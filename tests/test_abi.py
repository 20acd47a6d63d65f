"""CPU checks of the C ABI: the library loads, exports every declared entry
point, its host-side coefficient tables equal the oracle's, and it fails with
an error code (not a crash) where no GPU is present."""
import ctypes
import os
import re

import numpy as np
import pytest

import pyoracle as po
from canard_b200 import api, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(canard_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(api.LIBPATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


@pytest.mark.parametrize("fltk,fltrbc", [(0.85, 0.85), (0.65, 0.9), (0.5, 0.7)])
def test_coefficients_equal_oracle(fltk, fltrbc):
    np.testing.assert_array_equal(api.coeffs(fltk, fltrbc), po.coeffs(fltk, fltrbc))


@pytest.mark.parametrize("n", [13, 24, 65, 257])
def test_lu_factors_equal_oracle(n):
    for nt in (0, 1):
        for ns in (0, 1):
            for ne in (0, 1):
                u1, l1 = api.penta(0.85, 0.85, n, ns, ne, nt)
                u2, l2 = po.penta(0.85, 0.85, n, ns, ne, nt)
                np.testing.assert_array_equal(u1, u2)
                np.testing.assert_array_equal(l1, l2)


def test_argument_errors_are_codes():
    assert api.lib().canard_coeffs(0.85, -1.0, None) == api.ERR_ARG
    out = np.zeros(10)
    assert api.lib().canard_penta(0.85, 0.85, 4, 0, 0, 0, api._dp(out), api._dp(out)) == api.ERR_ARG
    h = ctypes.c_void_p()
    assert api.lib().canard_ctx_create(None, 0, None, 0, ctypes.byref(h)) == api.ERR_ARG


def test_context_without_gpu_reports_an_error():
    try:
        ctx = api.Context(cases.tgv(16), setup=False, upload_state=False)
    except api.CanardError as e:
        assert e.code in (api.ERR_CUDA, api.ERR_ARG)
        return
    ctx.close()
    pytest.skip("a GPU is present")


def test_unsupported_configurations_are_rejected_before_device_work():
    # boundary codes the reference does not have; precisions other than FP64
    # and FP32-mixed do not exist
    blk = cases.BlockSpec(16, 16, 16, [[50, 10], [10, 10], [45, 45]], [[0, -1], [-1, -1], [0, 0]])
    cs = cases.CaseSpec([blk])
    h = ctypes.c_void_p()
    c, b = api._structs([cs])
    for prec in (api.FP64, api.FP32_MIXED):
        rc = api.lib().canard_ctx_create(c, 1, b, prec, ctypes.byref(h))
        assert rc in (api.ERR_ARG, api.ERR_CUDA)
    c, b = api._structs([cases.tgv(16)])
    assert api.lib().canard_ctx_create(c, 1, b, 7, ctypes.byref(h)) == api.ERR_UNSUPPORTED


def test_noalloc_rejects_lines_beyond_the_tile_before_any_work():
    # the FP64 line tile holds at most 906 points along xi and 896 along eta or
    # zeta; longer lines are refused by the argument checks, before any device
    # call (the pointers are never touched)
    lib = api.lib()
    p = ctypes.c_void_p(256)
    assert lib.canard_deriv_noalloc(p, p, 906, 12, 12, 908, 1, 10, 10, 0.85, 0.85, None) == api.ERR_ARG
    assert lib.canard_deriv_noalloc(p, p, 12, 896, 12, 16, 2, 10, 10, 0.85, 0.85, None) == api.ERR_ARG
    assert lib.canard_deriv_noalloc(p, p, 12, 12, 896, 16, 3, 10, 10, 0.85, 0.85, None) == api.ERR_ARG


@pytest.mark.parametrize("prec", [0, 1])
def test_context_rejects_lines_longer_than_the_tile(prec):
    # FP64 tiles hold 906 points along xi and 896 along eta/zeta; the mixed
    # precision's tiles are half as wide and take longer lines
    h = ctypes.c_void_p()
    for dims in ((906, 12, 12), (12, 896, 12), (12, 12, 896)) if prec == 0 else ((1900, 12, 12),):
        blk = cases.BlockSpec(*dims, [[10, 10]] * 3, [[-1, -1]] * 3)
        c, b = api._structs([cases.CaseSpec([blk])])
        assert api.lib().canard_ctx_create(c, 1, b, prec, ctypes.byref(h)) == api.ERR_UNSUPPORTED, dims
