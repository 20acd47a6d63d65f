"""FP32-mixed precision path against the FP64 oracle.

In a CANARD_FP32_MIXED context the derivative and filter eliminations, the
flux components, the viscous stresses and the GCBC run in FP32 with FMA, while
the conserved state, the RK update, the metric and Jacobian masters, the
primitive computation and the LU factorisation stay FP64. The tolerance of the
specification is a relative L2 error <= 1e-5 against the FP64 oracle, per
conserved variable. A momentum component can be zero by symmetry (rho*w of a
Taylor-Green vortex) or a small perturbation riding on a frame velocity, and
then has no meaningful relative error of its own; momentum components are
therefore measured against the momentum scale ||rho|| * U_ref (U_ref = the
flow's velocity scale) whenever that exceeds their own norm. Unit operations
are checked at the FP32 rounding level they can reach.
"""
import numpy as np
import pytest

import pyoracle as po
from canard_b200 import api, cases

pytestmark = pytest.mark.gpu

TOL_STEPS = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def state_errors(qg, qo, uref):
    """Relative L2 error per conserved variable (see the module docstring)."""
    rho = np.linalg.norm(qo[0].ravel())
    out = []
    for v in range(5):
        den = np.linalg.norm(qo[v].ravel())
        if 1 <= v <= 3:
            den = max(den, rho * uref)
        out.append(float(np.linalg.norm((qg[v] - qo[v]).ravel()) / den))
    return out


def case_nonperiodic():
    blk = cases.BlockSpec(23, 18, 16, [[10, 10], [10, 10], [45, 45]], [[-1, -1], [-1, -1], [0, 0]])
    Z, Y, X = blk.shape
    x = np.linspace(-1, 1, X)
    y = np.linspace(-0.8, 0.9, Y)
    z = np.linspace(0, 1, Z)
    Zz, Yy, Xx = np.meshgrid(z, y, x, indexing="ij")
    xyz = np.stack([Xx + 0.02 * np.sin(3 * Yy), Yy + 0.03 * np.sin(2 * Xx), Zz])
    rho, u, v, w, p = cases.vortex_state(Xx, Yy, 0.3, 3.0, 0.3)
    return cases.CaseSpec([blk], viscous=1, reoo=2000.0, xyz=[xyz], qa=[cases._conserved(rho, u, v, w, p)],
                          name="np")


CASES = {
    "periodic": lambda: cases.tgv(nx=24, ny=20, nz=16),
    "nonperiodic": case_nonperiodic,
    "multiblock": lambda: cases.curvilinear_4block(24, 16, 14),
    "toy": lambda: cases.reference_toy(16, 14, 12),
}
UREF = {"periodic": 0.1, "nonperiodic": 0.3, "multiblock": 0.4, "toy": 0.3}


def smooth_fields(cs, seed):
    """Resolved test fields: a few low modes plus 1e-3 noise."""
    rng = np.random.default_rng(seed)
    out = []
    for b in cs.blocks:
        Z, Y, X = b.shape
        k, j, i = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
        f = (np.sin(2 * np.pi * i / (X - 1)) * np.cos(2 * np.pi * j / (Y - 1)) + 0.5 * np.sin(4 * np.pi * k / (Z - 1))
             + 1.0 + 1e-3 * rng.standard_normal(b.shape))
        out.append(f.ravel())
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_unit_deriv_fp32(name):
    cs = CASES[name]()
    o = po.Oracle(cs, setup=False)
    g = api.Context(cs, precision=api.FP32_MIXED, setup=False, upload_state=False)
    f = smooth_fields(cs, 3)
    o.mpigo([x.copy() for x in f], 0, 1, 0, 1, 1)
    g.mpigo([x.copy() for x in f], 0, 1, 0, 1, 1)
    for b, blk in enumerate(cs.blocks):
        for nn in (1, 2, 3):
            a = np.zeros(blk.npts)
            c = np.zeros(blk.npts)
            o.deriv(b, f[b], a, nn, 1)
            g.deriv(b, f[b], c, nn, 1)
            # FP32 rounding of the input, amplified by the one-sided closures
            # (coefficients up to 9) at non-periodic ends
            assert rel_l2(c, a) <= 5e-5, (name, b, nn, rel_l2(c, a))


@pytest.mark.parametrize("name", list(CASES))
def test_unit_filter_fp32(name):
    cs = CASES[name]()
    o = po.Oracle(cs, setup=False)
    g = api.Context(cs, precision=api.FP32_MIXED, setup=False, upload_state=False)
    fo = smooth_fields(cs, 5)
    fg = [x.copy() for x in fo]
    for m in (1, 2):
        for inn in (1, 2, 3):
            o.mpigo(fo, 1, 1, 0, 3 * (m - 1) + inn, m)
            g.mpigo(fg, 1, 1, 0, 3 * (m - 1) + inn, m)
            for b in range(len(cs.blocks)):
                o.filte(b, fo[b], inn, m)
                g.filte(b, fg[b], inn, m)
                # the FP64 field carries an FP32 increment: agreement far below FP32 rounding of the field
                assert rel_l2(fg[b], fo[b]) <= 1e-8, (name, m, inn, b, rel_l2(fg[b], fo[b]))


@pytest.mark.parametrize("name", list(CASES))
def test_steps_fp32_mixed_within_1e_5(name):
    cs = CASES[name]()
    o = po.Oracle(cs)
    g = api.Context(cs, precision=api.FP32_MIXED)
    o.step(12)
    g.step(12)
    np.testing.assert_array_equal(g.time()[:2], o.time()[:2])
    for b in range(len(cs.blocks)):
        errs = state_errors(g.state(b), o.state(b), UREF[name])
        print(name, b, ["%.2e" % e for e in errs])
        assert max(errs) <= TOL_STEPS, (name, b, errs)


def test_tgv64_fp32_mixed_ten_steps():
    cs = cases.tgv(64)
    o = po.Oracle(cs)
    g = api.Context(cs, precision=api.FP32_MIXED)
    o.step(10)
    g.step(10)
    errs = state_errors(g.state(0), o.state(0), 0.1)
    print("tgv64", ["%.2e" % e for e in errs])
    assert max(errs) <= TOL_STEPS, errs


def test_fp32_work_fields_are_readable():
    cs = CASES["multiblock"]()
    g = api.Context(cs, precision=api.FP32_MIXED)
    o = po.Oracle(cs)
    g.step(3)
    o.step(3)
    for b in range(len(cs.blocks)):
        de_g = g.field(api.F_DE, b).ravel()
        de_o = o.get(b, po.A_DE)
        assert rel_l2(de_g, de_o) <= 1e-3
        assert np.isfinite(g.field(api.F_DRVA[0], b)).all()


def test_autotuned_fp32_within_1e_5():
    cs = CASES["multiblock"]()
    g = api.Context(cs, precision=api.FP32_MIXED)
    rep = g.autotune(reps=2)
    assert len(rep) == 9
    o = po.Oracle(cs)
    g.step(12)
    o.step(12)
    for b in range(len(cs.blocks)):
        errs = state_errors(g.state(b), o.state(b), UREF["multiblock"])
        assert max(errs) <= TOL_STEPS, (b, errs, rep)


def test_face_only_stage_state_on_a_large_block():
    """On blocks whose faces hold under 5 % of the points (here 129^3) the
    FP32-mixed RK stages 1-3 store the FP64 stage state only on the block
    faces; 10 steps stay within the mixed-precision tolerance of FP64."""
    cs = cases.tgv(128)
    a = api.Context(cs)
    g = api.Context(cs, precision=api.FP32_MIXED)
    a.step(10)
    g.step(10)
    errs = state_errors(g.state(0), a.state(0), 0.1)
    assert max(errs) <= TOL_STEPS, errs


@pytest.mark.parametrize("name", list(CASES))
def test_streamed_filter_steps_within_1e_5(name):
    """The filter kind that streams the FP64 state into FP32 right-hand sides
    (k_filt2s), pinned on every direction: 12 steps within the tolerance."""
    cs = CASES[name]()
    o = po.Oracle(cs)
    g = api.Context(cs, precision=api.FP32_MIXED)
    for d in ("xi", "eta", "zeta"):
        g.set_line_kind("filter", d, "fp64-stream/fp32-split")
    o.step(12)
    g.step(12)
    for b in range(len(cs.blocks)):
        errs = state_errors(g.state(b), o.state(b), UREF[name])
        print(name, b, ["%.2e" % e for e in errs])
        assert max(errs) <= TOL_STEPS, (name, b, errs)


@pytest.mark.parametrize("nn", [1, 2, 3])
@pytest.mark.parametrize("name", ["periodic", "nonperiodic"])
def test_streamed_filter_unit(name, nn):
    """One filter pass of 5 smooth fields through canard_line_bench with the
    streamed kind, against the oracle's filte: the FP64 field carries an FP32
    increment, so the agreement is far below FP32 rounding of the field."""
    cs = CASES[name]()
    blk = cs.blocks[0]
    fields = np.stack([f.reshape(blk.shape) for f in (smooth_fields(cs, 11 + k)[0] for k in range(5))])
    g = api.Context(cs, precision=api.FP32_MIXED, setup=False, upload_state=False)
    g.set_line_kind("filter", "xi eta zeta".split()[nn - 1], "fp64-stream/fp32-split")
    out, ms = g.line_bench(1, nn, fields, reps=2)
    o = po.Oracle(cs, setup=False)
    inn = {2: 1, 3: 2, 1: 3}[nn]
    for k in range(5):
        f = fields[k].ravel().copy()
        o.mpigo([f], 1, 1, 0, k + 1, k + 1)
        o.filte(0, f, inn, k + 1)
        assert rel_l2(out[k].ravel(), f) <= 1e-8, (k, rel_l2(out[k].ravel(), f))
