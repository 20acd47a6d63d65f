"""Known-answer checks that pin the CPU oracle to the scheme's mathematics.

The reference ships no tests or golden vectors, so the oracle is pinned by
properties its formulas must have (src/mo_numerics.f90, src/mo_parameters.f90):

* interior compact derivative of sin(kx) = the 8th-order pentadiagonal
  modified wavenumber w'(w) = (2 aa sin w + 2 ab sin 2w) / (1 + 2 alpha cos w + 2 beta cos 2w);
* interior filter transfer function T(w) = 1 + [2fa(cos w - 1) + 2fb(cos 2w - 1)
  + 2fc(cos 3w - 1)] / (1 + 2 alphf cos w + 2 betf cos 2w), T(pi) = 0 at fltk = pi;
* constants: derivative 0 and filter identity (every closure row sums to 0);
* periodic closures: a periodic line gives the same derivative at its two
  shared end points and reproduces the modified wavenumber everywhere;
* golden fixtures in tests/golden/ (regenerated only by tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

import pyoracle as po
from canard_b200 import cases

ALPHA, BETA, AA, AB = 4 / 9.0, 1 / 36.0, 20 / 27.0, 25 / 216.0


def modified_wavenumber(w):
    return (2 * AA * np.sin(w) + 2 * AB * np.sin(2 * w)) / (1 + 2 * ALPHA * np.cos(w) + 2 * BETA * np.cos(2 * w))


def periodic_block(n=32, nz=16):
    per = [[cases.BC_PERIODIC] * 2] * 3
    return cases.BlockSpec(n, n, nz, [list(p) for p in per], [[0, 0]] * 3)


def nonperiodic_block(n=32, nz=16):
    bc = [[10, 10], [10, 10], [45, 45]]
    return cases.BlockSpec(n, n, nz, bc, [[-1, -1], [-1, -1], [0, 0]])


def make_oracle(blk, viscous=0):
    cs = cases.CaseSpec([blk], viscous=viscous)
    return po.Oracle(cs, setup=False)


def test_coefficient_identities():
    c = po.coeffs(0.85, 0.85)
    pbci = c[:48].reshape(2, 2, 12)
    pbco = c[48:96].reshape(2, 2, 12)
    pbcot = c[96:100].reshape(2, 2)
    alphf, betf, fa, fb, fc = c[100:105]
    # pbcot is the sum of pbco (src/mo_numerics.f90:127-132)
    assert np.allclose(pbcot, pbco.sum(axis=2), rtol=0, atol=1e-14)
    # derivative of a constant across an interface: pbci + pbco rows sum to 0
    assert np.allclose(pbci[0].sum(axis=1) + pbco[0].sum(axis=1), 0.0, atol=1e-12)
    # filter of a constant: closure rows sum to 0
    assert np.allclose(pbci[1].sum(axis=1) + pbco[1].sum(axis=1), 0.0, atol=1e-12)
    # interior filter (fcint, src/mo_numerics.f90:306-326): T(0) = 1,
    # T(pi) = 0 and T(fltk) = 1/2 at the cut-off
    for k in (0.5, 0.85, 0.95):
        a, b, fa1, fb1, fc1 = po.coeffs(k, 0.85)[100:105]

        def T(w):
            return 1 + (2 * fa1 * (np.cos(w) - 1) + 2 * fb1 * (np.cos(2 * w) - 1) + 2 * fc1 * (np.cos(3 * w) - 1)) / (
                1 + 2 * a * np.cos(w) + 2 * b * np.cos(2 * w))
        assert abs(T(0.0) - 1.0) < 1e-15
        assert abs(T(np.pi)) < 1e-11
        assert abs(T(k * np.pi) - 0.5) < 1e-11


def _line(arr, shape, nn, a, b):
    """line along direction nn at the other indices (a, b)"""
    v = arr.reshape(shape)
    if nn == 1:
        return v[b, a, :]
    if nn == 2:
        return v[b, :, a]
    return v[:, b, a]


@pytest.mark.parametrize("nn", [1, 2, 3])
def test_periodic_derivative_modified_wavenumber(nn):
    n = 32
    blk = periodic_block(n, n)
    o = make_oracle(blk)
    shape = blk.shape
    Z, Y, X = shape
    idx = [np.arange(X)[None, None, :], np.arange(Y)[None, :, None], np.arange(Z)[:, None, None]][nn - 1]
    for k in (1, 2, 3):
        w = 2 * np.pi * k / n
        f = np.broadcast_to(np.sin(w * idx), shape).copy().reshape(-1)
        o.mpigo([f.copy()], 0, 1, 0, 1, 1)
        out = np.zeros_like(f)
        o.deriv(0, f, out, nn, 1)
        exact = modified_wavenumber(w) * np.broadcast_to(np.cos(w * idx), shape).reshape(-1)
        err = np.abs(out - exact).reshape(shape)
        # the quasi-disjoint periodic closure (src/mo_numerics.f90:330-425) is a
        # truncated approximation at the shared end points; its error decays
        # geometrically into the line
        assert err.max() < 1e-6 * w, k
        mid = [np.s_[:, :, 14:-14], np.s_[:, 14:-14, :], np.s_[14:-14, :, :]][nn - 1]
        assert err[mid].max() < 1e-9 * w, k


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("nn", [1, 2, 3])
def test_derivative_solves_the_compact_system(nn, periodic):
    """The output satisfies every row of the pentadiagonal system of the
    reference (interior: src/mo_numerics.f90:761-763 with alpha, beta; one-sided
    closures: src/mo_parameters.f90:57-70), to rounding."""
    blk = periodic_block(26, 22) if periodic else nonperiodic_block(26, 22)
    o = make_oracle(blk)
    rng = np.random.default_rng(1)
    f = rng.standard_normal(blk.npts)
    o.mpigo([f.copy()], 0, 1, 0, 1, 1)
    d = np.zeros_like(f)
    o.deriv(0, f, d, nn, 1)
    shape = blk.shape
    for a, b in ((0, 0), (3, 5), (7, 2)):
        fl, dl = _line(f, shape, nn, a, b), _line(d, shape, nn, a, b)
        N = len(fl) - 1
        for i in range(2, N - 1):
            lhs = BETA * dl[i - 2] + ALPHA * dl[i - 1] + dl[i] + ALPHA * dl[i + 1] + (BETA * dl[i + 2] if i + 2 <= N else 0)
            if i + 2 > N:
                continue
            rhs = AA * (fl[i + 1] - fl[i - 1]) + AB * (fl[i + 2] - fl[i - 2])
            assert abs(lhs - rhs) < 1e-12 * (1 + abs(rhs)), (i, lhs, rhs)
        if not periodic and nn in (1, 2):
            a01, a02, a03, a04 = -6.666666667794732, 9.000000000052879, 1.333333333178555, -0.0833333333455545
            al01, be02 = 8.000000000449464, 6.000000000542
            lhs = dl[0] + al01 * dl[1] + be02 * dl[2]
            rhs = a01 * (fl[1] - fl[0]) + a02 * (fl[2] - fl[0]) + a03 * (fl[3] - fl[0]) + a04 * (fl[4] - fl[0])
            assert abs(lhs - rhs) < 1e-11 * (1 + abs(rhs))


@pytest.mark.parametrize("nn", [1, 2])
def test_nonperiodic_derivative_interior_and_accuracy(nn):
    n = 48
    blk = nonperiodic_block(n, 16)
    o = make_oracle(blk)
    Z, Y, X = blk.shape
    idx = [np.arange(X)[None, None, :], np.arange(Y)[None, :, None]][nn - 1]
    w = 2 * np.pi * 2 / n
    f = np.broadcast_to(np.sin(w * idx + 0.3), blk.shape).copy().reshape(-1)
    out = np.zeros_like(f)
    o.deriv(0, f, out, nn, 1)
    exact = w * np.broadcast_to(np.cos(w * idx + 0.3), blk.shape).reshape(-1)
    # smooth function: boundary closures are 4th order, interior 8th order
    assert np.max(np.abs(out - exact)) < 2e-4
    c = np.full_like(f, 3.25)
    o.deriv(0, c, out, nn, 1)
    assert np.max(np.abs(out)) < 1e-12


@pytest.mark.parametrize("inn", [1, 2, 3])
def test_filter_transfer_and_constants(inn):
    n = 32
    blk = periodic_block(n, n)
    o = make_oracle(blk)
    c = po.coeffs(0.85, 0.85)
    alphf, betf, fa, fb, fc = c[100:105]
    nn = [2, 3, 1][inn - 1]
    Z, Y, X = blk.shape
    idx = [np.arange(X)[None, None, :], np.arange(Y)[None, :, None], np.arange(Z)[:, None, None]][nn - 1]
    mid = [np.s_[:, :, 14:-14], np.s_[:, 14:-14, :], np.s_[14:-14, :, :]][nn - 1]
    # the periodic filter closure truncates the interface operator to 12
    # points, so away from the shared ends the response converges to T(w)
    for k in (2, 5):
        w = 2 * np.pi * k / n
        f = np.broadcast_to(np.cos(w * idx), blk.shape).copy().reshape(-1)
        o.mpigo([f], 1, 1, 0, 1, 1)
        g = f.copy()
        o.filte(0, g, inn, 1)
        T = 1 + (2 * fa * (np.cos(w) - 1) + 2 * fb * (np.cos(2 * w) - 1) + 2 * fc * (np.cos(3 * w) - 1)) / (
            1 + 2 * alphf * np.cos(w) + 2 * betf * np.cos(2 * w))
        err = np.abs(g - T * f).reshape(blk.shape)
        assert err.max() < 5e-4, k
        assert err[mid].max() < 2e-5, k
    # the increment solves the filter system row by row (src/mo_numerics.f90:946-951)
    rng = np.random.default_rng(3)
    f = rng.standard_normal(blk.npts)
    o.mpigo([f], 1, 1, 0, 1, 1)
    g = f.copy()
    o.filte(0, g, inn, 1)
    for a, b in ((0, 0), (4, 9)):
        fl, dl = _line(f, blk.shape, nn, a, b), _line(g - f, blk.shape, nn, a, b)
        for i in range(3, len(fl) - 3):
            lhs = betf * dl[i - 2] + alphf * dl[i - 1] + dl[i] + alphf * dl[i + 1] + betf * dl[i + 2]
            rhs = (fa * (fl[i - 1] + fl[i + 1] - 2 * fl[i]) + fb * (fl[i - 2] + fl[i + 2] - 2 * fl[i])
                   + fc * (fl[i - 3] + fl[i + 3] - 2 * fl[i]))
            assert abs(lhs - rhs) < 1e-12 * (1 + abs(rhs))
    const = np.full(blk.npts, 1.75)
    o.mpigo([const], 1, 1, 0, 1, 1)
    g = const.copy()
    o.filte(0, g, inn, 1)
    assert np.max(np.abs(g - 1.75)) < 1e-13


def test_tgv_conservation_and_decay():
    cs = cases.tgv(16)
    o = po.Oracle(cs)
    q0 = o.state(0)
    k0 = 0.5 * np.sum((q0[1] ** 2 + q0[2] ** 2 + q0[3] ** 2) / q0[0])
    o.step(20)
    q = o.state(0)
    # mass over the unique points (periodic duplicates excluded) is conserved
    m0 = q0[0][:-1, :-1, :-1].sum()
    m = q[0][:-1, :-1, :-1].sum()
    # compact closures are not exactly telescoping: mass holds to ~1e-8
    assert abs(m - m0) / m0 < 1e-6
    k = 0.5 * np.sum((q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0])
    assert k < k0
    t = o.time()
    assert t[0] == 20 and t[2] > 0


def test_uniform_flow_stays_uniform_on_curvilinear_grid():
    cs = cases.curvilinear_4block(24, 16, 14, noise=0.0)
    cs.szco = 0.0
    o = po.Oracle(cs)
    o.step(3)
    # filtered cofactor metrics satisfy the geometric identities only to the
    # scheme's truncation error: a uniform stream drifts by ~1e-6 in 3 steps
    for b in range(4):
        q = o.state(b)
        assert np.max(np.abs(q[0] - 1.0)) < 1e-5
        assert np.max(np.abs(q[2])) < 1e-5


GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["tgv16_step3", "curv4_step2"])
def test_golden_fixtures(name):
    from golden_cases import golden_case
    path = os.path.join(GOLDEN, name + ".npz")
    ref = np.load(path)
    cs, nsteps = golden_case(name)
    o = po.Oracle(cs)
    o.step(nsteps)
    for b in range(len(cs.blocks)):
        np.testing.assert_array_equal(o.state(b), ref[f"qa{b}"])


@pytest.mark.parametrize("name", __import__("golden_cases").DIGEST_CASES)
def test_golden_digests(name):
    """The oracle's states after 1, 10 and 100 steps and on split layouts equal
    the frozen digests bit for bit."""
    import hashlib
    import json
    from golden_cases import golden_case
    ref = json.load(open(os.path.join(GOLDEN, "digests.json")))[name]
    cs, nsteps = golden_case(name)
    o = po.Oracle(cs)
    o.step(nsteps)
    got = [hashlib.sha256(np.ascontiguousarray(o.state(b), np.float64).tobytes()).hexdigest()
           for b in range(len(cs.blocks))]
    assert got == ref

