"""GPU parity of the CUDA path against the CPU oracle, through the C ABI.

FP64 kernels evaluate the reference's expressions in the reference's order
without FMA contraction, so unit operations (mpigo, deriv, filte), the grid
metrics and every phase are compared BIT FOR BIT. The only library power on
the device, the Sutherland T^1.5, is correctly rounded on the GPU while the
oracle calls glibc's pow; the two can differ by one ulp, so after the
primitive phase the tests carry the oracle's viscosity over to stay bit exact,
and whole-step runs use the tolerance of the specification: relative L2
<= 1e-10 after 10 steps.
"""
import numpy as np
import pytest

import pyoracle as po
from canard_b200 import api, cases

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def case_periodic():
    return cases.tgv(nx=24, ny=20, nz=16)


def case_nonperiodic():
    # even and odd line lengths, non-reflecting xi/eta, periodic zeta
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


def case_multiblock():
    return cases.curvilinear_4block(24, 16, 14)


def case_toy():
    # the reference's run/exp.toy layout (six blocks from gridtoy_multi, straight
    # interfaces, periodic across the rows and in zeta, initialo's vortex), small
    return cases.reference_toy(16, 14, 12)


def case_validation():
    # the reference's run/exp.validation (gridtoy block, GCBC on four faces)
    return cases.reference_validation(24, 20, 12)


CASES = {"periodic": case_periodic, "nonperiodic": case_nonperiodic, "multiblock": case_multiblock,
         "toy": case_toy, "validation": case_validation}


def random_fields(cs, seed, ncols=1):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(ncols * b.npts) for b in cs.blocks]


@pytest.mark.parametrize("name", list(CASES))
def test_unit_deriv_bit_exact(name):
    cs = CASES[name]()
    o = po.Oracle(cs, setup=False)
    g = api.Context(cs, setup=False, upload_state=False)
    for m in (1, 4):
        f = random_fields(cs, 10 + m)
        o.mpigo([x.copy() for x in f], 0, 1, 0, m, m)
        g.mpigo([x.copy() for x in f], 0, 1, 0, m, m)
        for b, blk in enumerate(cs.blocks):
            for nn in (1, 2, 3):
                a = np.zeros(blk.npts)
                c = np.zeros(blk.npts)
                o.deriv(b, f[b], a, nn, m)
                g.deriv(b, f[b], c, nn, m)
                np.testing.assert_array_equal(c, a, err_msg=f"{name} b={b} nn={nn} m={m}")
                da = o.get(b, po.A_DRVA[nn - 1])
                dg = g.field(api.F_DRVA[nn - 1], b)
                np.testing.assert_array_equal(dg, da)


@pytest.mark.parametrize("name", list(CASES))
def test_unit_filter_chain_bit_exact(name):
    cs = CASES[name]()
    o = po.Oracle(cs, setup=False)
    g = api.Context(cs, setup=False, upload_state=False)
    fo = random_fields(cs, 7)
    fg = [x.copy() for x in fo]
    # the filter's third send component carries state from call to call
    # (src/mo_numerics.f90:509), so run the reference's sequence of passes
    for m in (1, 2, 3):
        for inn in (1, 2, 3):
            o.mpigo(fo, 1, 1, 0, 3 * (m - 1) + inn, m)
            g.mpigo(fg, 1, 1, 0, 3 * (m - 1) + inn, m)
            for b in range(len(cs.blocks)):
                o.filte(b, fo[b], inn, m)
                g.filte(b, fg[b], inn, m)
                np.testing.assert_array_equal(fg[b], fo[b], err_msg=f"{name} m={m} inn={inn} b={b}")


@pytest.mark.parametrize("name", list(CASES))
def test_grid_metrics_bit_exact(name):
    cs = CASES[name]()
    o = po.Oracle(cs)
    g = api.Context(cs)
    for b, blk in enumerate(cs.blocks):
        for fo, fg in ((po.A_XIM, api.F_XIM), (po.A_ETM, api.F_ETM), (po.A_ZEM, api.F_ZEM), (po.A_YACO, api.F_YACO)):
            np.testing.assert_array_equal(g.field(fg, b).ravel(), o.get(b, fo), err_msg=f"{name} b={b} f={fg}")
        for d in range(3):
            np.testing.assert_array_equal(g.field(api.F_CM[d], b), o.get(b, po.A_CM[d]))


PHASES = [
    (api.PH_PRIM, "prim"), (api.PH_VISCOUS, "viscous"), (api.PH_FLUXES, "fluxes"), (api.PH_GCBC, "gcbc"),
    (api.PH_SPONGE, "sponge"), (api.PH_RKUPDATE, "rk"), (api.PH_AVERAGE, "average"),
]


def compare_state(o, g, cs, what, exact=True, fields=(("qa", po.A_QA, api.F_QA), ("de", po.A_DE, api.F_DE))):
    for b in range(len(cs.blocks)):
        for label, fo, fg in fields:
            a = o.get(b, fo)
            c = g.field(fg, b).ravel()
            if exact:
                np.testing.assert_array_equal(c, a, err_msg=f"{what}: {label} block {b}")
            else:
                assert rel_l2(c, a) < 1e-13, (what, label, b, rel_l2(c, a))


@pytest.mark.parametrize("name", list(CASES))
def test_phases_bit_exact(name):
    cs = CASES[name]()
    o = po.Oracle(cs)
    g = api.Context(cs)
    t6 = [5, 1, 2.0e-3, 1.5e-3, 2.5e-3, 0.31]
    o.set_time(t6)
    g.set_time(t6)
    o.phase(po.PH_FILTER)
    g.phase(api.PH_FILTER)
    compare_state(o, g, cs, "filter", fields=(("qa", po.A_QA, api.F_QA),))
    o.phase(po.PH_COPYQO)
    g.phase(api.PH_COPYQO)
    for nk in (1, 2):
        o.phase(po.PH_MOVEF_A, nk)
        for ph, label in PHASES:
            o.phase(ph, nk)
            g.phase(ph, nk)
            if ph == api.PH_PRIM:
                for b in range(len(cs.blocks)):
                    np.testing.assert_array_equal(g.field(api.F_P, b).ravel(), o.get(b, po.A_P))
                    mo, mg = o.get(b, po.A_SS1), g.field(api.F_SS1, b).ravel()
                    assert np.max(np.abs(mg - mo) / np.abs(mo)) <= 2.3e-16, "Sutherland power beyond 1 ulp"
                    g.set_field(api.F_SS1, mo.reshape(g.field(api.F_SS1, b).shape), b)
            compare_state(o, g, cs, f"{label} nk={nk}")
            if ph == api.PH_VISCOUS and cs.viscous:
                for b in range(len(cs.blocks)):
                    np.testing.assert_array_equal(g.field(api.F_TAU, b).ravel(), o.get(b, po.A_TAU))
            if ph == api.PH_FLUXES:
                for b in range(len(cs.blocks)):
                    for d in range(3):
                        np.testing.assert_array_equal(g.field(api.F_DRVA[d], b), o.get(b, po.A_DRVA[d]))


@pytest.mark.parametrize("name", list(CASES))
def test_steps_match_oracle(name):
    cs = CASES[name]()
    o = po.Oracle(cs)
    g = api.Context(cs)
    o.step(12)
    g.step(12)
    np.testing.assert_array_equal(g.time()[:2], o.time()[:2])
    assert abs(g.time()[2] - o.time()[2]) <= 1e-12 * abs(o.time()[2])
    for b in range(len(cs.blocks)):
        err = rel_l2(g.state(b), o.state(b))
        assert err <= 1e-10, (name, b, err)


def test_tgv64_ten_steps_within_1e_10():
    """C1: 64^3 Taylor-Green vortex (65^3 stored points), Re 1600, Mach 0.1,
    FP64, 10 steps: relative L2 <= 1e-10 per conserved variable."""
    cs = cases.tgv(64)
    o = po.Oracle(cs)
    g = api.Context(cs)
    o.step(10)
    g.step(10)
    qo, qg = o.state(0), g.state(0)
    for v in range(5):
        err = rel_l2(qg[v], qo[v])
        assert err <= 1e-10, (v, err)


def test_error_status_instead_of_fault():
    cs = case_periodic()
    g = api.Context(cs)
    with pytest.raises(api.CanardError) as e:
        g.phase(99, 1)
    assert e.value.code == api.ERR_ARG
    with pytest.raises(api.CanardError) as e:
        g.deriv(5, np.zeros(10), np.zeros(10), 1, 1)
    assert e.value.code == api.ERR_ARG
    g.step(1)  # the context stays usable


def test_batched_context_equals_single_cases():
    """Independent cases advanced together in one context (one launch per phase
    and direction for all cases, per-case dt) give exactly the single-case
    results."""
    cs_list = cases.batched(3, seed=5, lo=20, hi=30)
    g = api.Context(cs_list)
    g.step(12)
    for i, cs in enumerate(cs_list):
        one = api.Context(cs)
        one.step(12)
        np.testing.assert_array_equal(g.state(0, case=i), one.state(0))
        np.testing.assert_array_equal(g.time(case=i), one.time())
        one.close()
    # and the oracle agrees for one of them
    o = po.Oracle(cs_list[1])
    o.step(12)
    assert rel_l2(g.state(0, case=1), o.state(0)) <= 1e-10


def test_graph_replay_equals_direct_launches():
    """canard_step replays a captured CUDA graph of the step; with the
    per-family timers on it launches the kernels one by one. Both give the
    same state bit for bit, across the dt-reduction steps (n % 10 == 1)."""
    cs = case_multiblock()
    a = api.Context(cs)
    b = api.Context(cs)
    b.set_timers(True)
    a.step(13)
    b.step(13)
    for blk in range(len(cs.blocks)):
        np.testing.assert_array_equal(a.state(blk), b.state(blk))
    np.testing.assert_array_equal(a.time(), b.time())
    assert a.launch_count() == b.launch_count()


def test_overflow_is_reported():
    """dt == 0 after step 2 is the reference's 'Canard: Overflow.' stop; made
    on the host by setting the time state, then reported by the step."""
    cs = case_periodic()
    g = api.Context(cs)
    g.set_time([5, 1, 0.0, 0.0, 0.0, 0.1])
    with pytest.raises(api.CanardError) as e:
        g.step(1)
    assert e.value.code == api.ERR_NAN


@pytest.mark.parametrize("name", ["periodic", "nonperiodic"])
def test_line_bench_matches_oracle(name):
    """The isolated line-solve bench (5 fields, one launch per direction)
    returns the oracle's derivative and filter bit for bit in FP64."""
    cs = CASES[name]()
    blk = cs.blocks[0]
    fields = cases.noise_fields(blk, 5, kmax=4)
    g = api.Context(cs, setup=False, upload_state=False)
    for op in (0, 1):
        o = po.Oracle(cs, setup=False)
        for nn in (1, 2, 3):
            out, ms = g.line_bench(op, nn, fields, reps=2)
            assert ms > 0
            for k in range(5):
                f = fields[k].ravel().copy()
                if op == 0:
                    o.mpigo([f.copy()], 0, 1, 0, k + 1, k + 1)
                    r = np.zeros_like(f)
                    o.deriv(0, f, r, nn, k + 1)
                else:
                    o.mpigo([f], 1, 1, 0, k + 1, k + 1)
                    o.filte(0, f, {2: 1, 3: 2, 1: 3}[nn], k + 1)
                    r = f
                np.testing.assert_array_equal(out[k].ravel(), r, err_msg=f"op {op} nn {nn} field {k}")


def test_autotune_keeps_results():
    """The line-tile autotuner changes only tile shapes and staging depths on
    the FP64 path: a tuned context steps bit-identically to an untuned one."""
    cs = case_multiblock()
    a = api.Context(cs)
    rep = a.autotune(reps=2)
    assert len(rep) == 9 and all(r["ms"] > 0 for r in rep)
    b = api.Context(cs)
    a.step(12)
    b.step(12)
    for blk in range(len(cs.blocks)):
        np.testing.assert_array_equal(a.state(blk), b.state(blk))


def test_non_finite_state_is_reported():
    """A NaN in the state (set from the host) is caught at the next dt
    reduction (every tenth step) and reported as the overflow error."""
    cs = case_periodic()
    g = api.Context(cs)
    q = g.state(0)
    q[0, 3, 4, 5] = np.nan
    g.set_state(0, q)
    with pytest.raises(api.CanardError) as e:
        g.step(2)  # the step with n % 10 == 1 reduces dt
    assert e.value.code == api.ERR_NAN


def test_bounded_wait_reports_timeout_and_context_stays_usable():
    """A device wait that can never complete (an mbarrier nothing arrives at)
    gives up after about half a second and is reported as ERR_TIMEOUT; the
    same context then steps exactly like a fresh one."""
    cs = case_periodic()
    a = api.Context(cs)
    b = api.Context(cs)
    code, sec = b.selftest_wait()
    assert code == api.ERR_TIMEOUT, code
    assert 0.3 < sec < 10.0, sec
    assert "bounded device wait" in api.lib().canard_last_error(b.h).decode()
    a.step(3)
    b.step(3)
    np.testing.assert_array_equal(b.state(0), a.state(0))


@pytest.mark.parametrize("shape", [(24, 20, 16), (16, 200, 140), (16, 256, 32)])
def test_tmem_line_kernel_bit_identical(shape):
    """The FP64 line kernel that keeps the elimination results in tensor
    memory (eta/zeta lines of 16..257 points) gives the same bits as the
    default shared-memory tiles. The shapes cover lines whose input boxes all
    load up front (L <= 128), the input ring's refill (L > 128) and L = 257,
    whose last row stays in registers."""
    nx, ny, nz = shape
    cs = cases.tgv(nx=nx, ny=ny, nz=nz)
    a = api.Context(cs)
    b = api.Context(cs)
    for grp in ("filter", "viscous", "flux"):
        for d in ("eta", "zeta"):
            b.set_line_kind(grp, d, "fp64-tmem")
    with pytest.raises(api.CanardError) as e:
        b.set_line_kind("flux", "xi", "fp64-tmem")  # xi lines stay in shared memory
    assert e.value.code == api.ERR_ARG
    a.step(3)
    b.step(3)
    np.testing.assert_array_equal(b.state(0), a.state(0))
    np.testing.assert_array_equal(b.field(api.F_DE, 0), a.field(api.F_DE, 0))


def test_restart_round_trip(tmp_path):
    """write_restart / read_restart move the state and the time state of every
    block exactly. The filter's persistent interface send chain is not in the
    reference's restart file (a restarted reference run starts it afresh too),
    so a restarted run agrees with the continued one to rounding, and the
    comparer finds no difference between two copies of the same files."""
    cs = case_multiblock()
    a = api.Context(cs)
    a.step(4)
    a.write_restart(str(tmp_path / "a"))
    b = api.Context(cs)
    b.read_restart(str(tmp_path / "a"))
    np.testing.assert_array_equal(b.time(), a.time())
    for blk in range(len(cs.blocks)):
        np.testing.assert_array_equal(b.state(blk), a.state(blk))
    b.write_restart(str(tmp_path / "b"))
    for blk, spec in enumerate(cs.blocks):
        f1, f2 = (str(tmp_path / d / api.restart_name(blk)) for d in ("a", "b"))
        assert open(f1, "rb").read() == open(f2, "rb").read()
        assert api.compare_restart(f1, f2, spec.npts, 1e-15) == 0
    a.step(3)
    b.step(3)
    for blk in range(len(cs.blocks)):
        assert rel_l2(b.state(blk), a.state(blk)) <= 1e-12


def case_walls():
    """Walls on three faces: xi side 1 and eta side 0 viscous (25), eta side 1
    inviscid (20); xi side 0 non-reflecting, zeta periodic. Wall faces meet
    along two edges (viscous then viscous, viscous then inviscid in the
    reference's face order), and the frame moves at Mach 0.3 along x, so the
    no-slip reset uses the frame velocity."""
    blk = cases.BlockSpec(22, 18, 16, [[10, 25], [25, 20], [45, 45]], [[-1, -1], [-1, -1], [0, 0]])
    Z, Y, X = blk.shape
    x = np.linspace(-1, 1, X)
    y = np.linspace(0, 1.2, Y)
    z = np.linspace(0, 1, Z)
    Zz, Yy, Xx = np.meshgrid(z, y, x, indexing="ij")
    xyz = np.stack([Xx + 0.02 * np.sin(3 * Yy), Yy + 0.02 * np.sin(2 * Xx), Zz])
    rho, u, v, w, p = cases.vortex_state(Xx, Yy, 0.0, 2.0, 0.3, 0.0, 0.6)
    return cases.CaseSpec([blk], viscous=1, reoo=2000.0, amach=(0.3, 0.0, 0.0), xyz=[xyz],
                          qa=[cases._conserved(rho, u, v, w, p)], name="walls")


def test_wall_phases_match_oracle():
    """The GCBC wall branch and wall_condition_update phase by phase. Every
    phase is bit-exact except the inviscid wall's energy reset, which takes
    rho^1.4 from the device's pow (the oracle: glibc's); there the two may
    differ by an ulp, so that phase is compared to 2.3e-16 relative and the
    oracle's state is carried over."""
    cs = case_walls()
    o = po.Oracle(cs)
    g = api.Context(cs)
    t6 = [5, 1, 2.0e-3, 1.5e-3, 2.5e-3, 0.31]
    o.set_time(t6)
    g.set_time(t6)
    for ph in (po.PH_FILTER, po.PH_COPYQO):
        o.phase(ph)
        g.phase(ph)
    compare_state(o, g, cs, "filter", fields=(("qa", po.A_QA, api.F_QA),))
    phases = PHASES[:6] + [(api.PH_WALL, "wall")] + PHASES[6:]
    for nk in (1, 2):
        o.phase(po.PH_MOVEF_A, nk)
        for ph, label in phases:
            o.phase(ph, nk)
            g.phase(ph, nk)
            if ph == api.PH_PRIM:
                mo = o.get(0, po.A_SS1)
                g.set_field(api.F_SS1, mo.reshape(g.field(api.F_SS1, 0).shape), 0)
            if ph == api.PH_WALL:
                a, c = o.get(0, po.A_QA), g.field(api.F_QA, 0).ravel()
                assert np.all(np.abs(c - a) <= 2.3e-16 * np.abs(a)), "wall reset beyond 1 ulp"
                g.set_state(0, a.reshape(g.state(0).shape))
            compare_state(o, g, cs, f"{label} nk={nk}")


def test_wall_steps_match_oracle():
    cs = case_walls()
    o = po.Oracle(cs)
    g = api.Context(cs)
    o.step(12)
    g.step(12)
    err = rel_l2(g.state(0), o.state(0))
    assert err <= 1e-10, err


def test_wall_steps_fp32_mixed():
    cs = case_walls()
    o = po.Oracle(cs)
    g = api.Context(cs, precision=api.FP32_MIXED)
    o.step(12)
    g.step(12)
    assert rel_l2(g.state(0), o.state(0)) <= 1e-5


def reference_recording(o, cs, nsteps):
    """The reference's time-averaged recording (src/mo_canard_driver.f90:373-402)
    restated in numpy over the oracle's steps, for a frame at rest (umf = 0)."""
    qb = [np.zeros(5 * b.npts) for b in cs.blocks]
    dtsum = 0.0
    for _ in range(nsteps):
        o.step(1)
        t = o.time()
        dtsum = dtsum + t[2]
        fctr = 0.5 * t[2]
        for b in range(len(cs.blocks)):
            qb[b] = qb[b] + fctr * (o.get(b, po.A_QO) + o.get(b, po.A_QA))
    out = []
    for b, blk in enumerate(cs.blocks):
        q = (o.get(b, po.A_QO) if int(t[0]) == 1 else (1.0 / dtsum) * qb[b]).reshape(5, -1)
        rr = 1.0 / q[0]
        v = np.empty(q.shape, np.float32)
        v[0] = q[0]
        v[1:4] = rr * q[1:4] + 0.0
        v[4] = (1.4 - 1.0) * (q[4] - (0.5 * rr) * ((q[1] * q[1] + q[2] * q[2]) + q[3] * q[3]))
        out.append(v.reshape((5,) + blk.shape))
    return out, t[5] - 0.5 * dtsum


@pytest.mark.parametrize("nsteps", [1, 4])
def test_recording_matches_the_reference_average(tmp_path, nsteps):
    """qb accumulated after every step, averaged over dtsum (qo after the first
    step), the FP32 output variables and the output time; a second output
    starts from a reset average; the Tecplot file holds what record_output
    returned."""
    cs = case_periodic()
    o = po.Oracle(cs)
    g = api.Context(cs)
    g.record_enable()
    for _ in range(nsteps):
        g.step(1)
        g.record_accumulate()
    arrs, t = g.record_output()
    ref, tref = reference_recording(o, cs, nsteps)
    np.testing.assert_allclose(arrs[0], ref[0], rtol=2.0 ** -23, atol=0)
    assert abs(t - tref) <= 1e-14 * abs(tref)
    # the next interval starts from zero
    g.step(2)
    g.record_accumulate()
    arrs2, t2 = g.record_output()
    assert t2 > t and np.all(np.isfinite(arrs2[0]))
    # file output of a multi-block case
    mb = api.Context(case_multiblock())
    mb.record_enable()
    for _ in range(4):  # dt is 0 for the first two steps (the reference's ramp)
        mb.step(1)
        mb.record_accumulate()
    mb.write_grid_plt(str(tmp_path))
    tt = mb.write_output(str(tmp_path), 0)
    data = open(tmp_path / api.plt_name(0), "rb").read()
    assert data[:8] == b"#!TDV112" and tt > 0
    npts = sum(b.npts for b in mb.cases[0].blocks)
    assert len(data) > 5 * 4 * npts
    assert (tmp_path / api.plt_name(-1)).exists()


@pytest.mark.parametrize("name", ["nonperiodic", "multiblock"])
def test_tmem_line_kernel_with_interfaces_and_gcbc(name):
    """The tensor-memory kernel where lines end on block interfaces (the
    receive buffers of the contraction) and on GCBC faces (the line-end values
    in drva): pinned on every eta/zeta group whose lines it takes, steps stay
    bit-identical to the default tiles."""
    cs = CASES[name]()
    a = api.Context(cs)
    b = api.Context(cs)
    pinned = 0
    for grp in ("filter", "viscous", "flux"):
        for d in ("eta", "zeta"):
            try:
                b.set_line_kind(grp, d, "fp64-tmem")
                pinned += 1
            except api.CanardError as e:
                assert e.code == api.ERR_ARG  # lines shorter than 16 points
    assert pinned >= 3
    a.step(4)
    b.step(4)
    for blk in range(len(cs.blocks)):
        np.testing.assert_array_equal(b.state(blk), a.state(blk))


def test_phase_with_caller_stage_scalars_equals_device_stage():
    """canard_phase_with takes dt, umf and dudtmf from the caller, as the
    reference's calc_fluxes / gcbc_update / RK update receive them; with the
    values the device's own movef gives (a constant moving frame, Mach 0.4
    along x) the phases give the same bits as canard_phase."""
    cs = case_multiblock()
    a, b = api.Context(cs), api.Context(cs)
    t6 = [5, 1, 2.0e-3, 1.5e-3, 2.5e-3, 0.31]
    umf = (cs.amach[0], cs.amach[1], cs.amach[2])
    for g in (a, b):
        g.set_time(t6)
        g.phase(api.PH_FILTER)
        g.phase(api.PH_COPYQO)
    for nk in (1, 2, 3):
        for g in (a, b):
            g.phase(api.PH_PRIM, nk)
            g.phase(api.PH_VISCOUS, nk)
        a.phase(api.PH_FLUXES, nk)
        b.phase_with(api.PH_FLUXES, nk, t6[2], umf)
        a.phase(api.PH_GCBC, nk)
        b.phase_with(api.PH_GCBC, nk, t6[2], umf)
        for g in (a, b):
            g.phase(api.PH_SPONGE, nk)
        a.phase(api.PH_RKUPDATE, nk)
        b.phase_with(api.PH_RKUPDATE, nk, t6[2], umf)
        for g in (a, b):
            g.phase(api.PH_AVERAGE, nk)
        for blk in range(len(cs.blocks)):
            np.testing.assert_array_equal(a.state(blk), b.state(blk), err_msg=f"nk={nk} block {blk}")
