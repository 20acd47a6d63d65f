"""The reader of the reference's input file (Fortran namelists) and the case
it describes, on the CPU (canard_b200.namelist, canard_b200.driver)."""
import os
import re

import numpy as np
import pytest

from canard_b200 import cases, driver, namelist

TOY = """&nml_driver
nio = 0
mbk = 5
ndata = 3
/
&nml_canard
nts = 0
nrestart = 1
cfl = 1.2d0
tmax = 0.25e0
ltimer = .false.
/
&nml_domdcomp
nbpc(:,1) = 2,2,2,2,2,2
nbpc(:,2) = 6*1
nbpc(:,3) = 1,1,1,1,1,1
lximb = 6*16
letmb = 6*14
lzemb = 6*12
nbbc(0,1,:) = 10,35
nbbc(0,2,:) = 45,35
nbbc(0,3,:) = 45,45
mbcd(0,1,:) = -1,1
mbcd(0,2,:) = 3,3
mbcd(0,3,:) =  0,0
nbbc(1,1,:) = 35,35
nbbc(1,2,:) = 45,35
nbbc(1,3,:) = 45,45
mbcd(1,1,:) = 0,2
mbcd(1,2,:) = 4,4
mbcd(1,3,:) =  1,1
nbbc(2,1,:) = 35,10
nbbc(2,2,:) = 45,35
nbbc(2,3,:) = 45,45
mbcd(2,1,:) = 1,-1
mbcd(2,2,:) = 5,5
mbcd(2,3,:) =  2,2
nbbc(3,1,:) = 10,35
nbbc(3,2,:) = 35,45
nbbc(3,3,:) = 45,45
mbcd(3,1,:) = -1,4
mbcd(3,2,:) = 0,0
mbcd(3,3,:) =  3,3
nbbc(4,1,:) = 35,35
nbbc(4,2,:) = 35,45
nbbc(4,3,:) = 45,45
mbcd(4,1,:) = 3,5
mbcd(4,2,:) = 1,1
mbcd(4,3,:) =  4,4
nbbc(5,1,:) = 35,10
nbbc(5,2,:) = 35,45
nbbc(5,3,:) = 45,45
mbcd(5,1,:) = 4,-1
mbcd(5,2,:) = 2,2
mbcd(5,3,:) =  5,5
/
&nml_numerics
fltk = 0.65e0
fltrbc = 0.9e0
/
&nml_physics
reoo = 500000.0e0  ! divided by the frame Mach number in the code
tempoo = 300.0e0
amach1 = 0.3e0
amach2 = 0.0e0
amach3 = 0.0e0
timf = 0.0e0
nsmf = 1
/
&nml_gridgen
gridtype = 1
lxi0 = 16, lxi1 = 16, lxi2 = 16
let0 = 14
lze0 = 12
doml0 = 0.5e0
doml1 = 1.0e0
domh = 0.5e0
span = 0.1e0
szth0 = 0.0e0
szth1 = 0.6e0
/
nml_sponge
szco = 10.0e0
/
"""


def test_scalars_arrays_and_the_group_without_ampersand():
    r = namelist.read(TOY)
    assert r["nml_driver"] == {"nio": 0, "mbk": 5, "ndata": 3}
    assert r["nml_canard"]["cfl"] == 1.2 and r["nml_canard"]["ltimer"] is False
    nbpc, lo = r["nml_domdcomp"]["nbpc"]
    assert lo == [0, 1] and nbpc.shape == (6, 3)
    np.testing.assert_array_equal(nbpc[:, 0], 2)
    np.testing.assert_array_equal(nbpc[:, 1:], 1)
    np.testing.assert_array_equal(r["nml_domdcomp"]["lximb"][0], 16)
    nbbc = r["nml_domdcomp"]["nbbc"][0]
    assert nbbc.shape == (6, 3, 2)
    assert list(nbbc[0, 0]) == [10, 35] and list(nbbc[5, 1]) == [35, 45]
    assert list(r["nml_domdcomp"]["mbcd"][0][4, 0]) == [3, 5]
    assert r["nml_gridgen"]["lxi1"] == 16 and r["nml_gridgen"]["span"] == 0.1
    # "nml_sponge" lacks its '&': the reference's READ never finds the group
    assert r["nml_sponge"]["szco"] == 0.0


def test_sections_repeat_counts_and_logicals():
    r = namelist.read("&nml_driver mbk = 2 /\n&nml_domdcomp lximb(1:2) = 2*7, letmb(2) = 5 /\n"
                      "&nml_canard ltimer = T, tmax = 1.5D-1 /")
    assert list(r["nml_domdcomp"]["lximb"][0]) == [0, 7, 7]
    assert list(r["nml_domdcomp"]["letmb"][0]) == [0, 0, 5]
    assert r["nml_canard"]["ltimer"] is True and r["nml_canard"]["tmax"] == 0.15


@pytest.mark.parametrize("text", ["&nml_canard cfl = 1.0, bogus = 2 /",
                                  "&nml_driver mbk = 1 /\n&nml_domdcomp lximb(3) = 5 /",
                                  "&nml_canard tmax = abc /"])
def test_errors(text):
    with pytest.raises(namelist.NamelistError):
        namelist.read(text)


def test_case_from_the_toy_input():
    warnings = []
    cs = driver.case_from_input(namelist.read(TOY), warn=warnings.append)
    assert len(warnings) == 1 and "nbpc" in warnings[0]
    assert len(cs.blocks) == 6 and cs.cfl == 1.2 and cs.fltk == 0.65 and cs.szco == 0.0
    ref = cases.reference_toy(16, 14, 12)
    for a, b in zip(cs.blocks, ref.blocks):
        assert [list(x) for x in a.nbc] == [list(x) for x in b.nbc]
        assert [list(x) for x in a.mbcd] == [list(x) for x in b.mbcd]
    for a, b in zip(cs.xyz, ref.xyz):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(cs.qa, ref.qa):
        np.testing.assert_array_equal(a, b)


def test_grid_sizes_must_match_the_blocks():
    bad = TOY.replace("lximb = 6*16", "lximb = 6*15")
    with pytest.raises(namelist.NamelistError):
        driver.case_from_input(namelist.read(bad), warn=lambda s: None)
    with pytest.raises(namelist.NamelistError):
        driver.case_from_input(namelist.read(TOY.replace("gridtype = 1", "gridtype = 2")), warn=lambda s: None)


# a checkout of the reference, named by CANARD_REFERENCE (skipped without one)
REF_RUN = os.path.join(os.environ.get("CANARD_REFERENCE", ""), "run") if os.environ.get("CANARD_REFERENCE") else ""


@pytest.mark.skipif(not REF_RUN or not os.path.isdir(REF_RUN), reason="CANARD_REFERENCE names no reference checkout")
@pytest.mark.parametrize("script,nblocks,points", [("exp.validation", 1, (17, 51, 51)), ("exp.aio", 1, (17, 51, 51)),
                                                   ("exp.toy", 6, (17, 101, 101)),
                                                   ("exp.toy.aio", 6, (17, 101, 101))])
def test_the_reference_run_inputs(script, nblocks, points):
    """The input.canard each of the reference's run scripts writes (its here
    document) reads and gives its case; every one splits blocks (nbpc > 1) and
    misspells the sponge group, so szco stays 0."""
    text = open(os.path.join(REF_RUN, script)).read()
    m = re.search(r"cat > input\.canard << EOF\n(.*?)\nEOF", text, re.S)
    assert m, script
    r = namelist.read(m.group(1))
    warnings = []
    cs = driver.case_from_input(r, warn=warnings.append)
    assert len(cs.blocks) == nblocks and all(b.shape == points for b in cs.blocks)
    assert r["nml_sponge"]["szco"] == 0.0 and len(warnings) == 1
    assert r["nml_numerics"]["fltk"] == 0.65 and r["nml_physics"]["amach1"] == 0.3


def test_output_writer_writes_in_order_and_reports_errors(tmp_path):
    """The writer thread that stands in for the reference's IO server writes
    the same bytes as a direct call, and a failed write surfaces at close()."""
    from canard_b200 import api
    rng = np.random.default_rng(3)
    outs = [[rng.standard_normal((5, 4, 3, 6)).astype(np.float32)] for _ in range(3)]
    w = driver.OutputWriter()
    for n, arrs in enumerate(outs):
        w.submit(str(tmp_path / "data" / ("n%03d.plt" % n)), n, arrs, 0.5 * n)
    w.close()
    for n, arrs in enumerate(outs):
        ref = tmp_path / ("ref%d.plt" % n)
        api.plt_write(str(ref), n, arrs, 0.5 * n)
        assert (tmp_path / "data" / ("n%03d.plt" % n)).read_bytes() == ref.read_bytes()
    w = driver.OutputWriter()
    w.submit(str(tmp_path / "x.plt"), 1000, outs[0], 0.0)  # three-digit names only
    with pytest.raises(api.CanardError):
        w.close()


class _FakeContext:
    """Stands in for api.Context on the CPU: the reference's dt ramp over a
    fixed dte (dt = 0 for the first two steps), no device."""

    def __init__(self, cs, precision=0, zero_dt_at=None):
        self.cs, self.t6, self.steps = cs, [0.0, 0.0, 0.0, 0.0, 0.0, 0.0], 0
        self.zero_dt_at, self.restarts, self.recorded = zero_dt_at, [], 0

    def time(self, case=0):
        return np.array(self.t6)

    def step(self, n=1):
        from canard_b200 import api
        k = int(self.t6[0])
        if self.zero_dt_at is not None and k >= self.zero_dt_at:
            raise api.CanardError(api.ERR_NAN, "Canard: Overflow.")
        dt = 0.0 if k < 2 else 0.01 * np.sin(0.05 * np.pi * min(k - 1, 10)) ** 2
        self.t6 = [k + 1, 1, dt, 0.0, 0.01, self.t6[5] + dt]
        self.steps += 1

    def set_timers(self, on):
        pass

    def record_enable(self, on=True):
        pass

    def record_accumulate(self):
        self.recorded += 1

    def record_output(self, case=0):
        return [np.zeros((5,) + b.shape, np.float32) for b in self.cs.blocks], self.t6[5]

    def write_restart(self, directory, case=0):
        self.restarts.append(directory)

    def read_restart(self, directory, case=0):
        pass

    def timers(self):
        return {}

    def close(self):
        pass


SMALL = TOY.replace("ndata = 3", "ndata = 4").replace("tmax = 0.25e0", "tmax = 0.05e0")


@pytest.mark.parametrize("zero_dt_at", [None, 7])
def test_driver_loop_on_a_stand_in_context(tmp_path, monkeypatch, zero_dt_at):
    import io
    made = []

    def fake(cs, precision=0):
        made.append(_FakeContext(cs, precision, zero_dt_at))
        return made[-1]

    monkeypatch.setattr(driver.api, "Context", fake)
    submitted = []
    monkeypatch.setattr(driver.OutputWriter, "submit", lambda self, p, n, a, t=0.0: submitted.append((p, n, t)))
    (tmp_path / "input.canard").write_text(SMALL)
    log = io.StringIO()
    res = driver.run(str(tmp_path / "input.canard"), out=log)
    ctx = made[0]
    if zero_dt_at is None:
        # stops at the first step that reaches tmax; outputs at 0, tmax/4, ..., tmax
        assert ctx.t6[5] >= 0.05 and ctx.t6[5] - ctx.t6[2] < 0.05
        assert [n for _, n, _ in submitted] == [-1, 0, 1, 2, 3, 4]
        assert "Overflow" not in log.getvalue()
        for (_, n, t), lo in zip(submitted[1:], [0.0, 0.0125, 0.025, 0.0375, 0.05]):
            assert t >= lo  # written at the first step whose end passes n tmax / ndata
    else:
        assert res["overflow"] and ctx.steps == zero_dt_at and "Canard: Overflow." in log.getvalue()
    assert res["outputs"][0] == "data/grid.plt" and len(res["outputs"]) == len(submitted)
    assert ctx.recorded == ctx.steps and ctx.restarts == [str(tmp_path)]
    assert "Canard: Finished." in log.getvalue()


class _SplitFake(_FakeContext):
    """The stand-in with per-rank states."""

    def __init__(self, cs, precision=0, zero_dt_at=None):
        super().__init__(cs, precision, zero_dt_at)
        self.q = [np.array(q) for q in cs.qa]
        self.t_set = None

    def step(self, n=1):
        super().step(n)
        for q in self.q:
            q *= 1.0 + 1e-3

    def state(self, b, case=0):
        return self.q[b].copy()

    def set_state(self, b, q, case=0):
        self.q[b] = np.array(q).reshape(self.q[b].shape)

    def set_time(self, t6, case=0):
        self.t_set = list(t6)
        self.t6 = list(t6)

    def record_output(self, case=0):
        return [q.astype(np.float32) for q in self.q], self.t6[5]


def test_driver_split_files_are_per_input_block(tmp_path, monkeypatch):
    """With split=True the context runs the input's ranks, and the restart and
    output files stay one per input block, assembled from its ranks; a restart
    read splits the block files back to the ranks."""
    import io
    from canard_b200 import api
    text = SMALL.replace("lximb = 6*16", "lximb = 6*26").replace("lxi0 = 16, lxi1 = 16, lxi2 = 16",
                                                                  "lxi0 = 26, lxi1 = 26, lxi2 = 26")
    (tmp_path / "input.canard").write_text(text)
    made = []

    def fake(cs, precision=0):
        made.append(_SplitFake(cs, precision))
        return made[-1]

    monkeypatch.setattr(driver.api, "Context", fake)
    submitted = []
    monkeypatch.setattr(driver.OutputWriter, "submit", lambda self, p, n, a, t=0.0: submitted.append((n, a)))
    log = io.StringIO()
    driver.run(str(tmp_path / "input.canard"), out=log, split=True)
    ctx = made[0]
    assert len(ctx.cs.blocks) == 12 and "nbpc > 1" not in log.getvalue()
    # restart files: per input block, equal to its ranks' states assembled
    blocks = cases.compose(ctx.cs.sub, ctx.q)
    assert len(blocks) == 6
    for m, q in enumerate(blocks):
        t6, got = api.read_restart_file(str(tmp_path / api.restart_name(m)), q[0].size)
        np.testing.assert_array_equal(got, q.reshape(5, -1))
    assert not (tmp_path / api.restart_name(6)).exists()
    # the grid and every output hold the six input blocks
    n, grid = submitted[0]
    assert n == -1 and len(grid) == 6 and grid[0].shape == (3, 13, 15, 27)
    for n, arrs in submitted[1:]:
        assert len(arrs) == 6 and arrs[1].shape == (5, 13, 15, 27)
    # restart: the block files split back to the ranks
    (tmp_path / "input.canard").write_text(text.replace("nts = 0", "nts = 1").replace("tmax = 0.05e0", "tmax = 0.07e0"))
    driver.run(str(tmp_path / "input.canard"), out=io.StringIO(), split=True, max_steps=0)
    ctx2 = made[1]
    assert ctx2.t_set is not None and ctx2.t_set[0] == ctx.t6[0]
    for r in range(12):
        np.testing.assert_array_equal(ctx2.q[r], ctx.q[r])


@pytest.mark.parametrize("ndata,nrestart,expect_outputs,expect_restart", [
    (-1, 1, [], True),          # ndata < 0: no output at all (loutput = .false.)
    (0, 0, ["data/grid.plt"], False),  # ndata = 0: the grid only; nrestart = 0: no restart file
])
def test_driver_output_and_restart_switches(tmp_path, monkeypatch, ndata, nrestart, expect_outputs, expect_restart):
    import io
    made = []
    monkeypatch.setattr(driver.api, "Context", lambda cs, precision=0: made.append(_FakeContext(cs)) or made[-1])
    submitted = []
    monkeypatch.setattr(driver.OutputWriter, "submit", lambda self, p, n, a, t=0.0: submitted.append(n))
    text = SMALL.replace("ndata = 4", "ndata = %d" % ndata).replace("nrestart = 1", "nrestart = %d" % nrestart)
    (tmp_path / "input.canard").write_text(text)
    res = driver.run(str(tmp_path / "input.canard"), out=io.StringIO())
    assert res["outputs"] == expect_outputs and len(submitted) == len(expect_outputs)
    assert bool(made[0].restarts) == expect_restart
    assert made[0].steps > 5  # the loop ran to tmax


def test_driver_restart_start_without_files_is_an_io_error(tmp_path):
    """nts /= 0 reads misc/restartzNNN.da; without them the run stops before
    its first step with the I/O error (the real context is needed for the
    read, so this runs the read path of the split-file helper on the CPU)."""
    from canard_b200 import api
    cs = cases.decompose(cases.reference_validation(26, 26, 12), [(2, 2, 1)])
    files = driver._Files(cs)
    with pytest.raises(api.CanardError) as e:
        files.read_restart(_SplitFake(cs), str(tmp_path))
    assert e.value.code == api.ERR_IO


def test_driver_stopped_early_is_not_an_overflow(tmp_path, monkeypatch):
    import io
    monkeypatch.setattr(driver.api, "Context", lambda cs, precision=0: _FakeContext(cs))
    monkeypatch.setattr(driver.OutputWriter, "submit", lambda self, p, n, a, t=0.0: None)
    (tmp_path / "input.canard").write_text(SMALL)
    log = io.StringIO()
    res = driver.run(str(tmp_path / "input.canard"), out=log, max_steps=1)  # dt is 0 for steps 0 and 1
    assert res["steps"] == 1 and "Overflow" not in log.getvalue()


def test_plan_devices_of_an_input(tmp_path):
    """--plan-devices: the input's ranks (nbpc) placed on devices, with the
    bytes per step that cross between them; no device is used."""
    import io
    text = SMALL.replace("lximb = 6*16", "lximb = 6*26").replace("lxi0 = 16, lxi1 = 16, lxi2 = 16",
                                                                  "lxi0 = 26, lxi1 = 26, lxi2 = 26")
    (tmp_path / "input.canard").write_text(text)
    log = io.StringIO()
    res = driver.plan_devices(str(tmp_path / "input.canard"), 3, out=log)
    assert res["ranks"] == 12 and res["devices"] == 3
    assert sorted(set(res["device_of_rank"])) == [0, 1, 2]
    assert all(b > 0 for b in res["bytes_per_step_out"])
    assert "12 ranks on 3 devices" in log.getvalue()
    f32 = driver.plan_devices(str(tmp_path / "input.canard"), 3, precision=1, out=io.StringIO())
    assert all(a < b for a, b in zip(f32["bytes_per_step_out"], res["bytes_per_step_out"]))


def test_nml_gpu_options(tmp_path, monkeypatch):
    """&nml_gpu carries this implementation's options (precision, split, a step
    limit, inviscid) in a group the reference never reads; arguments given to
    run() win over it; an input without the group keeps the defaults."""
    import io
    base = SMALL.replace("lximb = 6*16", "lximb = 6*26").replace("lxi0 = 16, lxi1 = 16, lxi2 = 16",
                                                                  "lxi0 = 26, lxi1 = 26, lxi2 = 26")
    text = base + "\n&nml_gpu nprecision = 1, lsplit = .true., nsteps = 3, linviscid = .true. /\n"
    r = namelist.read(text)
    assert int(r["nml_gpu"]["nprecision"]) == 1 and bool(r["nml_gpu"]["lsplit"]) and int(r["nml_gpu"]["nsteps"]) == 3
    assert driver.gpu_options(namelist.read(base)) == {"precision": 0, "viscous": 1, "max_steps": None,
                                                       "split": False}
    made = []

    def fake(cs, precision=0):
        made.append(_SplitFake(cs, precision))
        made[-1].precision = precision
        return made[-1]

    monkeypatch.setattr(driver.api, "Context", fake)
    monkeypatch.setattr(driver.OutputWriter, "submit", lambda self, p, n, a, t=0.0: None)
    (tmp_path / "input.canard").write_text(text)
    driver.run(str(tmp_path / "input.canard"), out=io.StringIO())
    ctx = made[-1]
    assert ctx.precision == 1 and len(ctx.cs.blocks) == 12 and ctx.steps == 3 and ctx.cs.viscous == 0
    driver.run(str(tmp_path / "input.canard"), out=io.StringIO(), precision=0, split=False, max_steps=2, viscous=1)
    ctx = made[-1]
    assert ctx.precision == 0 and len(ctx.cs.blocks) == 6 and ctx.steps == 2 and ctx.cs.viscous == 1
    with pytest.raises(namelist.NamelistError):
        driver.gpu_options(namelist.read(base + "\n&nml_gpu nprecision = 3 /\n"))
