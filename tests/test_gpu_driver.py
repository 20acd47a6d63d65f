"""The reference's program on the device path (canard_b200.driver): a small
copy of run/exp.validation read from its input file, run to tmax with two
outputs and a final restart file, then continued from that restart."""
import io
import os

import numpy as np
import pytest

from canard_b200 import api, cases, driver

pytestmark = pytest.mark.gpu

INPUT = """&nml_driver
nio = 0
mbk = 0
ndata = 2
/
&nml_canard
nts = {nts}
nrestart = 1
cfl = 1.4e0
tmax = {tmax!r}
ltimer = .true.
/
&nml_domdcomp
nbpc(:,1) = 2
nbpc(:,2) = 2
nbpc(:,3) = 1
lximb = 24
letmb = 20
lzemb = 12
nbbc(0,1,:) = 10,10
nbbc(0,2,:) = 10,10
nbbc(0,3,:) = 45,45
mbcd(0,1,:) = -1,-1
mbcd(0,2,:) = -1,-1
mbcd(0,3,:) =  0,0
/
&nml_numerics
fltk = 0.65e0
fltrbc = 0.9e0
/
&nml_physics
reoo = 500000.0e0
tempoo = 300.0e0
amach1 = 0.3e0
amach2 = 0.0e0
amach3 = 0.0e0
timf = 0.0e0
nsmf = 1
/
&nml_gridgen
gridtype = 0
lxi0 = 24
let0 = 20
lze0 = 12
doml0 = 0.5e0
doml1 = 1.0e0
domh = 0.5e0
span = 0.1e0
szth0 = 0.0e0
szth1 = 0.6e0
/
"""


def test_driver_runs_the_validation_input(tmp_path):
    cs = cases.reference_validation(24, 20, 12)
    a = api.Context(cs)
    a.step(8)
    tmax = float(a.time()[5])  # the time after 8 steps: the run stops exactly there
    q8 = a.state(0)
    a.step(3)
    t11 = float(a.time()[5])
    a.step(1)
    # within the 12th step: robust to the last-bit differences of the restart
    tmax2 = 0.5 * (t11 + float(a.time()[5]))
    q12 = a.state(0)
    a.close()
    inp = tmp_path / "input.canard"
    inp.write_text(INPUT.format(nts=0, tmax=tmax))
    log = io.StringIO()
    res = driver.run(str(inp), out=log)
    text = log.getvalue()
    assert "nbpc > 1" in text and "Canard: Finished." in text and "Overflow" not in text
    assert res["steps"] == 8 and res["n"] == 8 and res["time"] == tmax
    # the grid at start, then ndata + 1 outputs: at time 0 (the first step, the
    # output counter starts at -1), tmax/2 and tmax
    assert res["outputs"] == ["data/grid.plt", "data/n000.plt", "data/n001.plt", "data/n002.plt"]
    for f in res["outputs"] + [api.restart_name(0)]:
        assert os.path.getsize(tmp_path / f) > 0, f
    t6, q = api.read_restart_file(str(tmp_path / api.restart_name(0)), cs.blocks[0].npts)
    assert t6[0] == 8 and t6[5] == tmax
    np.testing.assert_array_equal(q.reshape(q8.shape), q8)
    # continue from the restart file into the 12th step
    inp.write_text(INPUT.format(nts=1, tmax=tmax2))
    res2 = driver.run(str(inp), out=io.StringIO())
    assert res2["n"] == 12 and res2["steps"] == 4
    _, q = api.read_restart_file(str(tmp_path / api.restart_name(0)), cs.blocks[0].npts)
    # the filter's interface send chain restarts afresh, as in the reference
    rel = np.linalg.norm((q.reshape(q12.shape) - q12).ravel()) / np.linalg.norm(q12.ravel())
    assert rel < 1e-13, rel
