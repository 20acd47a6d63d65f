"""Restart files in the reference's record format (src/mo_io.f90:184-271) and
the dcanard comparer (contrib/dcanard.f90:100-126), through the C ABI, on the
CPU: the format is pinned against an independent numpy restatement of the
record layout."""
import os

import numpy as np
import pytest

from canard_b200 import api


def numpy_restart_bytes(time6, qa):
    """Direct-access records of 5 float64: (n, ndt, dt, dts, dte), (timo, 0, 0,
    0, 0), then qa(l, 1..5) per point l."""
    head = np.array([time6[0], time6[1], time6[2], time6[3], time6[4], time6[5], 0, 0, 0, 0], np.float64)
    return head.tobytes() + np.ascontiguousarray(qa.T, np.float64).tobytes()


def sample(npts, seed):
    rng = np.random.default_rng(seed)
    qa = rng.standard_normal((5, npts))
    t6 = np.array([1234.0, 1200.0, 2.5e-3, 2.0e-3, 3.0e-3, 7.125])
    return t6, qa


def test_file_name_is_the_reference_truncation():
    # 'misc/restartz000.dat' assigned to character(19)
    assert api.restart_name(0) == "misc/restartz000.da"
    assert api.restart_name(7) == "misc/restartz007.da"


@pytest.mark.parametrize("npts", [1, 17 * 13 * 9, 5000])
def test_write_matches_the_record_layout_and_reads_back(tmp_path, npts):
    t6, qa = sample(npts, npts)
    p = str(tmp_path / "r.da")
    api.write_restart_file(p, t6, qa)
    assert open(p, "rb").read() == numpy_restart_bytes(t6, qa)
    t, q = api.read_restart_file(p, npts)
    np.testing.assert_array_equal(t, t6)
    np.testing.assert_array_equal(q, qa)


def test_reads_a_file_written_by_the_layout(tmp_path):
    t6, qa = sample(999, 3)
    p = tmp_path / "ref.da"
    p.write_bytes(numpy_restart_bytes(t6, qa))
    t, q = api.read_restart_file(str(p), 999)
    np.testing.assert_array_equal(t, t6)
    np.testing.assert_array_equal(q, qa)


def test_wrong_size_or_missing_file_is_an_io_error(tmp_path):
    t6, qa = sample(100, 1)
    p = str(tmp_path / "r.da")
    api.write_restart_file(p, t6, qa)
    for path, n in ((p, 99), (str(tmp_path / "absent.da"), 100)):
        with pytest.raises(api.CanardError) as e:
            api.read_restart_file(path, n)
        assert e.value.code == api.ERR_IO


def test_compare_reports_like_dcanard(tmp_path):
    npts = 50
    t6, qa = sample(npts, 9)
    qa[0, 3] = 1.0
    qb = qa.copy()
    qb[0, 3] = 1.0 + 2.0 ** -40        # relative 9.1e-13
    qb[4, 10] = qa[4, 10] * (1 + 1e-9)
    qb[2, 0] = qa[2, 0]                 # unchanged
    qa[1, 5] = 0.0
    qb[1, 5] = 0.0                      # 0/0: no line
    p1, p2, rep = (str(tmp_path / f) for f in ("a.da", "b.da", "report.dat"))
    api.write_restart_file(p1, t6, qa)
    api.write_restart_file(p2, t6, qb)
    assert api.compare_restart(p1, p1, npts, 1e-15) == 0
    assert api.compare_restart(p1, p2, npts, 1e-15, report=rep) == 2
    assert api.compare_restart(p1, p2, npts, 1e-10) == 1
    lines = open(rep).read().splitlines()
    assert len(lines) == 2
    # variable 1 first (j outer), Fortran (a,i8,a,i8,a,e15.7,...) fields
    assert lines[0].startswith(" i=       3 j=       1 v1=  0.1000000E+01 v2=  0.1000000E+01 abs=  0.9094947E-12")
    assert lines[1].startswith(" i=      10 j=       5 v1=")
    # a value of the first file equal to zero against a non-zero one is reported
    qc = qa.copy()
    qc[1, 5] = 1e-3
    api.write_restart_file(p2, t6, qc)
    assert api.compare_restart(p1, p2, npts, 1e-15) == 1


def test_fortran_e_format_of_negative_and_small_values(tmp_path):
    t6 = np.zeros(6)
    qa = np.zeros((5, 1))
    qb = np.zeros((5, 1))
    qa[0, 0], qb[0, 0] = -2.5e-3, -2.0e-3
    p1, p2, rep = (str(tmp_path / f) for f in ("a.da", "b.da", "r.dat"))
    api.write_restart_file(p1, t6, qa)
    api.write_restart_file(p2, t6, qb)
    assert api.compare_restart(p1, p2, 1, 0.0, report=rep) == 1
    line = open(rep).read().splitlines()[0]
    assert line == (" i=       0 j=       1 v1= -0.2500000E-02 v2= -0.2000000E-02 abs=  0.5000000E-03"
                    " rel=  0.2000000E+00")


def test_dcanard_command_compares_every_block(tmp_path, monkeypatch):
    """python -m canard_b200.dcanard: block sizes from input.canard, one report
    file per block under output/, the reference's summary line per block."""
    import io
    from canard_b200 import dcanard
    inp = ("&nml_driver\nmbk = 1\n/\n&nml_domdcomp\nlximb = 12, 13\nletmb = 12, 12\nlzemb = 12, 14\n/\n")
    (tmp_path / "input.canard").write_text(inp)
    sizes = [13 * 13 * 13, 14 * 13 * 15]
    for d in ("a", "b"):
        (tmp_path / d / "misc").mkdir(parents=True)
    for mb, npts in enumerate(sizes):
        t6, qa = sample(npts, 40 + mb)
        qb = qa.copy()
        if mb == 1:
            qb[2, 5] *= 1 + 1e-9
            qb[4, 7] *= 1 + 1e-12
        api.write_restart_file(str(tmp_path / "a" / api.restart_name(mb)), t6, qa)
        api.write_restart_file(str(tmp_path / "b" / api.restart_name(mb)), t6, qb)
    monkeypatch.chdir(tmp_path)
    out = io.StringIO()
    n = dcanard.compare("a", "b", 1e-15, out=out)
    assert n == 2
    lines = out.getvalue().splitlines()
    assert lines[-2] == "Compared %8d elements for %8d variables in block %8d" % (sizes[0], 5, 0)
    assert lines[-1] == "Compared %8d elements for %8d variables in block %8d" % (sizes[1], 5, 1)
    assert (tmp_path / "output" / "restart0.dat").read_text() == ""
    rep = (tmp_path / "output" / "restart1.dat").read_text().splitlines()
    assert len(rep) == 2 and rep[0].startswith(" i=       5 j=       3") and rep[1].startswith(" i=       7 j=       5")
    assert dcanard.compare("a", "b", 1e-10, out=io.StringIO()) == 1
    assert dcanard.compare("a", "b", 1e-8, out=io.StringIO()) == 0
    assert dcanard.main(["-d", "a", "b", "-t", "1e-15"]) == 0
