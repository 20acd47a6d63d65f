"""Grid files in the reference's record format (read_grid_parallel,
src/mo_io.f90:151-180; the generators' writes, src/mo_gridgen.f90:536-570)
through the C ABI, and the reference's own generators and initial condition
(gridtoy, gridtoy_multi, initialo), on the CPU."""
import math

import numpy as np
import pytest

from canard_b200 import api, cases


def record_bytes(xyz):
    """One 24-byte record (x, y, z) per point, i fastest: the plane records
    of the generators laid end to end."""
    g = np.asarray(xyz, np.float64).reshape(3, -1)
    return np.ascontiguousarray(g.T).tobytes()


def test_file_name():
    assert api.grid_name(0) == "misc/grid000.dat"
    assert api.grid_name(12) == "misc/grid012.dat"
    assert len(api.grid_name(999)) == 16  # character(16), no truncation


@pytest.mark.parametrize("shape", [(13, 13, 13), (17, 20, 31)])
def test_write_matches_the_record_layout_and_reads_back(tmp_path, shape):
    rng = np.random.default_rng(sum(shape))
    xyz = rng.standard_normal((3,) + shape)
    p = str(tmp_path / "g.dat")
    api.write_grid_file(p, xyz)
    assert open(p, "rb").read() == record_bytes(xyz)
    back = api.read_grid_file(p, int(np.prod(shape)))
    np.testing.assert_array_equal(back, xyz.reshape(3, -1))


def test_wrong_size_or_missing_file_is_an_io_error(tmp_path):
    xyz = np.zeros((3, 100))
    p = str(tmp_path / "g.dat")
    api.write_grid_file(p, xyz)
    for path, n in ((p, 99), (str(tmp_path / "absent.dat"), 100)):
        with pytest.raises(api.CanardError) as e:
            api.read_grid_file(path, n)
        assert e.value.code == api.ERR_IO


def test_gridtoy_coordinates():
    g = cases.gridtoy(50, 40, 16, 0.5, 1.0, 0.5, 0.1)
    assert g.shape == (3, 17, 41, 51)
    np.testing.assert_allclose(g[0, 0, 0, [0, 50]], [-0.5, 1.0], rtol=0, atol=1e-15)
    np.testing.assert_allclose(g[1, 0, [0, 40], 0], [-0.5, 0.5], rtol=0, atol=1e-15)
    # z runs from +span/2 at k = 0 down to -span/2
    np.testing.assert_allclose(g[2, [0, 16], 0, 0], [0.05, -0.05], rtol=0, atol=1e-15)
    assert np.all(np.diff(g[0], axis=2) > 0) and np.all(np.diff(g[2], axis=0) < 0)


def test_gridtoy_multi_blocks_share_their_interface_points():
    lxi0, lxi1, lxi2, let0 = 20, 14, 17, 12
    blocks = cases.gridtoy_multi(lxi0, lxi1, lxi2, let0, 12, 0.5, 1.0, 0.5, 0.1)
    assert [b.shape[3] - 1 for b in blocks] == [lxi0, lxi1, lxi2] * 2
    assert all(b.shape[1:3] == (13, let0 + 1) for b in blocks)
    for r in (0, 3):  # along x within a row
        for a, b in ((r, r + 1), (r + 1, r + 2)):
            np.testing.assert_array_equal(blocks[a][:, :, :, -1], blocks[b][:, :, :, 0])
    for a in range(3):  # the rows meet at y = 0
        np.testing.assert_array_equal(blocks[a][:, :, -1, :], blocks[a + 3][:, :, 0, :])
    np.testing.assert_allclose(blocks[0][0, 0, 0, 0], -0.5, atol=1e-15)
    np.testing.assert_allclose(blocks[2][0, 0, 0, -1], 1.0, atol=1e-14)
    np.testing.assert_allclose(blocks[3][1, 0, -1, 0], 0.5, atol=1e-15)


def test_initialo_is_the_reference_vortex():
    xyz = cases.gridtoy(30, 30, 12, 0.5, 1.0, 0.5, 0.1)
    q = cases.initialo(xyz)
    x, y = xyz[0], xyz[1]
    ao = 1.0 / (2 * math.pi) * np.sqrt(np.exp(1 - 12.5 ** 2 * (x ** 2 + y ** 2)))
    rho = (1 - 0.2 * ao ** 2) ** 2.5
    np.testing.assert_allclose(q[0], rho, rtol=1e-15)
    np.testing.assert_allclose(q[1], rho * 12.5 * y * ao, rtol=1e-14, atol=1e-16)
    np.testing.assert_allclose(q[2], -rho * 12.5 * x * ao, rtol=1e-14, atol=1e-16)
    assert np.all(q[3] == 0)
    ke = 0.5 * (q[1] ** 2 + q[2] ** 2) / q[0]
    np.testing.assert_allclose(q[4], rho ** 1.4 / (1.4 * 0.4) + ke, rtol=1e-14)


def test_reference_cases_build():
    v = cases.reference_validation(24, 20, 12)
    assert len(v.blocks) == 1 and v.xyz[0].shape == (3, 13, 21, 25)
    t = cases.reference_toy(16, 14, 12)
    assert len(t.blocks) == 6
    for m, b in enumerate(t.blocks):
        for d in range(3):
            for s in range(2):
                nb = b.mbcd[d][s]
                if nb >= 0:  # the neighbour points back, with the same code
                    assert t.blocks[nb].mbcd[d][1 - s] == m
                    assert t.blocks[nb].nbc[d][1 - s] == b.nbc[d][s]
