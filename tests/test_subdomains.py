"""Sub-domains (nbpc > 1) in the CPU oracle: the reference's decomposition of
blocks into ranks (domdcomp_init, src/mo_domdcomp.f90:85-232) with code-40
faces between them, and its junction search over the blocks with the owner
tests and rank numbering of search_point / search_line (src/mo_domdcomp.f90:
269-437, 588-605)."""
import numpy as np
import pytest

import pyoracle as po
from canard_b200 import cases


def test_one_subdomain_per_block_is_the_plain_case():
    cs = cases.curvilinear_4block(24, 16, 14)
    d = cases.decompose(cs, [(1, 1, 1)] * 4)
    assert [(b.lxi, b.let, b.lze, b.nbc, b.mbcd) for b in d.blocks] == \
        [(b.lxi, b.let, b.lze, [list(x) for x in b.nbc], [list(x) for x in b.mbcd]) for b in cs.blocks]
    a, b = po.Oracle(cs), po.Oracle(d)
    a.step(4)
    b.step(4)
    for m in range(4):
        np.testing.assert_array_equal(b.state(m), a.state(m))


def test_decomposition_bookkeeping():
    cs = cases.curvilinear_4block(40, 30, 28)
    nbpc = [(2, 1, 2), (2, 1, 2), (2, 1, 2), (2, 1, 2)]
    d = cases.decompose(cs, nbpc)
    assert len(d.blocks) == 16
    # the ranks tile their block
    for m, b in enumerate(cs.blocks):
        cover = np.zeros(b.shape, int)
        for (mm, *_), sl in zip(d.sub["ranks"], d.sub["slices"]):
            if mm == m:
                cover[sl[0]:sl[0] + sl[3], sl[1]:sl[1] + sl[4], sl[2]:sl[2] + sl[5]] += 1
        assert np.all(cover == 1)
    # neighbours point back with a matching face: code 40 between sub-domains
    for r, b in enumerate(d.blocks):
        for dd in range(3):
            for s in range(2):
                nb = b.mbcd[dd][s]
                if nb < 0:
                    continue
                assert d.blocks[nb].mbcd[dd][1 - s] == r
                assert d.blocks[nb].nbc[dd][1 - s] == b.nbc[dd][s]
                tr = [x for x in range(3) if x != dd]
                ext = lambda q: [(q.lxi, q.let, q.lze)[x] for x in tr]
                assert ext(d.blocks[nb]) == ext(b)
    np.testing.assert_array_equal(cases.compose(d.sub, d.qa)[2], cs.qa[2])
    with pytest.raises(ValueError):
        cases.decompose(cases.tgv(nx=24, ny=20, nz=16), [(2, 2, 2)])  # 12-point sub-domains
    with pytest.raises(ValueError, match="shared face"):  # blocks 0 and 1 meet along xi, split along eta
        cases.decompose(cs, [(1, 2, 1), (1, 1, 1), (1, 1, 1), (1, 1, 1)])


def split_vs_plain(cs, nbpc, steps):
    d = cases.decompose(cs, nbpc)
    o = po.Oracle(d)
    o.step(steps)
    q = cases.compose(d.sub, [o.state(r) for r in range(len(d.blocks))])
    a = po.Oracle(cs)
    a.step(steps)
    rels = []
    for m in range(len(cs.blocks)):
        assert np.isfinite(q[m]).all()
        ref = a.state(m)
        rels.append(float(np.linalg.norm((q[m] - ref).ravel()) / np.linalg.norm(ref.ravel())))
    return rels


@pytest.mark.parametrize("make,nbpc,steps", [
    # periodic box split 2 x 2 x 2: every corner, edge and face junction of the
    # box is shared by sub-domains of different ranks
    (lambda: cases.tgv(nx=48, ny=40, nz=32), [(2, 2, 2)], 6),
    # run/exp.validation's block (GCBC on four faces) split 2 x 2 x 1, like its input
    (lambda: cases.reference_validation(48, 40, 12), [(2, 2, 1)], 8),
    # run/exp.toy's six blocks split 4 x 2 x 1 each (48 ranks), like its input
    (lambda: cases.reference_toy(52, 26, 12), [(4, 2, 1)] * 6, 4),
])
def test_split_runs_stay_close_to_one_subdomain_per_block(make, nbpc, steps):
    """The split changes the scheme only at the code-40 faces, whose interface
    closures replace the coupled rows: the states stay close to the unsplit
    run's (and a wrong junction pairing would not)."""
    rels = split_vs_plain(make(), nbpc, steps)
    print("split vs one sub-domain per block, relative L2:", rels)
    assert max(rels) < 1e-5 and min(rels) > 0, rels


def _nonperiodic():
    blk = cases.BlockSpec(23, 18, 16, [[10, 10], [10, 10], [45, 45]], [[-1, -1], [-1, -1], [0, 0]])
    Z, Y, X = blk.shape
    Zz, Yy, Xx = np.meshgrid(np.linspace(0, 1, Z), np.linspace(-0.8, 0.9, Y), np.linspace(-1, 1, X), indexing="ij")
    rho, u, v, w, p = cases.vortex_state(Xx, Yy, 0.3, 3.0, 0.3)
    return cases.CaseSpec([blk], viscous=1, reoo=2000.0, xyz=[np.stack([Xx, Yy, Zz])],
                          qa=[cases._conserved(rho, u, v, w, p)])


def _walls():
    blk = cases.BlockSpec(22, 18, 16, [[10, 25], [25, 20], [45, 45]], [[-1, -1], [-1, -1], [0, 0]])
    Z, Y, X = blk.shape
    Zz, Yy, Xx = np.meshgrid(np.linspace(0, 1, Z), np.linspace(0, 1.2, Y), np.linspace(-1, 1, X), indexing="ij")
    rho, u, v, w, p = cases.vortex_state(Xx, Yy, 0.0, 2.0, 0.3, 0.0, 0.6)
    return cases.CaseSpec([blk], viscous=1, reoo=2000.0, amach=(0.3, 0.0, 0.0), xyz=[np.stack([Xx, Yy, Zz])],
                          qa=[cases._conserved(rho, u, v, w, p)])


@pytest.mark.parametrize("make,nbpc", [
    (lambda: cases.tgv(nx=24, ny=20, nz=16), None),
    (lambda: cases.tgv(64), None),
    (lambda: cases.curvilinear_4block(24, 16, 14), None),
    (lambda: cases.reference_toy(16, 14, 12), None),
    (lambda: cases.reference_validation(24, 20, 12), None),
    (_nonperiodic, None),
    (_walls, None),
    (lambda: cases.batched(4, lo=16, hi=24)[1], None),
    (lambda: cases.tgv(nx=48, ny=40, nz=32), [(2, 2, 2)]),
    (lambda: cases.reference_validation(48, 40, 12), [(2, 2, 1)]),
    (lambda: cases.reference_toy(52, 26, 12), [(4, 2, 1)] * 6),
    (lambda: cases.curvilinear_4block(40, 30, 28), [(2, 1, 2)] * 4),
])
def test_device_averaging_plans_match_the_oracle(make, nbpc):
    """The device's junction-averaging plans (point, line, surface), built by
    the library's plan builder and applied on the host with the device's
    arithmetic, give the oracle's averaging phase bit for bit, for plain and
    split cases."""
    from canard_b200 import api
    cs = make()
    if nbpc:
        cs = cases.decompose(cs, nbpc)
    rng = np.random.default_rng(len(cs.blocks))
    qa = [q * (1 + 1e-3 * rng.standard_normal(q.shape)) for q in cs.qa]
    o = po.Oracle(cs)
    for r, q in enumerate(qa):
        o.set_state(r, q)
    o.phase(po.PH_AVERAGE, 1)
    got = api.average_host(cs, qa)
    for r in range(len(cs.blocks)):
        np.testing.assert_array_equal(got[r].reshape(-1), o.state(r).reshape(-1), err_msg=f"rank {r}")
