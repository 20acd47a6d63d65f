"""A case's ranks placed on several devices (canard_b200.placement), with the
devices played by gloo processes on the CPU. Each process holds only the states
of its own ranks, receives the averaging sources that live on the other
processes through the plan's send lists, and applies the junction averaging
(average_point, average_line, average_surface: src/mo_domdcomp.f90:439-559,
src/mo_gcbc.f90:342-422) with the device kernels' arithmetic. Together the
processes must give the single-process result (canard_average_host) bit for
bit. Face links are checked as a partition of the reference's message pattern."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from canard_b200 import api, cases, placement


CASES = {
    "tgv_box": (lambda: cases.tgv(nx=26, ny=24, nz=26), [(2, 1, 2)]),
    "validation": (lambda: cases.reference_validation(48, 40, 12), [(2, 2, 1)]),
    "curv4": (lambda: cases.curvilinear_4block(40, 30, 28), [(2, 1, 2)] * 4),
    "toy": (lambda: cases.reference_toy(52, 26, 12), [(4, 2, 1)] * 6),
}


def free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def make_case(name):
    make, nbpc = CASES[name]
    cs = cases.decompose(make(), nbpc)
    rng = np.random.default_rng(len(cs.blocks))
    qa = [np.ascontiguousarray(q * (1 + 1e-3 * rng.standard_normal(q.shape))) for q in cs.qa]
    return cs, qa


def apply_pass(p, d, local, recv):
    """One averaging pass on device d: local[r] = rank r's (5, npts) state,
    recv = (n, 5) values from the other devices in slot order. Arithmetic as
    canard_average_host: a snapshot of every source first, then per target the
    mean of its sources (mode 0: ordered sum times 1/count) or the running
    average onto the point (mode 1), targets in plan order."""
    t = p.targets
    mine = np.flatnonzero(np.isin(t[:, 0], list(local)))
    snap = np.zeros((len(p.sources), 5))
    slot = p.slots[d]
    for ent in np.concatenate([np.arange(t[i, 2], t[i, 2] + t[i, 3]) for i in mine]) if len(mine) else []:
        r, l = p.sources[ent]
        snap[ent] = local[r][:, l] if slot[ent] < 0 else recv[slot[ent]]
    for i in mine:  # sequential: a point may be a target more than once
        r, l, first, count = t[i]
        src = snap[first:first + count]
        if p.mode == 0:
            acc = src[0].copy()
            for j in range(1, count):
                acc = acc + src[j]
            local[r][:, l] = (1.0 / float(count)) * acc
        else:
            x = local[r][:, l].copy()
            r1 = 1.0
            for j in range(count):
                r1 = r1 + 1.0
                r2 = 1.0 / r1
                x = r2 * ((r1 - 1.0) * x + src[j]) + 0.0 * x
            local[r][:, l] = x


def _worker(w, world, port, name, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=w, world_size=world)
    cs, qa = make_case(name)
    dev = placement.contiguous(cs, world)
    plan = placement.ExchangePlan(cs, dev)
    local = {r: qa[r].reshape(5, -1).copy() for r in np.flatnonzero(dev == w)}
    sent = 0
    for p in plan.passes:
        reqs = []
        for d in range(world):
            pts = p.sends.get((w, d))
            if d == w or pts is None:
                continue
            vals = np.stack([local[r][:, l] for r, l in pts]) if len(pts) else np.zeros((0, 5))
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(vals)), d))
            sent += vals.size
        parts = []
        for e in range(world):
            pts = p.sends.get((e, w))
            if e == w or pts is None:
                continue
            buf = torch.zeros((len(pts), 5), dtype=torch.float64)
            dist.recv(buf, e)
            parts.append(buf.numpy())
        for q in reqs:
            q.wait()
        recv = np.concatenate(parts) if parts else np.zeros((0, 5))
        apply_pass(p, w, local, recv)
    out.put((w, {int(r): v for r, v in local.items()}, sent))
    dist.barrier()
    dist.destroy_process_group()


def run_world(name, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(w, world, port, name, q)) for w in range(world)]
    for p in procs:
        p.start()
    got, sent = {}, 0
    for _ in range(world):
        w, loc, s = q.get(timeout=300)
        got.update(loc)
        sent += s
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return got, sent


@pytest.mark.parametrize("name,world", [("tgv_box", 2), ("curv4", 2), ("curv4", 3), ("toy", 3)])
def test_distributed_averaging_equals_the_single_process_plans(name, world):
    cs, qa = make_case(name)
    ref = api.average_host(cs, qa)
    got, sent = run_world(name, world)
    assert sorted(got) == list(range(len(cs.blocks)))
    for r in range(len(cs.blocks)):
        np.testing.assert_array_equal(got[r].reshape(-1), ref[r].reshape(-1), err_msg=f"rank {r}")
    plan = placement.ExchangePlan(cs, placement.contiguous(cs, world))
    assert sent == 5 * plan.summary()["averaging_remote_points"]
    assert sent > 0  # the placement does cut junctions


@pytest.mark.parametrize("name", list(CASES))
def test_face_links_are_the_reference_message_pattern(name):
    """Every interface or curved face of every rank receives from exactly one
    face, the one its neighbour entry names, over the same line count; the
    placement's crossing links are the links whose two ranks sit on different
    devices."""
    cs, _ = make_case(name)
    links = api.plan_export(cs, api.PLAN_FACES)
    want = set()
    for r, b in enumerate(cs.blocks):
        for d in range(3):
            for s in range(2):
                if b.nbc[d][s] in (30, 35, 40, 45):
                    want.add((r, d + 1, s))
    assert sorted(map(tuple, links[:, :3].tolist())) == sorted(want)
    for dst, nn, ds, src, ss, lines, code in links:
        assert cs.blocks[dst].mbcd[nn - 1][ds] == src and ss == 1 - ds
        assert code == cs.blocks[src].nbc[nn - 1][ss]
        ext = [(q.lxi + 1, q.let + 1, q.lze + 1) for q in (cs.blocks[src], cs.blocks[dst])]
        tr = [a for a in range(3) if a != nn - 1]
        assert lines == ext[0][tr[0]] * ext[0][tr[1]] and ext[0][tr[0]] == ext[1][tr[0]]
    for ndev in (2, 3):
        dev = placement.contiguous(cs, ndev)
        plan = placement.ExchangePlan(cs, dev)
        cross = {tuple(x) for x in plan.cross_links.tolist()}
        assert cross == {tuple(x) for x in links.tolist() if dev[x[0]] != dev[x[3]]}


def test_contiguous_placement_balances_points():
    cs = cases.decompose(cases.tgv(nx=64, ny=64, nz=64), [(1, 2, 4)])
    for ndev in (1, 2, 4, 8):
        dev = placement.contiguous(cs, ndev)
        assert sorted(set(dev.tolist())) == list(range(ndev))
        assert np.all(np.diff(dev) >= 0)  # runs of consecutive ranks
        pts = placement.rank_points(cs)
        load = np.array([pts[dev == d].sum() for d in range(ndev)])
        assert load.max() - load.min() <= pts.max()
    with pytest.raises(ValueError):
        placement.contiguous(cs, 9)


def test_bytes_of_one_zeta_cut():
    """TGV box split once along zeta on 2 devices: the periodic face and the
    sub-domain face each cross in both directions. Per crossing link and step:
    lines x (4 stages x 9 viscous fields x 2 values x 8 B + 5 filtered fields
    x 3 values x 8 B); averaging: the periodic face's points, 5 values per
    stage."""
    n = 32
    cs = cases.decompose(cases.tgv(nx=n, ny=n, nz=n), [(1, 1, 2)])
    plan = placement.ExchangePlan(cs, placement.contiguous(cs, 2))
    lines = (n + 1) ** 2
    assert len(plan.cross_links) == 4
    m = plan.bytes_per_step(viscous=True)
    per_link = lines * (4 * 9 * 2 * 8 + 5 * 3 * 8)
    avg_pts = sum(len(v) for p in plan.passes for (e, d), v in p.sends.items() if e == 0)
    assert m[0, 1] == 2 * per_link + 4 * 5 * 8 * avg_pts
    assert avg_pts >= lines  # the periodic face's points (and its edges and corners)
    m32 = plan.bytes_per_step(viscous=True, deriv_bytes=4)
    assert m[0, 1] - m32[0, 1] == 2 * lines * 4 * 9 * 2 * 4
    assert plan.bytes_per_step(viscous=False)[0, 1] == 2 * lines * (4 * 5 * 2 * 8 + 5 * 3 * 8) + 4 * 5 * 8 * avg_pts


def _mpigo_fields(cs):
    rng = np.random.default_rng(99)
    return [rng.standard_normal((b.lxi + 1) * (b.let + 1) * (b.lze + 1)) for b in cs.blocks]


def _recv(o, r, nt):
    """Rank r's receive buffers of the oracle, per direction (5 fields, 2 sides,
    2 or 3 values, lines)."""
    import pyoracle as po
    flat = o.get(r, po.A_RECV0 if nt == 0 else po.A_RECV1).reshape(-1)
    b = o.cs.blocks[r]
    out, at = [], 0
    for d in range(3):
        ext = [b.lxi + 1, b.let + 1, b.lze + 1]
        nb = ext[(d + 1) % 3] * ext[(d + 2) % 3]
        size = 5 * 2 * (2 + nt) * nb
        out.append(flat[at:at + size].reshape(5, 2, 2 + nt, nb))
        at += size
    return out


def _mpigo_worker(w, world, port, name, nt, out):
    import pyoracle as po
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=w, world_size=world)
    cs, _ = make_case(name)
    dev = placement.contiguous(cs, world)
    plan = placement.ExchangePlan(cs, dev)
    # this device's ranks only; the others' fields are unknown here
    f = [x if dev[r] == w else np.full_like(x, np.nan) for r, x in enumerate(_mpigo_fields(cs))]
    o = po.Oracle(cs, setup=False, threads=1)  # one process per device shares the cores
    m = 2
    o.mpigo(f, nt, 1, 0, 7, m)
    mine = {int(r): _recv(o, r, nt) for r in np.flatnonzero(dev == w)}
    reqs, sends = [], 0
    for dst, nn, ds, src, ss, lines, code in plan.cross_links:
        if code not in placement.INTERFACE_CODES:
            continue
        if dev[src] == w:  # computed here from this device's sender, owed to the receiver's device
            blk = np.ascontiguousarray(_recv(o, dst, nt)[nn - 1][m - 1, ds])
            reqs.append(dist.isend(torch.from_numpy(blk), int(dev[dst]), tag=int(dst * 6 + (nn - 1) * 2 + ds)))
            sends += 1
    for dst, nn, ds, src, ss, lines, code in plan.cross_links:
        if code in placement.INTERFACE_CODES and dev[dst] == w:
            buf = torch.zeros(mine[dst][nn - 1][m - 1, ds].shape, dtype=torch.float64)
            dist.recv(buf, int(dev[src]), tag=int(dst * 6 + (nn - 1) * 2 + ds))
            mine[dst][nn - 1][m - 1, ds] = buf.numpy()
    for q in reqs:
        q.wait()
    out.put((w, {r: [a.copy() for a in v] for r, v in mine.items()}, sends))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name,world,nt", [("tgv_box", 2, 0), ("curv4", 3, 1), ("toy", 2, 0)])
def test_distributed_interface_contractions(name, world, nt):
    """mpigo (src/mo_numerics.f90:429-705) with the ranks on gloo processes:
    each process forms the contractions of its own ranks' faces (the oracle
    stands in for the device kernel), sends those of the crossing links to the
    receiver's process, and then holds every receive buffer of its ranks as
    the single-process exchange fills it, bit for bit (derivative nt = 0 and
    filter nt = 1)."""
    import pyoracle as po
    cs, _ = make_case(name)
    o = po.Oracle(cs, setup=False)
    o.mpigo(_mpigo_fields(cs), nt, 1, 0, 7, 2)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_mpigo_worker, args=(w, world, port, name, nt, q)) for w in range(world)]
    for p in procs:
        p.start()
    got, sends = {}, 0
    for _ in range(world):
        _, loc, s = q.get(timeout=300)
        got.update(loc)
        sends += s
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sends > 0
    for r in range(len(cs.blocks)):
        want = _recv(o, r, nt)
        for d in range(3):
            np.testing.assert_array_equal(got[r][d][1], want[d][1], err_msg=f"rank {r} direction {d + 1}")


def _emulate(cs, qa, dev):
    """The devices of a placement one after the other in this process: each
    gets exactly its plan's send lists from the others' pre-pass states."""
    plan = placement.ExchangePlan(cs, dev)
    local = [{r: qa[r].reshape(5, -1).copy() for r in np.flatnonzero(dev == d)} for d in range(plan.ndev)]
    for p in plan.passes:
        recv = []
        for d in range(plan.ndev):
            parts = [np.stack([local[e][r][:, l] for r, l in p.sends[(e, d)]])
                     for e in range(plan.ndev) if e != d and (e, d) in p.sends]
            recv.append(np.concatenate(parts) if parts else np.zeros((0, 5)))
        for d in range(plan.ndev):
            apply_pass(p, d, local[d], recv[d])
    out = {}
    for loc in local:
        out.update(loc)
    return out


@pytest.mark.parametrize("seed", range(6))
def test_random_splits_and_placements(seed):
    """Random box sizes, splits and device counts (periodic TGV boxes and the
    4-block curvilinear case): the placed averaging equals the single-process
    plans bit for bit, and the crossing links are exactly the links between
    devices."""
    rng = np.random.default_rng(seed)
    if seed % 2 == 0:
        nbpc = [tuple(int(v) for v in rng.integers(1, 4, 3))]
        n = [int(26 + rng.integers(0, 8)) * k for k in nbpc[0]]
        base = cases.tgv(nx=max(n[0], 16), ny=max(n[1], 16), nz=max(n[2], 16))
    else:
        nbpc = [tuple(int(v) for v in rng.integers(1, 3, 3))] * 4
        base = cases.curvilinear_4block(44, 30, 28)
    cs = cases.decompose(base, nbpc)
    qa = [np.ascontiguousarray(q * (1 + 1e-3 * rng.standard_normal(q.shape))) for q in cs.qa]
    ndev = int(rng.integers(1, min(len(cs.blocks), 5) + 1))
    dev = placement.contiguous(cs, ndev) if seed < 4 else rng.permutation(np.arange(len(cs.blocks)) % ndev)
    got = _emulate(cs, qa, np.asarray(dev))
    ref = api.average_host(cs, qa)
    for r in range(len(cs.blocks)):
        np.testing.assert_array_equal(got[r].reshape(-1), ref[r].reshape(-1), err_msg=f"rank {r}")


def _stage_before_gcbc(cs):
    """An oracle one step into the case, then stage 1 up to the GCBC update
    (primitives, time step, viscous stresses, fluxes)."""
    import pyoracle as po
    o = po.Oracle(cs, threads=1)
    o.step(1)
    for ph in (po.PH_FILTER, po.PH_COPYQO, po.PH_PRIM, po.PH_TIMESTEP, po.PH_VISCOUS, po.PH_FLUXES):
        o.phase(ph, 1)
    return o


def _gcbc_worker(w, world, port, name, out):
    import pyoracle as po
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=w, world_size=world)
    cs, _ = make_case(name)
    dev = placement.contiguous(cs, world)
    plan = placement.ExchangePlan(cs, dev)
    o = _stage_before_gcbc(cs)
    # this device knows nothing of the other devices' ranks from here on
    for r in np.flatnonzero(dev != w):
        for a in (po.A_QA, po.A_DE, po.A_P) + po.A_DRVA:
            o.set(int(r), a, np.full(o.get(int(r), a).size, np.nan))
    o.phase(po.PH_GCBC_SETUP, 1)
    curved = [x for x in plan.cross_links.tolist() if x[6] == placement.CURVED_CODE]
    reqs = []
    for dst, nn, ds, src, ss, lines, code in curved:
        if dev[src] == w:  # the sender's characteristic values, (5, lines) of its side
            drva = o.get(src, po.A_DRVA[nn - 1]).reshape(2, 5, lines)
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(drva[ss])), int(dev[dst]),
                                   tag=int(dst * 6 + (nn - 1) * 2 + ds)))
    for dst, nn, ds, src, ss, lines, code in curved:
        if dev[dst] == w:  # into this device's mirror of the remote sender
            buf = torch.zeros((5, lines), dtype=torch.float64)
            dist.recv(buf, int(dev[src]), tag=int(dst * 6 + (nn - 1) * 2 + ds))
            drva = o.get(src, po.A_DRVA[nn - 1]).reshape(2, 5, lines)
            drva[ss] = buf.numpy()
            o.set(src, po.A_DRVA[nn - 1], drva.reshape(-1))
    for q in reqs:
        q.wait()
    o.phase(po.PH_GCBC_COMM_UPDATE, 1)
    out.put((w, {int(r): o.get(int(r), po.A_DE) for r in np.flatnonzero(dev == w)}, len(reqs)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_gcbc_exchange(world):
    """gcbc_comm (src/mo_gcbc.f90:186-220) with the ranks on gloo processes: each
    process forms the characteristic values (drva) of its own ranks' faces, the
    crossing curved-interface links carry them to the receiver's process, and
    the GCBC update of every rank then equals the single-process phase bit for
    bit (the 4-block curvilinear case, split 2 x 1 x 2 per block)."""
    import pyoracle as po
    cs, _ = make_case("curv4")
    o = _stage_before_gcbc(cs)
    o.phase(po.PH_GCBC, 1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_gcbc_worker, args=(w, world, port, "curv4", q)) for w in range(world)]
    for p in procs:
        p.start()
    got, sends = {}, 0
    for _ in range(world):
        _, loc, s = q.get(timeout=300)
        got.update(loc)
        sends += s
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sends > 0
    for r in range(len(cs.blocks)):
        np.testing.assert_array_equal(got[r], o.get(r, po.A_DE), err_msg=f"rank {r}")


class _DeviceHook:
    """Exchange hook of one process holding the ranks of one device: at each
    point where the single-process oracle reads another rank's data it moves
    exactly what the placement's plan says crosses devices, and no more. The
    other devices' ranks are mirrors whose state is NaN."""

    def __init__(self, o, plan, w):
        import pyoracle as po
        self.po, self.o, self.plan, self.w = po, o, plan, w
        self.dev = plan.device
        self.rounds = 0

    def _swap(self, items):
        """items: (src rank, dst rank, tag, get(), put(value)) of crossing
        pieces; sends those this device owns, receives those it needs."""
        reqs = []
        for src, dst, tag, get, _ in items:
            if self.dev[src] == self.w and self.dev[dst] != self.w:
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(get())), int(self.dev[dst]), tag=tag))
        for src, dst, tag, get, put in items:
            if self.dev[dst] == self.w and self.dev[src] != self.w:
                buf = torch.from_numpy(np.zeros_like(get()))
                dist.recv(buf, int(self.dev[src]), tag=tag)
                put(buf.numpy())
        for q in reqs:
            q.wait()
        self.rounds += 1

    def __call__(self, kind, a, b, data):
        po, o = self.po, self.o
        links = self.plan.cross_links
        if kind == 0:  # mpigo: the receiver's buffer slot, filled on the sender's device
            nt, m, which = a, b, (po.A_RECV0 if a == 0 else po.A_RECV1)
            cache = {}

            def buf(r):
                if r not in cache:
                    cache[r] = o.get(r, which)
                return cache[r]

            def slot(r, nn, side):
                blk = o.cs.blocks[r]
                ext = [blk.lxi + 1, blk.let + 1, blk.lze + 1]
                sizes = [5 * 2 * (2 + nt) * ext[(d + 1) % 3] * ext[(d + 2) % 3] for d in range(3)]
                at = sum(sizes[:nn - 1])
                return buf(r)[at:at + sizes[nn - 1]].reshape(5, 2, 2 + nt, -1)[m - 1, side]

            items = []
            for dst, nn, ds, src, ss, lines, code in links.tolist():
                if code in placement.INTERFACE_CODES:
                    def put(v, dst=dst, nn=nn, ds=ds):
                        slot(dst, nn, ds)[...] = v
                    items.append((src, dst, dst * 6 + (nn - 1) * 2 + ds, lambda dst=dst, nn=nn, ds=ds: slot(dst, nn, ds),
                                  put))
            self._swap(items)
            for r in cache:
                if self.dev[r] == self.w:
                    o.set(r, which, cache[r])
        elif kind == 1:  # gcbc_comm: the sender's drva, into this device's mirror of it
            items = []
            for dst, nn, ds, src, ss, lines, code in links.tolist():
                if code != placement.CURVED_CODE:
                    continue

                def get(src=src, nn=nn, ss=ss, lines=lines):
                    return o.get(src, po.A_DRVA[nn - 1]).reshape(2, 5, lines)[ss]

                def put(v, src=src, nn=nn, ss=ss, lines=lines):
                    d = o.get(src, po.A_DRVA[nn - 1]).reshape(2, 5, lines)
                    d[ss] = v
                    o.set(src, po.A_DRVA[nn - 1], d.reshape(-1))
                items.append((src, dst, dst * 6 + (nn - 1) * 2 + ds, get, put))
            self._swap(items)
        elif kind == 2:  # an averaging pass: the remote sources, into the mirrors
            p = self.plan.passes[a]
            reqs = []
            for (e, d), pts in p.sends.items():
                if e == self.w:
                    q = {r: o.get(int(r), po.A_QA).reshape(5, -1) for r in np.unique(pts[:, 0])}
                    vals = np.stack([q[r][:, l] for r, l in pts])
                    reqs.append(dist.isend(torch.from_numpy(vals), int(d), tag=100 + a))
            for (e, d), pts in p.sends.items():
                if d == self.w:
                    buf = torch.zeros((len(pts), 5), dtype=torch.float64)
                    dist.recv(buf, int(e), tag=100 + a)
                    for r in np.unique(pts[:, 0]):
                        q = o.get(int(r), po.A_QA).reshape(5, -1)
                        sel = pts[:, 0] == r
                        q[:, pts[sel, 1]] = buf.numpy()[sel].T
                        o.set(int(r), po.A_QA, q.reshape(-1))
            for q in reqs:
                q.wait()
            self.rounds += 1
        elif kind == 3:  # the time step's maxima: this device's ranks, then MAX over devices
            n = len(data) // 2
            mine = self.dev == self.w
            t = torch.tensor([data[:n][mine].max(), data[n:][mine].max()], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            data[:n] = t[0].item()
            data[n:] = t[1].item()
            self.rounds += 1


def _step_worker(w, world, port, name, steps, out):
    import pyoracle as po
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=w, world_size=world)
    cs, qa = make_case(name)
    dev = placement.contiguous(cs, world)
    plan = placement.ExchangePlan(cs, dev)
    o = po.Oracle(cs, threads=1)
    for r in range(len(cs.blocks)):
        o.set_state(r, qa[r] if dev[r] == w else np.full_like(qa[r], np.nan))
    hook = _DeviceHook(o, plan, w)
    o.set_hook(hook)
    o.step(steps)
    o.set_hook(None)
    out.put((w, {int(r): o.state(int(r)) for r in np.flatnonzero(dev == w)}, hook.rounds))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("tgv_box", 2), ("curv4", 3), ("toy", 3), ("validation", 2)])
def test_distributed_time_steps(name, world):
    """Whole time steps with the ranks on gloo processes: each process holds
    the state of its own device's ranks only (the others are NaN), and the
    plan's exchanges (interface contractions, curved-interface drva, averaging
    sources, the time step's maxima) are all that crosses between processes.
    After 4 steps every rank equals the single-process run bit for bit."""
    import pyoracle as po
    cs, qa = make_case(name)
    o = po.Oracle(cs)
    for r in range(len(cs.blocks)):
        o.set_state(r, qa[r])
    o.step(4)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_step_worker, args=(w, world, port, name, 4, q)) for w in range(world)]
    for p in procs:
        p.start()
    got, rounds = {}, []
    for _ in range(world):
        _, loc, n = q.get(timeout=600)
        got.update(loc)
        rounds.append(n)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert len(set(rounds)) == 1 and rounds[0] > 0  # every process took the same exchange steps
    for r in range(len(cs.blocks)):
        assert np.all(np.isfinite(got[r]))
        np.testing.assert_array_equal(got[r], o.state(r), err_msg=f"rank {r}")
