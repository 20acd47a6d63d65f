"""The reference's program, on the device path: reads ``input.canard``, builds
the blocks and their grid with the reference's generators, starts from
``initialo`` or a restart file, and runs the time loop of canard_driver
(src/mo_canard_driver.f90:34-459) with its stop rule, output schedule,
time-averaged recording, Tecplot files and final restart file, in the
reference's file formats and names under the run directory:

* ``data/grid.plt`` at start, ``data/nNNN.plt`` at each of the ``ndata``
  output times (``ndata < 0``: no output);
* ``misc/restartzNNN.da`` per block at the end when ``nrestart == 1``; a run
  with ``nts != 0`` starts from these files.

The output files are written by a writer thread (OutputWriter), the role of
the reference's IO server ranks (src/mo_io_server.f90): the stepping thread
copies an output's averages to the host and carries on while the file is
written.

By default every block runs as one sub-domain: an input with ``nbpc > 1`` is
run with one sub-domain per block (its interface closures then differ from the
reference's split run at the sub-domain faces), and a warning says so. With
``split=True`` the blocks are split as the input says (cases.decompose): the
ranks run as the reference's ranks do, and the restart and output files are
still per input block, assembled from its ranks. The reference's VISCOUS build
flag is the ``viscous`` argument.
"""
from __future__ import annotations

import os
import queue
import sys
import threading
import time
from typing import Optional

import numpy as np

from . import api, cases, namelist


class OutputWriter:
    """Writes Tecplot outputs (api.plt_write) on a host thread, in the order
    they are handed over. The library call releases the interpreter lock, so
    the writes overlap the steps. close() waits for every write and raises the
    first error."""

    def __init__(self):
        self._q: "queue.Queue" = queue.Queue()
        self._err: Optional[BaseException] = None
        self._t = threading.Thread(target=self._loop, name="canard-output", daemon=True)
        self._t.start()

    def _loop(self):
        while True:
            item = self._q.get()
            if item is None:
                return
            path, n, arrays, t = item
            if self._err is not None:
                continue
            try:
                os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
                api.plt_write(path, n, arrays, t)
            except BaseException as e:  # reported by close()
                self._err = e

    def submit(self, path: str, n: int, arrays, t: float = 0.0):
        self._q.put((path, n, arrays, t))

    def close(self):
        self._q.put(None)
        self._t.join()
        if self._err is not None:
            raise self._err


def case_from_input(nml, viscous: int = 1, warn=print, split: bool = False) -> cases.CaseSpec:
    """The case an ``input.canard`` describes (namelists as read by
    namelist.read): blocks and boundary codes from nml_domdcomp, the grid from
    nml_gridgen's generator, initialo's state, and the physics, numerics and
    sponge parameters; with ``split``, its blocks split into the ranks of nbpc."""
    drv, can, dd = nml["nml_driver"], nml["nml_canard"], nml["nml_domdcomp"]
    gg, num, phy, sp = nml["nml_gridgen"], nml["nml_numerics"], nml["nml_physics"], nml["nml_sponge"]
    nb = int(drv["mbk"]) + 1
    lxi, let, lze = (dd[k][0] for k in ("lximb", "letmb", "lzemb"))
    nbbc, mbcd, nbpc = dd["nbbc"][0], dd["mbcd"][0], dd["nbpc"][0]
    if np.any(nbpc > 1) and not split:
        warn("canard_b200: nbpc > 1 in the input; every block runs as one sub-domain here")
    gt = int(gg["gridtype"])
    if gt == 0:
        xyz = [cases.gridtoy(int(gg["lxi0"]), int(gg["let0"]), int(gg["lze0"]), float(gg["doml0"]),
                             float(gg["doml1"]), float(gg["domh"]), float(gg["span"]))]
    elif gt == 1:
        xyz = cases.gridtoy_multi(int(gg["lxi0"]), int(gg["lxi1"]), int(gg["lxi2"]), int(gg["let0"]),
                                  int(gg["lze0"]), float(gg["doml0"]), float(gg["doml1"]), float(gg["domh"]),
                                  float(gg["span"]))
    else:
        raise namelist.NamelistError(f"gridtype {gt}: only the reference's gridtoy (0) and gridtoy_multi (1)")
    if len(xyz) < nb:
        raise namelist.NamelistError(f"gridtype {gt} makes {len(xyz)} block(s), the input has {nb}")
    blocks = []
    for m in range(nb):
        b = cases.BlockSpec(int(lxi[m]), int(let[m]), int(lze[m]),
                            [[int(nbbc[m, d, s]) for s in range(2)] for d in range(3)],
                            [[int(mbcd[m, d, s]) for s in range(2)] for d in range(3)])
        if xyz[m].shape[1:] != b.shape:
            raise namelist.NamelistError(f"block {m}: the grid has {xyz[m].shape[1:][::-1]} points per direction, "
                                         f"nml_domdcomp {b.shape[::-1]}")
        blocks.append(b)
    xyz = xyz[:nb]
    cs = cases.CaseSpec(blocks, viscous=viscous, fltk=float(num["fltk"]), fltrbc=float(num["fltrbc"]),
                        reoo=float(phy["reoo"]), tempoo=float(phy["tempoo"]),
                        amach=(float(phy["amach1"]), float(phy["amach2"]), float(phy["amach3"])),
                        timf=float(phy["timf"]), nsmf=int(phy["nsmf"]), cfl=float(can["cfl"]),
                        szco=float(sp["szco"]), szth0=float(gg["szth0"]), szth1=float(gg["szth1"]),
                        doml0=float(gg["doml0"]), doml1=float(gg["doml1"]), xyz=xyz,
                        qa=[cases.initialo(g) for g in xyz], name="input.canard")
    if split and np.any(nbpc > 1):
        cs = cases.decompose(cs, [tuple(int(v) for v in nbpc[m]) for m in range(nb)])
    return cs


class _Files:
    """The per-input-block restart and output files of a case whose context
    blocks may be ranks of split blocks (cs.sub): states and outputs are
    assembled per input block, restart states split back to the ranks."""

    def __init__(self, cs):
        self.cs, self.sub = cs, cs.sub

    def per_block(self, arrays):
        return cases.compose(self.sub, arrays) if self.sub else list(arrays)

    def grid(self):
        return [np.asarray(x, np.float32) for x in self.per_block(self.cs.xyz)]

    def write_restart(self, ctx, directory):
        if not self.sub:
            ctx.write_restart(directory)
            return
        os.makedirs(os.path.join(directory, "misc"), exist_ok=True)
        t6 = ctx.time()
        for m, q in enumerate(self.per_block([ctx.state(r) for r in range(len(self.cs.blocks))])):
            api.write_restart_file(os.path.join(directory, api.restart_name(m)), t6, q)

    def read_restart(self, ctx, directory):
        if not self.sub:
            ctx.read_restart(directory)
            return
        blocks = []
        for m, shape in enumerate(self.sub["shapes"]):
            t6, q = api.read_restart_file(os.path.join(directory, api.restart_name(m)), int(np.prod(shape)))
            blocks.append(q.reshape((5,) + tuple(shape)))
        for r, ((m, *_), sl) in enumerate(zip(self.sub["ranks"], self.sub["slices"])):
            ctx.set_state(r, np.ascontiguousarray(blocks[m][:, sl[0]:sl[0] + sl[3], sl[1]:sl[1] + sl[4],
                                                               sl[2]:sl[2] + sl[5]]))
        ctx.set_time(t6)


def gpu_options(nml, precision=None, viscous=None, max_steps=None, split=None) -> dict:
    """The run's options: each argument that is not None, else the input's
    &nml_gpu value (defaults: FP64, viscous, no step limit, no split)."""
    g = nml["nml_gpu"]
    if precision is None:
        if int(g["nprecision"]) not in (api.FP64, api.FP32_MIXED, api.FP64_FAST):
            raise namelist.NamelistError(f"&nml_gpu: nprecision {int(g['nprecision'])} "
                                         "(0 FP64, 1 FP32-mixed, 2 fast FP64)")
        precision = int(g["nprecision"])
    if viscous is None:
        viscous = 0 if bool(g["linviscid"]) else 1
    if max_steps is None and int(g["nsteps"]) > 0:
        max_steps = int(g["nsteps"])
    if split is None:
        split = bool(g["lsplit"])
    return {"precision": precision, "viscous": viscous, "max_steps": max_steps, "split": split}


def plan_devices(input_path: str, ndev: int, viscous: Optional[int] = None, precision: Optional[int] = None,
                 out=sys.stdout) -> dict:
    """The input's ranks (its blocks split by nbpc) placed on ndev devices
    (placement.contiguous) and the bytes each device would send the others per
    time step (placement.ExchangePlan); printed and returned. No device is used."""
    from . import placement
    nml = namelist.read_file(input_path)
    opt = gpu_options(nml, precision=precision, viscous=viscous)
    viscous, precision = opt["viscous"], opt["precision"]
    cs = case_from_input(nml, viscous=viscous, warn=lambda s: print(s, file=out), split=True)
    plan = placement.ExchangePlan(cs, placement.contiguous(cs, ndev))
    res = plan.summary(viscous=bool(viscous), deriv_bytes=4 if precision == api.FP32_MIXED else 8)
    res["device_of_rank"] = plan.device.tolist()
    print(f" {res['ranks']} ranks on {ndev} devices: {res['cross_links']} face links cross devices", file=out)
    for d in range(ndev):
        ranks = [r for r, e in enumerate(res["device_of_rank"]) if e == d]
        print(f" device {d}: ranks {ranks[0]}-{ranks[-1]}, {res['points_per_device'][d]} points, "
              f"{res['bytes_per_step_out'][d] / 1e6:.3f} MB out per step", file=out)
    return res


def run(input_path: str = "input.canard", directory: Optional[str] = None, precision: Optional[int] = None,
        viscous: Optional[int] = None, max_steps: Optional[int] = None, out=sys.stdout,
        split: Optional[bool] = None) -> dict:
    """Runs the case of ``input_path`` in ``directory`` (default: the input's
    directory) like the reference's program; returns a summary (steps, time,
    outputs written, whether the run stopped on a zero time step). ``split``:
    run the input's sub-domains (nbpc) as the reference's ranks. Options left
    at None come from the input's &nml_gpu group (gpu_options)."""
    directory = directory or os.path.dirname(os.path.abspath(input_path))
    nml = namelist.read_file(input_path)
    opt = gpu_options(nml, precision=precision, viscous=viscous, max_steps=max_steps, split=split)
    precision, viscous, max_steps, split = opt["precision"], opt["viscous"], opt["max_steps"], opt["split"]
    cs = case_from_input(nml, viscous=viscous, warn=lambda s: print(s, file=out), split=split)
    files = _Files(cs)
    can, drv = nml["nml_canard"], nml["nml_driver"]
    tmax, ndata = float(can["tmax"]), int(drv["ndata"])
    loutput = ndata >= 0
    ctx = api.Context(cs, precision=precision)
    try:
        if int(can["nts"]) != 0:
            files.read_restart(ctx, directory)
        if bool(can["ltimer"]):
            ctx.set_timers(True)
        outputs = []
        writer = OutputWriter()
        if loutput:
            writer.submit(os.path.join(directory, api.plt_name(-1)), -1, files.grid())
            outputs.append(api.plt_name(-1))
            ctx.record_enable(True)
        t0 = time.perf_counter()
        try:
            steps, _, overflow = _loop(ctx, tmax, ndata, loutput, max_steps, directory, writer, outputs, out, files)
        finally:
            writer.close()  # every output file is complete when run() returns
        if int(can["nrestart"]) == 1:
            files.write_restart(ctx, directory)
        wall = time.perf_counter() - t0
        n, _, dt, _, _, timo = ctx.time()
        # the loop ends on a zero time step only after step 2 (dt is 0 before)
        if overflow or (dt == 0.0 and n > 2):
            print(" Canard: Overflow.", file=out)
        if bool(can["ltimer"]):
            for name, v in ctx.timers().items():
                if v["launches"]:
                    print(" %-18s %10.3f ms %8d launches" % (name, v["ms"], v["launches"]), file=out)
        print(" Canard: Finished.", file=out)
    finally:
        ctx.close()
    return {"steps": steps, "n": int(n), "time": float(timo), "outputs": outputs, "overflow": overflow,
            "wall_s": wall, "points": cs.npts}


def _loop(ctx, tmax, ndata, loutput, max_steps, directory, writer, outputs, out, files):
    """The time loop of canard_driver; returns (steps, output count - 1,
    whether it ended on a zero time step)."""
    ndati = -1
    steps = 0
    while True:
        n, _, dt, _, _, timo = ctx.time()
        # do while (timo < tmax .and. (dt /= 0 .or. n <= 2))
        if not (timo < tmax and (dt != 0.0 or n <= 2)):
            break
        if max_steps is not None and steps >= max_steps:
            break
        print(" n =%8d   time =%12.5f" % (int(n), timo), file=out)
        try:
            ctx.step(1)
        except api.CanardError as e:
            if e.code != api.ERR_NAN:
                raise
            return steps, ndati, True  # dt == 0 after step 2: the reference's loop ends here
        steps += 1
        if loutput:
            ctx.record_accumulate()
            timo_new = ctx.time()[5]  # timo + dt of this step
            # nout: the output time res falls within [timo, timo + dt]
            res = (ndati + 1) * tmax / ndata if ndata > 0 else np.inf
            if (timo - res) * (timo_new - res) <= 0.0:
                ndati += 1
                arrays, t_out = ctx.record_output()
                arrays = [np.asarray(a, np.float32) for a in files.per_block(arrays)]
                writer.submit(os.path.join(directory, api.plt_name(ndati)), ndati, arrays, t_out)
                outputs.append(api.plt_name(ndati))
    return steps, ndati, False
