"""Python host side of the C ABI (include/canard_gpu.h).

Mirrors the reference's interfaces for the time-step path:

* ``Context.mpigo / deriv / filte``      -> t_numerics (src/mo_numerics.f90:429-987)
* ``Context.phase(PH_FLUXES, nk)`` etc.  -> t_physics / mo_gcbc / mo_sponge routines
* ``Context.step(n)``                    -> the time loop body (src/mo_canard_driver.f90:226-431)

Arrays cross the boundary as host float64 arrays in the reference layout
``q(0:lmx, ncols)`` (NumPy shape ``(ncols, lze+1, let+1, lxi+1)``).
Errors come back as ``CanardError`` carrying the library's code and message,
the way the reference stops with a message.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Sequence

import numpy as np

from . import cases as _cases

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libcanard_b200.so")

OK, ERR_ARG, ERR_CUDA, ERR_NAN, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_STATE, ERR_IO = range(8)
FP64, FP32_MIXED, FP64_FAST = 0, 1, 2

F_QA, F_QO, F_DE, F_P, F_SS1, F_XIM, F_ETM, F_ZEM, F_YACO, F_TAU = range(10)
F_DRVA = (10, 11, 12)
F_CM = (13, 14, 15)
NCOLS = {F_QA: 5, F_QO: 5, F_DE: 5, F_P: 1, F_SS1: 1, F_XIM: 3, F_ETM: 3, F_ZEM: 3, F_YACO: 1, F_TAU: 9}

(PH_FILTER, PH_COPYQO, PH_PRIM, PH_TIMESTEP, PH_VISCOUS, PH_FLUXES, PH_GCBC, PH_SPONGE,
 PH_RKUPDATE, PH_WALL, PH_AVERAGE, PH_ADVANCE, PH_MOVEF_A) = range(13)


class CanardError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"canard error {code}: {msg}")
        self.code = code


class _Block(ctypes.Structure):
    _fields_ = [("lxi", ctypes.c_int32), ("let", ctypes.c_int32), ("lze", ctypes.c_int32),
                ("nbc", (ctypes.c_int32 * 2) * 3), ("mbcd", (ctypes.c_int32 * 2) * 3)]


class _Case(ctypes.Structure):
    _fields_ = [("nblocks", ctypes.c_int32), ("viscous", ctypes.c_int32),
                ("fltk", ctypes.c_double), ("fltrbc", ctypes.c_double),
                ("reoo", ctypes.c_double), ("tempoo", ctypes.c_double),
                ("amach1", ctypes.c_double), ("amach2", ctypes.c_double), ("amach3", ctypes.c_double),
                ("timf", ctypes.c_double), ("nsmf", ctypes.c_int32), ("cfl", ctypes.c_double),
                ("szco", ctypes.c_double), ("szth0", ctypes.c_double), ("szth1", ctypes.c_double),
                ("doml0", ctypes.c_double), ("doml1", ctypes.c_double)]


_lib = None
_DP = ctypes.POINTER(ctypes.c_double)
_FP = ctypes.POINTER(ctypes.c_float)


def lib():
    """Load the in-tree CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"{LIBPATH} is missing: build it with canard_b200/csrc/build.py")
        L = ctypes.CDLL(LIBPATH)
        vp = ctypes.c_void_p
        i32 = ctypes.c_int32
        L.canard_ctx_create.argtypes = [ctypes.POINTER(_Case), i32, ctypes.POINTER(_Block), i32,
                                        ctypes.POINTER(vp)]
        L.canard_ctx_destroy.argtypes = [vp]
        L.canard_last_error.restype = ctypes.c_char_p
        L.canard_last_error.argtypes = [vp]
        L.canard_set_stream.argtypes = [vp, vp]
        L.canard_upload_grid.argtypes = [vp, i32, i32, _DP]
        L.canard_setup.argtypes = [vp]
        L.canard_set_state.argtypes = [vp, i32, i32, _DP]
        L.canard_get_state.argtypes = [vp, i32, i32, _DP]
        L.canard_get_field.argtypes = [vp, i32, i32, i32, _DP, ctypes.c_int64]
        L.canard_set_field.argtypes = [vp, i32, i32, i32, _DP, ctypes.c_int64]
        L.canard_step.argtypes = [vp, i32]
        L.canard_step_host.argtypes = [vp, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32),
                                       ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        L.canard_phase.argtypes = [vp, i32, i32]
        L.canard_phase_with.argtypes = [vp, i32, i32, ctypes.c_double, _DP, _DP]
        L.canard_get_time.argtypes = [vp, i32, _DP]
        L.canard_restart_write_file.argtypes = [ctypes.c_char_p, _DP, _DP, ctypes.c_int64]
        L.canard_restart_read_file.argtypes = [ctypes.c_char_p, _DP, _DP, ctypes.c_int64]
        L.canard_grid_write_file.argtypes = [ctypes.c_char_p, _DP, ctypes.c_int64]
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.canard_average_host.argtypes = [i32, ctypes.c_void_p, i32, i32p, i32p, i32p, ctypes.POINTER(_DP)]
        L.canard_set_subdomains.argtypes = [vp, i32, i32, i32p, i32p, i32p]
        i64p = ctypes.POINTER(ctypes.c_int64)
        L.canard_plan_export.argtypes = [i32, ctypes.c_void_p, i32, i32p, i32p, i32p, i32, i64p, ctypes.c_int64,
                                         i64p]
        L.canard_grid_read_file.argtypes = [ctypes.c_char_p, _DP, ctypes.c_int64]
        L.canard_restart_compare.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int64, ctypes.c_double,
                                             ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        L.canard_write_restart.argtypes = [vp, i32, i32, ctypes.c_char_p]
        L.canard_record_enable.argtypes = [vp, i32]
        L.canard_record_accumulate.argtypes = [vp]
        L.canard_record_output.argtypes = [vp, i32, ctypes.POINTER(_FP), _DP]
        L.canard_plt_write.argtypes = [ctypes.c_char_p, i32, i32, ctypes.POINTER(ctypes.c_int32),
                                       ctypes.c_double, ctypes.POINTER(_FP)]
        L.canard_read_restart.argtypes = [vp, i32, i32, ctypes.c_char_p]
        L.canard_set_time.argtypes = [vp, i32, _DP]
        L.canard_mpigo.argtypes = [vp, ctypes.POINTER(_DP), i32, i32, i32, i32, i32, i32]
        L.canard_deriv.argtypes = [vp, i32, _DP, _DP, i32, i32]
        L.canard_filte.argtypes = [vp, i32, _DP, i32, i32]
        L.canard_set_timers.argtypes = [vp, i32]
        L.canard_set_graphs.argtypes = [vp, i32]
        L.canard_autotune.argtypes = [vp, i32, _DP, i32]
        L.canard_set_line_kind.argtypes = [vp, i32, i32, i32, i32]
        L.canard_line_bench.argtypes = [vp, i32, i32, i32, _DP, _DP, i32, ctypes.POINTER(ctypes.c_double)]
        L.canard_get_timers.argtypes = [vp, _DP, _DP, _DP, i32]
        L.canard_timer_name.restype = ctypes.c_char_p
        L.canard_timer_name.argtypes = [i32]
        L.canard_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.canard_selftest_wait.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.canard_deriv_noalloc.argtypes = [vp, vp, i32, i32, i32, i32, i32, i32, i32, ctypes.c_double,
                                           ctypes.c_double, vp]
        L.canard_deriv_noalloc_status.argtypes = [vp]
        L.canard_coeffs.argtypes = [ctypes.c_double, ctypes.c_double, _DP]
        L.canard_penta.argtypes = [ctypes.c_double, ctypes.c_double, i32, i32, i32, i32, _DP, _DP]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_DP)


def coeffs(fltk: float, fltrbc: float) -> np.ndarray:
    out = np.zeros(150)
    rc = lib().canard_coeffs(fltk, fltrbc, _dp(out))
    if rc:
        raise CanardError(rc, "canard_coeffs")
    return out


def penta(fltk, fltrbc, n, ns, ne, nt):
    xu = np.zeros(3 * n)
    xl = np.zeros(2 * n)
    rc = lib().canard_penta(fltk, fltrbc, n, ns, ne, nt, _dp(xu), _dp(xl))
    if rc:
        raise CanardError(rc, "canard_penta")
    return xu.reshape(3, n), xl.reshape(2, n)


def restart_name(mb: int) -> str:
    """The reference's restart file of block mb, relative to the run directory:
    'misc/restart' + 'z' + three digits + '.dat' assigned to a character(19)
    variable, which Fortran truncates to 19 characters (src/mo_io.f90:27,
    108-116), so the file is misc/restartzNNN.da."""
    return ("misc/restart" + "z%03d" % mb + ".dat")[:19]


def write_restart_file(path, time6, qa):
    """One block's restart file in the reference's format; qa is (5, ...) in
    the reference layout (qa(0:lmx, 5))."""
    q = np.ascontiguousarray(qa, np.float64).reshape(5, -1)
    t = np.ascontiguousarray(time6, np.float64)
    rc = lib().canard_restart_write_file(os.fsencode(path), _dp(t), _dp(q), q.shape[1])
    if rc:
        raise CanardError(rc, f"canard_restart_write_file {path}")


def read_restart_file(path, npts):
    """(time6, qa (5, npts)) of a restart file of a block of npts points."""
    t = np.zeros(6)
    q = np.zeros((5, npts))
    rc = lib().canard_restart_read_file(os.fsencode(path), _dp(t), _dp(q), npts)
    if rc:
        raise CanardError(rc, f"canard_restart_read_file {path}")
    return t, q


def grid_name(mb: int) -> str:
    """The reference's grid file of block mb, relative to the run directory:
    'misc/grid' + three digits + '.dat', 16 characters, which fit its
    character(16) variable (src/mo_io.f90:31, 115)."""
    return "misc/grid%03d.dat" % mb


def write_grid_file(path, xyz):
    """One block's grid file in the reference's format; xyz is (3, ...) in
    the reference layout (ss(0:lmx, 3))."""
    g = np.ascontiguousarray(xyz, np.float64).reshape(3, -1)
    rc = lib().canard_grid_write_file(os.fsencode(path), _dp(g), g.shape[1])
    if rc:
        raise CanardError(rc, f"canard_grid_write_file {path}")


def read_grid_file(path, npts):
    """xyz (3, npts) of the grid file of a block of npts points."""
    g = np.zeros((3, npts))
    rc = lib().canard_grid_read_file(os.fsencode(path), _dp(g), npts)
    if rc:
        raise CanardError(rc, f"canard_grid_read_file {path}")
    return g


def plt_name(n: int) -> str:
    """The reference's output file of output n (-1: the grid), relative to the
    run directory (src/mo_io.f90:96-106)."""
    return "data/grid.plt" if n == -1 else "data/n%03d.plt" % n


def plt_write(path, n, arrays, time=0.0):
    """write_output_file: one output (n >= 0: rho, u, v, w, p; n = -1: x, y, z)
    of every block, arrays[b] of shape (nvar, lze+1, let+1, lxi+1) float32."""
    arrs = [np.ascontiguousarray(a, np.float32) for a in arrays]
    dims = (ctypes.c_int32 * (3 * len(arrs)))()
    for b, a in enumerate(arrs):
        dims[3 * b], dims[3 * b + 1], dims[3 * b + 2] = a.shape[3], a.shape[2], a.shape[1]
    ptrs = (_FP * len(arrs))(*[a.ctypes.data_as(_FP) for a in arrs])
    rc = lib().canard_plt_write(os.fsencode(path), n, len(arrs), dims, time, ptrs)
    if rc:
        raise CanardError(rc, f"canard_plt_write {path}")


def compare_restart(path1, path2, npts, wtol=1e-15, report=None):
    """dcanard: the number of values whose difference relative to the first
    file's value exceeds wtol; their lines go to `report` if given."""
    n = ctypes.c_int64(0)
    rc = lib().canard_restart_compare(os.fsencode(path1), os.fsencode(path2), npts, wtol,
                                      os.fsencode(report) if report else None, ctypes.byref(n))
    if rc:
        raise CanardError(rc, f"canard_restart_compare {path1} {path2}")
    return n.value


def _structs(case_list: Sequence[_cases.CaseSpec]):
    cs_arr = (_Case * len(case_list))()
    blocks = [b for cs in case_list for b in cs.blocks]
    b_arr = (_Block * len(blocks))()
    for i, cs in enumerate(case_list):
        c = cs_arr[i]
        c.nblocks = len(cs.blocks)
        c.viscous = int(cs.viscous)
        c.fltk, c.fltrbc, c.reoo, c.tempoo = cs.fltk, cs.fltrbc, cs.reoo, cs.tempoo
        c.amach1, c.amach2, c.amach3 = (float(v) for v in cs.amach)
        c.timf, c.nsmf, c.cfl = cs.timf, int(cs.nsmf), cs.cfl
        c.szco, c.szth0, c.szth1, c.doml0, c.doml1 = cs.szco, cs.szth0, cs.szth1, cs.doml0, cs.doml1
    for i, b in enumerate(blocks):
        b_arr[i].lxi, b_arr[i].let, b_arr[i].lze = b.lxi, b.let, b.lze
        for d in range(3):
            for s in range(2):
                b_arr[i].nbc[d][s] = int(b.nbc[d][s])
                b_arr[i].mbcd[d][s] = int(b.mbcd[d][s])
    return cs_arr, b_arr


def _sub_args(cs: _cases.CaseSpec):
    i32p = ctypes.POINTER(ctypes.c_int32)
    if not cs.sub:
        return [], [0, None, None, None]
    keep = [np.ascontiguousarray(cs.sub[k], np.int32) for k in ("nbpc", "mbcd", "ranks")]
    return keep, [len(cs.sub["nbpc"])] + [a.ctypes.data_as(i32p) for a in keep]


def average_host(cs: _cases.CaseSpec, qa):
    """The junction averaging of one case (average_point, average_line,
    average_surface) on the host, through the plans the device builds and the
    device's arithmetic, for a case of blocks or of sub-domains
    (cases.decompose). qa: per block / rank (5, ...); returns the averaged
    copies."""
    _, blocks = _structs([cs])
    arrs = [np.ascontiguousarray(q, np.float64).copy() for q in qa]
    ptrs = (_DP * len(arrs))(*[_dp(a) for a in arrs])
    keep, args = _sub_args(cs)
    rc = lib().canard_average_host(len(arrs), ctypes.cast(blocks, ctypes.c_void_p), *args, ptrs)
    if rc:
        raise CanardError(rc, "canard_average_host")
    return arrs


PLAN_FACES, PLAN_POINTS, PLAN_LINES, PLAN_SURFACE = 0, 1, 2, 3
_PLAN_WIDTH = (7, 4, 4, 4, 2, 2, 2)


def plan_export(cs: _cases.CaseSpec, kind: int) -> np.ndarray:
    """One exchange list of a case (canard_plan_export) as an int64 array of
    rows: kind 0 the face links (receiving rank, nn, receiving side, sending
    rank, sending side, lines, sending face's code); 1-3 the point, line and
    surface averaging targets (rank, l, first, count); 4-6 their sources
    (rank, l). Host only."""
    _, blocks = _structs([cs])
    keep, args = _sub_args(cs)
    i64p = ctypes.POINTER(ctypes.c_int64)
    n = ctypes.c_int64(0)
    call = lambda out, cap: lib().canard_plan_export(len(cs.blocks), ctypes.cast(blocks, ctypes.c_void_p), *args,
                                                     kind, out, cap, ctypes.byref(n))
    rc = call(None, 0)
    if rc:
        raise CanardError(rc, "canard_plan_export")
    out = np.zeros(max(n.value, 1), np.int64)
    if n.value:
        rc = call(out.ctypes.data_as(i64p), out.size)
        if rc:
            raise CanardError(rc, "canard_plan_export")
    return out[:n.value].reshape(-1, _PLAN_WIDTH[kind])


class Context:
    """A device context holding one or more cases (several = batched)."""

    def __init__(self, case_list, precision: int = FP64, setup: bool = True, upload_state: bool = True):
        if isinstance(case_list, _cases.CaseSpec):
            case_list = [case_list]
        self.cases: List[_cases.CaseSpec] = list(case_list)
        self._c, self._b = _structs(self.cases)
        h = ctypes.c_void_p()
        rc = lib().canard_ctx_create(self._c, len(self.cases), self._b, int(precision), ctypes.byref(h))
        if rc:
            raise CanardError(rc, "canard_ctx_create failed")
        self.h = h
        i32p = ctypes.POINTER(ctypes.c_int32)
        for ci, cs in enumerate(self.cases):
            if cs.sub:  # sub-domains of split blocks (cases.decompose)
                a = [np.ascontiguousarray(cs.sub[k], np.int32) for k in ("nbpc", "mbcd", "ranks")]
                self._check(lib().canard_set_subdomains(self.h, ci, len(cs.sub["nbpc"]),
                                                        *[x.ctypes.data_as(i32p) for x in a]))
        if setup:
            for ci, cs in enumerate(self.cases):
                for bi, x in enumerate(cs.xyz):
                    self._check(lib().canard_upload_grid(self.h, ci, bi, _dp(np.ascontiguousarray(x, np.float64))))
            self._check(lib().canard_setup(self.h))
        if upload_state:
            for ci, cs in enumerate(self.cases):
                if cs.qa is not None:
                    for bi, q in enumerate(cs.qa):
                        self.set_state(bi, q, ci)

    def _check(self, rc):
        if rc:
            raise CanardError(rc, lib().canard_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().canard_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int):
        self._check(lib().canard_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def set_state(self, b, qa, case=0):
        self._check(lib().canard_set_state(self.h, case, b, _dp(np.ascontiguousarray(qa, np.float64))))

    def state(self, b=0, case=0):
        blk = self.cases[case].blocks[b]
        out = np.zeros((5,) + blk.shape)
        self._check(lib().canard_get_state(self.h, case, b, _dp(out)))
        return out

    def get_state_into(self, b, out, case=0):
        self._check(lib().canard_get_state(self.h, case, b, _dp(out)))

    def set_timers(self, on):
        self._check(lib().canard_set_timers(self.h, 1 if on else 0))

    def set_graphs(self, on):
        self._check(lib().canard_set_graphs(self.h, 1 if on else 0))

    def autotune(self, reps=5):
        """Times the line-tile candidates of every (group, direction) and
        installs the fastest; returns one dict per group and direction."""
        rep = np.zeros(6 * 16)
        k = lib().canard_autotune(self.h, reps, _dp(rep), 16)
        if k < 0:
            self._check(-k)
        kinds = {0: "fp64", 1: "fp32-split", 2: "fp64-tile/fp32-split", 3: "fp32-one-lane",
                 4: "fp64-tile/fp32-one-lane", 5: "fp64-tmem", 6: "fp64-stream/fp32-split", 7: "fp64-split",
                 8: "fp64-quad", 9: "fp32-quad", 10: "fp64-twist", 11: "fp32-twist", 12: "fp64-tile/fp32-twist"}
        out = []
        for i in range(k):
            g, d, kd, nc, best, dflt = rep[6 * i:6 * i + 6]
            out.append({"group": ("filter", "viscous", "flux")[int(g)], "dir": "xi eta zeta".split()[int(d)],
                        "kind": kinds.get(int(kd), str(int(kd))), "chunks": int(nc) or "default",
                        "ms": best, "default_ms": dflt})
        return out

    LINE_KINDS = {"default": -1, "fp64": 0, "fp32-split": 1, "fp64-tile/fp32-split": 2, "fp32-one-lane": 3,
                  "fp64-tile/fp32-one-lane": 4, "fp64-tmem": 5, "fp64-stream/fp32-split": 6, "fp64-split": 7,
                  "fp64-quad": 8, "fp32-quad": 9, "fp64-twist": 10, "fp32-twist": 11, "fp64-tile/fp32-twist": 12}

    def set_line_kind(self, group, direction, kind, chunks=0):
        """Pins the line kernel of a group ("filter", "viscous", "flux") and
        direction ("xi", "eta", "zeta"), by name from LINE_KINDS; "fp64",
        "fp64-tmem" give results bit-identical to the reference's order,
        "fp64-split" and "fp64-twist" (the fast FP64 mode's kinds) differ at
        rounding level."""
        g = ("filter", "viscous", "flux").index(group)
        d = ("xi", "eta", "zeta").index(direction)
        self._check(lib().canard_set_line_kind(self.h, g, d, self.LINE_KINDS[kind], chunks))

    def line_bench(self, op, nn, fields, reps=10):
        """One direction's derivative (op 0) or filter (op 1) over up to 5
        fields of block 0 (array (nfields, ...) in the reference layout):
        returns (result of one launch, average ms of `reps` timed launches)."""
        f = np.ascontiguousarray(fields, np.float64)
        out = np.zeros_like(f)
        ms = ctypes.c_double()
        self._check(lib().canard_line_bench(self.h, op, nn, f.shape[0], _dp(f), _dp(out), reps, ctypes.byref(ms)))
        return out, ms.value

    def timers(self):
        """Per kernel family: device ms, launches, algorithmic bytes since set_timers(True)."""
        n = 32
        ms, la, by = np.zeros(n), np.zeros(n), np.zeros(n)
        k = lib().canard_get_timers(self.h, _dp(ms), _dp(la), _dp(by), n)
        if k < 0:
            self._check(-k)
        return {lib().canard_timer_name(i).decode(): {"ms": ms[i], "launches": int(la[i]), "bytes": by[i]}
                for i in range(k)}

    def launch_count(self):
        v = ctypes.c_int64()
        self._check(lib().canard_launch_count(self.h, ctypes.byref(v)))
        return int(v.value)

    def selftest_wait(self):
        """Runs the bounded-wait self-test: returns (status code, seconds);
        the code is ERR_TIMEOUT when the device wait gave up as designed."""
        s = ctypes.c_double()
        code = lib().canard_selftest_wait(self.h, ctypes.byref(s))
        return code, s.value

    def field(self, which, b=0, case=0):
        blk = self.cases[case].blocks[b]
        if which in NCOLS:
            out = np.zeros((NCOLS[which],) + blk.shape)
        else:
            nbs = [(blk.let + 1) * (blk.lze + 1), (blk.lze + 1) * (blk.lxi + 1), (blk.lxi + 1) * (blk.let + 1)]
            d = (which - 10) % 3
            out = np.zeros((10 if which < 13 else 6) * nbs[d])
        self._check(lib().canard_get_field(self.h, case, b, which, _dp(out), out.size))
        return out

    def set_field(self, which, arr, b=0, case=0):
        a = np.ascontiguousarray(arr, np.float64)
        self._check(lib().canard_set_field(self.h, case, b, which, _dp(a), a.size))

    def step(self, n=1):
        self._check(lib().canard_step(self.h, n))

    def step_host(self, n, arrays, blocks=None):
        """n steps through host memory: arrays[k] (float64, the reference
        layout of block blocks[k] = (case, block), default (0, k)) is the
        step's input before every step and receives its result after it; the
        copies are pipelined in both directions (canard_step_host)."""
        if blocks is None:
            blocks = [(0, k) for k in range(len(arrays))]
        for a in arrays:
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("host states must be C-contiguous float64 arrays")
        nb = len(arrays)
        ic = (ctypes.c_int32 * nb)(*[c for c, _ in blocks])
        ib = (ctypes.c_int32 * nb)(*[b for _, b in blocks])
        ptrs = (ctypes.POINTER(ctypes.c_double) * nb)(*[_dp(a) for a in arrays])
        self._check(lib().canard_step_host(self.h, n, nb, ic, ib, ptrs))

    def phase(self, ph, nk=0):
        self._check(lib().canard_phase(self.h, ph, nk))

    def phase_with(self, ph, nk, dt, umf, dudtmf=(0.0, 0.0, 0.0)):
        """A fluxes / GCBC / RK update / wall phase with the stage's dt and
        moving frame given as the reference's routines receive them."""
        u = np.ascontiguousarray(umf, dtype=np.float64)
        a = np.ascontiguousarray(dudtmf, dtype=np.float64)
        self._check(lib().canard_phase_with(self.h, ph, nk, float(dt), _dp(u), _dp(a)))

    def time(self, case=0):
        out = np.zeros(6)
        self._check(lib().canard_get_time(self.h, case, _dp(out)))
        return out

    def set_time(self, t6, case=0):
        self._check(lib().canard_set_time(self.h, case, _dp(np.asarray(t6, np.float64))))

    def write_restart(self, directory, case=0):
        """write_restart_file for every block of a case: the state and the
        case's time state into directory/misc/restartzNNN.da (NNN = block)."""
        os.makedirs(os.path.join(directory, "misc"), exist_ok=True)
        for b in range(len(self.cases[case].blocks)):
            path = os.path.join(directory, restart_name(b))
            self._check(lib().canard_write_restart(self.h, case, b, os.fsencode(path)))

    def record_enable(self, on=True):
        """Time-averaged recording on (qb = 0, dtsum = 0) or off."""
        self._check(lib().canard_record_enable(self.h, 1 if on else 0))

    def record_accumulate(self):
        """qb += (dt/2)(qo + qa), dtsum += dt: after every step of a recorded run."""
        self._check(lib().canard_record_accumulate(self.h))

    def record_output(self, case=0):
        """(per block float32 arrays (5, lze+1, let+1, lxi+1) of rho, u, v, w, p
        of the average, output time); resets the average."""
        arrs = [np.zeros((5,) + b.shape, np.float32) for b in self.cases[case].blocks]
        ptrs = (_FP * len(arrs))(*[a.ctypes.data_as(_FP) for a in arrs])
        t = np.zeros(1)
        self._check(lib().canard_record_output(self.h, case, ptrs, _dp(t)))
        return arrs, float(t[0])

    def write_grid_plt(self, directory, case=0):
        """The grid file written at start-up (data/grid.plt: x, y, z in FP32)."""
        os.makedirs(os.path.join(directory, "data"), exist_ok=True)
        cs = self.cases[case]
        plt_write(os.path.join(directory, plt_name(-1)), -1, [np.asarray(x, np.float32) for x in cs.xyz])

    def write_output(self, directory, n, case=0):
        """An output of the recording: data/nNNN.plt of every block; returns the
        output time."""
        os.makedirs(os.path.join(directory, "data"), exist_ok=True)
        arrs, t = self.record_output(case)
        plt_write(os.path.join(directory, plt_name(n)), n, arrs, t)
        return t

    def read_restart(self, directory, case=0):
        """read_restart_file for every block of a case (pathbase = directory)."""
        for b in range(len(self.cases[case].blocks)):
            path = os.path.join(directory, restart_name(b))
            self._check(lib().canard_read_restart(self.h, case, b, os.fsencode(path)))

    # t_numerics
    def mpigo(self, fields, nt, nrt, n45, itag, m, ncols=1):
        arr = (_DP * len(fields))(*[_dp(f) for f in fields])
        self._check(lib().canard_mpigo(self.h, arr, ncols, nt, nrt, n45, itag, m))

    def deriv(self, b, fin, fout, nn, m):
        self._check(lib().canard_deriv(self.h, b, _dp(fin), _dp(fout), nn, m))

    def filte(self, b, f, inn, m):
        self._check(lib().canard_filte(self.h, b, _dp(f), inn, m))
