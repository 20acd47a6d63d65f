"""ctypes binding of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg to
check or time the reference algorithm on the CPU. The product package
(canard_b200) never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

A_QA, A_QO, A_DE, A_P, A_SS1 = 0, 1, 2, 3, 4
A_XIM, A_ETM, A_ZEM, A_YACO, A_TAU = 5, 6, 7, 8, 9
A_DRVA = (10, 11, 12)
A_CM = (13, 14, 15)
A_RECV0, A_RECV1, A_SEND1, A_SBCC, A_SPONGE = 16, 17, 18, 19, 20

PH_FILTER, PH_COPYQO, PH_PRIM, PH_TIMESTEP, PH_VISCOUS, PH_FLUXES = 0, 1, 2, 3, 4, 5
PH_GCBC, PH_SPONGE, PH_RKUPDATE, PH_WALL, PH_AVERAGE, PH_ADVANCE, PH_MOVEF_A = 6, 7, 8, 9, 10, 11, 12
PH_GCBC_SETUP, PH_GCBC_COMM_UPDATE = 13, 14  # PH_GCBC in two parts


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
# orc_hook_fn: (user, kind, a, b, data, n)
HOOK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                        ctypes.POINTER(ctypes.c_double), ctypes.c_int)


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_set_subdomains.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.POINTER(ctypes.c_int32)] * 3
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(_Case), ctypes.POINTER(_Block)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        for f in ("orc_set_grid", "orc_set_state"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.orc_setup.argtypes = [ctypes.c_void_p]
        L.orc_get_array.restype = ctypes.c_long
        L.orc_get_array.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.orc_set_array.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_phase.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_get_time.argtypes = [ctypes.c_void_p, dp]
        L.orc_set_time.argtypes = [ctypes.c_void_p, dp]
        L.orc_mpigo.argtypes = [ctypes.c_void_p, ctypes.POINTER(dp), ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_deriv.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int]
        L.orc_filte.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int]
        L.orc_set_hook.argtypes = [ctypes.c_void_p, HOOK, ctypes.c_void_p]
        L.orc_coeffs.argtypes = [ctypes.c_double, ctypes.c_double, dp]
        L.orc_penta.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_structs(cs):
    c = _Case()
    c.nblocks = len(cs.blocks)
    c.viscous = int(cs.viscous)
    c.fltk, c.fltrbc, c.reoo, c.tempoo = cs.fltk, cs.fltrbc, cs.reoo, cs.tempoo
    c.amach1, c.amach2, c.amach3 = (float(v) for v in cs.amach)
    c.timf, c.nsmf, c.cfl = cs.timf, int(cs.nsmf), cs.cfl
    c.szco, c.szth0, c.szth1, c.doml0, c.doml1 = cs.szco, cs.szth0, cs.szth1, cs.doml0, cs.doml1
    arr = (_Block * len(cs.blocks))()
    for i, b in enumerate(cs.blocks):
        arr[i].lxi, arr[i].let, arr[i].lze = b.lxi, b.let, b.lze
        for d in range(3):
            for s in range(2):
                arr[i].nbc[d][s] = int(b.nbc[d][s])
                arr[i].mbcd[d][s] = int(b.mbcd[d][s])
    return c, arr


def coeffs(fltk, fltrbc):
    out = np.zeros(150)
    n = lib().orc_coeffs(fltk, fltrbc, _dp(out))
    assert n == 150
    return out


def penta(fltk, fltrbc, n, ns, ne, nt):
    xu = np.zeros(3 * n)
    xl = np.zeros(2 * n)
    rc = lib().orc_penta(fltk, fltrbc, n, ns, ne, nt, _dp(xu), _dp(xl))
    assert rc == 0
    return xu.reshape(3, n), xl.reshape(2, n)


class Oracle:
    """One case (all blocks) on the CPU, with the reference's phase structure."""

    def __init__(self, cs, setup=True, threads=None):
        self.cs = cs
        self._c, self._b = make_structs(cs)
        L = lib()
        if threads is not None:
            L.orc_set_threads(int(threads))
        self.h = L.orc_create(ctypes.byref(self._c), self._b)
        if not self.h:
            raise RuntimeError("orc_create failed")
        if getattr(cs, "sub", None):
            sub = cs.sub
            nbpc = np.ascontiguousarray(sub["nbpc"], dtype=np.int32)
            mbcd = np.ascontiguousarray(sub["mbcd"], dtype=np.int32)
            ranks = np.ascontiguousarray(sub["ranks"], dtype=np.int32)
            i32p = ctypes.POINTER(ctypes.c_int32)
            rc = L.orc_set_subdomains(self.h, len(sub["nbpc"]), nbpc.ctypes.data_as(i32p),
                                      mbcd.ctypes.data_as(i32p), ranks.ctypes.data_as(i32p))
            if rc != 0:
                raise RuntimeError("orc_set_subdomains failed")
        if cs.xyz is not None:
            for i, x in enumerate(cs.xyz):
                self.set_grid(i, x)
        if setup and cs.xyz is not None:
            rc = L.orc_setup(self.h)
            if rc != 0:
                raise RuntimeError(f"orc_setup rc={rc}")
        if cs.qa is not None:
            for i, q in enumerate(cs.qa):
                self.set_state(i, q)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    def set_grid(self, b, xyz):
        lib().orc_set_grid(self.h, b, _dp(np.ascontiguousarray(xyz, dtype=np.float64)))

    def set_state(self, b, qa):
        lib().orc_set_state(self.h, b, _dp(np.ascontiguousarray(qa, dtype=np.float64)))

    def get(self, b, which):
        n = lib().orc_get_array(self.h, b, which, None)
        if n < 0:
            raise ValueError(which)
        out = np.zeros(n)
        lib().orc_get_array(self.h, b, which, _dp(out))
        return out

    def set(self, b, which, arr):
        rc = lib().orc_set_array(self.h, b, which, _dp(np.ascontiguousarray(arr, dtype=np.float64)))
        if rc != 0:
            raise ValueError(which)

    def state(self, b):
        return self.get(b, A_QA).reshape((5,) + self.cs.blocks[b].shape)

    def step(self, n=1):
        rc = lib().orc_step(self.h, n)
        if rc != 0:
            raise RuntimeError(f"orc_step rc={rc}")

    def phase(self, ph, nk=0):
        rc = lib().orc_phase(self.h, ph, nk)
        if rc != 0:
            raise RuntimeError(f"orc_phase({ph}) rc={rc}")

    def time(self):
        out = np.zeros(6)
        lib().orc_get_time(self.h, _dp(out))
        return out

    def set_time(self, t6):
        lib().orc_set_time(self.h, _dp(np.asarray(t6, dtype=np.float64)))

    def mpigo(self, fields, nt, nrt, n45, itag, m):
        """fields: list (one per block) of C-contiguous float64 arrays (ncols*npts)."""
        arr = (ctypes.POINTER(ctypes.c_double) * len(fields))(*[_dp(f) for f in fields])
        rc = lib().orc_mpigo(self.h, arr, 1, nt, nrt, n45, itag, m)
        if rc != 0:
            raise RuntimeError("orc_mpigo")

    def set_hook(self, fn):
        """fn(kind, a, b, data) at the oracle's exchange points (orc_set_hook);
        data is a NumPy view of the hook's doubles (empty for kinds 0-2).
        None removes it."""
        if fn is None:
            self._hook = None
            lib().orc_set_hook(self.h, HOOK(), None)
            return

        def tramp(_user, kind, a, b, data, n):
            view = np.ctypeslib.as_array(data, shape=(2 * n,)) if n else np.zeros(0)
            fn(kind, a, b, view)

        self._hook = HOOK(tramp)  # kept alive while registered
        lib().orc_set_hook(self.h, self._hook, None)

    def deriv(self, b, fin, fout, nn, m):
        rc = lib().orc_deriv(self.h, b, _dp(fin), _dp(fout), nn, m)
        assert rc == 0

    def filte(self, b, f, inn, m):
        rc = lib().orc_filte(self.h, b, _dp(f), inn, m)
        assert rc == 0
