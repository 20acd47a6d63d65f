"""Placement of one case's ranks on several devices, and the exchanges between
the devices that the placement implies.

A case's ranks are its blocks, or the sub-domains of its split blocks
(``cases.decompose``, the reference's ``nbpc > 1``, src/mo_domdcomp.f90:
85-232). In the reference every rank is an MPI process and every exchange a
message. Here the ranks that share a device exchange through device memory,
and only the exchanges between ranks on different devices cross NVLink:

* interface contractions (mpigo, src/mo_numerics.f90:429-705): per line of a
  face with code 35, 40 or 45, 2 values per derivative field (9 fields per RK
  stage when viscous: u, v, w, T and the 5 flux columns; 5 when inviscid) and
  3 per filtered field (5 fields per step);
* ``drva`` across curved interfaces (code 30, gcbc_comm, src/mo_gcbc.f90:
  186-220): 5 values per line per stage;
* sources of the junction averaging after every stage (average_point,
  average_line: src/mo_domdcomp.f90:439-559; average_surface: src/mo_gcbc.f90:
  342-422): 5 values per source point that lives on another device.

The lists come from the library's own plan builder (``canard_plan_export``),
the one the single-device context runs, so a multi-device run exchanges
exactly what the single-device run reads across ranks.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import api
from .cases import CaseSpec

INTERFACE_CODES = (35, 40, 45)  # faces whose lines take the interface closure (mpigo)
CURVED_CODE = 30                # curved interface: drva exchange (gcbc_comm)
STAGES = 4


def rank_points(cs: CaseSpec) -> np.ndarray:
    return np.array([(b.lxi + 1) * (b.let + 1) * (b.lze + 1) for b in cs.blocks], np.int64)


def contiguous(cs: CaseSpec, ndev: int) -> np.ndarray:
    """Device of every rank: ranks in their numbering order (xi fastest, then
    eta, zeta, block by block, as src/mo_domdcomp.f90:588-605 numbers them)
    cut into ndev runs of about equal point count, so that a device holds
    whole planes of sub-domains and its cuts are few. A rank goes to the
    device that holds the middle of its points."""
    if ndev < 1:
        raise ValueError("device count must be positive")
    pts = rank_points(cs)
    if ndev > len(pts):
        raise ValueError(f"{ndev} devices for {len(pts)} ranks: split the blocks further")
    start = np.concatenate([[0], np.cumsum(pts)[:-1]])
    mid = start + pts / 2.0
    dev = np.minimum((mid * ndev / pts.sum()).astype(np.int64), ndev - 1)
    # every device gets at least one rank
    for d in range(ndev):
        if not np.any(dev == d):
            raise ValueError(f"device {d} gets no rank: the ranks are too uneven for {ndev} devices")
    return dev


@dataclass
class AveragingPass:
    """One averaging pass (points, lines or surface) split over the devices.

    targets / sources: the plan rows (rank, l, first, count) and (rank, l).
    sends[(e, d)]: the (rank, l) points device e sends device d, sorted and
    without repeats. slots[d]: per source entry read by device d's targets,
    -1 for a source on device d itself, else its position in the
    concatenation of sends[(e, d)] over e = 0, 1, ... (e != d)."""
    kind: int
    mode: int  # 0: mean of the sources; 1: running average onto the point
    targets: np.ndarray
    sources: np.ndarray
    sends: Dict[Tuple[int, int], np.ndarray] = field(default_factory=dict)
    slots: Dict[int, np.ndarray] = field(default_factory=dict)

    def remote_points(self, e: int, d: int) -> int:
        return len(self.sends.get((e, d), ()))


class ExchangePlan:
    """The exchanges of case ``cs`` with its ranks on the devices ``device``."""

    def __init__(self, cs: CaseSpec, device: Sequence[int]):
        self.cs = cs
        self.device = np.asarray(device, np.int64)
        if self.device.shape != (len(cs.blocks),) or self.device.min() < 0:
            raise ValueError("one device index per rank")
        self.ndev = int(self.device.max()) + 1
        self.links = api.plan_export(cs, api.PLAN_FACES)
        dv = self.device
        self.cross_links = self.links[dv[self.links[:, 3]] != dv[self.links[:, 0]]]
        self.passes: List[AveragingPass] = []
        for kind in (api.PLAN_POINTS, api.PLAN_LINES, api.PLAN_SURFACE):
            p = AveragingPass(kind, 1 if kind == api.PLAN_SURFACE else 0, api.plan_export(cs, kind),
                              api.plan_export(cs, kind + 3))
            self._split(p)
            self.passes.append(p)

    def _split(self, p: AveragingPass):
        dv = self.device
        for d in range(self.ndev):
            t = p.targets[dv[p.targets[:, 0]] == d]
            # source entries read by d's targets, in plan order
            ent = np.concatenate([np.arange(f, f + c) for f, c in t[:, 2:4]]) if len(t) else \
                np.zeros(0, np.int64)
            src = p.sources[ent]
            sdev = dv[src[:, 0]] if len(src) else np.zeros(0, np.int64)
            slot = np.full(len(p.sources), -1, np.int64)
            base = 0
            for e in range(self.ndev):
                if e == d:
                    continue
                sel = sdev == e
                if not np.any(sel):
                    continue
                pts, inv = np.unique(src[sel], axis=0, return_inverse=True)
                p.sends[(e, d)] = pts
                slot[ent[sel]] = base + inv.reshape(-1)
                base += len(pts)
            p.slots[d] = slot

    def bytes_per_step(self, viscous: bool = True, deriv_bytes: int = 8) -> np.ndarray:
        """Bytes each device sends each other device per time step: [from, to].
        deriv_bytes is the width of an exchanged derivative value (8 FP64, 4
        with FP32 derivatives); filter and averaging values are FP64."""
        m = np.zeros((self.ndev, self.ndev))
        fields = 9 if viscous else 5
        dv = self.device
        for dst, _nn, _ds, src, _ss, lines, code in self.cross_links:
            e, d = dv[src], dv[dst]
            if code in INTERFACE_CODES:
                m[e, d] += lines * (STAGES * fields * 2 * deriv_bytes + 5 * 3 * 8)
            elif code == CURVED_CODE:
                m[e, d] += lines * STAGES * 5 * 8
        for p in self.passes:
            for (e, d), pts in p.sends.items():
                m[e, d] += STAGES * 5 * 8 * len(pts)
        return m

    def summary(self, viscous: bool = True, deriv_bytes: int = 8) -> dict:
        m = self.bytes_per_step(viscous, deriv_bytes)
        pts = rank_points(self.cs)
        load = np.array([pts[self.device == d].sum() for d in range(self.ndev)])
        return {
            "devices": self.ndev,
            "ranks": len(self.cs.blocks),
            "points_per_device": load.tolist(),
            "cross_links": int(len(self.cross_links)),
            "bytes_per_step_out": m.sum(axis=1).tolist(),
            "bytes_per_step_max_out": float(m.sum(axis=1).max()),
            "averaging_remote_points": sum(len(v) for p in self.passes for v in p.sends.values()),
        }
