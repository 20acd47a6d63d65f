"""Case descriptions and synthetic inputs for the Canard per-step hot path.

A case is the content of the reference's ``input.canard`` namelists for one run
(``nml_domdcomp``, ``nml_numerics``, ``nml_physics``, ``nml_canard``,
``nml_sponge``; see src/mo_io.f90:35-66, src/mo_physics.f90:86-111,
src/mo_numerics.f90:97-110, src/mo_sponge.f90:20-30, src/mo_gridgen.f90:49-71)
plus the grid coordinates and the initial conserved state of every block.

Every block is one sub-domain with ``nbpc = 1`` (one rank per block in the
reference); ``decompose`` splits blocks into the reference's sub-domains for
the oracle. Field arrays use the reference layout: a NumPy array of shape
``(ncols, lze+1, let+1, lxi+1)`` in C order is exactly the Fortran array
``q(0:lmx, ncols)`` with ``l = (k*(let+1)+j)*(lxi+1)+i`` (src/mo_utils.f90:54-69).

The workloads are seeded synthetic stand-ins for the configurations the
throughput metric is quoted on (the reference ships no data sets):

* ``tgv``: Taylor-Green vortex on [0, 2pi]^3, periodic on all faces.
* ``curvilinear_4block``: 4 blocks tiled 2x2 in (xi, eta) on a sine-perturbed
  grid, non-reflecting GCBC in/outflow, sponge, periodic in zeta.
* ``vortex``: isentropic vortex advected through a GCBC outflow.
* ``batched``: many independent single-block TGV / vortex cases.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

# boundary codes, src/mo_parameters.f90:34-40
BC_NON_REFLECTIVE = 10
BC_WALL_INVISCID = 20
BC_WALL_VISCOUS = 25
BC_INTER_CURV = 30
BC_INTER_STRAIGHT = 35
BC_INTER_SUBDOMAINS = 40
BC_PERIODIC = 45

GAM = 1.4


@dataclasses.dataclass
class BlockSpec:
    lxi: int
    let: int
    lze: int
    nbc: Sequence[Sequence[int]]   # [direction][side]
    mbcd: Sequence[Sequence[int]]  # [direction][side], neighbour block or -1

    @property
    def shape(self):
        return (self.lze + 1, self.let + 1, self.lxi + 1)

    @property
    def npts(self) -> int:
        return (self.lxi + 1) * (self.let + 1) * (self.lze + 1)


@dataclasses.dataclass
class CaseSpec:
    blocks: List[BlockSpec]
    viscous: int = 1
    fltk: float = 0.85          # namelist value; the code uses pi*fltk
    fltrbc: float = 0.85
    reoo: float = 16000.0
    tempoo: float = 300.0
    amach: Sequence[float] = (0.0, 0.0, 0.0)
    timf: float = 0.0
    nsmf: int = 1
    cfl: float = 0.8
    szco: float = 0.0
    szth0: float = 0.0
    szth1: float = 0.0
    doml0: float = 0.0
    doml1: float = 0.0
    xyz: Optional[List[np.ndarray]] = None   # per block (3, Z, Y, X)
    qa: Optional[List[np.ndarray]] = None    # per block (5, Z, Y, X)
    name: str = ""
    # set by decompose(): the blocks above are then sub-domains (ranks) of the
    # input's blocks; see decompose()
    sub: Optional[dict] = None

    @property
    def npts(self) -> int:
        return sum(b.npts for b in self.blocks)


def _conserved(rho, u, v, w, p):
    q = np.empty((5,) + rho.shape)
    q[0] = rho
    q[1] = rho * u
    q[2] = rho * v
    q[3] = rho * w
    q[4] = p / (GAM - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return q


def tgv(n: int = 64, mach: float = 0.1, re: float = 1600.0, viscous: int = 1,
        nx: Optional[int] = None, ny: Optional[int] = None, nz: Optional[int] = None) -> CaseSpec:
    """Taylor-Green vortex: u = V0 sin x cos y cos z, v = -V0 cos x sin y cos z,
    w = 0, p = 1/gamma + V0^2/16 (cos 2x + cos 2y)(cos 2z + 2), isothermal start
    (T = gamma p / rho = 1), V0 = Mach in units of the sound speed.

    The flow is at rest in the frame (amach = 0), so the reference uses reoo
    unscaled (src/mo_physics.f90:104-106): reoo = Re / M."""
    nx = nx or n
    ny = ny or n
    nz = nz or n
    per = [[BC_PERIODIC, BC_PERIODIC]] * 3
    blk = BlockSpec(nx, ny, nz, [list(p) for p in per], [[0, 0], [0, 0], [0, 0]])
    x = 2 * np.pi * np.arange(nx + 1) / nx
    y = 2 * np.pi * np.arange(ny + 1) / ny
    z = 2 * np.pi * np.arange(nz + 1) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    xyz = np.stack([X, Y, Z])
    v0 = mach
    u = v0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -v0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    p = 1.0 / GAM + v0 * v0 / 16.0 * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    rho = GAM * p
    return CaseSpec([blk], viscous=viscous, reoo=re / mach, xyz=[xyz], qa=[_conserved(rho, u, v, w, p)],
                    name=f"tgv{nx}x{ny}x{nz}")


def vortex_state(X, Y, mach, strength=5.0, radius=1.0, xc=0.0, yc=0.0):
    """Isentropic vortex (strength in units of the sound speed) in a uniform
    stream of Mach ``mach`` along x; returns rho, u, v, w, p."""
    r2 = ((X - xc) ** 2 + (Y - yc) ** 2) / radius ** 2
    eps = strength * mach / (2 * np.pi)   # peak swirl, Yee's beta scaled by the stream speed
    du = -eps * (Y - yc) / radius * np.exp(0.5 * (1 - r2))
    dv = eps * (X - xc) / radius * np.exp(0.5 * (1 - r2))
    T = 1.0 - 0.5 * (GAM - 1) * eps * eps * np.exp(1 - r2)   # cyclostrophic, isentropic
    rho = T ** (1.0 / (GAM - 1))
    p = rho * T / GAM
    return rho, mach + du, dv, np.zeros_like(du), p


def vortex(nx=384, ny=256, nz=128, mach=0.5, strength=5.0, radius=1.0, re=1e5, viscous=1,
           sponge_cells=20, xc=4.0, cfl=0.5) -> CaseSpec:
    """Isentropic vortex carried by a Mach ``mach`` stream through a
    non-reflecting (GCBC) outflow, in Canard's moving-frame form: the state
    holds the vortex around fluid at rest, the frame moves at Mach ``mach``
    along x (amach1 = mach, nsmf = 1), and sponges over ``sponge_cells`` cells
    at both x ends hold the far field (src/mo_sponge.f90:34-88; the sponge
    profile spans 2 szth, so szth = half the sponge width). Without them the
    all-non-reflecting box drifts and the reference algorithm itself stops
    being finite after a few hundred steps.

    Domain [-8, 8] x [-16/3, 16/3] x [0, 4] at 384x256x128 cells: xi faces
    BC 10 (inflow and outflow), eta and zeta periodic. With non-reflecting
    eta faces as well, errors grow at the edges where two non-reflecting
    faces meet a periodic seam, in FP64 too, within ~1000 steps.

    The vortex starts at x = ``xc`` (4) and the stream carries it towards
    the outflow at x = 8, which it reaches within 1000 steps at CFL 0.5 on
    the stated grid. At CFL 0.8 the same case grows slowly from about step
    600 in FP64 (the non-reflecting faces' time-step limit, as for the
    curvilinear case)."""
    bc = [[BC_NON_REFLECTIVE, BC_NON_REFLECTIVE], [BC_PERIODIC, BC_PERIODIC], [BC_PERIODIC, BC_PERIODIC]]
    mb = [[-1, -1], [0, 0], [0, 0]]
    blk = BlockSpec(nx, ny, nz, bc, mb)
    lx = 16.0
    dx = lx / nx
    x = -8.0 + dx * np.arange(nx + 1)
    y = -0.5 * ny * dx + dx * np.arange(ny + 1)  # periodic: the last point repeats the first
    z = dx * np.arange(nz + 1)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rho, u, v, w, p = vortex_state(X, Y, mach, strength, radius, xc=xc)
    szth = 0.5 * sponge_cells * dx
    return CaseSpec([blk], viscous=viscous, reoo=re, amach=(mach, 0.0, 0.0), nsmf=1, cfl=cfl,
                    szco=1.0, szth0=szth, szth1=szth, doml0=8.0, doml1=8.0,
                    xyz=[np.stack([X, Y, Z])], qa=[_conserved(rho, u - mach, v, w, p)],
                    name=f"vortex{nx}x{ny}x{nz}")


def curvilinear_4block(nxb=192, nyb=128, nzb=64, mach=0.4, re=1e5, noise=0.01, seed=7,
                       viscous=1, sponge_cells=20, inflow_sponge_cells=None, cfl=0.5) -> CaseSpec:
    """Four blocks tiled 2x2 in (xi, eta) on x = xi + 0.05 sin(2 pi eta) sin(2 pi zeta),
    y = eta + 0.05 sin(2 pi xi), z = zeta with unit index spacing h = 1/128.

    Block numbering: 0 (lower left), 1 (lower right), 2 (upper left), 3 (upper
    right). Faces: xi-min of 0/2 and xi-max of 1/3 are non-reflecting (10);
    the xi interface is a straight interface (35); the eta interface is a
    curved interface (30); the outer eta faces are periodic between the lower
    and the upper row (45); zeta is periodic on each block (45).

    The uniform stream (Mach ``mach`` along x) is carried by the moving frame
    (amach1 = mach, nsmf = 1), with 1% seeded white velocity noise between the
    sponges. The sponges cover the last ``sponge_cells`` cells before the
    outflow and the first ``inflow_sponge_cells`` (default: as many) after the
    inflow (szth1, szth0 = half of each, src/mo_sponge.f90:46-51).

    CFL 0.5: at the reference's usual 0.8 the scheme itself (the oracle, any
    size tried) grows without bound within 200-350 steps on this grid with
    its non-reflecting xi faces; the same case periodic in xi, or at CFL 0.5,
    stays bounded over 400 steps."""
    # x and y spacing 1/nyb (1/128 at the stated size): the two block rows span
    # eta in [0, 2], whole periods of sin(2 pi eta); zeta spans [0, 1] over the
    # nzb cells, one period of sin(2 pi zeta), so the grid is smooth across
    # both periodic seams
    h = 1.0 / nyb
    hz = 1.0 / nzb
    NX, NY, NZ = 2 * nxb, 2 * nyb, nzb
    blocks = []
    for bj in range(2):
        for bi in range(2):
            nbc = [[0, 0], [0, 0], [BC_PERIODIC, BC_PERIODIC]]
            mb = [[-1, -1], [-1, -1], [-1, -1]]
            me = 2 * bj + bi
            mb[2] = [me, me]
            if bi == 0:
                nbc[0] = [BC_NON_REFLECTIVE, BC_INTER_STRAIGHT]
                mb[0] = [-1, me + 1]
            else:
                nbc[0] = [BC_INTER_STRAIGHT, BC_NON_REFLECTIVE]
                mb[0] = [me - 1, -1]
            other = 2 * (1 - bj) + bi
            if bj == 0:
                nbc[1] = [BC_PERIODIC, BC_INTER_CURV]
            else:
                nbc[1] = [BC_INTER_CURV, BC_PERIODIC]
            mb[1] = [other, other]
            blocks.append(BlockSpec(nxb, nyb, nzb, nbc, mb))
    rng = np.random.default_rng(seed)
    ni = sponge_cells if inflow_sponge_cells is None else inflow_sponge_cells
    xyz, qa = [], []
    for bj in range(2):
        for bi in range(2):
            i = bi * nxb + np.arange(nxb + 1)
            j = bj * nyb + np.arange(nyb + 1)
            k = np.arange(nzb + 1)
            Kz, Jy, Ix = np.meshgrid(k, j, i, indexing="ij")
            xi, eta, zeta = Ix * h, Jy * h, Kz * hz
            X = xi + 0.05 * np.sin(2 * np.pi * eta) * np.sin(2 * np.pi * zeta)
            Y = eta + 0.05 * np.sin(2 * np.pi * xi)
            Z = zeta
            xyz.append(np.stack([X, Y, Z]))
            shape = X.shape
            rho = np.ones(shape)
            p = np.full(shape, 1.0 / GAM)
            # the noise vanishes inside the sponges at both xi ends: white
            # noise on the non-reflecting faces makes the reference scheme
            # itself grow without bound within ~200 steps (oracle runs)
            quiet = ((Ix >= ni) & (Ix <= NX - sponge_cells)).astype(float)
            u = noise * mach * rng.standard_normal(shape) * quiet
            v = noise * mach * rng.standard_normal(shape) * quiet
            w = noise * mach * rng.standard_normal(shape) * quiet
            qa.append(_conserved(rho, u, v, w, p))
    xmax = NX * h
    return CaseSpec(blocks, viscous=viscous, reoo=re, amach=(mach, 0.0, 0.0), nsmf=1, cfl=cfl,
                    szco=1.0, szth0=0.5 * ni * h, szth1=0.5 * sponge_cells * h, doml0=0.0, doml1=xmax,
                    xyz=xyz, qa=qa, name=f"curv4x{nxb}x{nyb}x{nzb}")


def batched(ncases=64, seed=11, lo=32, hi=96) -> List[CaseSpec]:
    """Independent single-block cases with seeded uneven sides in [lo, hi],
    alternating TGV and isentropic vortex, Mach in [0.1, 0.5], Re in [400, 3200]."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(ncases):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, size=3))
        mach = float(rng.uniform(0.1, 0.5))
        re = float(rng.uniform(400.0, 3200.0))
        if c % 2 == 0:
            cs = tgv(nx=nx, ny=ny, nz=nz, mach=mach, re=re)
        else:
            cs = _periodic_vortex(nx, ny, nz, mach, re)
        cs.name = f"b{c}:" + cs.name
        out.append(cs)
    return out


def _periodic_vortex(nx, ny, nz, mach, re):
    per = [[BC_PERIODIC, BC_PERIODIC]] * 3
    blk = BlockSpec(nx, ny, nz, [list(p) for p in per], [[0, 0], [0, 0], [0, 0]])
    L = 10.0
    x = -L / 2 + L * np.arange(nx + 1) / nx
    y = -L / 2 + L * np.arange(ny + 1) / ny
    z = L * np.arange(nz + 1) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rho, u, v, w, p = vortex_state(X, Y, mach, 5.0, 1.0)
    return CaseSpec([blk], viscous=1, reoo=re / mach, xyz=[np.stack([X, Y, Z])],
                    qa=[_conserved(rho, u, v, w, p)], name=f"pvortex{nx}x{ny}x{nz}")


def noise_fields(blk: BlockSpec, nfields: int = 5, seed: int = 20261203, kmax: int = 32) -> np.ndarray:
    """Seeded N(0,1) noise plus sum_{k=1..kmax} sin(k 2 pi i / N) along each
    direction, for the isolated derivative / filter benches."""
    rng = np.random.default_rng(seed)
    Z, Y, X = blk.shape
    out = rng.standard_normal((nfields,) + blk.shape)
    i = np.arange(X)[None, None, :]
    j = np.arange(Y)[None, :, None]
    k = np.arange(Z)[:, None, None]
    modes = np.zeros(blk.shape)
    for kk in range(1, kmax + 1):
        modes = modes + np.sin(kk * 2 * np.pi * i / max(X - 1, 1)) + np.sin(kk * 2 * np.pi * j / max(Y - 1, 1)) \
            + np.sin(kk * 2 * np.pi * k / max(Z - 1, 1))
    return out + modes[None]


# ---------------------------------------------------------------------------
# The reference's own grid generators and initial condition (host code: they
# run once, before the device holds anything). Coordinates are evaluated with
# the Fortran expressions in the same order, so the grid files they give
# (api.write_grid_file) match the reference's byte for byte where libm is not
# involved (these generators use only +, -, *, /).

def gridtoy(lxi0: int, let0: int, lze0: int, doml0: float, doml1: float, domh: float, span: float) -> np.ndarray:
    """gridtoy (src/mo_gridgen.f90:510-575): one Cartesian block of
    (lxi0+1) x (let0+1) x (lze0+1) points, x = -doml0 + i (doml1+doml0)/lxi0,
    y = -domh + j 2 domh/let0, z = span ((lze0-k)/lze0 - 1/2). Returns xyz
    (3, lze0+1, let0+1, lxi0+1) in the reference layout."""
    ra0 = (doml1 + doml0) / lxi0
    ra1 = 2.0 * domh / let0
    x = -doml0 + (np.arange(lxi0 + 1, dtype=np.float64) - 0.0) * ra0
    y = -domh + (np.arange(let0 + 1, dtype=np.float64) - 0.0) * ra1
    z = span * ((lze0 - np.arange(lze0 + 1, dtype=np.float64)) / lze0 - 0.5)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return np.stack([X, Y, Z])


def gridtoy_multi(lxi0: int, lxi1: int, lxi2: int, let0: int, lze0: int, doml0: float, doml1: float,
                  domh: float, span: float) -> List[np.ndarray]:
    """gridtoy_multi (src/mo_gridgen.f90:577-654): six Cartesian blocks, three
    along x (lxi0, lxi1, lxi2 cells) by two along y (let0 cells each), sharing
    their interface points. Block mb covers i in its column (mb % 3) and j in
    its row (mb // 3) of the global (lxi0+lxi1+lxi2+3) x (2 let0+2) point
    array. Returns xyz (3, lze0+1, let0+1, lxi_mb+1) per block."""
    lxit = lxi0 + lxi1 + lxi2 + 2
    lett = 2 * let0 + 1
    lxis1 = lxi0 + 1
    lxie1 = lxis1 + lxi1
    lxis2 = lxie1 + 1
    cols = [(0, lxi0, 0.0), (lxis1, lxie1, 1.0), (lxis2, lxit, 2.0)]
    rows = [(0, let0, 0.0), (let0 + 1, lett, 1.0)]
    ra0 = (doml1 + doml0) / (lxi0 + lxi1 + lxi2)
    ra1 = domh / (2.0 * let0) * 2.0
    z = span * ((lze0 - np.arange(lze0 + 1, dtype=np.float64)) / lze0 - 0.5)
    out = []
    for mb in range(6):
        is_, ie, ra2 = cols[mb % 3]
        js, je, ra3 = rows[mb // 3]
        x = -doml0 + (np.arange(is_, ie + 1, dtype=np.float64) - ra2) * ra0
        y = -domh + (np.arange(js, je + 1, dtype=np.float64) - ra3) * ra1
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        out.append(np.stack([X, Y, Z]))
    return out


def initialo(xyz: np.ndarray) -> np.ndarray:
    """The reference's initial condition (initialo, src/mo_physics.f90:117-140):
    a vortex at the origin, k1 = 12.5, radius 1, k2 = 1,
    ao = k2/(2 pi) sqrt(exp(1 - k1^2 (x^2 + y^2))), rho = (1 - (gamma-1)/2 ao^2)^(1/(gamma-1)),
    u = k1 y ao, v = -k1 x ao, w = 0, rho E = rho^gamma/(gamma(gamma-1)) + rho |u|^2/2.
    Returns qa (5, ...) on the points of xyz (3, ...)."""
    x, y = xyz[0], xyz[1]
    radv, k1, k2 = 1.0, 12.5, 1.0
    gamm1 = GAM - 1.0
    ao = k2 / 2.0 / math.pi * np.sqrt(np.exp(1 - k1 * k1 * (x * x + y * y) / (radv * radv)))
    bo = (1.0 - 0.5 * gamm1 * ao * ao) ** (1.0 / gamm1)
    v1 = k1 * y * ao / radv
    v2 = -k1 * x * ao / radv
    hv2 = 0.5 * ((v1 * v1 + v2 * v2) + 0.0)
    q = np.empty((5,) + x.shape)
    q[0] = bo
    q[1] = bo * v1
    q[2] = bo * v2
    q[3] = bo * 0.0
    q[4] = (1.0 / GAM) * (1.0 / gamm1) * bo ** GAM + hv2 * bo
    return q


def reference_validation(lxi0: int = 50, let0: int = 50, lze0: int = 16) -> CaseSpec:
    """The reference's validation run (run/exp.validation): one block from
    gridtoy (doml0 0.5, doml1 1.0, domh 0.5, span 0.1), non-reflecting GCBC on
    the xi and eta faces, periodic in zeta, initialo's vortex in a Mach 0.3
    frame, Re 5e5, Tinf 300 K, fltk 0.65, fltrbc 0.9, CFL 1.4. Its input file
    misspells the sponge namelist (no '&'), so szco keeps its zero default and
    there is no sponge. The reference splits the block into 2 x 2 sub-domains
    (nbpc); here it is one sub-domain."""
    blk = BlockSpec(lxi0, let0, lze0, [[BC_NON_REFLECTIVE] * 2, [BC_NON_REFLECTIVE] * 2, [BC_PERIODIC] * 2],
                    [[-1, -1], [-1, -1], [0, 0]])
    xyz = gridtoy(lxi0, let0, lze0, 0.5, 1.0, 0.5, 0.1)
    return CaseSpec([blk], viscous=1, fltk=0.65, fltrbc=0.9, reoo=500000.0, tempoo=300.0, amach=(0.3, 0.0, 0.0),
                    nsmf=1, cfl=1.4, doml0=0.5, doml1=1.0, xyz=[xyz], qa=[initialo(xyz)],
                    name=f"validation{lxi0}x{let0}x{lze0}")


def reference_toy(lxi: int = 100, let0: int = 100, lze0: int = 16) -> CaseSpec:
    """The reference's toy run (run/exp.toy): six blocks from gridtoy_multi
    (lxi0 = lxi1 = lxi2 = lxi; doml0 0.5, doml1 1.0, domh 0.5, span 0.1),
    straight interfaces (BC 35) between them, non-reflecting GCBC at the x
    ends, periodic in eta across the two rows and in zeta, initialo's vortex
    in a Mach 0.3 frame, Re 5e5, fltk 0.65, fltrbc 0.9, CFL 1.4; no sponge
    (the input misspells its namelist). The reference splits each block into
    4 x 2 sub-domains; here each block is one."""
    nr, st, pe = BC_NON_REFLECTIVE, BC_INTER_STRAIGHT, BC_PERIODIC
    # nbbc / mbcd of run/exp.toy, per block [direction][side]
    nbbc = [[[nr, st], [pe, st], [pe, pe]], [[st, st], [pe, st], [pe, pe]], [[st, nr], [pe, st], [pe, pe]],
            [[nr, st], [st, pe], [pe, pe]], [[st, st], [st, pe], [pe, pe]], [[st, nr], [st, pe], [pe, pe]]]
    mbcd = [[[-1, 1], [3, 3], [0, 0]], [[0, 2], [4, 4], [1, 1]], [[1, -1], [5, 5], [2, 2]],
            [[-1, 4], [0, 0], [3, 3]], [[3, 5], [1, 1], [4, 4]], [[4, -1], [2, 2], [5, 5]]]
    xyz = gridtoy_multi(lxi, lxi, lxi, let0, lze0, 0.5, 1.0, 0.5, 0.1)
    blocks = [BlockSpec(lxi, let0, lze0, nbbc[m], mbcd[m]) for m in range(6)]
    return CaseSpec(blocks, viscous=1, fltk=0.65, fltrbc=0.9, reoo=500000.0, tempoo=300.0, amach=(0.3, 0.0, 0.0),
                    nsmf=1, cfl=1.4, doml0=0.5, doml1=1.0, xyz=xyz, qa=[initialo(g) for g in xyz],
                    name=f"toy6x{lxi}x{let0}x{lze0}")


# ---------------------------------------------------------------------------
# Sub-domains (nbpc > 1): the reference's domain decomposition of its blocks
# into ranks (domdcomp_init, src/mo_domdcomp.f90:85-232). Only the CPU oracle
# runs such cases so far; the device context takes one sub-domain per block.

def decompose(cs: CaseSpec, nbpc: Sequence[Sequence[int]]) -> CaseSpec:
    """Splits block m of cs into nbpc[m] = (n_xi, n_eta, n_zeta) sub-domains as
    domdcomp_init does: along a direction of l cells split in n, the first
    sub-domain has l - ((l+1)/n)(n-1) cells and the others (l+1)/n - 1 (points
    are not shared); inner faces get code 40 (BC_INTER_SUBDOMAINS) and the
    neighbouring rank, faces on the block's boundary keep its code and face
    the neighbouring block's sub-domain at that end with the same transverse
    position. Ranks are numbered rank = mo(m) + (k n_eta + j) n_xi + i for the
    position (i, j, k). The result's blocks are the ranks; its ``sub`` holds
    the input's nbpc and mbcd, per rank (block, i, j, k), and per rank the
    slice of its block's points (z0, y0, x0, nz, ny, nx)."""
    nb = len(cs.blocks)
    nbpc = [tuple(int(v) for v in p) for p in nbpc]
    if len(nbpc) != nb or any(len(p) != 3 or min(p) < 1 for p in nbpc):
        raise ValueError("nbpc needs three positive counts per block")
    # a face's sub-domains meet the neighbouring block's at equal transverse
    # positions (idsd3 below), so both blocks split the face alike
    for m, b in enumerate(cs.blocks):
        for d in range(3):
            for mm in b.mbcd[d]:
                if mm >= 0 and any(nbpc[mm][t] != nbpc[m][t] for t in ((d + 1) % 3, (d + 2) % 3)):
                    raise ValueError(f"blocks {m} and {mm} split their shared face differently "
                                     f"({nbpc[m]} and {nbpc[mm]})")
    mo = [0]
    for p in nbpc:
        mo.append(mo[-1] + p[0] * p[1] * p[2])

    def rank(m, pos):
        return mo[m] + (pos[2] * nbpc[m][1] + pos[1]) * nbpc[m][0] + pos[0]

    def idsd3(i, j, k, mm, nn):  # src/mo_domdcomp.f90:588-605
        pos = [0, 0, 0]
        pos[nn - 1], pos[nn % 3], pos[(nn + 1) % 3] = i, j, k
        return rank(mm, pos)

    blocks, xyz, qa, ranks, slices = [], [], [], [], []
    for m, b in enumerate(cs.blocks):
        ll = (b.lxi, b.let, b.lze)
        n = nbpc[m]
        for kz in range(n[2]):
            for jy in range(n[1]):
                for ix in range(n[0]):
                    pos = (ix, jy, kz)
                    r = rank(m, pos)
                    lk, st, nbc, mcd = [0] * 3, [0] * 3, [None] * 3, [None] * 3
                    for d in range(3):
                        mak, lpk, mpk = n[d], pos[d], (1, n[0], n[0] * n[1])[d]
                        face = []
                        for ip in (0, 1):
                            mm = b.mbcd[d][ip]
                            face.append(-1 if mm == -1 else
                                        idsd3((1 - ip) * (nbpc[mm][d] - 1), pos[(d + 1) % 3], pos[(d + 2) % 3],
                                              mm, d + 1))
                        base = (ll[d] + 1) // mak
                        first = ll[d] - base * (mak - 1)
                        if mak == 1:
                            lk[d], nbc[d], mcd[d] = ll[d], [b.nbc[d][0], b.nbc[d][1]], face
                        elif lpk == 0:
                            lk[d], nbc[d], mcd[d] = first, [b.nbc[d][0], BC_INTER_SUBDOMAINS], [face[0], r + mpk]
                        elif lpk < mak - 1:
                            lk[d], nbc[d], mcd[d] = base - 1, [BC_INTER_SUBDOMAINS] * 2, [r - mpk, r + mpk]
                        else:
                            lk[d], nbc[d], mcd[d] = base - 1, [BC_INTER_SUBDOMAINS, b.nbc[d][1]], [r - mpk, face[1]]
                        st[d] = 0 if lpk == 0 else first + 1 + (lpk - 1) * base
                    assert r == len(blocks)
                    if min(lk) < 12:
                        raise ValueError(f"block {m}, sub-domain {pos}: {[v + 1 for v in lk]} points; the interface "
                                         "closures need at least 13 per direction")
                    blocks.append(BlockSpec(lk[0], lk[1], lk[2], nbc, mcd))
                    sl = (st[2], st[1], st[0], lk[2] + 1, lk[1] + 1, lk[0] + 1)
                    cut = (slice(None), slice(sl[0], sl[0] + sl[3]), slice(sl[1], sl[1] + sl[4]),
                           slice(sl[2], sl[2] + sl[5]))
                    if cs.xyz is not None:
                        xyz.append(np.ascontiguousarray(cs.xyz[m][cut]))
                    if cs.qa is not None:
                        qa.append(np.ascontiguousarray(cs.qa[m][cut]))
                    ranks.append((m, ix, jy, kz))
                    slices.append(sl)
    sub = {"nbpc": [list(p) for p in nbpc], "mbcd": [[list(f) for f in b.mbcd] for b in cs.blocks],
           "ranks": ranks, "slices": slices, "shapes": [b.shape for b in cs.blocks]}
    return dataclasses.replace(cs, blocks=blocks, xyz=xyz if cs.xyz is not None else None,
                               qa=qa if cs.qa is not None else None, sub=sub,
                               name=cs.name + ":" + "x".join("%d%d%d" % p for p in nbpc))


def compose(sub: dict, arrays: Sequence[np.ndarray]) -> List[np.ndarray]:
    """The input blocks' arrays (ncols, Z, Y, X) from the ranks' arrays of a
    decomposed case (decompose's ``sub``)."""
    out = [None] * len(sub["shapes"])
    for (m, *_), sl, a in zip(sub["ranks"], sub["slices"], arrays):
        if out[m] is None:
            out[m] = np.zeros((a.shape[0],) + tuple(sub["shapes"][m]))
        out[m][:, sl[0]:sl[0] + sl[3], sl[1]:sl[1] + sl[4], sl[2]:sl[2] + sl[5]] = a
    return out
