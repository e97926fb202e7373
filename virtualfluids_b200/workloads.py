"""Synthetic workloads of the benchmark and parity tests.

No dataset is involved; every input is generated from seeded formulas.

Taylor-Green vortex (periodic cube of n^3 fluid nodes on [-pi, pi]^3, the
set-up of apps/gpu/TaylorGreenVortex/TaylorGreenVortex.cpp:107-148):
    u  = u0 (sin x cos y cos z, -cos x sin y cos z, 0)
    drho = 3 (u0^2 / 16) (cos 2x + cos 2y) (cos 2z + 2)
with u0 = 0.05, uniform noise of +-1e-3 u0 on each velocity component
(seeded), viscosity for Re = 1600 on the length n / (2 pi).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .grid import taylor_green_grid


@dataclass
class TaylorGreen:
    n: int
    u0: float
    nu: float
    omega: float
    grid: dict
    rho: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray


def taylor_green_viscosity(n: int, u0: float = 0.05, reynolds: float = 1600.0) -> float:
    return u0 * (n / (2.0 * math.pi)) / reynolds


def taylor_green(n: int, u0: float = 0.05, reynolds: float = 1600.0, noise: float = 1e-3,
                 seed: int = 1234) -> TaylorGreen:
    g = taylor_green_grid(n)
    x, y, z = g["coordX"], g["coordY"], g["coordZ"]
    rho = 3.0 * ((u0 * u0) / 16.0 * (np.cos(2.0 * x) + np.cos(2.0 * y)) * (np.cos(2.0 * z) + 2.0))
    vx = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    vy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    vz = np.zeros_like(x)
    if noise > 0:
        rng = np.random.default_rng(seed)
        amp = noise * u0
        vx = vx + rng.uniform(-amp, amp, x.shape)
        vy = vy + rng.uniform(-amp, amp, x.shape)
        vz = vz + rng.uniform(-amp, amp, x.shape)
    solid = g["geo"] != 19
    for a in (rho, vx, vy, vz):
        a[solid] = 0.0
    nu = taylor_green_viscosity(n, u0, reynolds)
    omega = 1.0 / (3.0 * nu + 0.5)
    return TaylorGreen(n, u0, nu, omega, g, rho, vx, vy, vz)


def cavity_grid(n: int, lid: float = 0.05) -> dict:
    """Level 0 of the lid-driven cavity: n^3 nodes, interpolated no-slip
    (q = 1/2) on five faces and the lid velocity (lid, 0, 0) on +z, built by
    the library's grid builder."""
    from .grid import MultipleGridBuilder, SideType
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, n - 1, n - 1, n - 1, 1.0)
    b.buildGrids()
    for side in (SideType.MX, SideType.PX, SideType.MY, SideType.PY, SideType.MZ):
        b.setNoSlipBoundaryCondition(side)
    b.setVelocityBoundaryCondition(SideType.PZ, lid, 0.0, 0.0)
    return b.arrays()[0]


def interface_planes(ncg: int = 128, nfg: int = 256, cf_planes=(40, 41), fc_planes=(80,)):
    """Two periodic boxes (coarse ncg^3, fine nfg^3) with structured interface
    cells: coarse-to-fine cells on the coarse z planes `cf_planes`, each
    writing the fine 2x2x2 block at twice its coordinates, and fine-to-coarse
    cells on `fc_planes` reading the fine block there.  No two cells write the
    same node.  Returns (coarse grid, fine grid, {"cf": (coarse, fine),
    "fc": (coarse, fine)}) with uint32 cell index arrays."""
    gc, gf = taylor_green_grid(ncg), taylor_green_grid(nfg)
    flc, flf = gc["fluid"], gf["fluid"]
    ii, jj = np.meshgrid(np.arange(ncg), np.arange(ncg), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()
    cells = {}
    for tag, planes in (("cf", cf_planes), ("fc", fc_planes)):
        cc = [flc[ii + ncg * (jj + ncg * kk)] for kk in planes]
        ff = [flf[2 * ii + nfg * (2 * jj + nfg * 2 * kk)] for kk in planes]
        cells[tag] = (np.concatenate(cc).astype(np.uint32), np.concatenate(ff).astype(np.uint32))
    return gc, gf, cells


def wall_mounted_cube(seed: int = 1234, coarse=(256, 96, 96), box=(48, 24, 0, 128, 72, 40), cube_x: int = 64,
                      cube_side: int = 16, inlet: float = 0.04, noise: float = 0.01) -> list[dict]:
    """The wall-mounted cube in a channel on two levels, built by the
    library's grid builder: coarse grid nx x ny x nz (spacing 1), a refined
    box (level 1), a solid cube of side `cube_side` on the floor at x =
    cube_x centred in y with interpolated no-slip faces, velocity inlet
    `inlet` with seeded +-`noise` relative noise per node, non-equilibrium
    pressure outlet (drho = 0), no-slip floor, slip top, periodic span.
    Returns the per-level array dicts (the inlet noise applied), ready for
    Simulation."""
    from .grid import MultipleGridBuilder, SideType
    nx, ny, nz = coarse
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, nx - 1, ny - 1, nz - 1, 1.0)
    b.addGrid(box, 1)
    y0 = ny / 2 - cube_side / 2
    b.addGeometry((cube_x, y0, 0, cube_x + cube_side, y0 + cube_side, cube_side))
    b.setPeriodicBoundaryCondition(False, True, False)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, inlet, 0.0, 0.0)
    b.setPressureBoundaryCondition(SideType.PX, 0.0)
    b.setNoSlipBoundaryCondition(SideType.MZ)
    b.setSlipBoundaryCondition(SideType.PZ, 0.0, 0.0, 1.0)
    b.setNoSlipBoundaryCondition(SideType.GEOMETRY)
    levels = b.arrays()
    rng = np.random.default_rng(seed)
    for g in levels:
        vx = g["velocity.vx"]
        inflow = vx != 0
        vx[inflow] = vx[inflow] * (1.0 + rng.uniform(-noise, noise, int(inflow.sum())))
    return levels


# --------------------------------------------------------------------------- #
# The adjoint channel: velocity inlet with a per-node parabolic profile,
# non-equilibrium pressure outlet (rho = 1), interpolated no-slip walls and a
# solid cube obstacle, K17 with a global body force.  Full size: 128 x 64 x 64
# fluid nodes, a 12^3 cube at x = 40 centred in y and z, inlet peak 0.04 with
# +-2% seeded noise, g = (1e-6, 0, 0), nu = 0.02 (Re = 0.04 * 64 / 0.02 = 128;
# the benchmark configuration leaves nu open), objective J = mean u_x over the
# 16^3 box x in [80, 96), centred in y and z.  adjoint_channel_small() is a
# 16 x 8 x 8 version with a 2^3 cube.
# --------------------------------------------------------------------------- #
def adjoint_channel_builder(nx, ny, nz, cube):
    from .grid import MultipleGridBuilder, SideType
    b = MultipleGridBuilder()
    # nx x ny x nz fluid nodes at half-integer positions; the walls lie halfway
    # to the stoppers, at 0 and n
    b.addCoarseGrid(0, 0, 0, nx, ny, nz, 1.0)
    b.addGeometry(cube)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, 0.04, 0.0, 0.0)
    b.setPressureBoundaryCondition(SideType.PX, 0.0)
    for side in (SideType.MY, SideType.PY, SideType.MZ, SideType.PZ):
        b.setNoSlipBoundaryCondition(side)
    b.setNoSlipBoundaryCondition(SideType.GEOMETRY)
    return b


def adjoint_channel():
    return adjoint_channel_builder(128, 64, 64, (40, 26, 26, 52, 38, 38))


def adjoint_channel_small():
    return adjoint_channel_builder(16, 8, 8, (6, 3, 3, 8, 5, 5))


def inlet_entries(g) -> np.ndarray:
    """Indices into the velocity list of the inlet plane's entries (the
    entries whose node lies on the smallest x with a non-zero velocity)."""
    k = g["velocity.k"].astype(np.int64)
    x = g["coordX"][k]
    return np.nonzero((x == x.min()) & (g["velocity.vx"] != 0))[0]


def inlet_profile(g, peak=0.04, noise=0.02, seed=1234) -> np.ndarray:
    """Parabolic inlet velocity over the cross-section (zero on the walls),
    peak `peak`, with seeded relative noise; one value per inlet entry."""
    k = g["velocity.k"].astype(np.int64)
    idx = inlet_entries(g)
    prof = parabola(g, g["coordY"][k[idx]], g["coordZ"][k[idx]], peak)
    rng = np.random.default_rng(seed)
    return prof * (1.0 + rng.uniform(-noise, noise, prof.shape))


def parabola(g, y, z, peak=0.04):
    """peak * 16 yy (1 - yy) zz (1 - zz) with yy, zz the positions relative to
    the walls (halfway beyond the outermost fluid nodes)."""
    fl = g["fluid"]
    ly = g["coordY"][fl].max() + 0.5
    lz = g["coordZ"][fl].max() + 0.5
    yy, zz = y / ly, z / lz
    return np.clip(peak * 16.0 * yy * (1.0 - yy) * zz * (1.0 - zz), 0.0, None)


def objective_box(g, x0, x1, y0, y1, z0, z1):
    """Fluid nodes in [x0, x1) x [y0, y1) x [z0, z1) and the weights of their mean u_x."""
    fl = g["fluid"].astype(np.int64)
    x, y, z = g["coordX"][fl], g["coordY"][fl], g["coordZ"][fl]
    sel = fl[(x >= x0) & (x < x1) & (y >= y0) & (y < y1) & (z >= z0) & (z < z1)]
    return sel.astype(np.uint32), np.full(len(sel), 1.0 / len(sel))


def initial_fields(g):
    """drho = 0 and the noise-free parabolic profile extruded along x (zero in
    solid nodes); independent of the controlled parameters."""
    vx = parabola(g, g["coordY"], g["coordZ"])
    vx[g["geo"] != 19] = 0.0
    zero = np.zeros_like(vx)
    return zero, vx, zero.copy(), zero.copy()
