"""The channel of the adjoint benchmark configuration and a small version of
it (test infrastructure): velocity inlet with a per-node parabolic profile,
non-equilibrium pressure outlet (rho = 1), interpolated no-slip walls and a
solid cube obstacle, K17 with a global body force.

Full size: 128 x 64 x 64 nodes, a 12^3 cube at x = 40 centred in y and z,
inlet peak 0.04 with +-2% seeded noise, g = (1e-6, 0, 0), nu = 0.02
(the configuration leaves nu open; 0.02 gives Re = 0.04 * 64 / 0.02 = 128),
objective J = mean u_x over the 16^3 box x in [80, 96), centred in y and z.
"""
from __future__ import annotations

import numpy as np

from virtualfluids_b200.grid import MultipleGridBuilder, SideType


def channel_builder(nx, ny, nz, cube):
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


def full_channel():
    return channel_builder(128, 64, 64, (40, 26, 26, 52, 38, 38))


def small_channel():
    return channel_builder(16, 8, 8, (6, 3, 3, 8, 5, 5))


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
