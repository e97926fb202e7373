"""Shared definitions of the golden scenarios (grid specs and the lattice
update sequence), used both to generate the fixtures from the reference and
to replay them in the tests."""
from __future__ import annotations

import math

import numpy as np

MX, PX, MY, PY, MZ, PZ = range(6)
NONE, NOSLIP, VELOCITY, PRESSURE, SLIP, STRESS = range(6)


def _spec(coarse, periodic=(0, 0, 0), sides=(), thin_walls=False):
    s = np.zeros(64)
    s[0:7] = coarse
    s[7:10] = periodic
    for i, b in enumerate(sides):
        s[30 + 5 * i: 35 + 5 * i] = b
    s[60] = 1.0 if thin_walls else 0.0
    return s


def grid_spec(name: str) -> np.ndarray:
    if name.startswith("tgv"):
        n = int(name[3:])
        d = 2 * math.pi / n
        return _spec([-math.pi, -math.pi, -math.pi, math.pi, math.pi, math.pi, d], (1, 1, 1), thin_walls=True)
    if name == "cavity8":
        sides = [(s, NOSLIP, 0, 0, 0) for s in (MX, PX, MY, PY, MZ)] + [(PZ, VELOCITY, 0.05, 0, 0)]
        return _spec([0, 0, 0, 7, 7, 7, 1.0], sides=sides)
    if name == "cavity8_lidfirst":
        sides = [(PZ, VELOCITY, 0.05, 0, 0)] + [(s, NOSLIP, 0, 0, 0) for s in (MX, PX, MY, PY, MZ)]
        return _spec([0, 0, 0, 7, 7, 7, 1.0], sides=sides)
    if name == "channel":
        sides = [(MX, VELOCITY, 0.04, 0, 0), (PX, PRESSURE, 0.0, 0, 0), (MZ, NOSLIP, 0, 0, 0), (PZ, SLIP, 0, 0, 1)]
        return _spec([0, 0, 0, 11, 7, 7, 1.0], (0, 1, 0), sides=sides)
    if name == "sphere_channel":
        # a solid sphere in a channel: the geometry list's q values come from
        # the ray-sphere intersection (fractional q on most links)
        sides = [(MX, VELOCITY, 0.04, 0, 0), (PX, PRESSURE, 0.0, 0, 0), (MZ, NOSLIP, 0, 0, 0), (PZ, SLIP, 0, 0, 1)]
        s = _spec([0, 0, 0, 31, 15, 15, 1.0], (0, 1, 0), sides=sides)
        s[19] = 2.0
        s[20:24] = [12, 7.3, 7.6, 3.2]
        s[26] = 1.0
        return s
    if name in ("thin_wall_cube", "thin_wall_sphere"):
        # a solid half a node above the no-slip floor of a 16^3 box, built
        # with thin walls: the boundary nodes squeezed between the solid and
        # the floor have no fluid neighbour and become solid stoppers
        sides = [(MZ, NOSLIP, 0, 0, 0), (PZ, NOSLIP, 0, 0, 0)]
        s = _spec([0, 0, 0, 15, 15, 15, 1.0], (1, 1, 0), sides=sides, thin_walls=True)
        if name == "thin_wall_cube":
            s[19] = 1.0
            s[20:26] = [4, 4, 0.5, 10, 10, 6]
        else:
            s[19] = 2.0
            s[20:24] = [7.3, 7.1, 3.5, 3.0]
        s[26] = 1.0
        return s
    if name == "cylinder_channel":
        # a solid cylinder across a channel (axis y, the periodic direction)
        sides = [(MX, VELOCITY, 0.04, 0, 0), (PX, PRESSURE, 0.0, 0, 0), (MZ, NOSLIP, 0, 0, 0), (PZ, SLIP, 0, 0, 1)]
        s = _spec([0, 0, 0, 23, 11, 15, 1.0], (0, 1, 0), sides=sides)
        s[19] = 3.0
        s[20:26] = [8.4, 5.7, 7.3, 2.6, 6.0, 1]
        s[26] = 1.0
        return s
    if name == "abl_stress":
        # the atmospheric boundary layer's sides (apps/gpu/AtmosphericBoundaryLayer):
        # periodic x and y, the wall-model floor (normal +z, sampling offset 2,
        # z0 = 0.1, dx = 1) under a slip lid; the stress parameters of side
        # slot 0 in the spec's stress block (index 176 on)
        sides = [(MZ, STRESS, 0, 0, 1), (PZ, SLIP, 0, 0, -1)]
        s = np.concatenate([_spec([0, 0, 0, 15, 7, 11, 1.0], (1, 1, 0), sides=sides), np.zeros(194 - 64)])
        s[176:179] = [2, 0.1, 1.0]
        return s
    if name == "conglomerate_channel":
        # three primitives united, a sphere removed from the cuboid
        # (Conglomerate); parts as 7 values each from index 64 on
        sides = [(MX, VELOCITY, 0.04, 0, 0), (PX, PRESSURE, 0.0, 0, 0), (MZ, NOSLIP, 0, 0, 0), (PZ, SLIP, 0, 0, 1)]
        s = _spec([0, 0, 0, 27, 19, 17, 1.0], (0, 1, 0), sides=sides)
        parts = [[1, 4, 5, 3, 9, 12, 9], [2, 15.2, 9.6, 8.1, 3.1, 0, 0], [3, 21.4, 9.8, 8.7, 2.2, 7.0, 1],
                 [2, 6.5, 8.3, 7.0, 2.4, 0, 0]]
        s[19] = 5.0
        s[62:64] = [3, 1]
        s[26] = 1.0
        return np.concatenate([s, np.array(parts, float).ravel()])
    raise KeyError(name)


GRID_SCENARIOS = ["tgv6", "tgv8", "cavity8", "cavity8_lidfirst", "channel", "sphere_channel"]
# solids built with thin walls (MultipleGridBuilder::buildGrids(true))
THIN_WALL_SCENARIOS = ["thin_wall_cube", "thin_wall_sphere"]
# solids added after the first fixtures (generated with --extra-grids)
EXTRA_GRID_SCENARIOS = ["cylinder_channel", "conglomerate_channel"]
# the wall-model (stress) BC's lists (generated with --stress)
STRESS_GRID_SCENARIOS = ["abl_stress"]

# multi-level grids made by the reference's builder, which the repository's
# builder reproduces: a channel 24 x 16 x 16 with a refined box and the
# reference's default layer counts, inlet velocity and outlet pressure; the
# cube channel (below); a box refined twice (three levels) with its own layer
# counts (the reference's builder crashes for two layers between levels); a
# box on the floor and the inlet wall (odd starts, refinement into
# two walls) around a solid cuboid
REFINED_SCENARIOS = ["refined_channel", "cube_channel", "two_level_box", "wall_box_solid"]


def refined_spec(name: str) -> np.ndarray:
    if name == "refined_channel":
        sides = [(MX, VELOCITY, 0.02, 0, 0), (PX, PRESSURE, 0.0, 0, 0)]
        s = _spec([0, 0, 0, 23, 15, 15, 1.0], (0, 1, 1), sides=sides)
        s[10] = 1.0
        s[11:17] = [8, 5, 5, 15, 10, 10]
        return s
    if name == "cube_channel":
        # the wall-mounted cube of the two-level benchmark, scaled down: a
        # channel 48 x 16 x 16 (periodic span), inlet velocity, outlet pressure,
        # no-slip floor, slip top, a solid cube of side 4 on the floor inside a
        # refined box, no-slip (interpolated) on the cube faces
        sides = [(MX, VELOCITY, 0.04, 0, 0), (PX, PRESSURE, 0.0, 0, 0), (MZ, NOSLIP, 0, 0, 0), (PZ, SLIP, 0, 0, 1)]
        s = _spec([0, 0, 0, 47, 15, 15, 1.0], (0, 1, 0), sides=sides)
        s[10] = 1.0
        s[11:17] = [12, 4, 0, 28, 12, 8]
        s[19] = 1.0
        s[20:26] = [16, 6, 0, 20, 10, 4]
        s[26] = 1.0
        return s
    if name == "two_level_box":
        sides = [(MX, VELOCITY, 0.03, 0, 0), (PX, PRESSURE, 0.0, 0, 0), (MZ, NOSLIP, 0, 0, 0), (PZ, SLIP, 0, 0, 1)]
        s = _spec([0, 0, 0, 31, 23, 23, 1.0], (0, 1, 0), sides=sides)
        s[10] = 1.0
        s[11:17] = [12, 9, 9, 17, 14, 14]
        s[17:19] = [6, 4]
        s[61] = 2.0
        return s
    if name == "wall_box_solid":
        sides = [(PX, PRESSURE, 0.0, 0, 0), (MX, VELOCITY, 0.04, 0.0, 0), (MZ, NOSLIP, 0, 0, 0), (PZ, SLIP, 0, 0, 1)]
        s = _spec([0, 0, 0, 23, 13, 11, 1.0], (0, 1, 0), sides=sides)
        s[10] = 1.0
        s[11:17] = [0, 3, 0, 10, 10, 6]
        s[17:19] = [6, 3]
        s[19] = 1.0
        s[20:26] = [3, 5, 0, 6, 8, 3]
        s[26] = 1.0
        return s
    raise KeyError(name)


def lattice_sequence(impl, g: dict, precision: str, steps: int = 4) -> np.ndarray:
    """Init both parities, then per step: K17 with a force, the five
    post-collision BC kernels, the pressure BC, and a BGK pass of the other
    parity.  ``impl`` is the oracle or the reference binding."""
    real = np.float64 if precision == "f64" else np.float32
    N = len(g["geo"])
    nx, ny, nz, geo, fl = g["neighborX"], g["neighborY"], g["neighborZ"], g["geo"], g["fluid"]
    rng = np.random.default_rng(7)
    rho = rng.uniform(-1e-3, 1e-3, N).astype(real)
    ux = (0.04 + rng.uniform(-1e-3, 1e-3, N)).astype(real)
    uy = rng.uniform(-1e-3, 1e-3, N).astype(real)
    uz = rng.uniform(-1e-3, 1e-3, N).astype(real)
    d = np.zeros(27 * N, real)
    for ev in (0, 1):
        impl.init_eq(d, N, geo, nx, ny, nz, rho, ux, uy, uz, ev)
    vk = g["velocity.k"]
    vq = g["velocity.q"].astype(real)
    vvx, vvy, vvz = (g["velocity.vx"].astype(real), g["velocity.vy"].astype(real), g["velocity.vz"].astype(real))
    sk, sq = g["slip.k"], g["slip.q"].astype(real)
    pk, pkn = g["pressure0.k"], g["pressure0.kN"]
    prho, pdir = g["pressure0.rho"].astype(real), int(g["pressure0.dir"][0])
    even, om = True, 1.8
    for _ in range(steps):
        impl.collision_k17(d, N, nx, ny, nz, fl, om, forces=(1e-5, 0, 0), force_factor=1.0,
                           limiters=(0.01, 0.01, 0.01), is_even=even)
        impl.bc_post(2, d, N, nx, ny, nz, vk, vq, om, vvx, vvy, vvz, is_even=even)
        impl.bc_post(0, d, N, nx, ny, nz, vk, vq, om, is_even=even)
        impl.bc_post(4, d, N, nx, ny, nz, sk, sq, om, is_even=even)
        impl.bc_post(1, d, N, nx, ny, nz, vk, vq, om, is_even=even)
        impl.bc_post(3, d, N, nx, ny, nz, vk, vq, om, vvx, vvy, vvz, is_even=even)
        impl.bc_pressure(d, N, nx, ny, nz, pk, pkn, prho, pdir, is_even=not even)
        impl.collision_bgk(d, N, geo, nx, ny, nz, om, is_even=not even)
        even = not even
    return d
