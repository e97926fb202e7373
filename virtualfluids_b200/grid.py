"""Grid construction API (mirrors VirtualFluids' MultipleGridBuilder /
LevelGridBuilder, src/gpu/GridGenerator/grid/GridBuilder/).

The grid is built by the native library (csrc/grid_builder.cpp) through the C
ABI (vfb_grid_*).  The result is a list of levels, each a dict of numpy arrays
in the GPU layout of VirtualFluids' LBMSimulationParameter:

  neighborX/Y/Z, neighborNeg, geo   uint32, numberOfNodes (+1 dummy node 0)
  coordX/Y/Z                        float64 node coordinates
  fluid                             uint32 fluid-node list (+1 shifted)
  velocity.k / .vx / .vy / .vz / .q compacted velocity BC list (q direction-major)
  slip.k / .nx / .ny / .nz / .q     compacted slip BC list
  pressure<i>.k / .kN / .rho / .q / .dir   one list per pressure side
"""
from __future__ import annotations

import ctypes
import enum

import numpy as np

from . import _lib


class SideType(enum.IntEnum):
    """grid/BoundaryConditions/Side.h:62-65"""

    MX = 0
    PX = 1
    MY = 2
    PY = 3
    MZ = 4
    PZ = 5
    GEOMETRY = 6


_BC_NONE, _BC_NOSLIP, _BC_VELOCITY, _BC_PRESSURE, _BC_SLIP, _BC_STRESS = 0, 1, 2, 3, 4, 5
# the grid spec's stress block: side slot i holds its sampling offset, z0 and
# level-0 dx at STRESS_BASE + 3 i
STRESS_BASE = 176
SPEC_WITH_STRESS = STRESS_BASE + 18

_REAL_NAMES_PREFIX = ("coord",)


def _dtype(name: str, esize: int):
    base = name.split(".")[-1]
    if name in ("dims", "pressure.count") or base in ("k", "kN", "dir", "samplingOffset"):
        return np.int32
    if name in ("neighborX", "neighborY", "neighborZ", "neighborNeg", "geo", "fluid", "cf.coarse", "cf.fine",
                "fc.coarse", "fc.fine"):
        return np.uint32
    return np.float64 if esize == 8 else np.float32


GRID_ARRAY_NAMES = ["coordX", "coordY", "coordZ", "neighborX", "neighborY", "neighborZ", "neighborNeg", "geo", "dims",
                    "fluid", "velocity.k", "velocity.vx", "velocity.vy", "velocity.vz", "velocity.q", "slip.k",
                    "slip.nx", "slip.ny", "slip.nz", "slip.q", "geometry.k", "geometry.q", "geometry.vx",
                    "geometry.vy", "geometry.vz", "pressure.count", "stress.k", "stress.kN", "stress.nx",
                    "stress.ny", "stress.nz", "stress.q", "stress.samplingOffset", "stress.z0",
                    "cf.coarse", "cf.fine", "fc.coarse", "fc.fine", "cf.offX", "cf.offY", "cf.offZ", "fc.offX",
                    "fc.offY", "fc.offZ"]


class Cuboid:
    """Axis-aligned box between two corners (geometries/Cuboid)."""

    def __init__(self, minX, minY, minZ, maxX, maxY, maxZ):
        self.corners = (minX, minY, minZ, maxX, maxY, maxZ)

    def box(self):
        return self.corners


class Sphere:
    """Sphere of a centre and a radius (geometries/Sphere); as a solid its
    links' q values come from the ray-sphere intersection."""

    def __init__(self, centerX, centerY, centerZ, radius):
        self.centerX, self.centerY, self.centerZ, self.radius = centerX, centerY, centerZ, radius


class Axis:
    """Axis ids of a Cylinder (basics/geometry3d/Axis.h)."""
    x, y, z = 0, 1, 2


class Cylinder:
    """Cylinder parallel to a coordinate axis: centre, radius, length along
    the axis (geometries/Cylinder).  As a solid it has no ray intersection,
    so, like a cuboid, its links get q = 1/2 next to solid stoppers."""

    def __init__(self, centerX, centerY, centerZ, radius, height, rotationalAxis=Axis.z):
        if int(rotationalAxis) not in (0, 1, 2):
            raise ValueError("rotationalAxis must be Axis.x, Axis.y or Axis.z")
        self.centerX, self.centerY, self.centerZ = centerX, centerY, centerZ
        self.radius, self.height, self.rotationalAxis = radius, height, int(rotationalAxis)


class Conglomerate:
    """geometries/Conglomerate: primitives united (add) minus primitives
    removed (subtract); as a solid it has no ray intersection."""

    def __init__(self):
        self.added, self.subtracted = [], []

    def add(self, obj):
        self.added.append(obj)

    def subtract(self, obj):
        self.subtracted.append(obj)


def _primitive_values(obj) -> list[float]:
    """kind and the 6 parameters of a primitive, as the grid spec holds them."""
    if isinstance(obj, Sphere):
        return [2, obj.centerX, obj.centerY, obj.centerZ, obj.radius, 0, 0]
    if isinstance(obj, Cylinder):
        return [3, obj.centerX, obj.centerY, obj.centerZ, obj.radius, obj.height, obj.rotationalAxis]
    c = obj.box() if isinstance(obj, Cuboid) else tuple(obj)
    return [1, *c]


def VerticalCylinder(centerX, centerY, centerZ, radius, height):
    """geometries/VerticalCylinder: a cylinder about the z axis."""
    return Cylinder(centerX, centerY, centerZ, radius, height, Axis.z)


class MultipleGridBuilder:
    """Builder with the reference's call sequence: addCoarseGrid, (addGrid,
    addGeometry), setPeriodicBoundaryCondition, buildGrids, then the side
    boundary conditions."""

    def __init__(self):
        self.spec = np.zeros(64)
        self._extra = np.zeros(0)   # conglomerate parts, from spec index 64 on
        self._coarse = False
        self._built = False
        self._bcs: list[tuple[int, int, float, float, float]] = []
        self._stress: dict[int, tuple[float, float, float]] = {}  # side slot -> (offset, z0, dx)

    # --- grid ---------------------------------------------------------------
    def addCoarseGrid(self, startX, startY, startZ, endX, endY, endZ, delta):
        self.spec[0:7] = [startX, startY, startZ, endX, endY, endZ, delta]
        self._coarse = True

    def addGrid(self, box, level: int = 1):
        """Refinement box (minX, minY, minZ, maxX, maxY, maxZ) refined down to
        `level` (MultipleGridBuilder::addGrid(gridShape, levelFine)): one grid
        per level from the current finest + 1 to `level`."""
        if level < 1:
            raise ValueError("the refinement level must be at least 1")
        self.spec[10] = 1
        self.spec[11:17] = box
        self.spec[61] = level

    def setNumberOfLayers(self, fine: int, between: int):
        self.spec[17:19] = [fine, between]

    def addGeometry(self, solid):
        """Solid primitive, meshed on the finest level: a Sphere, a Cylinder,
        a Cuboid, or a plain (minX, minY, minZ, maxX, maxY, maxZ) cuboid."""
        if isinstance(solid, Conglomerate):
            if not solid.added:
                raise ValueError("a conglomerate needs at least one added object")
            self.spec[19] = 5
            self.spec[62:64] = [len(solid.added), len(solid.subtracted)]
            self._extra = np.array([v for o in solid.added + solid.subtracted for v in _primitive_values(o)], float)
        else:
            self.spec[19:26] = _primitive_values(solid)

    def setPeriodicBoundaryCondition(self, px: bool, py: bool, pz: bool):
        self.spec[7:10] = [float(px), float(py), float(pz)]

    def buildGrids(self, enableThinWalls: bool = False):
        if not self._coarse:
            raise RuntimeError("addCoarseGrid must be called first")
        self.spec[60] = 1.0 if enableThinWalls else 0.0
        self._built = True

    # --- boundary conditions (LevelGridBuilder.cpp:81-266) --------------------
    def _add(self, side, kind, v0=0.0, v1=0.0, v2=0.0):
        if not self._built:
            raise RuntimeError("buildGrids() has to be called before setting boundary conditions")
        side = SideType(side)
        if side == SideType.GEOMETRY:
            self.spec[26:30] = [kind, v0, v1, v2]
            return
        if len(self._bcs) >= 6:
            raise RuntimeError("at most six side boundary conditions")
        self._bcs.append((int(side), kind, v0, v1, v2))

    def setNoSlipBoundaryCondition(self, side):
        self._add(side, _BC_NOSLIP)

    def setVelocityBoundaryCondition(self, side, vx, vy, vz):
        self._add(side, _BC_VELOCITY, vx, vy, vz)

    def setPressureBoundaryCondition(self, side, rho):
        self._add(side, _BC_PRESSURE, rho)

    def setSlipBoundaryCondition(self, side, normalX, normalY, normalZ):
        self._add(side, _BC_SLIP, normalX, normalY, normalZ)

    def setStressBoundaryCondition(self, side, normalX, normalY, normalZ, samplingOffset: int, z0, dx):
        """Wall-model BC on a side (LevelGridBuilder::setStressBoundaryCondition,
        LevelGridBuilder.cpp:129-150): the wall normal, the velocity sampling
        node samplingOffset nodes inside, the roughness length z0 and the
        level-0 spacing dx in the units of z0."""
        if SideType(side) == SideType.GEOMETRY:
            raise ValueError("the stress BC is set on a domain side")
        if int(samplingOffset) != samplingOffset or samplingOffset < 0:
            raise ValueError("samplingOffset must be a whole number >= 0")
        self._add(side, _BC_STRESS, normalX, normalY, normalZ)
        self._stress[len(self._bcs) - 1] = (float(samplingOffset), float(z0), float(dx))

    # --- result ---------------------------------------------------------------
    def full_spec(self) -> np.ndarray:
        s = self.spec.copy()
        for i, b in enumerate(self._bcs):
            s[30 + 5 * i: 35 + 5 * i] = b
        s = np.concatenate([s, self._extra])
        if self._stress:
            s = np.concatenate([s, np.zeros(max(0, SPEC_WITH_STRESS - len(s)))])
            for i, v in self._stress.items():
                s[STRESS_BASE + 3 * i: STRESS_BASE + 3 * i + 3] = v
        return s

    def arrays(self) -> list[dict[str, np.ndarray]]:
        """Run the native builder and return the arrays of every level."""
        L = _lib.lib()
        s = self.full_spec()
        h = L.vfb_grid_build(s.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(s))
        if not h:
            raise _lib.VfbError(_lib.VFB_ERR_CONFIGURATION, _lib.last_error())
        try:
            return [export_level(L, h, lvl, "vfb_grid") for lvl in range(L.vfb_grid_levels(h))]
        finally:
            L.vfb_grid_free(h)


def export_level(L, h, level: int, prefix: str) -> dict[str, np.ndarray]:
    count = getattr(L, prefix + "_count")
    esize = getattr(L, prefix + "_elem_size")
    copy = getattr(L, prefix + "_copy")
    names = list(GRID_ARRAY_NAMES)
    if count(h, level, b"pressure.count") > 0:
        tmp = np.zeros(1, np.int32)
        copy(h, level, b"pressure.count", tmp.ctypes.data_as(ctypes.c_void_p))
        for i in range(int(tmp[0])):
            names += [f"pressure{i}.{s}" for s in ("k", "kN", "rho", "q", "dir")]
    out: dict[str, np.ndarray] = {}
    for name in names:
        n = count(h, level, name.encode())
        if n < 0:
            continue
        es = esize(h, level, name.encode())
        a = np.zeros(n, _dtype(name, es))
        if a.itemsize != es:
            raise RuntimeError(f"element size mismatch for {name}")
        copy(h, level, name.encode(), a.ctypes.data_as(ctypes.c_void_p))
        out[name] = a
    return out


def taylor_green_grid(n: int) -> dict[str, np.ndarray]:
    """Periodic cube of n^3 fluid nodes on [-pi, pi]^3 with spacing 2 pi / n,
    built as apps/gpu/TaylorGreenVortex/TaylorGreenVortex.cpp:107-114 does."""
    import math
    b = MultipleGridBuilder()
    d = 2.0 * math.pi / n
    b.addCoarseGrid(-math.pi, -math.pi, -math.pi, math.pi, math.pi, math.pi, d)
    b.setPeriodicBoundaryCondition(True, True, True)
    b.buildGrids(True)
    return b.arrays()[0]
