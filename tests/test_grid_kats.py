"""Known-answer tests of the reference's own grid-generator unit tests, run
against the library's builder:

- tests/unit-tests/gpu/GridGenerator/grid/SideTest.cpp: the q values a
  domain side gives a node whose neighbours are all boundary stoppers
  (q = 1/2 on the links along the side's normal) and the reset of links that
  also point across a side set before (through vfb_debug_side_qs), and the
  side -> D3Q27 direction map (through the pressure list's normal);
- tests/unit-tests/gpu/GridGenerator/grid/GridImpTest.cpp (findNeighbors
  integration tests): only the last layer of a box has missing neighbours,
  and every fluid node reaches its x, xy, xyz neighbours, for spacings that
  do not divide the box (0.15, 1/64, 0.17, 0.18).
The reference's periodic-shift tests cover a feature this builder does not
offer (shifted periodic wiring)."""
import ctypes
import itertools

import numpy as np
import pytest

from virtualfluids_b200 import _lib
from virtualfluids_b200 import grid as vgrid

MX, PX, MY, PY, MZ, PZ = range(6)
(d000, dP00, dM00, d0P0, d0M0, d00P, d00M, dPP0, dMM0, dPM0, dMP0, dP0P, dM0M, dP0M, dM0P, d0PP, d0MM, d0PM, d0MP,
 dPPP, dMPP, dPMP, dMMP, dPPM, dMPM, dPMM, dMMM) = range(27)


def side_qs(side, already=()):
    f = _lib.lib().vfb_debug_side_qs
    s = (ctypes.c_int * 6)(*already)
    q = (ctypes.c_double * 27)()
    _lib.check(f(side, s, len(already), q))
    return list(q)


def expected(*dirs, n=27):
    e = [-1.0] * n
    for d in dirs:
        e[d] = 0.5
    return e


# (side, sides set before, directions with q = 1/2), as the reference's SideTest expects them
SIDE_KATS = [
    (PX, (), (dP00, dPP0, dPM0, dP0P, dP0M, dPPP, dPMP, dPPM, dPMM)),
    (PX, (MX,), (dP00, dPP0, dPM0, dP0P, dP0M, dPPP, dPMP, dPPM, dPMM)),
    (PX, (PY,), (dP00, dPM0, dP0P, dP0M, dPMP, dPMM)),
    (PX, (MY,), (dP00, dPP0, dP0P, dP0M, dPPP, dPPM)),
    (MZ, (MY,), (d00M, dP0M, dM0M, d0PM, dPPM, dMPM)),
    (MZ, (PY,), (d00M, dP0M, dM0M, d0MM, dPMM, dMMM)),
    (PZ, (PY, PX), (d00P, dM0P, d0MP, dMMP)),
    (PZ, (PY, MX), (d00P, dP0P, d0MP, dPMP)),
]


@pytest.mark.parametrize("side,already,half", SIDE_KATS)
def test_side_qs_match_reference_side_test(side, already, half):
    assert side_qs(side, already) == expected(*half)


def test_side_qs_in_the_plane_match_reference_side_test():
    """setQs2D: the first eleven directions (the x-y plane and z)."""
    assert side_qs(PX)[:11] == expected(dP00, dPP0, dPM0, n=11)
    assert side_qs(PX, (PY,))[:11] == expected(dP00, dPM0, n=11)


def _normal(side):
    return [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)][side]


C = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0), (-1, -1, 0), (1, -1, 0),
     (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1), (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1),
     (1, 1, 1), (-1, 1, 1), (1, -1, 1), (-1, -1, 1), (1, 1, -1), (-1, 1, -1), (1, -1, -1), (-1, -1, -1)]


def _along(d, side):
    n = _normal(side)
    return sum(a * b for a, b in zip(C[d], n)) > 0


@pytest.mark.parametrize("side", range(6))
def test_side_qs_every_combination_of_earlier_sides(side):
    """The rule behind SideTest's cases for every side and every set of one
    or two perpendicular sides set before: 1/2 on the links along the
    normal that do not also point across an earlier side."""
    others = [s for s in range(6) if s // 2 != side // 2]
    for k in (0, 1, 2):
        for already in itertools.combinations(others, k):
            half = [d for d in range(27) if _along(d, side) and not any(_along(d, o) for o in already)]
            assert side_qs(side, already) == expected(*half), (side, already)


def test_geometry_side_is_rejected():
    f = _lib.lib().vfb_debug_side_qs
    q = (ctypes.c_double * 27)()
    assert f(PX, (ctypes.c_int * 1)(6), 1, q) == _lib.VFB_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("side,direction", [(MX, dM00), (PX, dP00), (MY, d0M0), (PY, d0P0), (MZ, d00M), (PZ, d00P)])
def test_side_direction_matches_reference_side_test(side, direction):
    """SideTest getD3Q27Direction_*: the pressure list carries its side's normal."""
    b = vgrid.MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 5, 5, 5, 1.0)
    b.buildGrids()
    b.setPressureBoundaryCondition(vgrid.SideType(side), 0.0)
    g = b.arrays()[0]
    assert int(g["pressure0.dir"][0]) == direction


def _box(dx, lo, hi):
    b = vgrid.MultipleGridBuilder()
    b.addCoarseGrid(lo, lo, lo, hi, hi, hi, dx)
    b.buildGrids()
    return b.arrays()[0]


@pytest.mark.parametrize("dx,lo,hi,n", [(0.15, 0.0, 1.0, 9), (1.0 / 64, -0.6, 0.6, 79)])
def test_only_the_last_layer_misses_neighbours(dx, lo, hi, n):
    """GridImpTest findNeighborsIntegrationTest grid1 / grid2: n x n nodes
    without an x (y, z) neighbour, all on the last layer."""
    g = _box(dx, lo, hi)
    assert list(g["dims"]) == [n, n, n]
    for axis in ("neighborX", "neighborY", "neighborZ"):
        assert int((g[axis][1:] == 0).sum()) == n * n


@pytest.mark.parametrize("dx,lo,hi", [(0.15, 0.0, 1.0), (1.0 / 64, -0.6, 0.6), (0.17, 0.0, 1.0), (0.18, 0.0, 1.0)])
def test_fluid_nodes_reach_their_neighbours(dx, lo, hi):
    """GridImpTest validFluidNeighbors: x, then y of that, then z of that."""
    g = _box(dx, lo, hi)
    nx, ny, nz = g["neighborX"], g["neighborY"], g["neighborZ"]
    fl = g["fluid"].astype(np.int64)
    a = nx[fl].astype(np.int64)
    assert (a > 0).all()
    b = ny[a].astype(np.int64)
    assert (b > 0).all()
    assert (nz[b] > 0).all()
