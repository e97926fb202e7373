"""The enstrophy analyzer (EnstrophyAnalyzer.cu:112-338) without a GPU.

The oracle restates the reference's node function by reading: the
analyzer's launcher holds a kernel launch and thrust device vectors, so the
file cannot be built for the host like the other reference kernels, and the
restatement is checked instead against analytic curls.  The library's node
code (the function its kernel runs, evaluated on the host) equals the oracle
bit for bit."""
import ctypes

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from virtualfluids_b200 import _lib
from virtualfluids_b200.grid import MultipleGridBuilder, SideType
from virtualfluids_b200.workloads import taylor_green

GOLDEN_GRIDS = ["channel", "cube_channel", "sphere_channel"]


def _level0(name):
    from pathlib import Path
    with np.load(Path(__file__).resolve().parent / "golden" / f"grid_{name}.npz") as z:
        return {k.split(":", 1)[1]: z[k] for k in z.files if k.startswith("L0:")}


def _lib_nodes(precision, g, fields):
    real = np.float64 if precision == "f64" else np.float32
    arrays = [np.ascontiguousarray(a, dtype=real) for a in fields]
    N = len(g["geo"])
    out = np.zeros(N)
    counted = np.zeros(N, np.int32)
    idx = [np.ascontiguousarray(g[k]) for k in ("geo", "neighborX", "neighborY", "neighborZ", "neighborNeg")]
    rc = _lib.lib().vfb_debug_enstrophy_nodes(_lib.FP64 if precision == "f64" else _lib.FP32,
                                              *[a.ctypes.data for a in arrays], N, *[a.ctypes.data for a in idx],
                                              out.ctypes.data, counted.ctypes.data)
    assert rc == 0, _lib.last_error()
    return out, counted.astype(bool)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("grid", GOLDEN_GRIDS)
def test_library_node_values_equal_the_oracle(precision, grid):
    g = _level0(grid)
    O = Oracle(precision)
    rng = np.random.default_rng(3)
    fields = [rng.uniform(-0.02, 0.02, len(g["geo"])).astype(O.real) for _ in range(4)]
    ref, cref = O.enstrophy_nodes(*fields, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], g["neighborNeg"])
    got, cgot = _lib_nodes(precision, g, fields)
    assert np.array_equal(cgot, cref) and cref.sum() > 0
    assert np.array_equal(got.astype(O.real), ref)


def test_stencil_orders_are_exact_for_polynomial_shear():
    """u = (a y^p, b z^p, c x^p) on a walled box: the curl's components are
    exact for the central differences of order >= p + 1 (odd p: order p + 1),
    so nodes whose stencils reach far enough give 1/2 (1 + drho) |curl u|^2
    exactly (to rounding), and nodes next to walls use shorter stencils."""
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 20, 20, 20, 1.0)
    b.buildGrids()
    for s in (SideType.MX, SideType.PX, SideType.MY, SideType.PY, SideType.MZ, SideType.PZ):
        b.setNoSlipBoundaryCondition(s)
    g = b.arrays()[0]
    x, y, z = g["coordX"], g["coordY"], g["coordZ"]
    O = Oracle("f64")
    drho = 0.01 * np.ones_like(x)
    # linear field: every stencil order is exact
    vx, vy, vz = 1e-3 * y, -2e-3 * z, 3e-3 * x
    vals, counted = O.enstrophy_nodes(drho, vx, vy, vz, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"],
                                      g["neighborNeg"])
    # curl of (a y, b z, c x) = (-b, -c, -a)
    expected = 0.5 * 1.01 * ((2e-3) ** 2 + (3e-3) ** 2 + (1e-3) ** 2)
    assert counted.sum() > 0
    assert np.allclose(vals[counted], expected, rtol=1e-12, atol=0)
    # a cubic field: only the nodes whose x, y, z stencils are at least
    # fourth order see the exact derivative 3 y^2
    vx = 1e-6 * (y - 10.0) ** 3
    vals, counted = O.enstrophy_nodes(drho, vx, 0 * vy, 0 * vz, g["geo"], g["neighborX"], g["neighborY"],
                                      g["neighborZ"], g["neighborNeg"])
    exact = 0.5 * 1.01 * (3e-6 * (y - 10.0) ** 2) ** 2
    interior = counted & (y > np.unique(y)[4]) & (y < np.unique(y)[-5])
    assert interior.sum() > 0
    assert np.allclose(vals[interior], exact[interior], rtol=1e-9, atol=1e-30)
    # next to a wall the second-order stencil is used, which is not exact for a cubic
    near = counted & ~interior
    assert near.sum() > 0 and not np.allclose(vals[near], exact[near], rtol=1e-6, atol=0)


def test_periodic_taylor_green_enstrophy_matches_the_analytic_value():
    """u = u0 (sin kx cos ky cos kz, -cos kx sin ky cos kz, 0) on a periodic
    box: every node uses the eighth-order stencil, and the node values agree
    with 1/2 (1 + drho) |curl u|^2 of the analytic curl at the node to the
    stencil's truncation error ((kh)^8 / 630)."""
    n = 32
    g = taylor_green(n).grid
    k = 2 * np.pi / n
    x, y, z = (g[c] for c in ("coordX", "coordY", "coordZ"))  # the box spans 2 pi: one node is k wide
    u0 = 0.05
    vx = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    vy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    wx = -u0 * k * np.cos(x) * np.sin(y) * np.sin(z)
    wy = -u0 * k * np.sin(x) * np.cos(y) * np.sin(z)
    wz = 2 * u0 * k * np.sin(x) * np.sin(y) * np.cos(z)
    drho = np.full_like(x, 0.002)
    O = Oracle("f64")
    vals, counted = O.enstrophy_nodes(drho, vx, vy, 0 * vx, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"],
                                      g["neighborNeg"])
    assert counted.sum() == n ** 3
    exact = 0.5 * 1.002 * (wx ** 2 + wy ** 2 + wz ** 2)
    assert np.abs(vals[counted] - exact[counted]).max() <= 1e-6 * exact.max()
    assert abs(vals[counted].mean() / (3.0 / 8.0 * 1.002 * u0 ** 2 * k ** 2) - 1) < 1e-6


def test_debug_hook_rejects_bad_precision():
    a = np.zeros(4)
    assert _lib.lib().vfb_debug_enstrophy_nodes(_lib.FP16, *([a.ctypes.data] * 10), 4, a.ctypes.data,
                                                a.ctypes.data) != 0
