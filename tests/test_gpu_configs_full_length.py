"""Parity of the benchmark configurations at their stated lengths.

- Lid-driven cavity: 64^3, FP64, lid u = (0.05, 0, 0) on +z, halfway walls
  elsewhere, nu = 0.0032, 2000 steps through the public Simulation API (graph
  replay), against the FP64 oracle running the same schedule: fields within
  1e-12 relative (max norm).
- Taylor-Green vortex: 128^3, u0 = 0.05, Re = 1600, seeded noise, 1000 steps
  of the planned default kernels.  FP64 K17 and BGK within 1e-12 relative of
  the FP64 oracle; FP32 storage and arithmetic within 1e-4 L2 of the FP64
  oracle (single-precision rounding, stated bound).
- Wall-mounted cube: the full-size two-level grid (coarse 256 x 96 x 96,
  refined box 48..128 x 24..72 x 0..40, cube of side 16), K17, velocity inlet
  0.04 with seeded +-1% noise, pressure outlet, slip top, periodic span,
  interpolated no-slip on the cube, nu = 0.04 * 16 / 2000, from rest, 200 coarse
  steps (400 fine substeps) of the C++ schedule against the host schedule (the
  oracle for collision and BCs, the library's host interpolation for the
  interface cells).  FP64 within 1e-12 relative; FP32 within 1e-4 L2 of the
  FP64 host result (stated bound).

The oracle's node loops run on all host threads (OpenMP); the oracle results
are computed once per module and shared by the FP64 and FP32 comparisons.
"""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import gpu_run, oracle_run, rel_l2, rel_max, tgv_state
from tests.test_gpu_multilevel import HostSchedule
from virtualfluids_b200.grid import MultipleGridBuilder, SideType
from virtualfluids_b200.simulation import (BoundaryConditionFactory, NoSlipBC, Parameter, PressureBC, Simulation,
                                           SlipBC)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TGV_N, TGV_STEPS = 128, 1000
CUBE_STEPS = 200
FP32_L2_BOUND = 1e-4


def test_cavity64_fp64_2000_steps_matches_oracle(cuda):
    n, nu, steps = 64, 0.0032, 2000
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, n - 1, n - 1, n - 1, 1.0)
    b.buildGrids()
    for side in (SideType.MX, SideType.PX, SideType.MY, SideType.PY, SideType.MZ):
        b.setNoSlipBoundaryCondition(side)
    b.setVelocityBoundaryCondition(SideType.PZ, 0.05, 0.0, 0.0)
    p = Parameter()
    p.set_storage("fp64")
    p.set_viscosity_LB(nu)
    sim = Simulation(p, b, BoundaryConditionFactory())
    g = sim.levels[0]
    zero = np.zeros(len(g["geo"]))
    sim.init_level(0, zero, zero, zero, zero)
    sim.run(steps)
    got = sim.macroscopic(0)
    sim.close()

    O = Oracle("f64")
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    d = np.zeros(27 * N)
    for ev in (0, 1):
        O.init_eq(d, N, g["geo"], *nb, zero, zero, zero, zero, ev)
    om = 1.0 / (3.0 * nu + 0.5)
    vel = [g[f"velocity.{c}"] for c in ("vx", "vy", "vz")]
    even = True
    for _ in range(steps):
        O.collision_k17(d, N, *nb, g["fluid"], om, forces=(0, 0, 0), force_factor=1.0, limiters=(0.01, 0.01, 0.01),
                        is_even=even)
        O.bc_post(2, d, N, *nb, g["velocity.k"], g["velocity.q"], om, *vel, is_even=even)
        even = not even
    ref = O.macroscopic(d, N, g["geo"], *nb, even)
    fl = g["fluid"]
    assert np.abs(ref[1][fl]).max() > 1e-2  # the lid has driven a vortex
    for a, r in zip(got, ref):
        assert rel_max(a[fl], r[fl]) <= 1e-12


@pytest.fixture(scope="module")
def tgv():
    return tgv_state(TGV_N)


_oracle_cache = {}


def tgv_oracle(w, kernel):
    if kernel not in _oracle_cache:
        _oracle_cache[kernel] = oracle_run(w, "f64", TGV_STEPS, kernel)[1]
    return _oracle_cache[kernel]


@pytest.mark.parametrize("kernel", ["K17", "BGK"])
def test_tgv128_1000_steps_fp64(cuda, tgv, kernel):
    ref = tgv_oracle(tgv, kernel)
    _, _, got, _ = gpu_run(tgv, torch.float64, TGV_STEPS, kernel, planned=True)
    fl = tgv.grid["fluid"]
    for a, b in zip(got, ref):
        assert rel_max(a[fl], b[fl]) < 1e-12


@pytest.mark.parametrize("kernel", ["K17", "BGK"])
def test_tgv128_1000_steps_fp32(cuda, tgv, kernel):
    ref = tgv_oracle(tgv, kernel)
    _, _, got, _ = gpu_run(tgv, torch.float32, TGV_STEPS, kernel, planned=True)
    fl = tgv.grid["fluid"]
    for a, b in zip(got, ref):
        assert rel_l2(a[fl], b[fl]) < FP32_L2_BOUND


@pytest.fixture(scope="module")
def cube_host():
    from virtualfluids_b200.workloads import wall_mounted_cube
    lv = wall_mounted_cube()
    nu = 0.04 * 16 / 2000
    inits = [[np.zeros(len(g["geo"])) for _ in range(4)] for g in lv]
    host = HostSchedule(lv, inits, slip=True, geometry=True, nu=nu)
    for _ in range(CUBE_STEPS):
        host.update(0)
    return lv, nu, [host.macroscopic(lvl) for lvl in range(len(lv))]


@pytest.mark.parametrize("storage", ["fp64", "fp32"])
def test_full_cube_two_levels_matches_host(cuda, cube_host, storage):
    lv, nu, ref = cube_host
    assert len(lv) == 2 and len(lv[1]["geometry.k"]) > 0 and len(lv[0]["cf.coarse"]) > 0
    p = Parameter()
    p.set_storage(storage)
    p.set_viscosity_LB(nu)
    bc = BoundaryConditionFactory()
    bc.set_slip_boundary_condition(SlipBC.SlipCompressible)
    bc.set_geometry_boundary_condition(NoSlipBC.NoSlipInterpolatedCompressible)
    bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
    sim = Simulation(p, lv, bc)
    for lvl, g in enumerate(lv):
        zero = np.zeros(len(g["geo"]))
        sim.init_level(lvl, zero, zero, zero, zero)
    sim.run(CUBE_STEPS)
    got = [sim.macroscopic(lvl) for lvl in range(len(lv))]
    sim.close()
    assert np.abs(ref[1][1][lv[1]["fluid"]]).max() > 1e-3  # the fine level has seen the flow
    for lvl, g in enumerate(lv):
        fl = g["fluid"]
        for a, r in zip(got[lvl], ref[lvl]):
            if storage == "fp64":
                assert rel_max(a[fl], r[fl]) < 1e-12, lvl
            else:
                assert rel_l2(a[fl], r[fl]) < FP32_L2_BOUND, lvl
