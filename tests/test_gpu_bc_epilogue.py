"""The BC epilogue of the planned collision (vfb_collision_plan_set_bc_epilogue,
an option of the simulation, off by default):
a simulation whose collision applies the post-collision BCs of its wall nodes
itself equals the same simulation with separate BC launches for every entry
-- the entries read the same post-collision values and write cells nobody
else touches in the step.  The collision kernel with the epilogue is a
separate compilation of the same source, which may round a few FP32
operations differently: FP64 is compared bit for bit, FP32 and the 16-bit
storages to a bound far below the size of a wrong boundary value.  Cavity (all six walls), channel
(inlet, outlet, no-slip floor, slip lid), the sphere channel (geometry list
with fractional q, whose clipping links keep some nodes out of the
epilogue), the two-level cube channel, every storage."""
from pathlib import Path

import numpy as np
import pytest

from virtualfluids_b200.grid import MultipleGridBuilder, SideType
from virtualfluids_b200.simulation import (BoundaryConditionFactory, NoSlipBC, Parameter, PressureBC, Simulation,
                                           SlipBC, VelocityBC)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GOLDEN = Path(__file__).resolve().parent / "golden"


def _golden(name):
    with np.load(GOLDEN / f"grid_{name}.npz") as z:
        levels = {}
        for key in z.files:
            lvl, arr = key.split(":", 1)
            levels.setdefault(int(lvl[1:]), {})[arr] = z[key]
    return [levels[i] for i in sorted(levels)]


def _cavity(n=24):
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, n - 1, n - 1, n - 1, 1.0)
    b.buildGrids()
    for s in (SideType.MX, SideType.PX, SideType.MY, SideType.PY, SideType.MZ):
        b.setNoSlipBoundaryCondition(s)
    b.setVelocityBoundaryCondition(SideType.PZ, 0.05, 0.0, 0.0)
    return b


def _channel():
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 31, 15, 15, 1.0)
    b.setPeriodicBoundaryCondition(False, True, False)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, 0.04, 0.0, 0.0)
    b.setPressureBoundaryCondition(SideType.PX, 0.0)
    b.setNoSlipBoundaryCondition(SideType.MZ)
    b.setSlipBoundaryCondition(SideType.PZ, 0.0, 0.0, 1.0)
    return b


def _run(grid, storage, epilogue, steps, velocity=VelocityBC.VelocityInterpolatedCompressible,
         no_slip=NoSlipBC.NoSlipInterpolatedCompressible, geometry=NoSlipBC.NoSlipInterpolatedCompressible,
         slip=SlipBC.SlipCompressible, nu=0.02, seed=4):
    p = Parameter()
    p.set_storage(storage)
    p.set_viscosity_LB(nu)
    p.use_bc_epilogue = epilogue
    bc = BoundaryConditionFactory()
    bc.set_velocity_boundary_condition(velocity)
    bc.set_no_slip_boundary_condition(no_slip)
    bc.set_geometry_boundary_condition(geometry)
    bc.set_slip_boundary_condition(slip)
    bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
    sim = Simulation(p, grid, bc)
    rng = np.random.default_rng(seed)
    for lvl, g in enumerate(sim.levels):
        N = len(g["geo"])
        f = [rng.uniform(-1e-3, 1e-3, N) for _ in range(4)]
        f[1] += 0.02
        solid = g["geo"] != 19
        for a in f:
            a[solid] = 0.0
        sim.init_level(lvl, *f)
    sim.run(steps)
    stats = [sim.bc_epilogue_stats(lvl) for lvl in range(len(sim.levels))]
    out = [sim.macroscopic(lvl) for lvl in range(len(sim.levels))]
    sim.close()
    return out, stats


@pytest.mark.parametrize("storage", ["fp32", "fp64", "fp16", "fx16", "fx16w"])
@pytest.mark.parametrize("case", ["cavity", "channel", "sphere_channel", "cube_channel"])
def test_epilogue_equals_separate_launches(cuda, storage, case):
    grid = {"cavity": _cavity, "channel": _channel}.get(case, lambda: _golden(case))()
    steps = 9  # odd: both parities, an odd number of coarse steps
    a, sa = _run(grid, storage, True, steps)
    b, sb = _run(grid, storage, False, steps)
    assert sum(s[0] for s in sa) > 0, sa       # the epilogue took nodes
    assert all(s[0] == 0 for s in sb)
    tol = {"fp64": 0.0, "fp32": 1e-5, "fp16": 2e-3, "fx16": 3e-3, "fx16w": 1e-2}[storage]
    for lvl in range(len(a)):
        for x, y in zip(a[lvl], b[lvl]):
            scale = max(np.abs(y).max(), 1e-300)
            assert np.abs(x.astype(np.float64) - y).max() <= tol * scale, (case, storage, lvl)
    if case == "sphere_channel":
        # the clipping links of the sphere keep some geometry entries out
        assert sa[0][2] > 0


def test_epilogue_with_bounce_back_kinds(cuda):
    grid = _cavity(16)
    kw = dict(velocity=VelocityBC.VelocityBounceBack, no_slip=NoSlipBC.NoSlipBounceBack)
    a, sa = _run(grid, "fp32", True, 7, **kw)
    b, _ = _run(grid, "fp32", False, 7, **kw)
    assert sa[0][0] > 0
    for x, y in zip(a[0], b[0]):
        assert np.abs(x.astype(np.float64) - y).max() <= 1e-5 * np.abs(y).max()
