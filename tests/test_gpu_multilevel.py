"""The recursive two-level schedule (UpdateGrid27::updateGrid with fine-to-coarse
and coarse-to-fine interpolation) on a grid made by the reference's own
builder, against the same schedule run on the host: the oracle for collision
and boundary conditions, and the library's host interpolation (pinned to the
reference's scaling kernels by tests/test_scaling_host.py)."""
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import rel_max
from tests.scaling_cases import scaling_args
from virtualfluids_b200 import _lib
from virtualfluids_b200.simulation import (BoundaryConditionFactory, NoSlipBC, Parameter, PressureBC, Simulation,
                                           SlipBC)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GOLDEN = Path(__file__).resolve().parent / "golden"
NU = 0.02


def levels(name="refined_channel"):
    with np.load(GOLDEN / f"grid_{name}.npz") as z:
        out = {}
        for key in z.files:
            lvl, name = key.split(":", 1)
            out.setdefault(int(lvl[1:]), {})[name] = z[key]
    return [out[i] for i in sorted(out)]


def initial(g, seed):
    rng = np.random.default_rng(seed)
    N = len(g["geo"])
    f = [rng.uniform(-1e-4, 1e-4, N), 0.02 + rng.uniform(-1e-3, 1e-3, N), rng.uniform(-1e-3, 1e-3, N),
         rng.uniform(-1e-3, 1e-3, N)]
    for a in f:
        a[g["geo"] != 19] = 0.0
    return f


class HostSchedule:
    """UpdateGrid27::updateGrid for all levels on the host."""

    def __init__(self, lv, inits, slip=False, geometry=False, nu=NU):
        self.slip, self.geometry = slip, geometry
        self.O = Oracle("f64")
        self.lv = lv
        self.d = []
        for g, init in zip(lv, inits):
            N = len(g["geo"])
            d = np.zeros(27 * N)
            for ev in (0, 1):
                self.O.init_eq(d, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], *init, ev)
            self.d.append(d)
        self.even = [True] * len(lv)
        self.omega = [1.0 / (3.0 * nu * 2 ** l + 0.5) for l in range(len(lv))]

    def update(self, level):
        O, g, d = self.O, self.lv[level], self.d[level]
        finest = len(self.lv) - 1
        if level != finest:
            self.update(level + 1)
            self.update(level + 1)
        N = len(g["geo"])
        nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
        om, ev = self.omega[level], self.even[level]
        O.collision_k17(d, N, *nb, g["fluid"], om, forces=(0, 0, 0), force_factor=1.0 / 2 ** level,
                        limiters=(0.01, 0.01, 0.01), is_even=ev)
        # post-collision BCs in the reference's order: velocity, (no-slip), slip, geometry
        if len(g["velocity.k"]):
            vel = [g[f"velocity.{c}"] for c in ("vx", "vy", "vz")]
            O.bc_post(2, d, N, *nb, g["velocity.k"], g["velocity.q"], om, *vel, is_even=ev)
        if self.slip and len(g["slip.k"]):
            O.bc_post(4, d, N, *nb, g["slip.k"], g["slip.q"], om, is_even=ev)
        if self.geometry and len(g["geometry.k"]):
            O.bc_post(0, d, N, *nb, g["geometry.k"], g["geometry.q"], om, is_even=ev)
        self.even[level] = not ev
        if "pressure0.k" in g and len(g["pressure0.k"]):
            O.bc_pressure(d, N, *nb, g["pressure0.k"], g["pressure0.kN"], g["pressure0.rho"],
                          int(g["pressure0.dir"][0]), is_even=self.even[level])
        if level != finest:
            self.scale(level, False)
            self.scale(level, True)

    def scale(self, level, coarse_to_fine):
        tag = "cf" if coarse_to_fine else "fc"
        gc, gf = self.lv[level], self.lv[level + 1]
        if len(gc[f"{tag}.coarse"]) == 0:
            return
        c = {"gc": gc, "gf": gf, f"coarse_{tag}": gc[f"{tag}.coarse"], f"fine_{tag}": gc[f"{tag}.fine"],
             "omegaC": self.omega[level], "omegaF": self.omega[level + 1]}
        offs = [np.ascontiguousarray(gc[f"{tag}.off{a}"]) for a in "XYZ"]
        arrays = {f"{k}.neighbor{a}": c[k][f"neighbor{a}"].ctypes.data for k in ("gc", "gf") for a in "XYZ"}
        arrays[f"coarse_{tag}"] = c[f"coarse_{tag}"].ctypes.data
        arrays[f"fine_{tag}"] = c[f"fine_{tag}"].ctypes.data
        arrays.update({f"off{a}": o.ctypes.data for a, o in zip("XYZ", offs)})
        a = scaling_args(c, coarse_to_fine, self.even[level], self.d[level].ctypes.data,
                         self.d[level + 1].ctypes.data, arrays)
        _lib.check(_lib.lib().vfb_debug_scale_host(int(coarse_to_fine), _lib.FP64, a))

    def macroscopic(self, level):
        g = self.lv[level]
        return self.O.macroscopic(self.d[level], len(g["geo"]), g["geo"], g["neighborX"], g["neighborY"],
                                  g["neighborZ"], self.even[level])


@pytest.mark.parametrize("use_plan", [True, False])
def test_two_level_schedule_matches_host(cuda, use_plan):
    lv = levels()
    assert len(lv) == 2 and len(lv[0]["cf.coarse"]) > 0 and len(lv[0]["fc.coarse"]) > 0
    inits = [initial(g, 10 + i) for i, g in enumerate(lv)]
    p = Parameter()
    p.set_viscosity_LB(NU)
    p.use_plan = use_plan
    bc = BoundaryConditionFactory()
    bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
    sim = Simulation(p, lv, bc)
    for lvl, init in enumerate(inits):
        sim.init_level(lvl, *init)
    host = HostSchedule(lv, inits)
    steps = 4
    sim.run(steps)
    for _ in range(steps):
        host.update(0)
    for lvl, g in enumerate(lv):
        got = sim.macroscopic(lvl)
        ref = host.macroscopic(lvl)
        fl = g["fluid"]
        for a, r in zip(got, ref):
            assert rel_max(a[fl], r[fl]) < 1e-12, lvl
    # the fine level ran two substeps per coarse step: parity back to the start
    assert sim.level_state(1)[2] is True
    assert sim.level_state(0)[2] is (steps % 2 == 0)


def test_two_level_graph_replay_equals_direct_launches(cuda):
    lv = levels()
    inits = [initial(g, 20 + i) for i, g in enumerate(lv)]
    outs = []
    for graphs in (False, True):
        p = Parameter()
        p.set_viscosity_LB(NU)
        p.use_graphs = graphs
        bc = BoundaryConditionFactory()
        bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
        sim = Simulation(p, lv, bc)
        for lvl, init in enumerate(inits):
            sim.init_level(lvl, *init)
        sim.run(9)
        outs.append([sim.macroscopic(l) for l in range(2)])
    for la, lb in zip(*outs):
        for a, b in zip(la, lb):
            assert np.array_equal(a, b)


def test_cube_channel_two_levels_matches_host(cuda):
    """The wall-mounted cube benchmark scaled down (two levels, solid cube with
    interpolated no-slip faces on the fine level, velocity inlet, pressure
    outlet, slip top, periodic span), grid made by the reference's builder."""
    lv = levels("cube_channel")
    assert len(lv) == 2 and len(lv[1]["geometry.k"]) > 0 and len(lv[0]["slip.k"]) > 0
    inits = [initial(g, 30 + i) for i, g in enumerate(lv)]
    p = Parameter()
    p.set_viscosity_LB(NU)
    bc = BoundaryConditionFactory()
    bc.set_slip_boundary_condition(SlipBC.SlipCompressible)
    bc.set_geometry_boundary_condition(NoSlipBC.NoSlipInterpolatedCompressible)
    bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
    sim = Simulation(p, lv, bc)
    for lvl, init in enumerate(inits):
        sim.init_level(lvl, *init)
    host = HostSchedule(lv, inits, slip=True, geometry=True)
    steps = 4
    sim.run(steps)
    for _ in range(steps):
        host.update(0)
    for lvl, g in enumerate(lv):
        got = sim.macroscopic(lvl)
        ref = host.macroscopic(lvl)
        fl = g["fluid"]
        for a, r in zip(got, ref):
            assert rel_max(a[fl], r[fl]) < 1e-12, lvl


def test_builder_api_feeds_the_schedule(cuda):
    """The scaled-down cube channel built through the library's own builder
    API (addGrid, addGeometry, geometry no-slip) runs exactly as the same grid
    handed over as the reference builder's arrays."""
    from virtualfluids_b200.grid import MultipleGridBuilder, SideType
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 47, 15, 15, 1.0)
    b.addGrid((12, 4, 0, 28, 12, 8), 1)
    b.addGeometry((16, 6, 0, 20, 10, 4))
    b.setPeriodicBoundaryCondition(False, True, False)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, 0.04, 0, 0)
    b.setPressureBoundaryCondition(SideType.PX, 0.0)
    b.setNoSlipBoundaryCondition(SideType.MZ)
    b.setSlipBoundaryCondition(SideType.PZ, 0, 0, 1)
    b.setNoSlipBoundaryCondition(SideType.GEOMETRY)
    lv = levels("cube_channel")
    inits = [initial(g, 40 + i) for i, g in enumerate(lv)]
    outs = []
    for source in (b, lv):
        p = Parameter()
        p.set_viscosity_LB(NU)
        bc = BoundaryConditionFactory()
        bc.set_slip_boundary_condition(SlipBC.SlipCompressible)
        bc.set_geometry_boundary_condition(NoSlipBC.NoSlipInterpolatedCompressible)
        bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
        sim = Simulation(p, source, bc)
        for lvl, init in enumerate(inits):
            sim.init_level(lvl, *init)
        sim.run(6)
        outs.append([sim.macroscopic(lvl) for lvl in range(2)])
    for la, lb in zip(*outs):
        for a, c in zip(la, lb):
            assert np.array_equal(a, c)
