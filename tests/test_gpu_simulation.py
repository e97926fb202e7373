"""The C++ time-step schedule (vfb_sim_*, driven through the pyfluids-style
Simulation) against the oracle running the reference's UpdateGrid27 order
(collision, post-collision BCs velocity / slip, parity swap, pressure BC) on
walled grids."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import rel_l2, rel_max
from virtualfluids_b200 import _lib
from virtualfluids_b200.grid import MultipleGridBuilder, SideType
from virtualfluids_b200.simulation import (BoundaryConditionFactory, Parameter, PressureBC, SlipBC, Simulation,
                                           VelocityBC)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def cavity(n):
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, n - 1, n - 1, n - 1, 1.0)
    b.buildGrids()
    for s in (SideType.MX, SideType.PX, SideType.MY, SideType.PY, SideType.MZ):
        b.setNoSlipBoundaryCondition(s)
    b.setVelocityBoundaryCondition(SideType.PZ, 0.05, 0.0, 0.0)
    return b


def channel():
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 15, 7, 7, 1.0)
    b.setPeriodicBoundaryCondition(False, True, False)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, 0.04, 0.0, 0.0)
    b.setPressureBoundaryCondition(SideType.PX, 0.0)
    b.setNoSlipBoundaryCondition(SideType.MZ)
    b.setSlipBoundaryCondition(SideType.PZ, 0.0, 0.0, 1.0)
    return b


def oracle_schedule(g, precision, nu, steps, init, slip=False, pressure=False, velocity_kind=2, init_neq=False,
                    pressure_kind=0, correction_factor=0.0):
    """UpdateGrid27::updateGrid for one level, on the oracle (initialised by
    the equilibrium, or with init_neq by the non-equilibrium init; the
    pressure list runs PressureNonEquilibriumCompressible for pressure_kind 0,
    the non-reflecting outflow for 1 and its pressure-corrected form for 2)."""
    O = Oracle(precision)
    real = O.real
    N = len(g["geo"])
    nx, ny, nz, geo, fl = g["neighborX"], g["neighborY"], g["neighborZ"], g["geo"], g["fluid"]
    d = np.zeros(27 * N, real)
    om = 1.0 / (3.0 * nu + 0.5)
    for ev in (0, 1):
        if init_neq:
            O.init_noneq(d, N, geo, nx, ny, nz, g["neighborNeg"], *[a.astype(real) for a in init], real(om), ev)
        else:
            O.init_eq(d, N, geo, nx, ny, nz, *[a.astype(real) for a in init], ev)
    vel = [g[f"velocity.{c}"].astype(real) for c in ("vx", "vy", "vz")]
    even = True
    for _ in range(steps):
        O.collision_k17(d, N, nx, ny, nz, fl, om, forces=(0, 0, 0), force_factor=1.0, limiters=(0.01, 0.01, 0.01),
                        is_even=even)
        O.bc_post(velocity_kind, d, N, nx, ny, nz, g["velocity.k"], g["velocity.q"].astype(real), om, *vel,
                  is_even=even)
        if slip:
            O.bc_post(4, d, N, nx, ny, nz, g["slip.k"], g["slip.q"].astype(real), om, is_even=even)
        even = not even
        if pressure and pressure_kind == 0:
            O.bc_pressure(d, N, nx, ny, nz, g["pressure0.k"], g["pressure0.kN"], g["pressure0.rho"].astype(real),
                          int(g["pressure0.dir"][0]), is_even=even)
        elif pressure:
            O.bc_outflow(d, N, nx, ny, nz, g["pressure0.k"], g["pressure0.kN"], int(g["pressure0.dir"][0]),
                         pressure_kind == 2, real(correction_factor), is_even=even)
    return O.macroscopic(d, N, geo, nx, ny, nz, even)


def _init(g, seed=2):
    rng = np.random.default_rng(seed)
    N = len(g["geo"])
    f = [rng.uniform(-1e-3, 1e-3, N) for _ in range(4)]
    for a in f:
        a[g["geo"] != 19] = 0.0
    return f


@pytest.mark.parametrize("storage", ["fp64", "fp32"])
@pytest.mark.parametrize("use_plan", [True, False])
def test_cavity_schedule_matches_oracle(cuda, storage, use_plan):
    b = cavity(12)
    p = Parameter()
    p.set_storage(storage)
    p.set_viscosity_LB(0.0032)
    p.use_plan = use_plan
    sim = Simulation(p, b, BoundaryConditionFactory())
    g = sim.levels[0]
    init = _init(g)
    sim.init_level(0, *init)
    steps = 30
    sim.run(steps)
    got = sim.macroscopic(0)
    ref = oracle_schedule(g, "f64" if storage == "fp64" else "f32", 0.0032, steps, init)
    fl = g["fluid"]
    for a, r in zip(got, ref):
        if storage == "fp64":
            assert rel_max(a[fl], r[fl]) < 1e-12
        else:
            assert rel_l2(a[fl], r[fl]) < 1e-5
    _, _, bad = sim.mass_and_energy(0)
    assert bad == 0


def test_channel_schedule_with_slip_and_pressure(cuda):
    b = channel()
    p = Parameter()
    p.set_viscosity_LB(0.01)
    bc = BoundaryConditionFactory()
    bc.set_velocity_boundary_condition(VelocityBC.VelocityInterpolatedCompressible)
    bc.set_slip_boundary_condition(SlipBC.SlipCompressible)
    bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
    sim = Simulation(p, b, bc)
    g = sim.levels[0]
    init = _init(g, 5)
    sim.init_level(0, *init)
    sim.run(20)
    got = sim.macroscopic(0)
    ref = oracle_schedule(g, "f64", 0.01, 20, init, slip=True, pressure=True)
    fl = g["fluid"]
    for a, r in zip(got, ref):
        assert rel_max(a[fl], r[fl]) < 1e-12


def test_velocity_bounce_back_selection(cuda):
    b = cavity(8)
    p = Parameter()
    p.set_viscosity_LB(0.01)
    bc = BoundaryConditionFactory()
    bc.set_velocity_boundary_condition(VelocityBC.VelocityBounceBack)
    sim = Simulation(p, b, bc)
    g = sim.levels[0]
    init = _init(g, 9)
    sim.init_level(0, *init)
    sim.run(10)
    got = sim.macroscopic(0)
    ref = oracle_schedule(g, "f64", 0.01, 10, init, velocity_kind=_lib.BC_VELOCITY_BOUNCE_BACK)
    fl = g["fluid"]
    for a, r in zip(got, ref):
        assert rel_max(a[fl], r[fl]) < 1e-12


def test_initial_condition_function_and_parity(cuda):
    b = cavity(8)
    p = Parameter()
    p.set_viscosity_LB(0.01)
    p.set_initial_condition(lambda x, y, z: (0.0 * x, 0.01 * np.sin(z), 0.0 * x, 0.0 * x))
    sim = Simulation(p, b, BoundaryConditionFactory())
    rho, vx, vy, vz = sim.macroscopic(0)
    g = sim.levels[0]
    fl = g["fluid"]
    assert np.abs(vx[fl] - 0.01 * np.sin(g["coordZ"][fl])).max() < 1e-12
    assert sim.level_state(0)[2] is True
    sim.run(3)
    assert sim.level_state(0)[2] is False


@pytest.mark.parametrize("steps", [7, 10])
def test_graph_replay_equals_direct_launches(cuda, steps):
    """Two coarse steps captured into a CUDA graph and replayed give the same
    populations as launching every kernel from the host."""
    outs = []
    for graphs in (False, True):
        b = channel()
        p = Parameter()
        p.set_viscosity_LB(0.01)
        p.use_graphs = graphs
        bc = BoundaryConditionFactory()
        bc.set_slip_boundary_condition(SlipBC.SlipCompressible)
        bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
        sim = Simulation(p, b, bc)
        sim.init_level(0, *_init(sim.levels[0], 4))
        sim.run(3)
        sim.run(steps)
        outs.append((sim.macroscopic(0), sim.level_state(0)[2]))
    for a, b in zip(outs[0][0], outs[1][0]):
        assert np.array_equal(a, b)
    assert outs[0][1] == outs[1][1]


def test_kinetic_energy_analyzer_definition(cuda):
    """vfb_sim_kinetic_energy: the mean of (1 + drho) |u|^2 / 2 over the fluid
    nodes whose six axis neighbours are fluid, as KineticEnergyAnalyzer selects
    them (the walls of a channel exclude the nodes next to them)."""
    b = channel()
    p = Parameter()
    p.set_viscosity_LB(0.01)
    sim = Simulation(p, b, BoundaryConditionFactory())
    g = sim.levels[0]
    sim.init_level(0, *_init(g, 8))
    sim.run(5)
    ke, count = sim.kinetic_energy(0)
    geo, nx, ny, nz, nn = (g[k].astype(np.int64) for k in ("geo", "neighborX", "neighborY", "neighborZ",
                                                           "neighborNeg"))
    fluid = geo == 19
    k = np.nonzero(fluid)[0]
    w = nn[k]
    sel = fluid[nx[k]] & fluid[ny[k]] & fluid[nz[k]] & fluid[w] & fluid[nz[ny[w]]] & fluid[nz[nx[w]]] & fluid[ny[nx[w]]]
    nodes = k[sel]
    assert 0 < count == len(nodes) < len(k)
    drho, vx, vy, vz = sim.macroscopic(0)
    want = np.sum(0.5 * (vx[nodes] ** 2 + vy[nodes] ** 2 + vz[nodes] ** 2) * (drho[nodes] + 1.0)) / len(nodes)
    assert abs(ke - want) <= 1e-12 * abs(want)
