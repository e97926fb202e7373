"""A velocity BC on the geometry (setVelocityBoundaryCondition(GEOMETRY, ...))
through the schedule: the geometry list runs a velocity kind with the
per-node geometry velocities, divided by the velocity ratio at upload as
GridGenerator.cpp:507-513 divides them, and the result equals the oracle
running UpdateGrid27's post-collision order (velocity, then geometry)."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import rel_l2, rel_max
from virtualfluids_b200 import _lib
from virtualfluids_b200.grid import MultipleGridBuilder, SideType, Sphere
from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation, VelocityBC

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GEOMETRY_VELOCITY = (0.01, -0.02, 0.005)


def moving_sphere_channel(geometry_velocity=True):
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 23, 11, 11, 1.0)
    b.addGeometry(Sphere(10.3, 5.6, 5.4, 2.7))
    b.setPeriodicBoundaryCondition(False, True, True)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, 0.02, 0.0, 0.0)
    b.setVelocityBoundaryCondition(SideType.PX, 0.02, 0.0, 0.0)
    if geometry_velocity:
        b.setVelocityBoundaryCondition(SideType.GEOMETRY, *GEOMETRY_VELOCITY)
    else:
        b.setNoSlipBoundaryCondition(SideType.GEOMETRY)
    return b


def bc_post_simultaneous(O, kind, d, N, nb, k, q, omega, vel, is_even):
    """A post-collision BC over a list whose nodes neighbour each other (around
    a sphere one node's bounce-back lands in a cell that another BC node
    reads): the GPU kernels read every node's values before writing, so the
    oracle applies each node to the state before the kernel and the written
    cells are merged (no two nodes write one cell)."""
    n = len(k)
    q = q.reshape(27, n)
    out = d.copy()
    written = np.zeros(d.shape, bool)
    for i in range(n):
        one = d.copy()
        O.bc_post(kind, one, N, *nb, k[i:i + 1], np.ascontiguousarray(q[:, i]), omega,
                  *[v[i:i + 1] for v in vel], is_even=is_even)
        changed = one != d
        assert not (changed & written).any()
        out[changed] = one[changed]
        written |= changed
    d[:] = out


def oracle_run(g, precision, nu, steps, init, ratio):
    O = Oracle(precision)
    real = O.real
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    d = np.zeros(27 * N, real)
    for ev in (0, 1):
        O.init_eq(d, N, g["geo"], *nb, *[a.astype(real) for a in init], ev)
    om = 1.0 / (3.0 * nu + 0.5)
    vel = [g[f"velocity.{c}"].astype(real) for c in ("vx", "vy", "vz")]
    # the reference divides the geometry velocities in the working precision
    gvel = [g[f"geometry.{c}"].astype(real) / real(ratio) for c in ("vx", "vy", "vz")]
    even = True
    for _ in range(steps):
        O.collision_k17(d, N, *nb, g["fluid"], om, is_even=even)
        O.bc_post(_lib.BC_VELOCITY_INTERPOLATED, d, N, *nb, g["velocity.k"], g["velocity.q"].astype(real), om, *vel,
                  is_even=even)
        bc_post_simultaneous(O, _lib.BC_VELOCITY_INTERPOLATED, d, N, nb, g["geometry.k"],
                             g["geometry.q"].astype(real), real(om), gvel, even)
        even = not even
    return O.macroscopic(d, N, g["geo"], *nb, even)


@pytest.mark.parametrize("storage", ["fp64", "fp32"])
@pytest.mark.parametrize("ratio", [1.0, 2.5])
def test_geometry_velocity_schedule_matches_oracle(cuda, storage, ratio):
    p = Parameter()
    p.set_storage(storage)
    p.set_viscosity_LB(0.01)
    p.set_velocity_ratio(ratio)
    bc = BoundaryConditionFactory()
    bc.set_geometry_boundary_condition(VelocityBC.VelocityInterpolatedCompressible)
    sim = Simulation(p, moving_sphere_channel(), bc)
    g = sim.levels[0]
    assert len(g["geometry.k"]) > 50 and np.all(g["geometry.vy"] == GEOMETRY_VELOCITY[1])
    rng = np.random.default_rng(11)
    N = len(g["geo"])
    init = [rng.uniform(-1e-3, 1e-3, N) for _ in range(4)]
    for a in init:
        a[g["geo"] != 19] = 0.0
    sim.init_level(0, *init)
    steps = 12
    sim.run(steps)
    got = sim.macroscopic(0)
    ref = oracle_run(g, "f64" if storage == "fp64" else "f32", 0.01, steps, init, ratio)
    fl = g["fluid"]
    for a, r in zip(got, ref):
        if storage == "fp64":
            assert rel_max(a[fl], r[fl]) < 1e-12
        else:
            assert rel_l2(a[fl], r[fl]) < 1e-5
    sim.close()


def test_velocity_geometry_bc_needs_geometry_velocities(cuda):
    """A velocity kind on a geometry list that carries no velocities is a
    configuration error of vfb_sim_create."""
    bc = BoundaryConditionFactory()
    bc.set_geometry_boundary_condition(VelocityBC.VelocityInterpolatedCompressible)
    p = Parameter()
    p.set_viscosity_LB(0.01)
    with pytest.raises(_lib.VfbError) as e:
        Simulation(p, moving_sphere_channel(geometry_velocity=False), bc)
    assert e.value.code == _lib.VFB_ERR_CONFIGURATION
    assert "geometry velocities" in str(e.value)
