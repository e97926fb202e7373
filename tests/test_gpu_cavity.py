"""The lid-driven cavity of the benchmark configurations (64^3, FP64, lid
u = (0.05, 0, 0) on +z, halfway walls on the other faces, nu = 0.0032) through
the public Simulation API with CUDA-graph replay, against the FP64 oracle
running the same schedule (K17, the velocity BC over all six walls, the parity
swap) for 200 steps."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from virtualfluids_b200.grid import MultipleGridBuilder, SideType
from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_cavity64_fp64_200_steps_matches_oracle(cuda):
    n, nu, steps = 64, 0.0032, 200
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
    assert np.abs(ref[1][fl]).max() > 1e-3  # the lid has set the fluid in motion
    for a, r in zip(got, ref):
        assert np.abs(a[fl] - r[fl]).max() <= 1e-12 * np.abs(r[fl]).max()
