"""The enstrophy analyzer on the GPU (vfb_enstrophy, vfb_sim_enstrophy)
against the oracle's node values summed in FP64.  The node arithmetic is the
library's host-checked code (tests/test_enstrophy_host.py); here the kernel,
its FP64 reduction and the schedule's entry are checked.  Tolerances: FP64
1e-12 relative, FP32 1e-5 relative; the node count is exact."""
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.test_gpu_simulation import _init, cavity, oracle_schedule
from virtualfluids_b200 import kernels as K
from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GOLDEN = Path(__file__).resolve().parent / "golden"


def _level0(name):
    with np.load(GOLDEN / f"grid_{name}.npz") as z:
        return {k.split(":", 1)[1]: z[k] for k in z.files if k.startswith("L0:")}


@pytest.mark.parametrize("grid", ["channel", "cube_channel", "sphere_channel"])
@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_enstrophy_matches_oracle(cuda, grid, precision, tol):
    g = _level0(grid)
    O = Oracle(precision)
    rng = np.random.default_rng(9)
    fields = [rng.uniform(-0.02, 0.02, len(g["geo"])).astype(O.real) for _ in range(4)]
    vals, counted = O.enstrophy_nodes(*fields, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"],
                                      g["neighborNeg"])
    lat = K.DeviceLattice.from_arrays(g)
    mean, count = K.enstrophy(lat, *[torch.from_numpy(a).cuda() for a in fields])
    assert count == int(counted.sum()) > 0
    ref = vals[counted].astype(np.float64).sum() / count
    assert abs(mean - ref) <= tol * abs(ref)


def test_simulation_enstrophy_matches_oracle(cuda):
    p = Parameter()
    p.set_storage("fp64")
    p.set_viscosity_LB(0.0032)
    sim = Simulation(p, cavity(12), BoundaryConditionFactory())
    g = sim.levels[0]
    init = _init(g)
    sim.init_level(0, *init)
    sim.run(10)
    mean, count = sim.enstrophy(0)
    rho, vx, vy, vz = oracle_schedule(g, "f64", 0.0032, 10, init)
    vals, counted = Oracle("f64").enstrophy_nodes(rho, vx, vy, vz, g["geo"], g["neighborX"], g["neighborY"],
                                                  g["neighborZ"], g["neighborNeg"])
    assert count == int(counted.sum()) > 0
    ref = vals[counted].sum() / count
    assert abs(mean - ref) <= 1e-8 * abs(ref)
