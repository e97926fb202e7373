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


@pytest.mark.parametrize("grid", ["channel", "cube_channel", "sphere_channel", "tgv8"])
@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32", 2e-6)])
def test_oracle_enstrophy_matches_reference_kernel(cuda, grid, precision, tol):
    """Pins the oracle's enstrophy restatement to the reference's own kernel:
    EnstrophyAnalyzer.cu compiled unmodified for sm_100a (oracle/_ref), run on
    the same fields; the per-node values and the fluid flags against the
    oracle's (the node function has no transcendental, so FP64 agrees to the
    rounding of contracted multiply-adds)."""
    from oracle.pyoracle import ReferenceGpu, ref_gpu_available

    if not ref_gpu_available(precision):
        pytest.skip("the reference's GPU kernels were not built (oracle/_ref)")
    g = _level0(grid)
    O = Oracle(precision)
    rng = np.random.default_rng(13)
    N = len(g["geo"])
    fields = [rng.uniform(-0.02, 0.02, N).astype(O.real) for _ in range(4)]  # rho, vx, vy, vz
    vals, counted = O.enstrophy_nodes(*fields, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"],
                                      g["neighborNeg"])
    dt = torch.float64 if precision == "f64" else torch.float32
    t = {name: torch.from_numpy(np.ascontiguousarray(g[name]).astype(np.uint32)).cuda()
         for name in ("geo", "neighborX", "neighborY", "neighborZ", "neighborNeg")}
    rho, vx, vy, vz = (torch.from_numpy(a).to("cuda", dt) for a in fields)
    ens = torch.zeros(N, dtype=dt, device="cuda")
    flag = torch.zeros(N, dtype=torch.int32, device="cuda")
    ReferenceGpu(precision).enstrophy(vx, vy, vz, rho, t["neighborX"], t["neighborY"], t["neighborZ"],
                                      t["neighborNeg"], t["geo"], ens, flag)
    torch.cuda.synchronize()
    ref_vals = ens.cpu().numpy().astype(np.float64)
    ref_flag = flag.cpu().numpy() != 0
    assert np.array_equal(ref_flag, counted.astype(bool))
    assert ref_flag.sum() > 0
    v = vals.astype(np.float64)
    assert np.abs(v - ref_vals).max() <= tol * np.abs(ref_vals).max()
