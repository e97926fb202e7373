"""The non-reflecting outflow (vfb_bc_outflow_nonreflecting: the
counterparts of OutflowNonReflecting and OutflowNonReflectingPressureCorrection)
on the GPU against the oracle, whose arithmetic equals the reference's kernels
bit for bit (tests/test_oracle_vs_ref.py), and in the schedule as the
pressure-list kind.

Lists are planes normal to the list's axis, as grids make them: then the
positions one BC node reads are never written by another, and the GPU result
does not depend on the order of the threads.  Tolerances: FP64 1e-12 relative
to the largest population, FP32 1e-6 relative L2."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import rel_l2, rel_max, tgv_state
from tests.test_gpu_simulation import _init, channel, oracle_schedule
from virtualfluids_b200 import kernels as K
from virtualfluids_b200.simulation import (BoundaryConditionFactory, Parameter, PressureBC, SlipBC, Simulation,
                                           VelocityBC)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_AXIS = {1: ("coordX", 1), 2: ("coordX", -1), 3: ("coordY", 1), 4: ("coordY", -1), 5: ("coordZ", 1),
         6: ("coordZ", -1)}


def _plane_list(g, direction, rng):
    """The fluid nodes of one lattice plane normal to the direction's axis,
    with random inner neighbours."""
    name, _ = _AXIS[direction]
    c = g[name]
    level = np.unique(c[1:])[3]
    k = np.intersect1d(np.flatnonzero(c == level), g["fluid"]).astype(np.int32)
    kN = rng.integers(1, len(c), len(k)).astype(np.int32)
    return k, kN


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("correction", [False, True])
@pytest.mark.parametrize("direction", [1, 2, 3, 4, 5, 6])
def test_outflow_matches_oracle(cuda, dtype, correction, direction):
    w = tgv_state(12)
    g = w.grid
    N = len(g["geo"])
    O = Oracle("f64" if dtype == "float64" else "f32")
    rng = np.random.default_rng(direction)
    k, kN = _plane_list(g, direction, rng)
    d0 = rng.uniform(-0.02, 0.02, 27 * N).astype(O.real)
    lat = K.DeviceLattice.from_arrays(g)
    for even in (True, False):
        ref = d0.copy()
        O.bc_outflow(ref, N, g["neighborX"], g["neighborY"], g["neighborZ"], k, kN, direction, correction,
                     O.real(0.3), even)
        dist = torch.from_numpy(d0.copy()).cuda()
        K.bc_outflow(dist, lat, torch.from_numpy(k).cuda(), torch.from_numpy(kN).cuda(), direction, even,
                     pressure_correction=correction, correction_factor=0.3)
        got = dist.cpu().numpy()
        assert (ref != d0).sum() == 9 * len(k) and (got != d0).sum() > 0
        if dtype == "float64":
            assert rel_max(got, ref) < 1e-12
        else:
            assert rel_l2(got, ref) < 1e-6


@pytest.mark.parametrize("kind", [PressureBC.OutflowNonReflective, PressureBC.OutflowNonReflectivePressureCorrection])
def test_channel_schedule_with_outflow(cuda, kind):
    """The channel (velocity inlet, outflow plane, no-slip floor, slip top)
    for 20 steps with the outflow as the pressure-list kind, against the
    oracle's schedule."""
    p = Parameter()
    p.set_viscosity_LB(0.01)
    p.set_outflow_pressure_correction_factor(0.25)
    bc = BoundaryConditionFactory()
    bc.set_velocity_boundary_condition(VelocityBC.VelocityInterpolatedCompressible)
    bc.set_slip_boundary_condition(SlipBC.SlipCompressible)
    bc.set_pressure_boundary_condition(kind)
    sim = Simulation(p, channel(), bc)
    g = sim.levels[0]
    init = _init(g, 5)
    sim.init_level(0, *init)
    sim.run(20)
    got = sim.macroscopic(0)
    ref = oracle_schedule(g, "f64", 0.01, 20, init, slip=True, pressure=True, pressure_kind=int(kind),
                          correction_factor=0.25)
    fl = g["fluid"]
    for a, r in zip(got, ref):
        assert rel_max(a[fl], r[fl]) < 1e-12
