"""The non-equilibrium initialisation (vfb_init_nonequilibrium, the
counterpart of InitNavierStokesCompressibleNonEquilibrium_Device) on the GPU
against the oracle, whose node arithmetic equals the reference's kernel bit for
bit (tests/test_oracle_vs_ref.py), and through the Simulation's
set_use_init_neq switch.

Tolerances: FP64 1e-12 relative to the largest population; FP32 1e-6
relative L2 (fused multiply-adds are the only difference); FP16 / BF16 a few
units of the format's rounding (2e-3 and 1e-2 relative L2)."""
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import rel_l2, rel_max, tgv_state
from tests.test_gpu_simulation import _init, cavity, oracle_schedule
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K
from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GOLDEN = Path(__file__).resolve().parent / "golden"
_TOL = {"float64": 1e-12, "float32": 1e-6, "float16": 2e-3, "bfloat16": 1e-2}


def _level0(name):
    with np.load(GOLDEN / f"grid_{name}.npz") as z:
        return {k.split(":", 1)[1]: z[k] for k in z.files if k.startswith("L0:")}


@pytest.mark.parametrize("grid", ["channel", "sphere_channel"])
@pytest.mark.parametrize("dtype", ["float64", "float32", "float16", "bfloat16"])
def test_init_noneq_matches_oracle(cuda, grid, dtype):
    g = _level0(grid)
    N = len(g["geo"])
    O = Oracle("f64" if dtype == "float64" else "f32")
    rng = np.random.default_rng(8)
    fields = [rng.uniform(-0.02, 0.02, N).astype(O.real) for _ in range(4)]
    omega = 1.6
    ref = np.zeros(27 * N, O.real)
    for ev in (0, 1):
        O.init_noneq(ref, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], g["neighborNeg"], *fields,
                     O.real(omega), ev)
    lat = K.DeviceLattice.from_arrays(g)
    dt = getattr(torch, dtype)
    dist = K.new_distributions(lat, dt)
    dev = [torch.from_numpy(a).cuda() for a in fields]
    for ev in (False, True):
        K.init_nonequilibrium(dist, lat, *dev, omega, ev)
    got = dist.to(torch.float64).cpu().numpy() / K.storage_scale(dt)
    solid = np.flatnonzero((g["geo"] == 15) | (g["geo"] == 16))
    keep = np.ones(27 * N, bool)
    keep[solid] = False  # the rest population of solid nodes holds a marker
    if dtype == "float64":
        assert rel_max(got[keep], ref[keep]) < _TOL[dtype]
    else:
        assert rel_l2(got[keep], ref[keep]) < _TOL[dtype]
    marker = 65504.0 / K.HALF_STORAGE_SCALE if dtype == "float16" else 96.0
    assert np.all(got[solid] == marker)


@pytest.mark.parametrize("dtype,atol", [("float64", 1e-13), ("float32", 1e-6)])
def test_init_noneq_keeps_the_macroscopic_fields(cuda, dtype, atol):
    """The strain-rate part carries no mass and no momentum: the macroscopic
    fields read back from the populations are the ones given (to the rounding
    of the 27-term sums, absolute: the velocity scale is 0.05), while the
    populations differ from the equilibrium init's."""
    w = tgv_state(48)
    lat = K.DeviceLattice.from_arrays(w.grid)
    dt = getattr(torch, dtype)
    fields = [torch.from_numpy(a).to("cuda", dt) for a in (w.rho, w.vx, w.vy, w.vz)]
    dist = K.new_distributions(lat, dt)
    eq = K.new_distributions(lat, dt)
    for ev in (False, True):
        K.init_nonequilibrium(dist, lat, *fields, w.omega, ev)
        K.init_equilibrium(eq, lat, *fields, ev)
    macro = [m.cpu().numpy() for m in K.macroscopic(dist, lat, True)]
    fl = w.grid["fluid"]
    for m, a in zip(macro, (w.rho, w.vx, w.vy, w.vz)):
        assert np.abs(m[fl] - a[fl]).max() <= atol
    geo = w.grid["geo"]
    keep = np.ones(27 * lat.N, bool)
    keep[np.flatnonzero((geo == 15) | (geo == 16))] = False  # rest populations of non-fluid nodes hold the marker
    assert rel_l2(dist.cpu().numpy()[keep], eq.cpu().numpy()[keep]) > 1e-2


def test_init_noneq_needs_the_inverse_neighbour(cuda):
    w = tgv_state(8)
    lat = K.DeviceLattice.from_arrays(w.grid)
    lat.neighborInverse = None
    dist = K.new_distributions(lat, torch.float64)
    f = [torch.zeros(lat.N, dtype=torch.float64, device="cuda") for _ in range(4)]
    with pytest.raises(_lib.VfbError):
        K.init_nonequilibrium(dist, lat, *f, 1.0, True)
    lat = K.DeviceLattice.from_arrays(w.grid)
    with pytest.raises(_lib.VfbError):
        K.init_nonequilibrium(dist, lat, *f, 2.5, True)


def test_simulation_with_init_neq_matches_oracle(cuda):
    """Parameter.set_use_init_neq: the schedule starts from the
    non-equilibrium populations; 20 steps of the lid-driven cavity against the
    oracle started the same way."""
    p = Parameter()
    p.set_storage("fp64")
    p.set_viscosity_LB(0.0032)
    p.set_use_init_neq(True)
    sim = Simulation(p, cavity(12), BoundaryConditionFactory())
    g = sim.levels[0]
    init = _init(g)
    sim.init_level(0, *init)
    sim.run(20)
    got = sim.macroscopic(0)
    ref = oracle_schedule(g, "f64", 0.0032, 20, init, init_neq=True)
    plain = oracle_schedule(g, "f64", 0.0032, 20, init)
    fl = g["fluid"]
    for a, r in zip(got, ref):
        assert rel_max(a[fl], r[fl]) < 1e-12
    assert max(rel_max(a[fl], r[fl]) for a, r in zip(got, plain)) > 1e-9
