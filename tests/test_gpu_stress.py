"""GPU wall-model (stress) BC kernels (vfb_bc_stress) against the oracle.

The oracle's restatement (vfo_bc_stress) equals the reference's three
kernel sources built for the host bit for bit (tests/test_oracle_vs_ref.py).
Here the library's kernels run through the C ABI on stress lists made from
committed golden grids (tests/stress_cases.py) and are compared in the
populations, both filter states and the monitors.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import STRESS_MONITORS, STRESS_STATE, Oracle
from tests.gpu_helpers import rel_l2, rel_max
from tests.stress_cases import copy_list, make_stress_list, turbulent_viscosity, velocity_fields
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GOLDEN = Path(__file__).resolve().parent / "golden"
KINDS = [_lib.BC_STRESS_INTERPOLATED, _lib.BC_STRESS_BOUNCE_BACK, _lib.BC_STRESS_BOUNCE_BACK_PRESSURE]
# oracle list names -> vfb_stress_list names
TO_ABI = {"vxEl": "Vx", "vyEl": "Vy", "vzEl": "Vz", "vxWMean": "Vx1", "vyWMean": "Vy1", "vzWMean": "Vz1"}


def _grid(name):
    with np.load(GOLDEN / f"grid_{name}.npz") as z:
        return {k.split(":", 1)[1]: z[k] for k in z.files if k.startswith("L0:")}


def _state(g, seed=3):
    """FP64 populations near equilibrium with a non-equilibrium part of up to
    5% of each weight (inside FX16's range of a quarter of the weight)."""
    O = Oracle("f64")
    N = len(g["geo"])
    rng = np.random.default_rng(seed)
    d = np.zeros(27 * N)
    rho = rng.uniform(-1e-2, 1e-2, N)
    u = [rng.uniform(-2e-2, 2e-2, N) for _ in range(3)]
    for ev in (0, 1):
        O.init_eq(d, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], rho, *u, ev)
    w = np.repeat(np.asarray(K.WEIGHTS, float), N)
    d += rng.uniform(-0.05, 0.05, d.shape) * w * (d != 0)
    return d


def _device_list(lst, cd, monitor, locations=None):
    out = {}
    for name, a in lst.items():
        if name in STRESS_MONITORS and not monitor:
            continue
        t = torch.from_numpy(np.ascontiguousarray(a))
        t = t.cuda() if a.dtype.kind == "i" else t.to("cuda", cd)
        out[TO_ABI.get(name, name)] = t
    if locations is not None:
        out["locations"] = locations
    return out


def _run_gpu(g, d, lst, kind, dtype, is_even, vel, turb, monitor=True, table=False):
    """One launch on the GPU; returns (populations unscaled as float64, list arrays)."""
    cd = K.compute_dtype(dtype)
    lat = K.DeviceLattice.from_arrays(g)
    dist = K.new_distributions(lat, dtype)
    dist.copy_(K.encode(d, dtype))
    loc = None
    if table:
        loc = K.bc_locations(lat, torch.from_numpy(lst["k"]).cuda())
    dl = _device_list(lst, cd, monitor, loc)
    v = [torch.from_numpy(a).to("cuda", cd) for a in vel]
    t = None if turb is None else torch.from_numpy(turb).to("cuda", cd)
    K.bc_stress(kind, dist, lat, dl, 1.7, is_even, *v, turbulent_viscosity=t)
    torch.cuda.synchronize()
    got = K.decode(dist)
    back = {name: dl[TO_ABI.get(name, name)].cpu().to(torch.float64).numpy() for name in lst
            if name in STRESS_STATE or (monitor and name in STRESS_MONITORS)}
    return got, back


def _run_oracle_merged(g, d, lst, kind, is_even, vel, turb):
    """The oracle entry by entry on the state before the launch, the written
    cells merged (the GPU reads every entry's values before any write lands
    when the list is resident in one wave; no two entries write one cell)."""
    O = Oracle("f64")
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    n = len(lst["k"])
    want = d.copy()
    written = np.zeros(d.shape, bool)
    out = copy_list(lst)
    for i in range(n):
        one = {key: (np.ascontiguousarray(v.reshape(27, n)[:, i]) if key == "q" else v[i:i + 1].copy())
               for key, v in lst.items()}
        dd = d.copy()
        O.bc_stress(kind, dd, N, *nb, one, 1.7, *vel, turb=turb, monitor=True, is_even=is_even)
        changed = dd != d
        assert not (changed & written).any()
        want[changed] = dd[changed]
        written |= changed
        for key in STRESS_STATE + STRESS_MONITORS:
            out[key][i] = one[key][0]
    return want, out


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("grid,lst_name", [("channel", "slip"), ("sphere_channel", "geometry")])
@pytest.mark.parametrize("is_even", [True, False])
def test_stress_fp64_matches_oracle(cuda, kind, grid, lst_name, is_even):
    g = _grid(grid)
    N = len(g["geo"])
    lst = make_stress_list(g, lst_name, np.float64, seed=11 + kind)
    vel = velocity_fields(N, np.float64, 5)
    turb = turbulent_viscosity(N, np.float64, 6)
    d = _state(g)
    got, back = _run_gpu(g, d, lst, kind, torch.float64, is_even, vel, turb)
    want, ref = _run_oracle_merged(g, d, lst, kind - _lib.BC_STRESS_INTERPOLATED, is_even, vel, turb)
    assert (got != d).sum() > len(lst["k"])
    assert rel_max(got, want) < 1e-12
    for name in back:
        assert rel_max(back[name], ref[name]) < 1e-11, name


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("dtype,tol", [("float32", 1e-6), ("float16", 2e-3), ("int16", 3e-4), ("bfloat16", 2e-2)])
def test_stress_reduced_storage(cuda, kind, dtype, tol):
    """FP32 arithmetic on FP32 and 16-bit storage against the FP64 oracle
    (the populations within the storage's rounding, the wall model's state
    within single precision)."""
    g = _grid("channel")
    N = len(g["geo"])
    lst = make_stress_list(g, "slip", np.float64, seed=23, axis_normal=True)
    vel = velocity_fields(N, np.float64, 5)
    d = _state(g)
    got, back = _run_gpu(g, d, {k: (v.astype(np.float32) if v.dtype == np.float64 else v) for k, v in lst.items()},
                         kind, getattr(torch, dtype), True, vel, None)
    want, ref = _run_oracle_merged(g, d, lst, kind - _lib.BC_STRESS_INTERPOLATED, True, vel, None)
    assert rel_l2(got, want) < tol
    for name in STRESS_STATE + ("uStar",):
        assert rel_l2(back[name], ref[name]) < 5e-5, name


@pytest.mark.parametrize("kind", KINDS)
def test_stress_location_table_and_no_monitor(cuda, kind):
    """The location table writes exactly what the neighbour walk writes, and a
    launch without the monitor writes the same populations and states."""
    g = _grid("sphere_channel")
    N = len(g["geo"])
    lst = make_stress_list(g, "geometry", np.float64, seed=5)
    vel = velocity_fields(N, np.float64, 5)
    d = _state(g)
    a, sa = _run_gpu(g, d, lst, kind, torch.float64, False, vel, None, monitor=True, table=False)
    b, sb = _run_gpu(g, d, lst, kind, torch.float64, False, vel, None, monitor=False, table=True)
    assert np.array_equal(a, b)
    for name in STRESS_STATE:
        assert np.array_equal(sa[name], sb[name])


def test_stress_argument_errors(cuda):
    g = _grid("channel")
    N = len(g["geo"])
    lat = K.DeviceLattice.from_arrays(g)
    dist = K.new_distributions(lat, torch.float64)
    lst = _device_list(make_stress_list(g, "slip", np.float64, seed=1), torch.float64, True)
    v = [torch.zeros(N, dtype=torch.float64, device="cuda") for _ in range(3)]
    with pytest.raises(_lib.VfbError):
        K.bc_stress(5, dist, lat, lst, 1.7, True, *v)  # not a stress kind
    part = dict(lst)
    del part["Fy"]
    with pytest.raises(_lib.VfbError):
        K.bc_stress(_lib.BC_STRESS_BOUNCE_BACK, dist, lat, part, 1.7, True, *v)  # a partial monitor
    with pytest.raises(_lib.VfbError):
        K.bc_stress(_lib.BC_STRESS_INTERPOLATED, dist, lat, lst, 1.0, True, *v)  # omega 1
    empty = {key: t[:0] for key, t in lst.items()}
    K.bc_stress(_lib.BC_STRESS_BOUNCE_BACK, dist, lat, empty, 1.7, True, *v)  # an empty list is a no-op


def _abl(n=(15, 7, 11), offset=2, z0=0.1):
    """The atmospheric boundary layer's set-up (apps/gpu/AtmosphericBoundaryLayer):
    periodic x and y, the wall-model floor under a slip lid."""
    from virtualfluids_b200.grid import MultipleGridBuilder, SideType

    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, *n, 1.0)
    b.setPeriodicBoundaryCondition(True, True, False)
    b.buildGrids()
    b.setStressBoundaryCondition(SideType.MZ, 0.0, 0.0, 1.0, offset, z0, 1.0)
    b.setSlipBoundaryCondition(SideType.PZ, 0.0, 0.0, -1.0)
    return b


def _log_law_init(g, u_star=0.004, z0=0.1, seed=9):
    """A log-law mean flow in x with seeded perturbations, drho small."""
    rng = np.random.default_rng(seed)
    z = g["coordZ"] - g["coordZ"][g["fluid"]].min() + 0.5
    ux = u_star / 0.4 * np.log(np.maximum(z, 1e-3) / z0 + 1.0)
    f = [rng.uniform(-1e-4, 1e-4, len(z)), ux + rng.uniform(-2e-3, 2e-3, len(z)),
         rng.uniform(-2e-3, 2e-3, len(z)), rng.uniform(-1e-3, 1e-3, len(z))]
    solid = g["geo"] != 19
    for a in f:
        a[solid] = 0.0
    return f


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("storage", ["fp64", "fp32"])
def test_abl_schedule_with_stress_matches_oracle(cuda, kind, storage):
    """The scheduled step with the stress floor (after the slip lid, before the
    geometry: UpdateGrid27.cpp:243-249) against the oracle running the same
    order; the wall model samples the level's velocity arrays, which hold the
    initial field until an output pass refreshes them (the launchers pass
    velocityY as vz, Stress.cu:42-160); the monitor's u* and momentum too."""
    from virtualfluids_b200.simulation import (BoundaryConditionFactory, Parameter, Simulation, SlipBC, StressBC)

    b = _abl()
    p = Parameter()
    p.set_storage(storage)
    p.set_viscosity_LB(0.01)
    p.set_has_wall_model_monitor(True)
    p.use_graphs = True
    bc = BoundaryConditionFactory()
    bc.set_slip_boundary_condition(SlipBC.SlipCompressible)
    bc.set_stress_boundary_condition(StressBC(kind))
    sim = Simulation(p, b, bc)
    g = sim.levels[0]
    init = _log_law_init(g)
    sim.init_level(0, *init)
    steps = 12
    sim.run(steps)
    got = sim.macroscopic(0)
    wm = sim.wall_model(0)

    prec = "f64" if storage == "fp64" else "f32"
    O = Oracle(prec)
    real = O.real
    N = len(g["geo"])
    nx, ny, nz, geo, fl = g["neighborX"], g["neighborY"], g["neighborZ"], g["geo"], g["fluid"]
    om = real(1.0 / (3.0 * 0.01 + 0.5))
    d = np.zeros(27 * N, real)
    for ev in (0, 1):
        O.init_eq(d, N, geo, nx, ny, nz, *[a.astype(real) for a in init], ev)
    n = len(g["stress.k"])
    lst = {"k": g["stress.k"], "kN": g["stress.kN"], "q": g["stress.q"].astype(real),
           "normalX": g["stress.nx"].astype(real), "normalY": g["stress.ny"].astype(real),
           "normalZ": g["stress.nz"].astype(real), "samplingOffset": g["stress.samplingOffset"],
           "z0": g["stress.z0"].astype(real)}
    for name in STRESS_STATE + STRESS_MONITORS:
        lst[name] = np.zeros(n, real)
    vx, vy = init[1].astype(real), init[2].astype(real)
    even = True
    for _ in range(steps):
        O.collision_k17(d, N, nx, ny, nz, fl, om, forces=(0, 0, 0), force_factor=1.0, limiters=(0.01, 0.01, 0.01),
                        is_even=even)
        O.bc_post(4, d, N, nx, ny, nz, g["slip.k"], g["slip.q"].astype(real), om, is_even=even)
        O.bc_stress(kind - _lib.BC_STRESS_INTERPOLATED, d, N, nx, ny, nz, lst, om, vx, vy, vy, monitor=True,
                    is_even=even)
        even = not even
    want = O.macroscopic(d, N, geo, nx, ny, nz, even)
    # FP32: drho is of order 1e-4 here, and the GPU's FP32 arithmetic
    # (contracted multiply-adds, logf) rounds along other paths than the
    # oracle's; 1e-4 L2 on every field
    tol = 1e-11 if storage == "fp64" else 1e-4
    for a, w in zip(got, want):
        assert (rel_max if storage == "fp64" else rel_l2)(a[fl], w[fl]) < tol
    for abi, name in [("Vx", "vxEl"), ("Vy", "vyEl"), ("Vz", "vzEl"), ("Vx1", "vxWMean"), ("Vy1", "vyWMean"),
                      ("Vz1", "vzWMean"), ("uStar", "uStar"), ("Fx", "Fx"), ("Fy", "Fy"), ("Fz", "Fz")]:
        assert rel_l2(wm[abi], lst[name]) < (1e-10 if storage == "fp64" else 1e-4), abi
    assert np.all(wm["uStar"] > 0)
