"""The planned (bulk-copy, warp-tiled) collision path against the oracle and
against the generic kernel, on periodic and walled grids."""
import numpy as np
import pytest

from tests.gpu_helpers import gpu_run, oracle_run, rel_l2, rel_max, tgv_state
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K
from virtualfluids_b200.grid import MultipleGridBuilder, SideType

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("n", [16, 10, 33])
@pytest.mark.parametrize("kernel", ["K17", "BGK"])
def test_planned_fp64_matches_oracle(cuda, n, kernel):
    w = tgv_state(n)
    steps = 12
    _, ref, _ = oracle_run(w, "f64", steps, kernel)
    _, _, got, _ = gpu_run(w, torch.float64, steps, kernel, planned=True)
    fl = w.grid["fluid"]
    for a, b in zip(got, ref):
        assert rel_max(a[fl], b[fl]) < 1e-12


@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16", "int16"])
def test_planned_matches_generic(cuda, dtype):
    w = tgv_state(24)
    dt = getattr(torch, dtype)
    d1, _, m1, _ = gpu_run(w, dt, 10, planned=True)
    d2, _, m2, _ = gpu_run(w, dt, 10, planned=False)
    fl = w.grid["fluid"]
    # The planned default multiplies and adds two nodes at once in paired FP32
    # arithmetic, which rounds some products the scalar kernel fuses.  FP32:
    # the FP32 contract (1e-5 L2, the tolerance against the FP64 oracle).  FP16
    # / BF16: a store may then round to the neighbouring 16-bit value, so the
    # bound is a few units of the format's rounding (2^-11 for FP16, 2^-8 for
    # BF16) after 10 steps.
    # FX16 (int16): a store may round to the neighbouring step of 2^-17 of
    # the weight, an absolute step; on drho (about 1e-3 here) a few such
    # steps summed over the node's populations come to a few 1e-3 relative.
    tol = {"float32": 1e-5, "float16": 2e-3, "bfloat16": 1e-2, "int16": 3e-3}[dtype]
    for a, b in zip(m1, m2):
        assert rel_l2(a[fl], b[fl]) < tol


def test_plan_statistics_for_periodic_cube(cuda):
    w = tgv_state(64)
    lat = K.DeviceLattice.from_arrays(w.grid)
    plan = K.CollisionPlan(torch.float32, lat)
    st = plan.stats()
    # every node of a periodic box is served by the bulk tiles, the nodes on
    # the last x, y or z layer through their wrap offsets
    assert st["bulk_nodes"] == 64 ** 3
    assert st["lane_nodes"] == 0
    assert st["wrap_nodes"] == 64 ** 3 - 63 ** 3


def _walled_grid(periodic_y=False):
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 20, 13, 11, 1.0)
    b.setPeriodicBoundaryCondition(False, periodic_y, False)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, 0.03, 0, 0)
    b.setNoSlipBoundaryCondition(SideType.MZ)
    return b.arrays()[0]


@pytest.mark.parametrize("periodic_y", [False, True])
def test_planned_on_walled_grid_matches_generic(cuda, periodic_y):
    g = _walled_grid(periodic_y)
    lat = K.DeviceLattice.from_arrays(g)
    rng = np.random.default_rng(5)
    N = lat.N
    fields = [torch.from_numpy(rng.uniform(-1e-3, 1e-3, N)).cuda() for _ in range(4)]
    outs = []
    for planned in (True, False):
        dist = K.new_distributions(lat, torch.float64)
        for ev in (False, True):
            K.init_equilibrium(dist, lat, *fields, ev)
        plan = K.CollisionPlan(torch.float64, lat) if planned else None
        even = True
        for _ in range(8):
            K.collision("K17", dist, lat, 1.7, even, plan=plan, forces=(1e-5, 0, 0))
            even = not even
        outs.append(dist.cpu().numpy())
    assert rel_max(outs[0], outs[1]) < 1e-13


@pytest.mark.parametrize("template", [1, 2, 3])
def test_planned_templates_match_generic(cuda, template):
    w = tgv_state(12)
    lat = K.DeviceLattice.from_arrays(w.grid)
    N = lat.N
    rng = np.random.default_rng(11)
    body0 = [rng.uniform(-1e-5, 1e-5, N) for _ in range(3)]
    res = []
    for planned in (True, False):
        dist = K.new_distributions(lat, torch.float64)
        fields = [torch.from_numpy(a).cuda() for a in (w.rho, w.vx, w.vy, w.vz)]
        for ev in (False, True):
            K.init_equilibrium(dist, lat, *fields, ev)
        macro = [torch.zeros(N, dtype=torch.float64, device="cuda") for _ in range(4)]
        body = [torch.from_numpy(b.copy()).cuda() for b in body0]
        plan = K.CollisionPlan(torch.float64, lat) if planned else None
        K.collision("K17", dist, lat, w.omega, True, plan=plan, template=template, macro=macro, body=body,
                    forces=(2e-6, 0, -1e-6), force_factor=0.5)
        res.append([dist.cpu().numpy()] + [m.cpu().numpy() for m in macro] + [b.cpu().numpy() for b in body])
    for a, b in zip(*res):
        assert rel_max(a, b) < 1e-13 if np.abs(b).max() > 0 else np.array_equal(a, b)


def test_plan_rejects_other_arrays(cuda):
    w = tgv_state(8)
    lat = K.DeviceLattice.from_arrays(w.grid)
    plan = K.CollisionPlan(torch.float32, lat)
    dist = K.new_distributions(lat, torch.float32)
    other = lat.fluid.clone()
    with pytest.raises(_lib.VfbError):
        K.collision("K17", dist, lat, w.omega, True, plan=plan, fluid=other)


@pytest.mark.parametrize("n", [16, 13])
def test_planned_fp32_matches_fp64_oracle(cuda, n):
    w = tgv_state(n)
    _, ref, _ = oracle_run(w, "f64", 12)
    _, _, got, _ = gpu_run(w, torch.float32, 12, planned=True)
    fl = w.grid["fluid"]
    for a, b in zip(got, ref):
        assert rel_l2(a[fl], b[fl]) < 1e-5


@pytest.mark.parametrize("dtype", ["float32", "float16"])
def test_planned_bgk_matches_generic(cuda, dtype):
    w = tgv_state(20)
    dt = getattr(torch, dtype)
    _, _, m1, _ = gpu_run(w, dt, 8, "BGK", planned=True)
    _, _, m2, _ = gpu_run(w, dt, 8, "BGK", planned=False)
    fl = w.grid["fluid"]
    # the planned BGK pairs two nodes' arithmetic (paired FP32), which rounds
    # some products the scalar kernel fuses: the FP32 contract, 1e-5 L2
    tol = 1e-5 if dtype == "float32" else 2e-3
    for a, b in zip(m1, m2):
        assert rel_l2(a[fl], b[fl]) < tol


# every compiled tile configuration (VFB_TILE_CONFIG, read at plan creation):
# index -> storages it serves
_CONFIGS_FP64 = [1, 6, 10, 11, 17, 18]
_CONFIGS_FP32 = [0, 2, 3, 4, 5, 7, 8, 9, 12, 13, 14, 15, 16, 19, 20]
_CONFIGS_HALF = [9, 12, 19, 20]


@pytest.mark.parametrize("config,dtype", [(c, "float64") for c in _CONFIGS_FP64] +
                         [(c, "float32") for c in _CONFIGS_FP32] + [(c, "float16") for c in _CONFIGS_HALF] +
                         [(c, "int16") for c in _CONFIGS_HALF])
def test_every_tile_configuration_matches_oracle(cuda, monkeypatch, config, dtype):
    """Each tuning configuration on a box whose rows and tiles do not line up
    (13^3: wrap lanes and partial warps), 6 steps against the FP64 oracle."""
    monkeypatch.setenv("VFB_TILE_CONFIG", str(config))
    w = tgv_state(13)
    _, ref, _ = oracle_run(w, "f64", 6)
    _, _, got, _ = gpu_run(w, getattr(torch, dtype), 6, planned=True)
    fl = w.grid["fluid"]
    for a, b in zip(got, ref):
        if dtype == "float64":
            assert rel_max(a[fl], b[fl]) < 1e-12
        else:
            # int16 (FX16): the absolute step 2^-17 w on fields of about 1e-3 (drho)
            assert rel_l2(a[fl], b[fl]) < {"float32": 1e-5, "float16": 5e-3, "int16": 4e-3}[dtype]
