"""The FX16 storage (int16 q with f_d - w_d = q w_d 2^-17, FP32 arithmetic):
the stored codes of an equilibrium init equal the host's rounding of the
oracle's FP32 init to within one code, values beyond a quarter of the weight
saturate, solid nodes hold the saturated marker, and the Taylor-Green vortex
at 64^3 after 250 steps stays within 5e-4 L2 of the FP64 oracle (IEEE FP16
storage: about 1e-3)."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import gpu_run, oracle_run, rel_l2, tgv_state
from virtualfluids_b200 import kernels as K
from virtualfluids_b200.workloads import cavity_grid

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_init_codes_match_host_rounding(cuda):
    w = tgv_state(12)
    g = w.grid
    N = len(g["geo"])
    O = Oracle("f32")
    ref = np.zeros(27 * N, np.float32)
    for ev in (0, 1):
        O.init_eq(ref, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"],
                  *[a.astype(np.float32) for a in (w.rho, w.vx, w.vy, w.vz)], ev)
    lat = K.DeviceLattice.from_arrays(g)
    dist = K.new_distributions(lat, torch.int16)
    fields = [torch.from_numpy(a).to("cuda", torch.float32) for a in (w.rho, w.vx, w.vy, w.vz)]
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    got = dist.cpu().numpy().astype(np.int64)
    want = K.encode(ref.astype(np.float64), torch.int16, "cpu").numpy().astype(np.int64)
    fluid_rows = np.zeros(N, bool)
    fluid_rows[g["fluid"]] = True
    mask = np.tile(fluid_rows, 27)
    assert np.abs(got[mask] - want[mask]).max() <= 1
    assert np.mean(got[mask] == want[mask]) > 0.99
    assert np.abs(got[mask]).max() < 32767  # u0 = 0.05 is inside the range


def test_saturation_and_decode(cuda):
    w = tgv_state(8)
    lat = K.DeviceLattice.from_arrays(w.grid)
    dist = K.new_distributions(lat, torch.int16)
    big = [torch.full((lat.N,), v, dtype=torch.float32, device="cuda") for v in (0.0, 0.3, 0.0, 0.0)]
    K.init_equilibrium(dist, lat, *big, True)
    q = dist.view(27, -1)[:, w.grid["fluid"].astype(np.int64)].cpu().numpy()
    # with u = 0.3 the positive-x directions exceed a quarter of their weight: saturated codes
    assert q[1].max() == 32767 and q[2].min() == -32768
    vals = K.decode(dist).reshape(27, -1)
    assert abs(vals[1].max() - 0.25 * K.WEIGHTS[1] * 32767 / 32768) < 1e-12


def test_solid_marker(cuda):
    """The non-equilibrium init marks the rest population of solid and void
    nodes (the reference writes 96, InitNavierStokesCompressible_Device.cu:490-499);
    FX16 holds its saturated code there."""
    g = cavity_grid(8)
    lat = K.DeviceLattice.from_arrays(g)
    dist = K.new_distributions(lat, torch.int16)
    zero = torch.zeros(lat.N, dtype=torch.float32, device="cuda")
    for ev in (False, True):
        K.init_nonequilibrium(dist, lat, zero, zero, zero, zero, 1.6, ev)
    solid = np.flatnonzero((g["geo"] == 15) | (g["geo"] == 16))
    assert len(solid) > 0
    rest = dist.view(27, -1)[0].cpu().numpy()
    assert np.all(rest[solid] == 32767)


def test_tgv64_250_steps_accuracy(cuda):
    w = tgv_state(64)
    _, ref, _ = oracle_run(w, "f64", 250)
    fl = w.grid["fluid"]
    u_ref = np.concatenate([ref[i][fl] for i in (1, 2, 3)])
    errs = {}
    for dt in (torch.int16, torch.float16):
        _, _, got, _ = gpu_run(w, dt, 250, planned=True)
        errs[dt] = rel_l2(np.concatenate([got[i][fl] for i in (1, 2, 3)]), u_ref)
    print("L2(u) after 250 steps at 64^3:", {str(k): v for k, v in errs.items()})
    assert errs[torch.int16] < 5e-4
    assert errs[torch.int16] < errs[torch.float16]
