"""VelocityWithPressureInterpolatedCompressible (VFB_BC_VELOCITY_WITH_PRESSURE)
on the GPU: the velocity BC's interpolation minus w drho
(KernelUtilities.h:208-214).  The oracle's version of it equals the
reference's kernel source built for the host bit for bit
(tests/test_oracle_vs_ref.py); here the library's kernel is checked against
the oracle on wall lists (FP64 1e-12, FP32 1e-5 L2) and against the
reference's own GPU kernel compiled for sm_100a."""
import numpy as np
import pytest

from oracle.pyoracle import ReferenceGpu, ref_gpu_available
from tests.gpu_helpers import rel_l2, rel_max
from tests.test_gpu_bc import GpuImpl, _grid, _random_state
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
KIND = _lib.BC_VELOCITY_WITH_PRESSURE


def _velocities(n, real, seed=31):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-0.03, 0.03, n).astype(real) for _ in range(3)]


@pytest.mark.parametrize("is_even", [True, False])
@pytest.mark.parametrize("grid", ["cavity8", "channel"])
def test_velocity_with_pressure_matches_oracle_fp64(cuda, grid, is_even):
    g = _grid(grid)
    k, q = g["velocity.k"], g["velocity.q"].astype(np.float64)
    vel = _velocities(len(k), np.float64)
    O, d = _random_state(g, "f64")
    N = len(g["geo"])
    imp = GpuImpl(g, torch.float64)
    imp.load(d)
    got = d.copy()
    imp.bc_post(KIND, got, N, None, None, None, k, q, 1.7, *vel, is_even=is_even)
    before = d.copy()
    O.bc_post(KIND, d, N, g["neighborX"], g["neighborY"], g["neighborZ"], k, q, 1.7, *vel, is_even=is_even)
    assert (d != before).any()
    assert rel_max(got, d) < 1e-12


def test_velocity_with_pressure_matches_oracle_fp32(cuda):
    g = _grid("channel")
    k, q = g["velocity.k"], g["velocity.q"].astype(np.float32)
    vel = _velocities(len(k), np.float32)
    O, d = _random_state(g, "f32")
    N = len(g["geo"])
    imp = GpuImpl(g, torch.float32)
    imp.load(d)
    got = d.copy()
    imp.bc_post(KIND, got, N, None, None, None, k, q, 1.7, *vel, is_even=True)
    O.bc_post(KIND, d, N, g["neighborX"], g["neighborY"], g["neighborZ"], k, q, 1.7, *vel, is_even=True)
    assert rel_l2(got, d) < 1e-5


@pytest.mark.skipif(not ref_gpu_available("f64"), reason="reference GPU kernels not built")
def test_velocity_with_pressure_matches_reference_gpu_kernel(cuda):
    g = _grid("channel")
    _, d = _random_state(g, "f64")
    lat = K.DeviceLattice.from_arrays(g)
    ours = torch.from_numpy(d).cuda()
    ref = ours.clone()
    k = torch.from_numpy(g["velocity.k"].astype(np.int32)).cuda()
    q = torch.from_numpy(g["velocity.q"].astype(np.float64)).cuda()
    vel = [torch.from_numpy(v).cuda() for v in _velocities(k.numel(), np.float64)]
    for ev in (True, False):
        K.bc_post(KIND, ours, lat, k, q, 1.7, ev, *vel, stream=0)
        ReferenceGpu("f64").bc_post(KIND, ref, lat, k, q, 1.7, ev, *vel)
    torch.cuda.synchronize()
    a, b = ours.cpu().numpy(), ref.cpu().numpy()
    assert rel_max(a, b) < 1e-12
