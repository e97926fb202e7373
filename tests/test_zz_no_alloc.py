"""vfb_mass_and_energy_static: the mass / kinetic-energy sums without any
allocation, for callers that cannot allocate device memory where they want the
sums (a host whose pool allocator owns all of HBM, or a monitor inside a
solver loop whose memory footprint must stay fixed).

Its output must equal that of vfb_mass_and_energy (which takes its scratch
from cudaMallocAsync) on the same populations, on two calls in a row: the
second call reuses the static scratch the first one left behind.  This file
is collected last so that a stop at the first failure has run every other
test already."""
import ctypes

import pytest

from tests.gpu_helpers import tgv_state
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

REL_TOL = 1e-12  # both sum the same FP64 block partials in block order


def _sums(fn, dist, lat, even):
    out = (ctypes.c_double * 3)()
    rc = fn(K.STORAGE_OF_DTYPE[dist.dtype], dist.data_ptr(), lat.N, lat.neighborX.data_ptr(),
            lat.neighborY.data_ptr(), lat.neighborZ.data_ptr(), lat.fluid.data_ptr(), lat.numberOfFluidNodes,
            int(even), out, torch.cuda.current_stream().cuda_stream)
    _lib.check(rc)
    return list(out)


def _close(a, b):
    return all(abs(x - y) <= REL_TOL * max(abs(y), 1e-300) for x, y in zip(a, b))


@pytest.mark.parametrize("n", [8, 64])
@pytest.mark.parametrize("dtype", ["float32", "float64", "float16", "bfloat16", "int16"])
def test_static_sums_match_allocating_entry_point(cuda, n, dtype):
    dtype = getattr(torch, dtype)
    w = tgv_state(n)
    lat = K.DeviceLattice.from_arrays(w.grid)
    cd = K.compute_dtype(dtype)
    fields = [torch.from_numpy(a).to("cuda", cd) for a in (w.rho, w.vx, w.vy, w.vz)]
    dist = K.new_distributions(lat, dtype)
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    L = _lib.lib()
    even = True
    for call in range(2):
        K.collision("K17", dist, lat, w.omega, even)
        even = not even
        ref = _sums(L.vfb_mass_and_energy, dist, lat, even)
        got = _sums(L.vfb_mass_and_energy_static, dist, lat, even)
        assert ref[1] > 0.0 and ref[2] == 0.0
        assert _close(got, ref), (call, got, ref)


def test_static_empty_list_and_null_output(cuda):
    L = _lib.lib()
    out = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    assert L.vfb_mass_and_energy_static(0, None, 0, None, None, None, None, 0, 1, out, None) == _lib.VFB_OK
    assert list(out) == [0.0, 0.0, 0.0]
    assert L.vfb_mass_and_energy_static(0, None, 0, None, None, None, None, 1, 1, None, None) == \
        _lib.VFB_ERR_INVALID_ARGUMENT
