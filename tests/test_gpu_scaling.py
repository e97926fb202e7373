"""GPU interface interpolation (vfb_scale_coarse_to_fine / _fine_to_coarse)
against the reference's own kernels compiled on the host (oracle/_ref) and
against the library's host execution of the same arithmetic."""
import numpy as np
import pytest

from oracle.pyoracle import Reference, ref_available
from tests.gpu_helpers import rel_l2, rel_max
from tests.scaling_cases import case, host_arrays, scaling_args
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def device_arrays(c, real):
    out, keep = {}, []
    for key in ("gc", "gf"):
        for ax in "XYZ":
            t = torch.from_numpy(c[key][f"neighbor{ax}"].view(np.int32)).cuda()
            keep.append(t)
            out[f"{key}.neighbor{ax}"] = t.data_ptr()
    for name in ("coarse_cf", "fine_cf", "coarse_fc", "fine_fc"):
        t = torch.from_numpy(c[name].view(np.int32)).cuda()
        keep.append(t)
        out[name] = t.data_ptr()
    for i, ax in enumerate("XYZ"):
        t = torch.from_numpy(np.ascontiguousarray(c["off"][i]).astype(real)).cuda()
        keep.append(t)
        out[f"off{ax}"] = t.data_ptr()
    return out, keep


def run_gpu(c, coarse_to_fine, is_even, dtype):
    cd = K.compute_dtype(dtype)
    real = np.float64 if cd == torch.float64 else np.float32
    scale = K.storage_scale(dtype)
    dC = (torch.from_numpy(c["distC"].astype(np.float64)) * scale).to("cuda", dtype)
    dF = (torch.from_numpy(c["distF"].astype(np.float64)) * scale).to("cuda", dtype)
    arrays, keep = device_arrays(c, real)
    a = scaling_args(c, coarse_to_fine, is_even, dC.data_ptr(), dF.data_ptr(), arrays)
    fn = _lib.lib().vfb_scale_coarse_to_fine if coarse_to_fine else _lib.lib().vfb_scale_fine_to_coarse
    _lib.check(fn(K.STORAGE_OF_DTYPE[dtype], a, None))
    torch.cuda.synchronize()
    return [t.cpu().to(torch.float64).numpy() / scale for t in (dC, dF)]


def run_host(c, coarse_to_fine, is_even, precision):
    arrays = host_arrays(c)
    mc, mf = c["distC"].copy(), c["distF"].copy()
    a = scaling_args(c, coarse_to_fine, is_even, mc.ctypes.data, mf.ctypes.data, arrays)
    _lib.check(_lib.lib().vfb_debug_scale_host(int(coarse_to_fine), precision, a))
    return mc, mf


@pytest.mark.parametrize("is_even", [True, False])
@pytest.mark.parametrize("coarse_to_fine", [True, False])
def test_gpu_interpolation_fp64(cuda, coarse_to_fine, is_even):
    c = case(3)
    got = run_gpu(c, coarse_to_fine, is_even, torch.float64)
    host = run_host(c, coarse_to_fine, is_even, _lib.FP64)
    for g, h in zip(got, host):
        assert rel_max(g, h) < 1e-13
    if ref_available("f64"):
        ref_c, ref_f = c["distC"].copy(), c["distF"].copy()
        tag = "cf" if coarse_to_fine else "fc"
        Reference("f64").scale(coarse_to_fine, ref_c, ref_f, c["gc"], c["gf"], is_even, c[f"coarse_{tag}"],
                               c[f"fine_{tag}"], c["omegaC"], c["omegaF"], c["offX"], c["offY"], c["offZ"])
        for g, r in zip(got, (ref_c, ref_f)):
            assert rel_max(g, r) < 1e-13


@pytest.mark.parametrize("coarse_to_fine", [True, False])
@pytest.mark.parametrize("dtype,tol", [("float32", 1e-6), ("float16", 3e-3), ("bfloat16", 3e-2)])
def test_gpu_interpolation_reduced_storage(cuda, coarse_to_fine, dtype, tol):
    c = case(4)
    dt = getattr(torch, dtype)
    got = run_gpu(c, coarse_to_fine, True, dt)
    host = run_host(c, coarse_to_fine, True, _lib.FP64)
    for g, h in zip(got, host):
        assert rel_l2(g, h) < tol


@pytest.mark.parametrize("coarse_to_fine", [True, False])
def test_block_tables_equal_the_neighbour_walk(cuda, coarse_to_fine):
    """With the cells' block tables (vfb_scaling_blocks) the interpolation
    reads the same nodes as through the neighbour walk: FP64 results equal bit
    for bit."""
    c = case(3)
    outs = []
    for tables in (False, True):
        dC = torch.from_numpy(c["distC"].astype(np.float64)).cuda()
        dF = torch.from_numpy(c["distF"].astype(np.float64)).cuda()
        arrays, keep = device_arrays(c, np.float64)
        a = scaling_args(c, coarse_to_fine, True, dC.data_ptr(), dF.data_ptr(), arrays)
        if tables:
            tag = "cf" if coarse_to_fine else "fc"
            n = len(c[f"coarse_{tag}"])
            bc = torch.empty(27 * n, dtype=torch.int32, device="cuda")
            bf = torch.empty(27 * n, dtype=torch.int32, device="cuda")
            lib = _lib.lib()
            _lib.check(lib.vfb_scaling_blocks(arrays[f"coarse_{tag}"], n, arrays["gc.neighborX"], arrays["gc.neighborY"],
                                              arrays["gc.neighborZ"], bc.data_ptr(), None))
            _lib.check(lib.vfb_scaling_blocks(arrays[f"fine_{tag}"], n, arrays["gf.neighborX"], arrays["gf.neighborY"],
                                              arrays["gf.neighborZ"], bf.data_ptr(), None))
            keep += [bc, bf]
            a.coarseBlocks, a.fineBlocks = bc.data_ptr(), bf.data_ptr()
        fn = _lib.lib().vfb_scale_coarse_to_fine if coarse_to_fine else _lib.lib().vfb_scale_fine_to_coarse
        _lib.check(fn(_lib.FP64, a, None))
        torch.cuda.synchronize()
        outs.append([t.cpu().numpy() for t in (dC, dF)])
    for x, y in zip(*outs):
        assert np.array_equal(x, y)
