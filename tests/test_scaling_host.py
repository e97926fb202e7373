"""The interface interpolation arithmetic of the library (run on the host
through vfb_debug_scale_host) against the reference's own
scaleCoarseToFineCompressible / scaleFineToCoarseCompressible kernels
compiled on the host (oracle/_ref)."""
import numpy as np
import pytest

from oracle.pyoracle import Reference, ref_available
from tests.gpu_helpers import rel_l2, rel_max
from tests.scaling_cases import case, host_arrays, scaling_args
from virtualfluids_b200 import _lib

REAL = {"f64": np.float64, "f32": np.float32}


def run_both(precision, coarse_to_fine, is_even, seed=1):
    real = REAL[precision]
    c = case(seed, real=real)
    arrays = host_arrays(c)
    mine_c, mine_f = c["distC"].copy(), c["distF"].copy()
    a = scaling_args(c, coarse_to_fine, is_even, mine_c.ctypes.data, mine_f.ctypes.data, arrays)
    _lib.check(_lib.lib().vfb_debug_scale_host(int(coarse_to_fine), _lib.FP64 if precision == "f64" else _lib.FP32,
                                               a))
    R = Reference(precision)
    ref_c, ref_f = c["distC"].copy(), c["distF"].copy()
    tag = "cf" if coarse_to_fine else "fc"
    R.scale(coarse_to_fine, ref_c, ref_f, c["gc"], c["gf"], is_even, c[f"coarse_{tag}"], c[f"fine_{tag}"],
            c["omegaC"], c["omegaF"], c["offX"], c["offY"], c["offZ"])
    return c, (mine_c, mine_f), (ref_c, ref_f)


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("is_even", [True, False])
@pytest.mark.parametrize("coarse_to_fine", [True, False])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_interpolation_matches_reference(precision, coarse_to_fine, is_even):
    c, mine, ref = run_both(precision, coarse_to_fine, is_even)
    changed = mine[1] if coarse_to_fine else mine[0]
    original = c["distF"] if coarse_to_fine else c["distC"]
    assert np.count_nonzero(changed != original) > 0
    for m, r in zip(mine, ref):
        if precision == "f64":
            assert rel_max(m, r) < 1e-13
        else:
            assert rel_l2(m, r) < 1e-6


def test_scaling_rejects_bad_arguments():
    a = _lib.ScalingArgs()
    a.numberOfCells = 3
    assert _lib.lib().vfb_debug_scale_host(1, _lib.FP64, a) == _lib.VFB_ERR_INVALID_ARGUMENT
    assert _lib.lib().vfb_debug_scale_host(1, _lib.FP16, a) == _lib.VFB_ERR_INVALID_ARGUMENT
