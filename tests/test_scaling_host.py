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


def _refined_case(precision):
    """Coarse-to-fine cells of the reference-built two-level grid, with
    perturbed equilibrium populations on both levels."""
    from pathlib import Path
    from tests.scaling_cases import populations
    z = np.load(Path(__file__).resolve().parent / "golden" / "grid_refined_channel.npz")
    lv = [{k.split(":", 1)[1]: z[k] for k in z.files if k.startswith(f"L{l}:")} for l in (0, 1)]
    real = REAL[precision]
    c = dict(gc=lv[0], gf=lv[1], distC=populations(lv[0], 5, real), distF=populations(lv[1], 6, real),
             coarse_cf=lv[0]["cf.coarse"], fine_cf=lv[0]["cf.fine"], coarse_fc=lv[0]["fc.coarse"],
             fine_fc=lv[0]["fc.fine"], off=np.stack([lv[0]["cf.offX"], lv[0]["cf.offY"], lv[0]["cf.offZ"]]).astype(real),
             omegaC=1.7, omegaF=1.8)
    return c


def test_write_mask_reproduces_the_sequential_result():
    """Cells of the reference-built grid write some memory cells more than once
    (periodic seams, edge stoppers): with the mask every memory cell keeps its
    last writer, so masked writes equal the cells applied one by one."""
    c = _refined_case("f64")
    arrays = host_arrays(c)
    nx, ny, nz = (c["gf"][f"neighbor{a}"] for a in "XYZ")
    mask = np.zeros(27 * len(c["fine_cf"]), np.uint8)
    _lib.check(_lib.lib().vfb_scaling_write_mask(c["fine_cf"].ctypes.data, len(c["fine_cf"]), nx.ctypes.data,
                                                 ny.ctypes.data, nz.ctypes.data, len(nx), mask.ctypes.data))
    assert (mask != 0xFF).sum() > 0  # the grid really has repeated writes
    outs = []
    for use_mask in (False, True):
        dC, dF = c["distC"].copy(), c["distF"].copy()
        a = scaling_args(c, True, True, dC.ctypes.data, dF.ctypes.data, arrays)
        if use_mask:
            a.fineWriteMask = mask.ctypes.data
        _lib.check(_lib.lib().vfb_debug_scale_host(1, _lib.FP64, a))
        outs.append(dF)
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
def test_sequential_result_matches_reference_on_refined_grid():
    c = _refined_case("f64")
    arrays = host_arrays(c)
    dC, dF = c["distC"].copy(), c["distF"].copy()
    a = scaling_args(c, True, True, dC.ctypes.data, dF.ctypes.data, arrays)
    _lib.check(_lib.lib().vfb_debug_scale_host(1, _lib.FP64, a))
    rC, rF = c["distC"].copy(), c["distF"].copy()
    Reference("f64").scale(True, rC, rF, c["gc"], c["gf"], True, c["coarse_cf"], c["fine_cf"], c["omegaC"],
                           c["omegaF"], c["offX"], c["offY"], c["offZ"])
    assert rel_max(dF, rF) < 1e-13
