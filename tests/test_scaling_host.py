"""The interface interpolation arithmetic of the library (run on the host
through vfb_debug_scale_host) against the reference's own
scaleCoarseToFineCompressible / scaleFineToCoarseCompressible kernels
compiled on the host (oracle/_ref)."""
import ctypes
from pathlib import Path

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


def _golden_levels(name):
    with np.load(Path(__file__).resolve().parent / "golden" / f"grid_{name}.npz") as z:
        levels = {}
        for key in z.files:
            lvl, arr = key.split(":", 1)
            levels.setdefault(int(lvl[1:]), {})[arr] = z[key]
    return [levels[i] for i in sorted(levels)]


def _independent(g, gf, cf_mask=None, fc_fine=None):
    u = lambda a: np.ascontiguousarray(a, dtype=np.uint32)
    fcc, fcf = u(g["fc.coarse"]), u(g["fc.fine"] if fc_fine is None else fc_fine)
    cfc, cff = u(g["cf.coarse"]), u(g["cf.fine"])
    nc = [u(g[f"neighbor{a}"]) for a in "XYZ"]
    nf = [u(gf[f"neighbor{a}"]) for a in "XYZ"]
    mask = None
    if cf_mask:
        mask = np.zeros(27 * len(cff), np.uint8)
        _lib.check(_lib.lib().vfb_scaling_write_mask(cff.ctypes.data, len(cff), nf[0].ctypes.data, nf[1].ctypes.data,
                                                     nf[2].ctypes.data, len(nf[0]), mask.ctypes.data))
    out = ctypes.c_int(-1)
    _lib.check(_lib.lib().vfb_scaling_independent(
        fcc.ctypes.data, fcf.ctypes.data, len(fcc), cfc.ctypes.data, cff.ctypes.data, len(cfc),
        None if mask is None else mask.ctypes.data, *[a.ctypes.data for a in nc], len(nc[0]),
        *[a.ctypes.data for a in nf], len(nf[0]), ctypes.byref(out)))
    return out.value


@pytest.mark.parametrize("name", ["cube_channel", "two_level_box", "refined_channel"])
def test_interface_lists_independence(name):
    """vfb_scaling_independent: on the refinement grids the builder makes, the
    fine-to-coarse cells read no fine cell the coarse-to-fine cells write and
    the coarse-to-fine cells read no coarse cell the fine-to-coarse cells
    write, so one launch may serve both lists (vfb_scale_interface); with the
    fine-to-coarse cells moved onto the coarse-to-fine cells' fine nodes the
    check reports the dependence (grids with both lists)."""
    lv = _golden_levels(name)
    g, gf = lv[0], lv[1]
    assert _independent(g, gf, cf_mask=True) == 1
    if len(g["fc.fine"]):
        assert _independent(g, gf, cf_mask=True, fc_fine=np.asarray(g["cf.fine"])[: len(g["fc.fine"])]) == 0
