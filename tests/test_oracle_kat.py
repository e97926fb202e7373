"""Known-answer tests of the oracle's primitives, taken from the reference's
own unit tests:
  tests/unit-tests/lbm/ChimeraTests.cpp
  tests/unit-tests/lbm/MacroscopicQuantitiesTests.cpp
  tests/unit-tests/gpu/core/Utilities/KernelUtilitiesTests.cpp:44-120
"""
import ctypes

import numpy as np
import pytest

from oracle.pyoracle import Oracle

D = dict(d000=0, dP00=1, dM00=2, d0P0=3, d0M0=4, d00P=5, d00M=6, dPP0=7, dMM0=8, dPM0=9, dMP0=10, dP0P=11,
         dM0M=12, dP0M=13, dM0P=14, d0PP=15, d0MM=16, d0PM=17, d0MP=18, dPPP=19, dMPP=20, dPMP=21, dMMP=22,
         dPPM=23, dMPM=24, dPMM=25, dMMM=26)


@pytest.fixture(params=["f64", "f32"])
def oracle(request):
    O = Oracle(request.param)
    R = O.R
    O.fn("vfo_chimera").argtypes = [ctypes.c_int, ctypes.c_void_p, R, R, R, R]
    O.fn("vfo_macros").argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    O.fn("vfo_slot").argtypes = [ctypes.c_int, ctypes.c_int]
    return O


def chimera(O, which, abc, vv=1.0, v2=1.0, kinv=1.0, k=1.0):
    a = np.asarray(abc, dtype=O.real).copy()
    O.fn("vfo_chimera")(which, a.ctypes.data, vv, v2, kinv, k)
    return a


def test_forward_inverse_chimera_with_k(oracle):
    assert chimera(oracle, 0, [1, 1, 1]).tolist() == [3.0, -4.0, 6.0]


def test_backward_inverse_chimera_with_k(oracle):
    assert chimera(oracle, 1, [3, -4, 6]).tolist() == [1.0, 1.0, 1.0]


def test_forward_chimera(oracle):
    assert chimera(oracle, 2, [1, 1, 1]).tolist() == [3.0, -3.0, 5.0]


def test_backward_chimera(oracle):
    assert chimera(oracle, 3, [3, -3, 5]).tolist() == [1.0, 1.0, 1.0]


def macros(O, f):
    f = np.asarray(f, dtype=O.real)
    out = np.zeros(8, O.real)
    O.fn("vfo_macros")(f.ctypes.data, out.ctypes.data)
    return out


def test_density_of_ones_is_27(oracle):
    m = macros(oracle, np.ones(27))
    assert m[0] == 27.0
    assert m[1] == 0.0 and m[2] == 0.0 and m[3] == 0.0


@pytest.mark.parametrize("d,axis", [("dP00", 1), ("d0P0", 2), ("d00P", 3)])
def test_unit_velocity_when_one_population_is_two(oracle, d, axis):
    f = np.ones(27)
    f[D[d]] = 2.0
    m = macros(oracle, f)
    assert m[axis] == 1.0
    for other in {1, 2, 3} - {axis}:
        assert m[other] == 0.0


def test_compressible_values(oracle):
    f = np.ones(27)
    f[D["dP00"]] = 2.0
    m = macros(oracle, f)
    assert m[4] == 28.0
    assert m[5] == pytest.approx(1.0 / 29.0, rel=1e-6)
    assert m[6] == 0.0 and m[7] == 0.0


def test_even_view_is_identity(oracle):
    for d in range(27):
        assert oracle.fn("vfo_slot")(d, 1) == d


ODD_VIEW = {"dM00": "dP00", "dP00": "dM00", "d0M0": "d0P0", "d0P0": "d0M0", "d00M": "d00P", "d00P": "d00M",
            "dMM0": "dPP0", "dPP0": "dMM0", "dMP0": "dPM0", "dPM0": "dMP0", "dM0M": "dP0P", "dP0P": "dM0M",
            "dM0P": "dP0M", "dP0M": "dM0P", "d0MM": "d0PP", "d0PP": "d0MM", "d0MP": "d0PM", "d0PM": "d0MP",
            "d000": "d000", "dMMM": "dPPP", "dPPM": "dMMP", "dMPM": "dPMP", "dPMM": "dMPP", "dMMP": "dPPM",
            "dPPP": "dMMM", "dMPP": "dPMM", "dPMP": "dMPM"}


def test_odd_view_swaps_with_inverse(oracle):
    for d, src in ODD_VIEW.items():
        assert oracle.fn("vfo_slot")(D[d], 0) == D[src]
