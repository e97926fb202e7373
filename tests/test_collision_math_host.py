"""The library's collision arithmetic (csrc/collision_math.cuh, evaluated on
the host through vfb_debug_collide_node) against the oracle, node by node.

The library arranges the reference's operator for the GPU's issue rate
(multiply-add forms, shared sums), so agreement is to rounding: FP64 within
1e-13 relative to the largest population, FP32 within 2e-6.
"""
import ctypes

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from virtualfluids_b200 import _lib

D = ctypes.POINTER(ctypes.c_double)


def lib_node(op, precision, f, omega, lim, force):
    f = np.ascontiguousarray(f, dtype=np.float64).copy()
    lim = np.asarray(lim, dtype=np.float64)
    force = np.asarray(force, dtype=np.float64)
    out = np.zeros(4)
    rc = _lib.lib().vfb_debug_collide_node(op, precision, f.ctypes.data_as(D), omega, lim.ctypes.data_as(D),
                                           force.ctypes.data_as(D), out.ctypes.data_as(D))
    assert rc == 0, _lib.last_error()
    return f, out


@pytest.mark.parametrize("precision,tol", [("f64", 1e-13), ("f32", 2e-6)])
@pytest.mark.parametrize("limited", [True, False])
def test_k17_node_matches_oracle(precision, tol, limited):
    O = Oracle(precision)
    p = _lib.FP64 if precision == "f64" else _lib.FP32
    rng = np.random.default_rng(2024)
    for t in range(200):
        f = rng.uniform(-0.02, 0.02, 27)
        omega = rng.uniform(0.5, 1.995)
        lim = (0.01, 0.02, 0.005) if limited else (1e6, 1e6, 1e6)
        force = rng.uniform(-1e-4, 1e-4, 3)
        ref, mref = O.k17_node(f.astype(O.real), omega, lim, tuple(force))
        got, m = lib_node(0, p, f.astype(O.real).astype(np.float64), omega, lim, force)
        scale = max(np.abs(ref).max(), 1e-30)
        assert np.abs(got - ref).max() / scale < tol, t
        assert np.abs(m - mref).max() / max(np.abs(mref).max(), 1e-30) < tol, t


@pytest.mark.parametrize("precision,tol", [("f64", 1e-13), ("f32", 2e-6)])
def test_bgk_node_matches_oracle(precision, tol):
    O = Oracle(precision)
    p = _lib.FP64 if precision == "f64" else _lib.FP32
    rng = np.random.default_rng(7)
    for t in range(100):
        f = rng.uniform(-0.02, 0.02, 27).astype(O.real)
        omega = rng.uniform(0.5, 1.99)
        ref = O.bgk_node(f, omega)
        got, _ = lib_node(1, p, f.astype(np.float64), omega, (0.01,) * 3, (0, 0, 0))
        assert np.abs(got - ref).max() / np.abs(ref).max() < tol, t


def test_rest_state_is_a_fixed_point():
    got, m = lib_node(0, _lib.FP64, np.zeros(27), 1.9, (0.01,) * 3, (0, 0, 0))
    assert np.abs(got).max() < 1e-17
    assert np.abs(m).max() < 1e-17


def lib_noneq_node(precision, drho_u, grad, omega):
    dv = np.ascontiguousarray(drho_u, dtype=np.float64)
    g = np.ascontiguousarray(grad, dtype=np.float64).reshape(9)
    f = np.zeros(27)
    rc = _lib.lib().vfb_debug_init_nonequilibrium_node(precision, dv.ctypes.data_as(D), g.ctypes.data_as(D), omega,
                                                       f.ctypes.data_as(D))
    assert rc == 0, _lib.last_error()
    return f


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_noneq_init_node_matches_oracle_bit_for_bit(precision):
    """The non-equilibrium init's node arithmetic (the kernel's own code, run
    on the host) equals the oracle exactly: it performs the reference's
    operations in the reference's order, double products included in FP32.
    Mass and momentum of the non-equilibrium part vanish."""
    O = Oracle(precision)
    p = _lib.FP64 if precision == "f64" else _lib.FP32
    rng = np.random.default_rng(31)
    c = np.array([[0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1],
                  [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1],
                  [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1]])
    for t in range(200):
        drho_u = rng.uniform(-0.03, 0.03, 4).astype(O.real)
        grad = rng.uniform(-1e-2, 1e-2, 9).astype(O.real)
        omega = O.real(rng.uniform(0.3, 1.99))
        ref = O.noneq_node(*drho_u, grad.reshape(3, 3), omega)
        got = lib_noneq_node(p, drho_u, grad, float(omega))
        assert np.array_equal(got.astype(O.real), ref), t
        neq = ref.astype(np.float64) - O.noneq_node(*drho_u, np.zeros((3, 3)), omega).astype(np.float64)
        scale = np.abs(neq).max()
        assert abs(neq.sum()) <= 1e-5 * scale and np.abs(c @ neq).max() <= 1e-5 * scale, t


def test_noneq_init_node_rejects_bad_arguments():
    f = np.zeros(27)
    assert _lib.lib().vfb_debug_init_nonequilibrium_node(_lib.FP16, f.ctypes.data_as(D), f.ctypes.data_as(D), 1.0,
                                                         f.ctypes.data_as(D)) != 0
    assert _lib.lib().vfb_debug_init_nonequilibrium_node(_lib.FP64, None, f.ctypes.data_as(D), 1.0,
                                                         f.ctypes.data_as(D)) != 0
