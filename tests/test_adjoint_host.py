"""The generated reverse sweep of the K17 collision (adjoint_ops.gen.cuh, the
code the collision adjoint kernel runs) on the host, against central finite
differences of the library's own forward node arithmetic
(vfb_debug_collide_node): lam . dPhi/da_d and lam . dPhi/df for random
pre-collision states, FP64 to 1e-6 relative (finite-difference truncation),
FP32 against the FP64 sweep to 1e-4."""
import ctypes

import numpy as np
import pytest

from virtualfluids_b200 import _lib

D = ctypes.POINTER(ctypes.c_double)
W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1])


def state(rng):
    drho = rng.uniform(-0.01, 0.01)
    u = rng.uniform(-0.05, 0.05, 3)
    cu = CX * u[0] + CY * u[1] + CZ * u[2]
    feq = W * (drho + (1 + drho) * (3 * cu + 4.5 * cu ** 2 - 1.5 * (u @ u)))
    return feq + rng.uniform(-1e-3, 1e-3, 27) * W


def forward(a, omega, lim, force, precision=_lib.FP64):
    f = np.ascontiguousarray(a, dtype=np.float64).copy()
    out = np.zeros(4)
    lim = np.asarray(lim, np.float64)
    force = np.asarray(force, np.float64)
    _lib.check(_lib.lib().vfb_debug_collide_node(0, precision, f.ctypes.data_as(D), omega, lim.ctypes.data_as(D),
                                                 force.ctypes.data_as(D), out.ctypes.data_as(D)))
    return f


def adjoint(a, lam, omega, lim, force, precision=_lib.FP64):
    a = np.ascontiguousarray(a, dtype=np.float64)
    l = np.ascontiguousarray(lam, dtype=np.float64).copy()
    g = np.zeros(3)
    lim = np.asarray(lim, np.float64)
    force = np.asarray(force, np.float64)
    _lib.check(_lib.lib().vfb_debug_k17_adjoint_node(precision, a.ctypes.data_as(D), l.ctypes.data_as(D), omega,
                                                     lim.ctypes.data_as(D), force.ctypes.data_as(D),
                                                     g.ctypes.data_as(D)))
    return l, g


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("omega,lim", [(1.786, (0.01, 0.01, 0.01)), (1.98, (1e6, 1e6, 1e6)), (1.2, (0.01, 0.02, 0.005))])
def test_k17_adjoint_matches_finite_differences(seed, omega, lim):
    rng = np.random.default_rng(seed)
    a = state(rng)
    lam = rng.standard_normal(27)
    force = rng.uniform(-1e-5, 1e-5, 3)
    got, gforce = adjoint(a, lam, omega, lim, force)
    eps = 1e-7
    fd = np.zeros(27)
    for d in range(27):
        ap, am = a.copy(), a.copy()
        ap[d] += eps
        am[d] -= eps
        fd[d] = lam @ (forward(ap, omega, lim, force) - forward(am, omega, lim, force)) / (2 * eps)
    assert np.abs(got - fd).max() <= 1e-6 * np.abs(fd).max()
    fdf = np.zeros(3)
    for c in range(3):
        fp, fm = force.copy(), force.copy()
        fp[c] += eps
        fm[c] -= eps
        fdf[c] = lam @ (forward(a, omega, lim, fp) - forward(a, omega, lim, fm)) / (2 * eps)
    assert np.abs(gforce - fdf).max() <= 1e-6 * np.abs(fdf).max()


def test_k17_adjoint_fp32_matches_fp64():
    rng = np.random.default_rng(42)
    for _ in range(5):
        a = state(rng)
        lam = rng.standard_normal(27)
        force = rng.uniform(-1e-5, 1e-5, 3)
        g64, f64 = adjoint(a, lam, 1.786, (0.01, 0.01, 0.01), force)
        g32, f32 = adjoint(a, lam, 1.786, (0.01, 0.01, 0.01), force, _lib.FP32)
        assert np.abs(g32 - g64).max() <= 1e-4 * np.abs(g64).max()
        assert np.abs(f32 - f64).max() <= 1e-4 * np.abs(f64).max()


def test_k17_adjoint_is_linear_in_lam():
    rng = np.random.default_rng(3)
    a = state(rng)
    l1, l2 = rng.standard_normal(27), rng.standard_normal(27)
    g1, _ = adjoint(a, l1, 1.786, (0.01,) * 3, (0, 0, 0))
    g2, _ = adjoint(a, l2, 1.786, (0.01,) * 3, (0, 0, 0))
    g12, _ = adjoint(a, 2.0 * l1 - 3.0 * l2, 1.786, (0.01,) * 3, (0, 0, 0))
    assert np.allclose(g12, 2.0 * g1 - 3.0 * g2, rtol=0, atol=1e-13 * np.abs(g12).max())


def test_generated_header_is_current(tmp_path):
    """The committed reverse sweep (csrc/adjoint_ops.gen.cuh) is what the
    generator makes from the current operator source."""
    from virtualfluids_b200 import build
    out = build.generate_adjoint(tmp_path / "adjoint_ops.gen.cuh")
    assert out.read_bytes() == build.GEN_OUT.read_bytes()
