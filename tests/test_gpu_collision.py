"""GPU parity of the collision kernels against the oracle (through the C ABI).

Tolerances:
  FP64 storage    rho and u within 1e-12 relative (max norm, relative to the
                  field's maximum) of the FP64 oracle after N steps;
  FP32 storage    u within 1e-5 relative L2 of the FP32 oracle after N steps
                  (FMA contraction on the GPU is the only difference);
  FP16 / BF16     u within 5e-3 / 3e-2 relative L2 of the FP64 oracle after N
                  steps (storage rounding of f - w).
"""
import numpy as np
import pytest

from tests.gpu_helpers import gpu_run, oracle_run, rel_l2, rel_max, tgv_state

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("kernel", ["K17", "BGK"])
@pytest.mark.parametrize("limiters", [(0.01, 0.01, 0.01), (1e6, 1e6, 1e6)])
def test_fp64_matches_oracle(cuda, kernel, limiters):
    w = tgv_state(16)
    steps = 40
    _, ref, _ = oracle_run(w, "f64", steps, kernel, limiters)
    _, _, got, _ = gpu_run(w, torch.float64, steps, kernel, limiters)
    fluid = w.grid["fluid"]
    for a, b in zip(got, ref):
        assert rel_max(a[fluid], b[fluid]) < 1e-12


@pytest.mark.parametrize("kernel", ["K17", "BGK"])
def test_fp32_matches_oracle(cuda, kernel):
    w = tgv_state(16)
    steps = 40
    _, ref, _ = oracle_run(w, "f32", steps, kernel)
    _, _, got, _ = gpu_run(w, torch.float32, steps, kernel)
    fluid = w.grid["fluid"]
    u_ref = np.concatenate([ref[i][fluid] for i in (1, 2, 3)])
    u_got = np.concatenate([got[i][fluid] for i in (1, 2, 3)])
    assert rel_l2(u_got, u_ref) < 1e-5
    assert rel_max(got[0][fluid], ref[0][fluid]) < 1e-4


@pytest.mark.parametrize("dtype,tol", [("float16", 5e-3), ("bfloat16", 3e-2), ("int16", 1e-3)])
def test_low_precision_storage_against_fp64(cuda, dtype, tol):
    w = tgv_state(16)
    steps = 40
    _, ref, _ = oracle_run(w, "f64", steps)
    _, _, got, _ = gpu_run(w, getattr(torch, dtype), steps)
    fluid = w.grid["fluid"]
    u_ref = np.concatenate([ref[i][fluid] for i in (1, 2, 3)])
    u_got = np.concatenate([got[i][fluid] for i in (1, 2, 3)])
    err = rel_l2(u_got, u_ref)
    print(f"{dtype} L2(u) after {steps} steps: {err:.3e}")
    assert err < tol


def test_force_and_odd_size(cuda):
    w = tgv_state(10)
    _, ref, _ = oracle_run(w, "f64", 11, forces=(1e-5, -2e-5, 3e-6))
    _, _, got, _ = gpu_run(w, torch.float64, 11, forces=(1e-5, -2e-5, 3e-6))
    fluid = w.grid["fluid"]
    for a, b in zip(got, ref):
        assert rel_max(a[fluid], b[fluid]) < 1e-12


def test_distributions_match_after_one_step(cuda):
    w = tgv_state(8)
    d_ref, _, _ = oracle_run(w, "f64", 1)
    dist, _, _, _ = gpu_run(w, torch.float64, 1)
    d = dist.cpu().numpy()
    assert rel_max(d, d_ref) < 1e-13
