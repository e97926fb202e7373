"""Long-run parity: the periodic Taylor-Green vortex of the benchmark
configurations (u0 = 0.05, Re = 1600, seeded noise) at 32^3 for 500 steps of
the planned default kernels against the oracle: FP64 fields within 1e-12
relative; FP32 storage and arithmetic within 1e-4 L2 of the FP64 oracle (the
stated FP32 bound for 500 steps: single-precision rounding accumulates to a few
1e-5 by then, 7.7e-5 after 2000 steps at 512^3)."""
import numpy as np
import pytest

from tests.gpu_helpers import gpu_run, oracle_run, rel_l2, rel_max, tgv_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("kernel", ["K17", "BGK"])
def test_tgv32_500_steps_fp64(cuda, kernel):
    w = tgv_state(32)
    _, ref, _ = oracle_run(w, "f64", 500, kernel)
    _, _, got, _ = gpu_run(w, torch.float64, 500, kernel, planned=True)
    fl = w.grid["fluid"]
    for a, b in zip(got, ref):
        assert rel_max(a[fl], b[fl]) < 1e-12


def test_tgv32_500_steps_fp32(cuda):
    w = tgv_state(32)
    _, ref, _ = oracle_run(w, "f64", 500)
    _, _, got, _ = gpu_run(w, torch.float32, 500, planned=True)
    fl = w.grid["fluid"]
    for a, b in zip(got, ref):
        assert rel_l2(a[fl], b[fl]) < 1e-4
