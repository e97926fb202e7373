"""The PyTorch transcription of the time step (tests/adjoint_torch.py, the FP64
autograd reference of the adjoint) pinned to the oracle on the host: the K17
node operator on random states, and whole steps of the small adjoint channel
(velocity inlet with a per-node profile, walls, a solid cube, pressure outlet,
body force) against the oracle running UpdateGrid27's order."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle.pyoracle import Oracle  # noqa: E402
from tests import adjoint_torch as AT  # noqa: E402
from virtualfluids_b200.workloads import adjoint_channel_small, inlet_entries, inlet_profile, initial_fields  # noqa: E402,E501
from tests.test_adjoint_host import state  # noqa: E402


@pytest.mark.parametrize("seed", range(4))
def test_torch_k17_equals_oracle(seed):
    rng = np.random.default_rng(seed)
    O = Oracle("f64")
    fs = [state(rng) for _ in range(8)]
    force = (1e-6, -2e-6, 5e-7)
    lim = (0.01, 0.02, 0.005)
    got = AT.k17([torch.tensor([f[d] for f in fs], dtype=torch.float64) for d in range(27)], 1.786, lim, *force)
    for i, f in enumerate(fs):
        want, _ = O.k17_node(f, 1.786, limiter=lim, force=force)
        g = np.array([float(got[d][i]) for d in range(27)])
        assert np.abs(g - want).max() <= 1e-13 * np.abs(want).max()


def test_torch_step_equals_oracle_schedule():
    g = adjoint_channel_small().arrays()[0]
    vx = g["velocity.vx"].copy()
    vx[inlet_entries(g)] = inlet_profile(g)
    g["velocity.vx"] = vx
    nu, force, steps = 0.02, (1e-6, 2e-7, -3e-7), 6
    om = 1.0 / (3.0 * nu + 0.5)
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    init = initial_fields(g)
    O = Oracle("f64")
    d = np.zeros(27 * N)
    for ev in (0, 1):
        O.init_eq(d, N, g["geo"], *nb, *init, ev)
    D = torch.from_numpy(d.copy())
    vel = [g[f"velocity.{c}"] for c in ("vx", "vy", "vz")]
    even = True
    for _ in range(steps):
        O.collision_k17(d, N, *nb, g["fluid"], om, forces=force, force_factor=1.0, limiters=(0.01, 0.01, 0.01),
                        is_even=even)
        O.bc_post(2, d, N, *nb, g["velocity.k"], g["velocity.q"], om, *vel, is_even=even)
        O.bc_post(0, d, N, *nb, g["geometry.k"], g["geometry.q"], om, is_even=even)
        even = not even
        O.bc_pressure(d, N, *nb, g["pressure0.k"], g["pressure0.kN"], g["pressure0.rho"], int(g["pressure0.dir"][0]),
                      is_even=even)
    step = AT.Step(g, om)
    U = [torch.from_numpy(v) for v in vel]
    ev = True
    for _ in range(steps):
        D, ev = step.step(D, ev, U, [0.5 * f for f in force])
    assert ev == even
    assert np.abs(D.numpy() - d).max() <= 1e-13 * np.abs(d).max()
