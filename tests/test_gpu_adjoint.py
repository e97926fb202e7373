"""The adjoint of the time step (vfb_sim_adjoint_*, the hand-written adjoint
kernels) behind virtualfluids_b200.adjoint.FlowObjective.

- Small channel (16 x 8 x 8 fluid nodes, a 2^3 cube, velocity inlet with a
  parabolic profile, walls, pressure outlet, body force), FP64, 24 steps with
  a checkpoint every 5: J equals the PyTorch transcription of the step
  (tests/adjoint_torch.py, pinned to the oracle) to 1e-12, and the gradients
  of J with respect to every velocity-list value and the force equal FP64
  autograd through that transcription to 1e-9 relative.
- The FP32 adjoint agrees with the FP64 adjoint on the small channel to 1e-3.
- The benchmark channel (128 x 64 x 64, 12^3 cube, T = 1000, checkpoints every
  32, FP64): dJ/d(inlet profile) on 8 seeded inlet nodes and dJ/dg for all
  three force components agree with central finite differences
  (eps = 1e-4 * max(|p|, 1e-6)) to 1e-3 relative.
"""
import numpy as np
import pytest

from virtualfluids_b200.workloads import (adjoint_channel, adjoint_channel_small, inlet_entries, inlet_profile,
                                         initial_fields, objective_box)
from virtualfluids_b200 import _lib
from virtualfluids_b200.simulation import BoundaryConditionFactory, NoSlipBC, Parameter, PressureBC, Simulation

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

NU = 0.02
G = (1e-6, 0.0, 0.0)


def make_sim(builder, storage="fp64", force=G):
    p = Parameter()
    p.set_storage(storage)
    p.set_viscosity_LB(NU)
    p.set_forcing(*force)
    bc = BoundaryConditionFactory()
    bc.set_geometry_boundary_condition(NoSlipBC.NoSlipInterpolatedCompressible)
    bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
    return Simulation(p, builder, bc)


def problem(sim, steps, interval, box):
    from virtualfluids_b200.adjoint import FlowProblem
    g = sim.levels[0]
    nodes, w = objective_box(g, *box)
    return FlowProblem(sim, inlet_entries(g), initial_fields(g), steps, interval, nodes, (w, None, None))


SMALL_BOX = (10, 14, 2, 6, 2, 6)


def torch_reference(g, steps, profile, force):
    """J and its gradients by FP64 autograd through the transcription."""
    from oracle.pyoracle import Oracle
    from tests import adjoint_torch as AT
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    d = np.zeros(27 * N)
    for ev in (0, 1):
        Oracle("f64").init_eq(d, N, g["geo"], *nb, *initial_fields(g), ev)
    om = 1.0 / (3.0 * NU + 0.5)
    entries = inlet_entries(g)
    U = [torch.tensor(g[f"velocity.{c}"], dtype=torch.float64, requires_grad=True) for c in ("vx", "vy", "vz")]
    p = torch.tensor(profile, dtype=torch.float64, requires_grad=True)
    gforce = torch.tensor(force, dtype=torch.float64, requires_grad=True)
    ux = U[0].index_put((torch.from_numpy(entries),), p)
    step = AT.Step(g, om)
    D = torch.from_numpy(d)
    even = True
    for _ in range(steps):
        D, even = step.step(D, even, [ux, U[1], U[2]], [0.5 * gforce[c] for c in range(3)])
    nodes, w = objective_box(g, *SMALL_BOX)
    J = step.objective(D, even, nodes, w)
    J.backward()
    # the gradient of every velocity-list value: x component with the inlet entries from p
    gx = U[0].grad.clone()
    gx[torch.from_numpy(entries)] = p.grad
    return float(J.detach()), np.stack([gx.numpy(), U[1].grad.numpy(), U[2].grad.numpy()]), gforce.grad.numpy()


def test_small_channel_fp64_matches_torch_autograd(cuda):
    sim = make_sim(adjoint_channel_small())
    g = sim.levels[0]
    profile = inlet_profile(g)
    pb = problem(sim, 24, 5, SMALL_BOX)
    J = pb.evaluate(profile, G)
    dv, df = sim.adjoint_backward(1.0)
    g_ref = dict(g)
    vx = g["velocity.vx"].copy()
    vx[inlet_entries(g)] = profile
    g_ref["velocity.vx"] = vx
    J_ref, dv_ref, df_ref = torch_reference(g_ref, 24, profile, G)
    assert abs(J - J_ref) <= 1e-12 * abs(J_ref)
    assert np.abs(dv_ref).max() > 0 and np.abs(df_ref).max() > 0
    assert np.abs(dv - dv_ref).max() <= 1e-9 * np.abs(dv_ref).max()
    assert np.abs(df - df_ref).max() <= 1e-9 * np.abs(df_ref).max()
    sim.close()


def test_flow_objective_autograd_function(cuda):
    """FlowObjective.apply: J.backward() fills the gradients of the inlet
    profile and the force; the gradient equals the direct adjoint call, also
    after another evaluation ran in between."""
    from virtualfluids_b200.adjoint import FlowObjective
    sim = make_sim(adjoint_channel_small())
    g = sim.levels[0]
    pb = problem(sim, 12, 4, SMALL_BOX)
    prof = torch.tensor(inlet_profile(g), dtype=torch.float64, requires_grad=True)
    force = torch.tensor(G, dtype=torch.float64, requires_grad=True)
    J = FlowObjective.apply(prof, force, pb)
    J2 = FlowObjective.apply(prof * 1.01, force, pb)  # a second evaluation before the backward pass
    (2.0 * J).backward()
    pb.evaluate(inlet_profile(g), G)
    dv, df = pb.gradient(2.0)
    # equal to 1e-12 of each gradient's largest entry: the BC scatters add with
    # atomics, whose order may change the last bits of entries that cancel
    assert np.allclose(prof.grad.numpy(), dv, rtol=0, atol=1e-12 * np.abs(dv).max())
    assert np.allclose(force.grad.numpy(), df, rtol=0, atol=1e-12 * np.abs(df).max())
    assert float(J2) != float(J)
    sim.close()


def test_schedules_give_the_same_gradient(cuda, monkeypatch):
    """The checkpointed schedule (each segment recomputed with tapes), the
    taped one (interval >= steps: the forward pass records the tapes) and one
    launch per BC list instead of the lists together give the same J (bit for
    bit: the same forward arithmetic) and the same gradients (to the order of
    the scatters' atomic additions)."""
    out = []
    for separate, interval in ((True, 5), (False, 5), (False, 24), (False, 100), (True, 24)):
        if separate:
            monkeypatch.setenv("VFB_ADJOINT_SEPARATE_LISTS", "1")
        else:
            monkeypatch.delenv("VFB_ADJOINT_SEPARATE_LISTS", raising=False)
        sim = make_sim(adjoint_channel_small())
        pb = problem(sim, 24, interval, SMALL_BOX)
        J = pb.evaluate(inlet_profile(sim.levels[0]), G)
        dv, df = pb.gradient(1.0)
        sched = sim.adjoint_schedule()
        assert sched == {"lists_together": not separate, "taped_forward": interval >= 24}, sched
        out.append((J, dv, df))
        sim.close()
    J0, dv0, df0 = out[0]
    for J, dv, df in out[1:]:
        assert J == J0
        assert np.abs(dv - dv0).max() <= 1e-12 * np.abs(dv0).max()
        assert np.abs(df - df0).max() <= 1e-12 * np.abs(df0).max()


def test_small_channel_fp32_adjoint_close_to_fp64(cuda):
    out = []
    for storage in ("fp64", "fp32"):
        sim = make_sim(adjoint_channel_small(), storage)
        pb = problem(sim, 24, 5, SMALL_BOX)
        pb.evaluate(inlet_profile(sim.levels[0]), G)
        out.append(pb.gradient(1.0))
        sim.close()
    (v64, f64), (v32, f32) = out
    assert np.abs(v32 - v64).max() <= 1e-3 * np.abs(v64).max()
    assert np.abs(f32 - f64).max() <= 1e-3 * np.abs(f64).max()


def test_adjoint_errors(cuda):
    p = Parameter()
    p.set_viscosity_LB(NU)
    p.configure_main_kernel("BGKCompSP27")
    sim = Simulation(p, adjoint_channel_small(), BoundaryConditionFactory())
    with pytest.raises(_lib.VfbError) as e:
        sim.adjoint_forward(4, 2, [1], [1.0])
    assert e.value.code == _lib.VFB_ERR_UNSUPPORTED
    sim.close()
    sim = make_sim(adjoint_channel_small())
    with pytest.raises(_lib.VfbError) as e:
        sim.adjoint_backward()
    assert e.value.code == _lib.VFB_ERR_CONFIGURATION
    with pytest.raises(_lib.VfbError):
        sim.adjoint_forward(4, 0, [1], [1.0])
    with pytest.raises(_lib.VfbError) as e:
        sim.adjoint_forward(4, 2, [len(sim.levels[0]["geo"])], [1.0])
    assert e.value.code == _lib.VFB_ERR_OUT_OF_RANGE
    sim.close()


@pytest.fixture(scope="module")
def full_problem():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sim = make_sim(adjoint_channel())
    g = sim.levels[0]
    pb = problem(sim, 1000, 32, (80, 96, 24, 40, 24, 40))
    yield sim, g, pb
    sim.close()


def test_full_channel_gradients_match_finite_differences(cuda, full_problem):
    sim, g, pb = full_problem
    assert len(pb.entries) == 64 * 64 and len(pb.nodes) == 16 ** 3
    profile = inlet_profile(g)
    J0 = pb.evaluate(profile, G)
    dv, df = pb.gradient(1.0)
    assert J0 > 0
    rng = np.random.default_rng(77)
    # eight seeded inlet nodes away from the walls (zero velocity there)
    interior = np.nonzero(profile > 0.25 * profile.max())[0]
    picks = rng.choice(interior, 8, replace=False)
    for j in picks:
        eps = 1e-4 * max(abs(profile[j]), 1e-6)
        plus, minus = profile.copy(), profile.copy()
        plus[j] += eps
        minus[j] -= eps
        fd = (pb.evaluate(plus, G) - pb.evaluate(minus, G)) / (2 * eps)
        assert abs(dv[j] - fd) <= 1e-3 * abs(fd), (j, dv[j], fd)
    for c in range(3):
        eps = 1e-4 * max(abs(G[c]), 1e-6)
        gp, gm = list(G), list(G)
        gp[c] += eps
        gm[c] -= eps
        fd = (pb.evaluate(profile, gp) - pb.evaluate(profile, gm)) / (2 * eps)
        assert abs(df[c] - fd) <= 1e-3 * max(abs(fd), 1e-3 * abs(df[0])), (c, df[c], fd)
