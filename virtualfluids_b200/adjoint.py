"""Gradients of a flow objective through the library's adjoint time step,
as a torch.autograd.Function.

The reference (pyfluids) has no adjoint.  Here a single-level Simulation is
the forward model: the controlled parameters are velocity values of the
velocity-BC list (an inlet profile) and the global body force; the objective
is a weighted sum of node velocities after `steps` time steps from a fixed
initial state.  forward() runs the steps with checkpoints
(vfb_sim_adjoint_forward), backward() runs the hand-written adjoint kernels
backwards through the checkpoint segments (vfb_sim_adjoint_backward).

    problem = FlowProblem(sim, entries, initial, steps=1000, checkpoint_interval=32,
                          objective_nodes=nodes, objective_weights=(wx, None, None))
    J = FlowObjective.apply(profile, force, problem)
    J.backward()          # profile.grad, force.grad
"""
from __future__ import annotations

import numpy as np
import torch

from .simulation import Simulation


class FlowProblem:
    """The forward model of FlowObjective.

    sim                 a single-level Simulation (FP32 or FP64 storage)
    entries             indices into the level's velocity list whose velocity
                        component `component` is controlled (e.g. the inlet)
    initial             (drho, vx, vy, vz) host arrays: the state every
                        evaluation starts from (independent of the parameters)
    objective_nodes     node indices of the objective
    objective_weights   (wx, wy, wz), each an array over the nodes or None
    """

    def __init__(self, sim: Simulation, entries, initial, steps: int, checkpoint_interval: int, objective_nodes,
                 objective_weights, component: int = 0):
        self.sim = sim
        self.entries = np.asarray(entries, dtype=np.int64)
        self.initial = [np.asarray(a, dtype=np.float64) for a in initial]
        self.steps = int(steps)
        self.interval = int(checkpoint_interval)
        self.nodes = np.asarray(objective_nodes, dtype=np.uint32)
        self.weights = objective_weights
        self.component = int(component)
        g = sim.levels[0]
        self.base = [g[f"velocity.{c}"].astype(np.float64).copy() for c in ("vx", "vy", "vz")]
        self.evaluations = 0

    def evaluate(self, values, force) -> float:
        """J for the controlled velocity values and the global force (the
        simulation's state is reset to the initial fields first)."""
        vel = [b.copy() for b in self.base]
        vel[self.component][self.entries] = np.asarray(values, dtype=np.float64)
        self.sim.set_velocity_bc(*vel)
        self.sim.set_forces(*[float(f) for f in force])
        self.sim.init_level(0, *self.initial)
        wx, wy, wz = self.weights
        self.evaluations += 1
        return self.sim.adjoint_forward(self.steps, self.interval, self.nodes, wx, wy, wz)

    def gradient(self, seed: float = 1.0):
        """(dL/d values, dL/d force) of the last evaluate(), dL/dJ = seed."""
        dv, df = self.sim.adjoint_backward(seed)
        return dv[self.component][self.entries], df


class FlowObjective(torch.autograd.Function):
    """J(values, force) of a FlowProblem, differentiable in both inputs."""

    @staticmethod
    def forward(ctx, values: torch.Tensor, force: torch.Tensor, problem: FlowProblem):
        v = values.detach().cpu().double().numpy().copy()
        f = force.detach().cpu().double().numpy().copy()
        J = problem.evaluate(v, f)
        ctx.problem = problem
        ctx.inputs = (v, f, problem.evaluations)
        ctx.meta = (values.dtype, values.device, force.dtype, force.device)
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_output):
        vdt, vdev, fdt, fdev = ctx.meta
        v, f, evaluation = ctx.inputs
        if ctx.problem.evaluations != evaluation:
            # the problem ran another evaluation since: redo this one's forward pass
            ctx.problem.evaluate(v, f)
        dv, df = ctx.problem.gradient(float(grad_output))
        return (torch.from_numpy(np.ascontiguousarray(dv)).to(vdev, vdt), torch.from_numpy(df).to(fdev, fdt), None)
