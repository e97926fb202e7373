"""Helpers shared by the GPU parity tests: run the same update on the GPU
(through the C ABI) and on the oracle, and compare."""
from __future__ import annotations

import numpy as np

from oracle.pyoracle import Oracle
from virtualfluids_b200 import kernels as K
from virtualfluids_b200.workloads import taylor_green


def rel_max(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def tgv_state(n: int, seed: int = 1234):
    return taylor_green(n, seed=seed)


def oracle_run(w, precision: str, steps: int, kernel="K17", limiters=(0.01, 0.01, 0.01), forces=(0, 0, 0)):
    """Initialise both parities and run `steps` collisions on the oracle."""
    O = Oracle(precision)
    real = O.real
    g = w.grid
    N = len(g["geo"])
    d = np.zeros(27 * N, real)
    args = (g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"])
    for ev in (0, 1):
        O.init_eq(d, N, *args, w.rho.astype(real), w.vx.astype(real), w.vy.astype(real), w.vz.astype(real), ev)
    even = True
    for _ in range(steps):
        if kernel == "K17":
            O.collision_k17(d, N, g["neighborX"], g["neighborY"], g["neighborZ"], g["fluid"], w.omega,
                            forces=forces, limiters=limiters, is_even=even)
        else:
            O.collision_bgk(d, N, *args, w.omega, is_even=even)
        even = not even
    macro = O.macroscopic(d, N, *args, even)
    return d, macro, even


def gpu_run(w, dtype, steps: int, kernel="K17", limiters=(0.01, 0.01, 0.01), forces=(0, 0, 0), planned=False):
    import torch
    lat = K.DeviceLattice.from_arrays(w.grid)
    plan = K.CollisionPlan(dtype, lat) if planned else None
    cd = K.compute_dtype(dtype)
    dist = K.new_distributions(lat, dtype)
    fields = [torch.from_numpy(a).to("cuda", cd) for a in (w.rho, w.vx, w.vy, w.vz)]
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    even = True
    for _ in range(steps):
        K.collision(kernel, dist, lat, w.omega, even, limiters=limiters, forces=forces, plan=plan)
        even = not even
    macro = [m.cpu().numpy() for m in K.macroscopic(dist, lat, even)]
    torch.cuda.synchronize()
    if plan is not None:
        plan.check()
    return dist, lat, macro, even
