"""Wall-model (stress) BC cases shared by the oracle pins and the GPU tests.

A stress list is built from a BC list of a committed golden grid (its nodes
and q), with seeded values for what the builder does not fix: unit normals,
sampling nodes, sampling offsets, roughness lengths and the two filter
states.  The kernels only read the sampling node's velocity, so any node
index exercises them.
"""
from __future__ import annotations

import numpy as np

from oracle.pyoracle import STRESS_MONITORS, STRESS_STATE


def make_stress_list(g: dict, lst: str, real, seed: int, axis_normal: bool = False) -> dict:
    rng = np.random.default_rng(seed)
    k = g[f"{lst}.k"].astype(np.int32)
    n = len(k)
    N = len(g["geo"])
    fluid = g["fluid"].astype(np.int64)
    out = {"k": k, "q": g[f"{lst}.q"].astype(real)}
    out["kN"] = rng.choice(fluid, n).astype(np.int32)
    if axis_normal:
        nrm = np.zeros((3, n))
        nrm[2] = 1.0
    else:
        nrm = rng.normal(size=(3, n))
        nrm /= np.linalg.norm(nrm, axis=0)
    out["normalX"], out["normalY"], out["normalZ"] = (a.astype(real) for a in nrm)
    for name in STRESS_STATE:
        out[name] = rng.uniform(-0.04, 0.04, n).astype(real)
    out["samplingOffset"] = rng.integers(1, 5, n).astype(np.int32)
    out["z0"] = rng.uniform(0.01, 0.5, n).astype(real)
    for name in STRESS_MONITORS:
        out[name] = np.zeros(n, real)
    assert out["kN"].max() < N
    return out


def copy_list(lst: dict) -> dict:
    return {key: np.array(v, copy=True) for key, v in lst.items()}


def velocity_fields(N: int, real, seed: int):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-0.05, 0.05, N).astype(real) for _ in range(3)]


def turbulent_viscosity(N: int, real, seed: int):
    """Per-node eddy viscosities, a few negative ones to reach max(0, nu_t)."""
    return np.random.default_rng(seed).uniform(-0.01, 0.05, N).astype(real)


def stress_populations(N: int, real):
    """Seeded populations for the wall-model fixtures."""
    return np.random.default_rng(80).uniform(-0.02, 0.02, 27 * N).astype(real)
