"""Synthetic two-level inputs for the interface interpolation tests: two
periodic lattices with perturbed equilibrium populations and interface cells
chosen so that no two cells write the same node."""
from __future__ import annotations

import ctypes

import numpy as np

from oracle.pyoracle import Oracle
from virtualfluids_b200 import _lib
from virtualfluids_b200.grid import taylor_green_grid

_GRIDS: dict[int, dict] = {}


def grid(n: int) -> dict:
    if n not in _GRIDS:
        _GRIDS[n] = taylor_green_grid(n)
    return _GRIDS[n]


def populations(g: dict, seed: int, real=np.float64) -> np.ndarray:
    O = Oracle("f64")
    N = len(g["geo"])
    rng = np.random.default_rng(seed)
    d = np.zeros(27 * N)
    fields = [rng.uniform(-2e-2, 2e-2, N) for _ in range(4)]
    for ev in (0, 1):
        O.init_eq(d, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], *fields, ev)
    d += rng.uniform(-1e-3, 1e-3, d.shape) * (d != 0)
    return d.astype(real)


def case(seed: int = 1, nc: int = 8, nf: int = 12, cells: int = 40, real=np.float64) -> dict:
    """Coarse n=nc and fine n=nf periodic boxes, `cells` interface cells:
    coarse-to-fine cells write disjoint 2x2x2 fine blocks (even fine
    coordinates), fine-to-coarse cells write distinct coarse nodes; about a
    third of the cells have a zero offset (the pressure-Laplacian branch)."""
    rng = np.random.default_rng(seed)
    gc, gf = grid(nc), grid(nf)
    flc, flf = gc["fluid"], gf["fluid"]
    half = nf // 2
    evens = [flf[2 * i + nf * (2 * j + nf * 2 * k)] for i in range(half) for j in range(half) for k in range(half)]
    fine_cf = rng.choice(np.array(evens, np.uint32), cells, replace=False).astype(np.uint32)
    coarse_cf = rng.choice(flc, cells).astype(np.uint32)
    coarse_fc = rng.choice(flc, cells, replace=False).astype(np.uint32)
    fine_fc = rng.choice(flf, cells).astype(np.uint32)
    off = rng.choice([-1.0, 0.0, 1.0], (3, cells)).astype(real)
    off[:, : cells // 3] = 0.0
    return dict(gc=gc, gf=gf, distC=populations(gc, seed, real), distF=populations(gf, seed + 1, real),
                coarse_cf=coarse_cf, fine_cf=fine_cf, coarse_fc=coarse_fc, fine_fc=fine_fc, off=off,
                omegaC=1.7, omegaF=1.8)


def scaling_args(c: dict, coarse_to_fine: bool, is_even: bool, distC_ptr: int, distF_ptr: int, arrays) -> _lib.ScalingArgs:
    """vfb_scaling_args over pointers; `arrays` maps the index / offset names
    to objects with a data pointer (numpy .ctypes.data or torch .data_ptr())."""
    a = _lib.ScalingArgs()
    a.distributionsCoarse = distC_ptr
    a.distributionsFine = distF_ptr
    for side, key in (("coarse", "gc"), ("fine", "gf")):
        for ax in "XYZ":
            setattr(a, f"neighbor{ax}{side}", arrays[f"{key}.neighbor{ax}"])
    a.numberOfLBnodesCoarse = len(c["gc"]["geo"])
    a.numberOfLBnodesFine = len(c["gf"]["geo"])
    a.isEvenTimestep = int(bool(is_even))
    tag = "cf" if coarse_to_fine else "fc"
    a.coarseCells = arrays[f"coarse_{tag}"]
    a.fineCells = arrays[f"fine_{tag}"]
    a.numberOfCells = len(c[f"coarse_{tag}"])
    a.omegaCoarse = c["omegaC"]
    a.omegaFine = c["omegaF"]
    a.offsetX, a.offsetY, a.offsetZ = arrays["offX"], arrays["offY"], arrays["offZ"]
    return a


def host_arrays(c: dict) -> dict:
    out = {}
    for key in ("gc", "gf"):
        for ax in "XYZ":
            out[f"{key}.neighbor{ax}"] = c[key][f"neighbor{ax}"].ctypes.data
    for name in ("coarse_cf", "fine_cf", "coarse_fc", "fine_fc"):
        out[name] = c[name].ctypes.data
    for i, ax in enumerate("XYZ"):
        c[f"off{ax}"] = np.ascontiguousarray(c["off"][i])
        out[f"off{ax}"] = c[f"off{ax}"].ctypes.data
    return out
