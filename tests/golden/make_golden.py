"""Generate the golden fixtures of tests/golden from the reference itself.

Runs the reference's own sources compiled on the host (oracle/_ref, built by
``make -C oracle ref`` from the reference tree) and stores small inputs and
outputs as .npz files.  The parity tests compare the oracle and the
repository's grid builder against these files, so the pin also holds on a
machine without the reference tree.

    python tests/golden/make_golden.py                 (all fixtures)
    python tests/golden/make_golden.py --init-noneq    (the non-equilibrium init only)
    python tests/golden/make_golden.py --outflow       (the non-reflecting outflow only)
    python tests/golden/make_golden.py --thin-walls    (the thin-wall grids only)
    python tests/golden/make_golden.py --extra-grids   (the cylinder and conglomerate grids only)
    python tests/golden/make_golden.py --stress        (the wall-model grid and kernels only)
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import subprocess

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.pyoracle import Reference  # noqa: E402
from tests.golden.scenarios import (EXTRA_GRID_SCENARIOS, GRID_SCENARIOS, REFINED_SCENARIOS,  # noqa: E402
                                    STRESS_GRID_SCENARIOS, THIN_WALL_SCENARIOS, grid_spec, lattice_sequence,
                                    refined_spec)
from tests.stress_cases import (copy_list, make_stress_list, stress_populations,  # noqa: E402
                                turbulent_viscosity, velocity_fields)

OUT = Path(__file__).resolve().parent


def k17_nodes(precision: str) -> None:
    R = Reference(precision)
    rng = np.random.default_rng(20241203)
    n = 64
    fin = rng.uniform(-0.02, 0.02, (n, 27))
    omega = rng.uniform(0.5, 1.99, n)
    lim = np.where(rng.uniform(size=(n, 1)) < 0.5, 0.01, 1e6) * np.ones((n, 3))
    lim[::7] = [0.02, 0.005, 0.1]
    force = rng.uniform(-1e-4, 1e-4, (n, 3))
    fout = np.zeros_like(fin)
    macro = np.zeros((n, 4))
    for i in range(n):
        f, m = R.k17_node(fin[i], omega[i], tuple(lim[i]), tuple(force[i]))
        fout[i], macro[i] = f, m
    real = np.float64 if precision == "f64" else np.float32
    np.savez_compressed(OUT / f"k17_nodes_{precision}.npz", fin=fin.astype(real), omega=omega.astype(real),
                        lim=lim.astype(real), force=force.astype(real), fout=fout.astype(real),
                        macro=macro.astype(real))


def grids() -> None:
    R = Reference("f64")
    for name in GRID_SCENARIOS:
        levels = R.grid(grid_spec(name))
        arrays = {f"L{lvl}:{k}": v for lvl, d in levels.items() for k, v in d.items()}
        np.savez_compressed(OUT / f"grid_{name}.npz", **arrays)


def thin_wall_grids(names=THIN_WALL_SCENARIOS) -> None:
    """Solids built with thin walls (and the later solid scenarios), from the
    reference builder."""
    R = Reference("f64")
    for name in names:
        levels = R.grid(grid_spec(name))
        arrays = {f"L{lvl}:{k}": v for lvl, d in levels.items() for k, v in d.items()}
        np.savez_compressed(OUT / f"grid_{name}.npz", **arrays)


def refined_grid(name: str) -> None:
    """One multi-level grid with its interface cells, from the reference builder."""
    levels = Reference("f64").grid(refined_spec(name))
    arrays = {f"L{lvl}:{k}": v for lvl, d in levels.items() for k, v in d.items()}
    np.savez_compressed(OUT / f"grid_{name}.npz", **arrays)


def refined_grids() -> None:
    """Every multi-level scenario, each built in a fresh process: the
    reference's builder is not reliable across several multi-level builds in
    one process (it has crashed there)."""
    for name in REFINED_SCENARIOS:
        subprocess.run([sys.executable, __file__, "--refined", name], check=True)


def lattice(precision: str) -> None:
    R = Reference(precision)
    levels = R.grid(grid_spec("channel"))
    dist = lattice_sequence(R, levels[0], precision)
    np.savez_compressed(OUT / f"lattice_channel_{precision}.npz", dist=dist)


def init_noneq(precision: str) -> None:
    """InitNavierStokesCompressibleNonEquilibrium_Device over the channel
    grid (walls, inflow and outflow planes) for both parity views, from
    seeded fields."""
    R = Reference(precision)
    real = np.float64 if precision == "f64" else np.float32
    g = R.grid(grid_spec("channel"))[0]
    N = len(g["geo"])
    rng = np.random.default_rng(20261203)
    fields = [rng.uniform(-0.02, 0.02, N).astype(real) for _ in range(4)]
    omega = real(1.6)
    dist = np.zeros(27 * N, real)
    for ev in (0, 1):
        R.init_noneq(dist, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], g["neighborNeg"], *fields,
                     omega, ev)
    np.savez_compressed(OUT / f"init_noneq_channel_{precision}.npz", rho=fields[0], vx=fields[1], vy=fields[2],
                        vz=fields[3], omega=np.array(omega), dist=dist)


def outflow(precision: str) -> None:
    """OutflowNonReflecting_Device and its pressure-corrected form over the
    channel grid's outflow list (both parity views), from seeded populations;
    the outputs are stored at the positions the kernels write."""
    R = Reference(precision)
    real = np.float64 if precision == "f64" else np.float32
    g = R.grid(grid_spec("channel"))[0]
    N = len(g["geo"])
    rng = np.random.default_rng(20261204)
    dist0 = rng.uniform(-0.02, 0.02, 27 * N).astype(real)
    factor = real(0.3)
    out = {"dist": dist0, "factor": np.array(factor)}
    for correction in (0, 1):
        for ev in (0, 1):
            d = dist0.copy()
            R.bc_outflow(d, N, g["neighborX"], g["neighborY"], g["neighborZ"], g["pressure0.k"], g["pressure0.kN"],
                         int(g["pressure0.dir"][0]), bool(correction), factor, bool(ev))
            idx = np.flatnonzero(d != dist0)
            out[f"idx_c{correction}_e{ev}"] = idx
            out[f"val_c{correction}_e{ev}"] = d[idx]
    np.savez_compressed(OUT / f"outflow_channel_{precision}.npz", **out)


def stress(precision: str) -> None:
    """The three wall-model kernels (StressCompressible,
    StressBounceBackCompressible, StressBounceBackPressureCompressible) of
    the reference, two launches each (both parities) on a stress list made
    from the sphere channel's geometry list (fractional q) with seeded
    normals, sampling nodes, states and an eddy-viscosity field; stored: the
    written positions and values, and the list's states and monitors."""
    R = Reference(precision)
    real = np.float64 if precision == "f64" else np.float32
    g = Reference("f64").grid(grid_spec("sphere_channel"))[0]  # the grid of grid_sphere_channel.npz
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    base = make_stress_list(g, "geometry", real, seed=77)
    vel = velocity_fields(N, real, seed=78)
    turb = turbulent_viscosity(N, real, seed=79)
    dist0 = stress_populations(N, real)
    # the inputs are regenerated from their seeds by the test; their first
    # values and sums are stored to detect a change of the generator
    out = {"dist_head": dist0[:16], "dist_sum": np.array(dist0.astype(np.float64).sum()),
           "vx_head": vel[0][:16], "turb_head": turb[:16], "kN_head": base["kN"][:16]}
    for kind in (0, 1, 2):
        d = dist0.copy()
        lst = copy_list(base)
        for ev in (1, 0):
            R.bc_stress(kind, d, N, *nb, lst, real(1.7), *vel, turb=turb, monitor=True, is_even=bool(ev))
        idx = np.flatnonzero(d != dist0)
        out[f"idx_{kind}"] = idx
        out[f"val_{kind}"] = d[idx]
        for k in ("vxEl", "vyEl", "vzEl", "vxWMean", "vyWMean", "vzWMean", "uStar", "Fx", "Fy", "Fz"):
            out[f"out{kind}.{k}"] = lst[k]
    np.savez_compressed(OUT / f"stress_sphere_{precision}.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "--refined":
        refined_grid(sys.argv[2])
        sys.exit(0)
    if len(sys.argv) == 2 and sys.argv[1] == "--init-noneq":
        for p in ("f64", "f32"):
            init_noneq(p)
        outflow(p)
        sys.exit(0)
    if len(sys.argv) == 2 and sys.argv[1] == "--thin-walls":
        thin_wall_grids()
        sys.exit(0)
    if len(sys.argv) == 2 and sys.argv[1] == "--extra-grids":
        thin_wall_grids(EXTRA_GRID_SCENARIOS)
        sys.exit(0)
    if len(sys.argv) == 2 and sys.argv[1] == "--stress":
        thin_wall_grids(STRESS_GRID_SCENARIOS)
        for p in ("f64", "f32"):
            stress(p)
        sys.exit(0)
    if len(sys.argv) == 2 and sys.argv[1] == "--outflow":
        for p in ("f64", "f32"):
            outflow(p)
        sys.exit(0)
    for p in ("f64", "f32"):
        k17_nodes(p)
        lattice(p)
        init_noneq(p)
    grids()
    thin_wall_grids()
    thin_wall_grids(EXTRA_GRID_SCENARIOS)
    refined_grids()
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)
