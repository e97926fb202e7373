"""The oracle pinned to the reference.

Against the committed golden fixtures (tests/golden, generated by
tests/golden/make_golden.py from the reference's own sources) always, and
against the live reference build (oracle/_ref) when it is present.  The bar
is bit-exact equality: the oracle performs the reference's operations in the
reference's order.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import Oracle, Reference, ref_available
from tests.golden.scenarios import grid_spec, lattice_sequence

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_k17_node_matches_golden(precision):
    g = np.load(GOLDEN / f"k17_nodes_{precision}.npz")
    O = Oracle(precision)
    for i in range(len(g["omega"])):
        f, m = O.k17_node(g["fin"][i], g["omega"][i], tuple(g["lim"][i]), tuple(g["force"][i]))
        assert np.array_equal(f, g["fout"][i]), i
        assert np.array_equal(m, g["macro"][i]), i


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_lattice_sequence_matches_golden(precision):
    from virtualfluids_b200.grid import MultipleGridBuilder  # noqa: F401  (builder checked separately)
    grid = dict(np.load(GOLDEN / "grid_channel.npz"))
    g = {k.split(":", 1)[1]: v for k, v in grid.items() if k.startswith("L0:")}
    d = lattice_sequence(Oracle(precision), g, precision)
    ref = np.load(GOLDEN / f"lattice_channel_{precision}.npz")["dist"]
    assert np.array_equal(d, ref)


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_k17_node_matches_live_reference(precision):
    O, R = Oracle(precision), Reference(precision)
    rng = np.random.default_rng(99)
    for t in range(100):
        f = rng.uniform(-0.03, 0.03, 27)
        om = rng.uniform(0.2, 1.999)
        lim = (0.01, 0.01, 0.01) if t % 3 else (1e6, 1e6, 1e6)
        force = tuple(rng.uniform(-1e-4, 1e-4, 3))
        a, ma = O.k17_node(f, om, lim, force)
        b, mb = R.k17_node(f, om, lim, force)
        assert np.array_equal(a, b) and np.array_equal(ma, mb)


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_lattice_sequence_matches_live_reference(precision):
    R = Reference(precision)
    g = R.grid(grid_spec("channel"))[0]
    a = lattice_sequence(Oracle(precision), g, precision, steps=6)
    b = lattice_sequence(R, g, precision, steps=6)
    assert np.array_equal(a, b)


def _sphere_grid():
    with np.load(GOLDEN / "grid_sphere_channel.npz") as z:
        return {k.split(":", 1)[1]: z[k] for k in z.files if k.startswith("L0:")}


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("kind", [0, 1, 4])
@pytest.mark.parametrize("is_even", [True, False])
def test_bc_on_fractional_q_matches_live_reference(kind, is_even):
    """The solid sphere's geometry list, whose q come from the ray-sphere
    intersection (fractional on most links): the oracle's no-slip
    (interpolated, bounce-back) and slip BCs equal the reference's kernels
    bit for bit."""
    g = _sphere_grid()
    k, q = g["geometry.k"], g["geometry.q"].astype(np.float64)
    assert ((q > 0) & (q < 1) & (q != 0.5)).sum() > 1000
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    rng = np.random.default_rng(17)
    fields = [rng.uniform(-1e-2, 1e-2, N) for _ in range(4)]
    out = []
    for impl in (Oracle("f64"), Reference("f64")):
        d = np.zeros(27 * N)
        for ev in (0, 1):
            impl.init_eq(d, N, g["geo"], *nb, *fields, ev)
        d += np.random.default_rng(3).uniform(-1e-3, 1e-3, d.shape) * (d != 0)
        impl.bc_post(kind, d, N, *nb, k, q, 1.7, is_even=is_even)
        out.append(d)
    assert np.array_equal(out[0], out[1])


def _golden_level0(name):
    with np.load(GOLDEN / f"grid_{name}.npz") as z:
        return {k.split(":", 1)[1]: z[k] for k in z.files if k.startswith("L0:")}


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("grid,lst", [("cavity8", "velocity"), ("channel", "velocity"), ("sphere_channel", "geometry")])
@pytest.mark.parametrize("is_even", [True, False])
def test_velocity_with_pressure_bc_matches_live_reference(precision, grid, lst, is_even):
    """VelocityWithPressureInterpolatedCompressible (kind 5): the oracle equals
    the reference's kernel source built for the host, bit for bit, on wall
    lists (q = 1/2) and on the sphere's fractional q."""
    g = _golden_level0(grid)
    real = np.float64 if precision == "f64" else np.float32
    k, q = g[f"{lst}.k"], g[f"{lst}.q"].astype(real)
    n = len(k)
    rng = np.random.default_rng(21)
    vel = [rng.uniform(-0.03, 0.03, n).astype(real) for _ in range(3)]
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    fields = [rng.uniform(-1e-2, 1e-2, N).astype(real) for _ in range(4)]
    out = []
    for impl in (Oracle(precision), Reference(precision)):
        d = np.zeros(27 * N, real)
        for ev in (0, 1):
            impl.init_eq(d, N, g["geo"], *nb, *fields, ev)
        d += (np.random.default_rng(5).uniform(-1e-3, 1e-3, d.shape) * (d != 0)).astype(real)
        before = d.copy()
        impl.bc_post(5, d, N, *nb, k, q, real(1.7), *vel, is_even=is_even)
        assert (d != before).sum() > n
        out.append(d)
    assert np.array_equal(out[0], out[1])


def _channel_level0():
    with np.load(GOLDEN / "grid_channel.npz") as z:
        return {k.split(":", 1)[1]: z[k] for k in z.files if k.startswith("L0:")}


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_init_noneq_matches_golden(precision):
    """The non-equilibrium init (both parity views) on the channel grid
    equals the fixture made by the reference's kernel built for the host."""
    g = _channel_level0()
    ref = np.load(GOLDEN / f"init_noneq_channel_{precision}.npz")
    O = Oracle(precision)
    N = len(g["geo"])
    d = np.zeros(27 * N, O.real)
    for ev in (0, 1):
        O.init_noneq(d, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], g["neighborNeg"], ref["rho"],
                     ref["vx"], ref["vy"], ref["vz"], ref["omega"][()], ev)
    assert np.array_equal(d, ref["dist"])
    # the rest population of every solid node carries the reference's marker
    solid = (g["geo"] == 15) | (g["geo"] == 16)
    assert solid.any() and np.all(d[:N][solid] == 96)


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("grid", ["channel", "sphere_channel", "cavity8"])
@pytest.mark.parametrize("omega", [1.6, 0.7])
def test_init_noneq_matches_live_reference(precision, grid, omega):
    """InitNavierStokesCompressibleNonEquilibrium_Device: the oracle equals
    the reference's kernel built for the host, bit for bit, including the
    double-literal products of the single-precision build."""
    g = _golden_level0(grid)
    O, R = Oracle(precision), Reference(precision)
    N = len(g["geo"])
    rng = np.random.default_rng(41)
    fields = [rng.uniform(-0.02, 0.02, N).astype(O.real) for _ in range(4)]
    out = []
    for impl in (O, R):
        d = np.zeros(27 * N, O.real)
        for ev in (0, 1):
            impl.init_noneq(d, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], g["neighborNeg"], *fields,
                            O.real(omega), ev)
        out.append(d)
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("correction", [0, 1])
@pytest.mark.parametrize("is_even", [0, 1])
def test_outflow_matches_golden(precision, correction, is_even):
    """OutflowNonReflecting (and its pressure-corrected form) on the channel
    grid's outflow plane equals the fixture made by the reference's kernels
    built for the host: the written positions and values, nothing else."""
    g = _channel_level0()
    ref = np.load(GOLDEN / f"outflow_channel_{precision}.npz")
    O = Oracle(precision)
    N = len(g["geo"])
    d = ref["dist"].copy()
    O.bc_outflow(d, N, g["neighborX"], g["neighborY"], g["neighborZ"], g["pressure0.k"], g["pressure0.kN"],
                 int(g["pressure0.dir"][0]), bool(correction), ref["factor"][()], bool(is_even))
    idx = np.flatnonzero(d != ref["dist"])
    assert np.array_equal(idx, ref[f"idx_c{correction}_e{is_even}"])
    assert np.array_equal(d[idx], ref[f"val_c{correction}_e{is_even}"])
    assert len(idx) == 9 * len(g["pressure0.k"])


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("correction", [False, True])
def test_outflow_matches_live_reference_every_direction(precision, correction):
    """All six normals, both parities, on random node pairs of a periodic box
    and on the outflow planes of the channel and cube grids."""
    from virtualfluids_b200.workloads import taylor_green
    O, R = Oracle(precision), Reference(precision)
    g = taylor_green(9).grid
    N = len(g["geo"])
    rng = np.random.default_rng(2)
    k = rng.choice(np.arange(1, N), 40, replace=False).astype(np.int32)
    kN = rng.integers(1, N, 40).astype(np.int32)
    cases = [(g, k, kN, direction) for direction in range(1, 7)]
    for name in ("channel", "cube_channel"):
        h = _golden_level0(name)
        cases.append((h, h["pressure0.k"], h["pressure0.kN"], int(h["pressure0.dir"][0])))
    for grid, kk, kkN, direction in cases:
        M = len(grid["geo"])
        for ev in (True, False):
            out = []
            for impl in (O, R):
                d = np.random.default_rng(5).uniform(-0.02, 0.02, 27 * M).astype(O.real)
                impl.bc_outflow(d, M, grid["neighborX"], grid["neighborY"], grid["neighborZ"], kk, kkN, direction,
                                correction, O.real(0.7), ev)
                out.append(d)
            assert np.array_equal(out[0], out[1]), (direction, ev)


@pytest.mark.skipif(not ref_available("f64"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("grid,lst", [("channel", "slip"), ("sphere_channel", "geometry")])
@pytest.mark.parametrize("is_even", [True, False])
def test_stress_bc_matches_live_reference(precision, kind, grid, lst, is_even):
    """The wall-model BCs (StressCompressible, StressBounceBack,
    StressBounceBackPressure with the iMEM model): the oracle equals the
    reference's kernel sources built for the host bit for bit, in the
    populations, both filter states and the monitors, on a flat wall (q = 1/2)
    and on the sphere's fractional q, with random unit normals and an eddy
    viscosity field."""
    from tests.stress_cases import copy_list, make_stress_list, turbulent_viscosity, velocity_fields

    g = _golden_level0(grid)
    real = np.float64 if precision == "f64" else np.float32
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    base = make_stress_list(g, lst, real, seed=31 + kind)
    vel = velocity_fields(N, real, seed=7)
    turb = turbulent_viscosity(N, real, seed=8)
    rng = np.random.default_rng(41)
    fields = [rng.uniform(-1e-2, 1e-2, N).astype(real) for _ in range(4)]
    out = []
    for impl in (Oracle(precision), Reference(precision)):
        d = np.zeros(27 * N, real)
        for ev in (0, 1):
            impl.init_eq(d, N, g["geo"], *nb, *fields, ev)
        d += (np.random.default_rng(5).uniform(-1e-3, 1e-3, d.shape) * (d != 0)).astype(real)
        lst_i = copy_list(base)
        before = d.copy()
        for step in range(2):
            impl.bc_stress(kind, d, N, *nb, lst_i, real(1.7), *vel, turb=turb, monitor=True,
                           is_even=is_even ^ bool(step))
        assert (d != before).sum() > len(base["k"])
        out.append((d, lst_i))
    (d0, l0), (d1, l1) = out
    assert np.array_equal(d0, d1)
    for name in l0:
        assert np.array_equal(l0[name], l1[name]), name
    assert np.all(np.isfinite(l0["uStar"])) and np.any(l0["Fx"] != 0)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_stress_bc_matches_golden(precision, kind):
    """The oracle's wall-model BCs against the fixture made by the reference's
    three kernel sources built for the host (tests/golden/make_golden.py
    --stress): two launches on the sphere channel's geometry list with
    seeded states, compared in the written populations, states and monitors."""
    from tests.stress_cases import copy_list, make_stress_list, stress_populations, turbulent_viscosity, velocity_fields

    ref = np.load(GOLDEN / f"stress_sphere_{precision}.npz")
    g = _golden_level0("sphere_channel")
    real = np.float64 if precision == "f64" else np.float32
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    base = make_stress_list(g, "geometry", real, seed=77)
    vel = velocity_fields(N, real, seed=78)
    turb = turbulent_viscosity(N, real, seed=79)
    dist0 = stress_populations(N, real)
    assert np.array_equal(dist0[:16], ref["dist_head"]) and dist0.astype(np.float64).sum() == ref["dist_sum"]
    assert np.array_equal(vel[0][:16], ref["vx_head"]) and np.array_equal(turb[:16], ref["turb_head"])
    assert np.array_equal(base["kN"][:16], ref["kN_head"])
    O = Oracle(precision)
    d = dist0.copy()
    lst = copy_list(base)
    for ev in (1, 0):
        O.bc_stress(kind, d, N, *nb, lst, real(1.7), *vel, turb=turb, monitor=True, is_even=bool(ev))
    idx = np.flatnonzero(d != dist0)
    assert np.array_equal(idx, ref[f"idx_{kind}"])
    assert np.array_equal(d[idx], ref[f"val_{kind}"])
    for k in ("vxEl", "vyEl", "vzEl", "vxWMean", "vyWMean", "vzWMean", "uStar", "Fx", "Fy", "Fz"):
        assert np.array_equal(lst[k], ref[f"out{kind}.{k}"]), k
