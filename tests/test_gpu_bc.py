"""GPU boundary-condition kernels (vfb_bc_post, vfb_bc_pressure_noneq)
against the oracle, kind by kind, and the whole golden lattice sequence
(collision + five post-collision BCs + pressure BC + BGK) against the
fixture generated from the reference's own kernels."""
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import rel_l2, rel_max
from tests.golden.scenarios import lattice_sequence
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GOLDEN = Path(__file__).resolve().parent / "golden"
TORCH_REAL = {"f64": torch.float64, "f32": torch.float32}


def _grid(name):
    """Level 0 of a committed golden grid (the grid the reference's builder made)."""
    with np.load(GOLDEN / f"grid_{name}.npz") as z:
        return {k.split(":", 1)[1]: z[k] for k in z.files if k.startswith("L0:")}


class GpuImpl:
    """The lattice-sequence interface of the oracle, run on the GPU through
    the C ABI; after every call the numpy array is refreshed from the device."""

    def __init__(self, g, dtype):
        self.g = g
        self.dtype = dtype
        self.cd = K.compute_dtype(dtype)
        self.lat = K.DeviceLattice.from_arrays(g)
        self.dist = K.new_distributions(self.lat, dtype)

    def _t(self, a, dt=None):
        return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt or self.cd)

    def _i(self, a):
        return torch.from_numpy(np.ascontiguousarray(a).astype(np.int32)).cuda()

    def _back(self, d):
        d[:] = self.dist.cpu().to(torch.float64).numpy().astype(d.dtype) / K.storage_scale(self.dtype)

    def load(self, d):
        """The (unscaled) populations d into the device array."""
        self.dist.copy_((torch.from_numpy(d).to(torch.float64) * K.storage_scale(self.dtype)).to("cuda", self.dtype))

    def init_eq(self, d, N, geo, nx, ny, nz, rho, ux, uy, uz, ev):
        K.init_equilibrium(self.dist, self.lat, *[self._t(a) for a in (rho, ux, uy, uz)], bool(ev))
        self._back(d)

    def collision_k17(self, d, N, nx, ny, nz, fl, om, forces, force_factor, limiters, is_even):
        K.collision("K17", self.dist, self.lat, om, is_even, forces=forces, force_factor=force_factor,
                    limiters=limiters)
        self._back(d)

    def collision_bgk(self, d, N, geo, nx, ny, nz, om, is_even):
        K.collision("BGK", self.dist, self.lat, om, is_even)
        self._back(d)

    def bc_post(self, kind, d, N, nx, ny, nz, k, q, om, vx=None, vy=None, vz=None, is_even=True):
        v = [None if a is None else self._t(a) for a in (vx, vy, vz)]
        K.bc_post(kind, self.dist, self.lat, self._i(k), self._t(q), om, is_even, *v)
        self._back(d)

    def bc_pressure(self, d, N, nx, ny, nz, k, kN, rho, direction, is_even=True):
        K.bc_pressure(self.dist, self.lat, self._i(k), self._i(kN), self._t(rho), direction, is_even)
        self._back(d)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_lattice_sequence_matches_reference_golden(cuda, precision):
    g = _grid("channel")
    ref = np.load(GOLDEN / f"lattice_channel_{precision}.npz")["dist"]
    got = lattice_sequence(GpuImpl(g, TORCH_REAL[precision]), g, precision)
    if precision == "f64":
        assert rel_max(got, ref) < 1e-12
    else:
        assert rel_l2(got, ref) < 1e-5


def _random_state(g, precision, seed=3):
    O = Oracle(precision)
    real = O.real
    N = len(g["geo"])
    rng = np.random.default_rng(seed)
    d = np.zeros(27 * N, real)
    rho = rng.uniform(-1e-2, 1e-2, N).astype(real)
    u = [rng.uniform(-2e-2, 2e-2, N).astype(real) for _ in range(3)]
    for ev in (0, 1):
        O.init_eq(d, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], rho, *u, ev)
    # non-equilibrium parts so that the interpolated formulas see f != feq
    d += rng.uniform(-1e-3, 1e-3, d.shape).astype(real) * (d != 0)
    return O, d


CASES = [(_lib.BC_NOSLIP_INTERPOLATED, "velocity"), (_lib.BC_NOSLIP_BOUNCE_BACK, "velocity"),
         (_lib.BC_VELOCITY_INTERPOLATED, "velocity"), (_lib.BC_VELOCITY_BOUNCE_BACK, "velocity"),
         (_lib.BC_SLIP, "slip")]


@pytest.mark.parametrize("kind,lst", CASES)
@pytest.mark.parametrize("is_even", [True, False])
@pytest.mark.parametrize("grid", ["cavity8", "channel"])
def test_bc_post_matches_oracle_fp64(cuda, kind, lst, is_even, grid):
    g = _grid(grid)
    if len(g[f"{lst}.k"]) == 0:
        pytest.skip(f"no {lst} list in {grid}")
    O, d = _random_state(g, "f64")
    N = len(g["geo"])
    k, q = g[f"{lst}.k"], g[f"{lst}.q"].astype(np.float64)
    vel = [g[f"velocity.{c}"].astype(np.float64) for c in ("vx", "vy", "vz")] if lst == "velocity" else [None] * 3
    om = 1.7
    imp = GpuImpl(g, torch.float64)
    imp.load(d)
    got = d.copy()
    imp.bc_post(kind, got, N, None, None, None, k, q, om, *vel, is_even=is_even)
    O.bc_post(kind, d, N, g["neighborX"], g["neighborY"], g["neighborZ"], k, q, om, *vel, is_even=is_even)
    assert np.any(got != _random_state(g, "f64")[1])  # the kernel wrote something
    assert rel_max(got, d) < 1e-13


@pytest.mark.parametrize("kind,lst", CASES)
@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
def test_bc_post_reduced_storage(cuda, kind, lst, dtype):
    g = _grid("cavity8" if lst == "velocity" else "channel")
    O, d = _random_state(g, "f64")
    N = len(g["geo"])
    k, q = g[f"{lst}.k"], g[f"{lst}.q"]
    vel = [g[f"velocity.{c}"] for c in ("vx", "vy", "vz")] if lst == "velocity" else [None] * 3
    dt = getattr(torch, dtype)
    imp = GpuImpl(g, dt)
    imp.load(d)
    got = np.zeros_like(d)
    imp.bc_post(kind, got, N, None, None, None, k, q, 1.7, *vel, is_even=True)
    O.bc_post(kind, d, N, g["neighborX"], g["neighborY"], g["neighborZ"], k, q.astype(np.float64), 1.7,
              *[None if v is None else v.astype(np.float64) for v in vel], is_even=True)
    tol = {"float32": 1e-6, "float16": 2e-3, "bfloat16": 2e-2}[dtype]
    assert rel_l2(got, d) < tol


@pytest.mark.parametrize("is_even", [True, False])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_pressure_bc_matches_oracle(cuda, is_even, precision):
    g = _grid("channel")
    O, d = _random_state(g, precision)
    N = len(g["geo"])
    k, kN = g["pressure0.k"], g["pressure0.kN"]
    rho = np.full(len(k), 2e-3, O.real)
    direction = int(g["pressure0.dir"][0])
    imp = GpuImpl(g, TORCH_REAL[precision])
    imp.load(d)
    got = d.copy()
    imp.bc_pressure(got, N, None, None, None, k, kN, rho, direction, is_even=is_even)
    O.bc_pressure(d, N, g["neighborX"], g["neighborY"], g["neighborZ"], k, kN, rho, direction, is_even=is_even)
    if precision == "f64":
        assert rel_max(got, d) < 1e-13
    else:
        assert rel_l2(got, d) < 1e-6


def test_bc_argument_errors(cuda):
    g = _grid("cavity8")
    imp = GpuImpl(g, torch.float64)
    k = imp._i(g["velocity.k"])
    q = imp._t(g["velocity.q"])
    with pytest.raises(_lib.VfbError):
        K.bc_post(_lib.BC_VELOCITY_INTERPOLATED, imp.dist, imp.lat, k, q, 1.7, True)  # no velocities
    with pytest.raises(_lib.VfbError):
        K.bc_post(9, imp.dist, imp.lat, k, q, 1.7, True)
    with pytest.raises(_lib.VfbError):
        K.bc_pressure(imp.dist, imp.lat, k, k, q, 7, True)


@pytest.mark.parametrize("kind", [_lib.BC_NOSLIP_INTERPOLATED, _lib.BC_NOSLIP_BOUNCE_BACK, _lib.BC_SLIP])
@pytest.mark.parametrize("is_even", [True, False])
def test_geometry_bc_with_fractional_q_matches_oracle(cuda, kind, is_even):
    """The solid sphere's geometry list, q from the ray-sphere intersection
    (fractional on most links), FP64 against the oracle.

    Unlike the walls, the BC nodes around a sphere are neighbours of each
    other: a node's bounce-back value lands in a cell from which a
    neighbouring BC node reads its post-collision population.  The GPU
    kernels (the reference's and this library's) read every node's values
    before writing, so the oracle is applied node by node to the state before
    the kernel and the written cells merged (no two nodes write one cell).
    The list (276 nodes) is resident in one wave, so every read precedes every
    write on the GPU too."""
    g = _grid("sphere_channel")
    k, q = g["geometry.k"], g["geometry.q"].astype(np.float64)
    assert ((q > 0) & (q < 1) & (q != 0.5)).sum() > 1000
    O, d = _random_state(g, "f64")
    N = len(g["geo"])
    nb = (g["neighborX"], g["neighborY"], g["neighborZ"])
    imp = GpuImpl(g, torch.float64)
    imp.load(d)
    got = d.copy()
    imp.bc_post(kind, got, N, None, None, None, k, q, 1.7, None, None, None, is_even=is_even)
    n = len(k)
    want = d.copy()
    written = np.zeros(d.shape, bool)
    for i in range(n):
        one = d.copy()
        O.bc_post(kind, one, N, *nb, k[i:i + 1], np.ascontiguousarray(q.reshape(27, n)[:, i]), 1.7, is_even=is_even)
        changed = one != d
        assert not (changed & written).any()
        want[changed] = one[changed]
        written |= changed
    assert rel_max(got, want) < 1e-12


@pytest.mark.parametrize("kind,lst", CASES)
@pytest.mark.parametrize("is_even", [True, False])
def test_location_table_equals_neighbour_chain(cuda, kind, lst, is_even):
    """A BC list with its location table (vfb_bc_locations) writes exactly what
    the walk through the neighbour arrays writes."""
    g = _grid("cavity8" if lst == "velocity" else "channel")
    _, d = _random_state(g, "f64")
    k, q = g[f"{lst}.k"], g[f"{lst}.q"]
    vel = [g[f"velocity.{c}"] for c in ("vx", "vy", "vz")] if lst == "velocity" else [None] * 3
    out = []
    for with_table in (False, True):
        imp = GpuImpl(g, torch.float64)
        imp.load(d)
        kk = imp._i(k)
        locs = K.bc_locations(imp.lat, kk) if with_table else None
        v = [None if a is None else imp._t(a) for a in vel]
        K.bc_post(kind, imp.dist, imp.lat, kk, imp._t(q), 1.7, is_even, *v, locations=locs)
        out.append(imp.dist.cpu().numpy())
    assert np.array_equal(out[0], out[1])
