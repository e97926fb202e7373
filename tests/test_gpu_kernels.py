"""GPU parity of init, macroscopic output, collision templates and FP64
reductions against the oracle."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.gpu_helpers import rel_max, tgv_state
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def setup(n=8, dtype=None):
    dtype = dtype or torch.float64
    w = tgv_state(n)
    lat = K.DeviceLattice.from_arrays(w.grid)
    cd = K.compute_dtype(dtype)
    fields = [torch.from_numpy(a).to("cuda", cd) for a in (w.rho, w.vx, w.vy, w.vz)]
    dist = K.new_distributions(lat, dtype)
    return w, lat, fields, dist


def oracle_init(w):
    O = Oracle("f64")
    g = w.grid
    N = len(g["geo"])
    d = np.zeros(27 * N)
    for ev in (0, 1):
        O.init_eq(d, N, g["geo"], g["neighborX"], g["neighborY"], g["neighborZ"], w.rho, w.vx, w.vy, w.vz, ev)
    return O, d


def test_init_equilibrium_matches_oracle(cuda):
    w, lat, fields, dist = setup()
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    _, d = oracle_init(w)
    assert rel_max(dist.cpu().numpy(), d) < 1e-15


def test_macroscopic_recovers_initial_fields(cuda):
    w, lat, fields, dist = setup()
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    rho, vx, vy, vz = [m.cpu().numpy() for m in K.macroscopic(dist, lat, True)]
    fl = w.grid["fluid"]
    assert np.abs(vx[fl] - w.vx[fl]).max() < 1e-6
    assert np.abs(rho[fl] - w.rho[fl]).max() < 1e-6
    solid = w.grid["geo"] != 19
    assert (rho[solid] == 0).all()


@pytest.mark.parametrize("template", [1, 2, 3])
def test_collision_templates(cuda, template):
    w, lat, fields, dist = setup()
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    O, d = oracle_init(w)
    g = w.grid
    N = lat.N
    macro_ref = [np.zeros(N) for _ in range(4)]
    rng = np.random.default_rng(3)
    body = [rng.uniform(-1e-5, 1e-5, N) for _ in range(3)]
    body_ref = [b.copy() for b in body]
    O.collision_k17(d, N, g["neighborX"], g["neighborY"], g["neighborZ"], g["fluid"], w.omega,
                    forces=(1e-6, 0, 0), force_factor=0.5, is_even=True, flags=template, macro=macro_ref,
                    body=body_ref)
    macro = [torch.zeros(N, dtype=torch.float64, device="cuda") for _ in range(4)]
    bdev = [torch.from_numpy(b).cuda() for b in body]
    K.collision("K17", dist, lat, w.omega, True, forces=(1e-6, 0, 0), force_factor=0.5, template=template,
                macro=macro, body=bdev)
    assert rel_max(dist.cpu().numpy(), d) < 1e-13
    if template & 1:
        for a, b in zip(macro, macro_ref):
            assert rel_max(a.cpu().numpy(), b) < 1e-13
    if template & 2:
        for a, b in zip(bdev, body_ref):
            assert np.array_equal(a.cpu().numpy(), b)  # both reset to zero on fluid nodes


def test_mass_and_energy_fp64(cuda):
    w, lat, fields, dist = setup()
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    m, e, bad = K.mass_and_energy(dist, lat, True)
    fl = w.grid["fluid"]
    O, d = oracle_init(w)
    rho, vx, vy, vz = O.macroscopic(d, lat.N, w.grid["geo"], w.grid["neighborX"], w.grid["neighborY"],
                                    w.grid["neighborZ"], True)
    assert bad == 0
    assert m == pytest.approx(rho[fl].sum(), rel=1e-12, abs=1e-15)
    ke = (0.5 * (vx ** 2 + vy ** 2 + vz ** 2) * (rho + 1.0))[fl].sum()
    assert e == pytest.approx(ke, rel=1e-12)


def test_bad_template_reports_error(cuda):
    w, lat, fields, dist = setup()
    with pytest.raises(_lib.VfbError):
        K.collision("K17", dist, lat, w.omega, True, template=7)
