"""The FX16 range check (vfb_saturated_populations) and the wide format FX16W.

FX16 stores f - w = q w 2^-17 with q an int16, so deviations beyond a quarter
of the weight are clipped on store.  The count of clipped codes equals a
count over the downloaded array; it is zero for a flow inside the range
(Taylor-Green, u0 = 0.05) and positive for one outside it (a cavity whose lid
moves at 0.3, where the diagonal populations leave the range), and zero for
FP32 storage.  FX16W (f - w = q w R 2^-15, R = 1/4, 1/2, 1, 1 by the number
of non-zero components) holds a cavity with a 0.1 lid that FX16 clips, and
its velocities stay close to FP32's there while FX16's do not."""
import ctypes

import numpy as np
import pytest

from virtualfluids_b200 import _lib
from virtualfluids_b200.grid import MultipleGridBuilder, SideType
from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _cavity(n, lid):
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, n - 1, n - 1, n - 1, 1.0)
    b.buildGrids()
    for s in (SideType.MX, SideType.PX, SideType.MY, SideType.PY, SideType.MZ):
        b.setNoSlipBoundaryCondition(s)
    b.setVelocityBoundaryCondition(SideType.PZ, lid, 0.0, 0.0)
    return b


def _periodic(n):
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, n - 1, n - 1, n - 1, 1.0)
    b.setPeriodicBoundaryCondition(True, True, True)
    b.buildGrids()
    return b


def _sim(grid, storage, init=None):
    p = Parameter()
    p.set_storage(storage)
    p.set_viscosity_LB(0.02)
    sim = Simulation(p, grid, BoundaryConditionFactory())
    g = sim.levels[0]
    N = len(g["geo"])
    f = init(g) if init else [np.zeros(N)] * 4
    sim.init_level(0, *f)
    return sim


def _count_on_host(sim):
    ptr, N, _, _ = sim.level_state(0)
    a = np.empty(27 * N, np.int16)
    _lib.check(_lib.lib().vfb_copy_device_to_host(a.ctypes.data, ctypes.c_void_p(ptr), a.nbytes, None))
    tail = a[N:]
    return int(np.count_nonzero((tail == 32767) | (tail == -32768)))


def _taylor_green(n, u0=0.05):
    def init(g):
        x = 2 * np.pi * g["coordX"] / n
        y = 2 * np.pi * g["coordY"] / n
        z = 2 * np.pi * g["coordZ"] / n
        vx = u0 * np.sin(x) * np.cos(y) * np.cos(z)
        vy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
        return [np.zeros_like(x), vx, vy, np.zeros_like(x)]
    return init


def test_inside_the_range_nothing_is_clipped(cuda):
    sim = _sim(_periodic(32), "fx16", _taylor_green(32))
    sim.run(40)
    assert sim.saturated_populations(0) == 0 == _count_on_host(sim)
    sim.close()


def test_fast_lid_clips_and_the_count_matches_the_array(cuda):
    sim = _sim(_cavity(24, 0.3), "fx16")
    sim.run(60)
    n = sim.saturated_populations(0)
    assert n > 0
    assert n == _count_on_host(sim)
    sim.close()
    sim = _sim(_cavity(24, 0.3), "fp32")
    sim.run(60)
    assert sim.saturated_populations(0) == 0
    sim.close()


def _velocity(sim):
    fl = sim.levels[0]["fluid"]
    return np.stack([a[fl].astype(np.float64) for a in sim.macroscopic(0)[1:]])


def test_wide_format_holds_what_fx16_clips(cuda):
    out = {}
    for storage in ("fp32", "fx16", "fx16w"):
        sim = _sim(_cavity(24, 0.1), storage)
        sim.run(200)
        out[storage] = (sim.saturated_populations(0), _velocity(sim))
        sim.close()
    assert out["fx16"][0] > 0
    assert out["fx16w"][0] == 0
    ref = out["fp32"][1]
    scale = np.abs(ref).max()
    err_w = np.abs(out["fx16w"][1] - ref).max() / scale
    err_n = np.abs(out["fx16"][1] - ref).max() / scale
    assert err_w < 1e-2, err_w
    assert err_w < err_n, (err_w, err_n)


def test_wide_format_inside_the_range(cuda):
    """On Taylor-Green both fixed-point formats stay inside their ranges and
    close to FP32 (FX16W at about twice FX16's step on the faces)."""
    out = {}
    for storage in ("fp32", "fx16", "fx16w"):
        sim = _sim(_periodic(32), storage, _taylor_green(32))
        sim.run(100)
        out[storage] = (sim.saturated_populations(0), _velocity(sim))
        sim.close()
    assert out["fx16"][0] == 0 == out["fx16w"][0]
    ref = out["fp32"][1]
    scale = np.abs(ref).max()
    for storage in ("fx16", "fx16w"):
        assert np.abs(out[storage][1] - ref).max() <= 2e-3 * scale, storage
