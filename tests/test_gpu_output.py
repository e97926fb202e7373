"""The output pass (vfb_sim_output / vfb_output_pass): one read of the
populations gives the fields of vfb_macroscopic bit for bit and the FP64
sums of vfb_sim_mass_and_energy, vfb_sim_kinetic_energy and vfb_sim_enstrophy
to 1e-12 (summation order), and it takes less time than those separate calls."""
import time

import numpy as np
import pytest

from virtualfluids_b200.grid import MultipleGridBuilder, SideType
from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def channel(nx=48, ny=24, nz=24):
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, nx, ny, nz, 1.0)
    b.setPeriodicBoundaryCondition(False, True, False)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, 0.04, 0.0, 0.0)
    b.setPressureBoundaryCondition(SideType.PX, 0.0)
    b.setNoSlipBoundaryCondition(SideType.MZ)
    b.setNoSlipBoundaryCondition(SideType.PZ)
    return b


def _close(a, b, tol=1e-12):
    return abs(a - b) <= tol * max(abs(b), 1e-300)


@pytest.mark.parametrize("storage", ["fp64", "fp32", "fx16"])
def test_output_pass_equals_separate_passes(cuda, storage):
    p = Parameter()
    p.set_storage(storage)
    p.set_viscosity_LB(0.01)
    sim = Simulation(p, channel(), BoundaryConditionFactory())
    g = sim.levels[0]
    rng = np.random.default_rng(5)
    N = len(g["geo"])
    init = [rng.uniform(-1e-3, 1e-3, N), 0.03 + rng.uniform(-1e-3, 1e-3, N), rng.uniform(-1e-3, 1e-3, N),
            rng.uniform(-1e-3, 1e-3, N)]
    for a in init:
        a[g["geo"] != 19] = 0.0
    sim.init_level(0, *init)
    sim.run(7)
    out = sim.output(0)
    fields = sim.macroscopic(0)
    for a, b in zip(out["fields"], fields):
        assert np.array_equal(a, b)
    mass, energy, bad = sim.mass_and_energy(0)
    ke, ken = sim.kinetic_energy(0)
    ens, ensn = sim.enstrophy(0)
    assert bad == out["nonfinite"] == 0 and out["fluid_nodes"] == len(g["fluid"])
    assert _close(out["mass"], mass) and _close(out["energy"], energy)
    assert _close(out["kinetic_energy"], ke) and out["kinetic_energy_nodes"] == ken
    assert _close(out["enstrophy"], ens) and out["enstrophy_nodes"] == ensn
    assert 0 < ken < len(g["fluid"])
    sim.close()


def test_output_pass_is_faster_than_the_separate_calls(cuda):
    from virtualfluids_b200.workloads import taylor_green
    n = 192
    w = taylor_green(n)
    b = MultipleGridBuilder()
    d = 2.0 * np.pi / n
    b.addCoarseGrid(-np.pi, -np.pi, -np.pi, np.pi, np.pi, np.pi, d)
    b.setPeriodicBoundaryCondition(True, True, True)
    b.buildGrids(True)
    p = Parameter()
    p.set_storage("fp32")
    p.set_viscosity_LB(w.nu)
    sim = Simulation(p, b, BoundaryConditionFactory())
    sim.init_level(0, w.rho, w.vx, w.vy, w.vz)
    sim.run(2)

    def separate():
        sim.mass_and_energy(0)
        sim.kinetic_energy(0)
        sim.enstrophy(0)

    def fused():
        sim.output(0, fields=False)

    for fn in (separate, fused):
        fn()
    times = {}
    for name, fn in (("separate", separate), ("fused", fused)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        times[name] = (time.perf_counter() - t0) / 5
    print(f"output pass {n}^3: fused {1e3 * times['fused']:.2f} ms, separate {1e3 * times['separate']:.2f} ms")
    assert times["fused"] < times["separate"]
    sim.close()
