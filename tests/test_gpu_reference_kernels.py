"""The library's kernels against the reference's own GPU kernels, compiled
unmodified by nvcc for sm_100a (oracle/_ref/libvfref_gpu_{f64,f32}.so,
launchers in oracle/ref/ref_gpu_device.cu) and run on the same device with the
same inputs: runCollision<K17> (RunCollision.cuh:74-143), the B92 BGK kernel,
the post-collision BC kernels and both interface kernels.

The last test is the same-device baseline: both sides event-timed on the
same arrays (TGV 256^3 FP32 for the collisions, the 256^3 cavity walls for
the BC kernels, 32k / 16k interface cells), one JSON line per kernel on
stdout.  The reference's pressure BC kernel is not run on the GPU (a
__syncthreads() under divergent control flow); its parity rests on the host
build of the same source."""
import json

import numpy as np
import pytest

from oracle.pyoracle import ReferenceGpu, ref_gpu_available
from tests.gpu_helpers import rel_l2, rel_max, tgv_state
from tests.scaling_cases import case
from tests.test_gpu_bc import CASES, _grid, _random_state
from virtualfluids_b200 import _lib
from virtualfluids_b200 import kernels as K
from virtualfluids_b200.workloads import cavity_grid, interface_planes, taylor_green

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu_available("f64") or not ref_gpu_available("f32"),
                                 reason="reference GPU kernels not built (oracle/_ref needs the reference tree)")]
torch = pytest.importorskip("torch")

TORCH_REAL = {"f64": torch.float64, "f32": torch.float32}
FORCES = (2e-6, -1e-6, 5e-7)
LIMITERS = (0.01, 0.01, 0.01)


def _tgv_pair(n, precision):
    """Two identical initialised population arrays of the TGV n^3 state."""
    w = tgv_state(n)
    dt = TORCH_REAL[precision]
    lat = K.DeviceLattice.from_arrays(w.grid)
    dist = K.new_distributions(lat, dt)
    fields = [torch.from_numpy(a).to("cuda", dt) for a in (w.rho, w.vx, w.vy, w.vz)]
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    return w, lat, dist, dist.clone()


def _close(got, ref, precision):
    a, b = got.cpu().double().numpy(), ref.cpu().double().numpy()
    if precision == "f64":
        return rel_max(a, b) < 1e-12
    return rel_l2(a, b) < 1e-5


@pytest.mark.parametrize("planned", [True, False])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_k17_matches_reference_gpu_kernel(cuda, precision, planned):
    """12 steps with a body force: the planned / generic K17 against runCollision<K17>."""
    R = ReferenceGpu(precision)
    dt = TORCH_REAL[precision]
    w, lat, ours, ref = _tgv_pair(32, precision)
    plan = K.CollisionPlan(dt, lat) if planned else None
    forces = torch.tensor(FORCES, dtype=dt, device="cuda")
    limiters = torch.tensor(LIMITERS, dtype=dt, device="cuda")
    even = True
    for _ in range(12):
        K.collision("K17", ours, lat, w.omega, even, plan=plan, forces=FORCES, limiters=LIMITERS, stream=0)
        R.collision_k17(ref, lat, w.omega, even, forces, limiters)
        even = not even
    torch.cuda.synchronize()
    if plan is not None:
        plan.check()
    assert _close(ours, ref, precision)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_bgk_matches_reference_gpu_kernel(cuda, precision):
    R = ReferenceGpu(precision)
    w, lat, ours, ref = _tgv_pair(24, precision)
    even = True
    for _ in range(12):
        K.collision("BGK", ours, lat, w.omega, even, stream=0)
        R.collision_bgk(ref, lat, w.omega, even)
        even = not even
    torch.cuda.synchronize()
    assert _close(ours, ref, precision)


@pytest.mark.parametrize("kind,lst", CASES)
@pytest.mark.parametrize("is_even", [True, False])
@pytest.mark.parametrize("grid", ["cavity8", "channel"])
def test_bc_kernels_match_reference_gpu_kernels(cuda, kind, lst, is_even, grid):
    g = _grid(grid)
    if len(g[f"{lst}.k"]) == 0:
        pytest.skip(f"no {lst} list in {grid}")
    _, d = _random_state(g, "f64")
    lat = K.DeviceLattice.from_arrays(g)
    ours = torch.from_numpy(d).cuda()
    ref = ours.clone()
    k = torch.from_numpy(g[f"{lst}.k"].astype(np.int32)).cuda()
    q = torch.from_numpy(g[f"{lst}.q"].astype(np.float64)).cuda()
    vel = ([torch.from_numpy(g[f"velocity.{c}"].astype(np.float64)).cuda() for c in ("vx", "vy", "vz")]
           if lst == "velocity" else [None] * 3)
    K.bc_post(kind, ours, lat, k, q, 1.7, is_even, *vel, stream=0)
    ReferenceGpu("f64").bc_post(kind, ref, lat, k, q, 1.7, is_even, *vel)
    torch.cuda.synchronize()
    assert _close(ours, ref, "f64")


@pytest.mark.parametrize("kind", [_lib.BC_NOSLIP_INTERPOLATED, _lib.BC_SLIP])
def test_bc_kernels_on_fractional_q_match_reference_gpu_kernels(cuda, kind):
    """The solid sphere's geometry list (q from the ray-sphere intersection)."""
    g = _grid("sphere_channel")
    _, d = _random_state(g, "f64")
    lat = K.DeviceLattice.from_arrays(g)
    ours = torch.from_numpy(d).cuda()
    ref = ours.clone()
    k = torch.from_numpy(g["geometry.k"].astype(np.int32)).cuda()
    q = torch.from_numpy(g["geometry.q"].astype(np.float64)).cuda()
    for ev in (True, False):
        K.bc_post(kind, ours, lat, k, q, 1.7, ev, stream=0)
        ReferenceGpu("f64").bc_post(kind, ref, lat, k, q, 1.7, ev)
    torch.cuda.synchronize()
    assert _close(ours, ref, "f64")


@pytest.mark.parametrize("is_even", [True, False])
@pytest.mark.parametrize("coarse_to_fine", [True, False])
def test_interface_kernels_match_reference_gpu_kernels(cuda, coarse_to_fine, is_even):
    """Cells that write disjoint nodes, a third of them with zero offset."""
    c = case(3)
    latc, latf = K.DeviceLattice.from_arrays(c["gc"]), K.DeviceLattice.from_arrays(c["gf"])
    tag = "cf" if coarse_to_fine else "fc"

    def t(a, dt=None):
        a = np.ascontiguousarray(a)
        return torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).to("cuda", dt)
    cells_c, cells_f = t(c[f"coarse_{tag}"]), t(c[f"fine_{tag}"])
    off = [t(o, torch.float64) for o in c["off"]]
    out = []
    for side in ("ours", "ref"):
        dC, dF = t(c["distC"], torch.float64), t(c["distF"], torch.float64)
        if side == "ref":
            ReferenceGpu("f64").scale(coarse_to_fine, dC, dF, latc, latf, is_even, cells_c, cells_f, c["omegaC"],
                                      c["omegaF"], *off)
        else:
            a = _lib.ScalingArgs()
            a.distributionsCoarse, a.distributionsFine = dC.data_ptr(), dF.data_ptr()
            a.neighborXcoarse, a.neighborYcoarse, a.neighborZcoarse = (x.data_ptr() for x in (
                latc.neighborX, latc.neighborY, latc.neighborZ))
            a.neighborXfine, a.neighborYfine, a.neighborZfine = (x.data_ptr() for x in (
                latf.neighborX, latf.neighborY, latf.neighborZ))
            a.numberOfLBnodesCoarse, a.numberOfLBnodesFine = latc.N, latf.N
            a.isEvenTimestep = int(is_even)
            a.coarseCells, a.fineCells = cells_c.data_ptr(), cells_f.data_ptr()
            a.numberOfCells = cells_c.numel()
            a.omegaCoarse, a.omegaFine = c["omegaC"], c["omegaF"]
            a.offsetX, a.offsetY, a.offsetZ = (o.data_ptr() for o in off)
            fn = _lib.lib().vfb_scale_coarse_to_fine if coarse_to_fine else _lib.lib().vfb_scale_fine_to_coarse
            _lib.check(fn(_lib.FP64, a, None))
        torch.cuda.synchronize()
        out.append((dC, dF))
    for g, r in zip(*out):
        assert _close(g, r, "f64")


def _event_ms(fn, reps=10, warmup=3):
    """Mean device time of one call, CUDA events on the legacy stream, where
    both sides launch."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    s = torch.cuda.default_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def test_same_device_baseline_timing(cuda):
    """Event-timed: the reference's kernels and the library's on the same
    arrays.  Both sides leave the populations in a valid state after every
    launch (parity alternates), so each timed loop is a real time-stepping
    loop; the inputs (1.8 GB at TGV 256^3 FP32) exceed L2."""
    rows = []

    def row(name, units, unit, ours_ms, ref_ms, bytes_per_unit):
        r = {"kernel": name, unit: int(units), "ours_ms": round(ours_ms, 4), "reference_ms": round(ref_ms, 4),
             "speedup": round(ref_ms / ours_ms, 3), "bytes_per_unit": bytes_per_unit,
             "ours_gbs": round(units * bytes_per_unit / ours_ms / 1e6, 1),
             "reference_gbs": round(units * bytes_per_unit / ref_ms / 1e6, 1)}
        rows.append(r)
        print(json.dumps(r), flush=True)

    # collisions, TGV 256^3
    for precision, n in (("f32", 256), ("f64", 256)):
        dt = TORCH_REAL[precision]
        s = 4 if precision == "f32" else 8
        w = taylor_green(n)
        lat = K.DeviceLattice.from_arrays(w.grid)
        dist = K.new_distributions(lat, dt)
        fields = [torch.from_numpy(a).to("cuda", dt) for a in (w.rho, w.vx, w.vy, w.vz)]
        for ev in (False, True):
            K.init_equilibrium(dist, lat, *fields, ev)
        del fields
        R = ReferenceGpu(precision)
        forces = torch.zeros(3, dtype=dt, device="cuda")
        limiters = torch.tensor(LIMITERS, dtype=dt, device="cuda")
        plan = K.CollisionPlan(dt, lat)
        st = {"even": True}

        def step(fn):
            def go():
                fn(st["even"])
                st["even"] = not st["even"]
            return go
        nf = lat.numberOfFluidNodes
        for kernel in ("K17", "BGK"):
            ours = _event_ms(step(lambda ev: K.collision(kernel, dist, lat, w.omega, ev, plan=plan, stream=0)))
            if kernel == "K17":
                ref = _event_ms(step(lambda ev: R.collision_k17(dist, lat, w.omega, ev, forces, limiters)))
            else:
                ref = _event_ms(step(lambda ev: R.collision_bgk(dist, lat, w.omega, ev)))
            row(f"{kernel.lower()}_{precision}_tgv{n}", nf, "nodes", ours, ref, 54 * s + 16)
        plan.check()
        plan.close()
        del dist, plan, lat, w
        torch.cuda.empty_cache()

    # BC kernels on the 256^3 cavity walls, FP32
    g = cavity_grid(256)
    lat = K.DeviceLattice.from_arrays(g)
    dist = K.new_distributions(lat, torch.float32)
    dist.uniform_(-1e-3, 1e-3)
    k = torch.from_numpy(g["velocity.k"].astype(np.int32)).cuda()
    q = torch.from_numpy(g["velocity.q"].astype(np.float32)).cuda()
    v = [torch.from_numpy(g[f"velocity.{c}"].astype(np.float32)).cuda() for c in ("vx", "vy", "vz")]
    active = int((g["velocity.q"].reshape(27, -1) >= 0).sum())
    R = ReferenceGpu("f32")
    for kind, name in ((_lib.BC_VELOCITY_INTERPOLATED, "velocity_bc"), (_lib.BC_NOSLIP_INTERPOLATED, "noslip_bc")):
        vel = v if kind == _lib.BC_VELOCITY_INTERPOLATED else [None] * 3
        ours = _event_ms(lambda: K.bc_post(kind, dist, lat, k, q, 1.9, True, *vel, stream=0))
        ref = _event_ms(lambda: R.bc_post(kind, dist, lat, k, q, 1.9, True, *vel))
        extra = 12 if kind == _lib.BC_VELOCITY_INTERPOLATED else 0
        row(f"{name}_fp32_cavity256", k.numel(), "bc_nodes", ours, ref,
            round(27 * 4 + 27 * 4 + 4 + extra + active * 4 / k.numel(), 2))
    del dist, lat
    torch.cuda.empty_cache()

    # interface kernels, FP32: 2 x 128^2 coarse-to-fine and 128^2 fine-to-coarse cells
    gc, gf, cells = interface_planes(128, 256)
    latc, latf = K.DeviceLattice.from_arrays(gc), K.DeviceLattice.from_arrays(gf)
    dc, df = K.new_distributions(latc, torch.float32), K.new_distributions(latf, torch.float32)
    dc.uniform_(-1e-3, 1e-3)
    df.uniform_(-1e-3, 1e-3)
    for tag in ("cf", "fc"):
        cc, ff = (torch.from_numpy(x.view(np.int32)).cuda() for x in cells[tag])
        zeros = torch.zeros(cc.numel(), dtype=torch.float32, device="cuda")
        a = _lib.ScalingArgs()
        a.distributionsCoarse, a.distributionsFine = dc.data_ptr(), df.data_ptr()
        a.neighborXcoarse, a.neighborYcoarse, a.neighborZcoarse = (x.data_ptr() for x in (
            latc.neighborX, latc.neighborY, latc.neighborZ))
        a.neighborXfine, a.neighborYfine, a.neighborZfine = (x.data_ptr() for x in (
            latf.neighborX, latf.neighborY, latf.neighborZ))
        a.numberOfLBnodesCoarse, a.numberOfLBnodesFine = latc.N, latf.N
        a.isEvenTimestep = 1
        a.coarseCells, a.fineCells = cc.data_ptr(), ff.data_ptr()
        a.numberOfCells = cc.numel()
        a.omegaCoarse, a.omegaFine = 1.9, 1.85
        a.offsetX = a.offsetY = a.offsetZ = zeros.data_ptr()
        fn = _lib.lib().vfb_scale_coarse_to_fine if tag == "cf" else _lib.lib().vfb_scale_fine_to_coarse
        ours = _event_ms(lambda: _lib.check(fn(_lib.FP32, a, None)))
        ref = _event_ms(lambda: R.scale(tag == "cf", dc, df, latc, latf, True, cc, ff, 1.9, 1.85, zeros, zeros,
                                        zeros))
        write = 8 * 27 * 4 if tag == "cf" else 27 * 4
        row("coarse_to_fine_fp32" if tag == "cf" else "fine_to_coarse_fp32", cc.numel(), "cells", ours, ref,
            8 * 27 * 4 + write + 20)

    by = {r["kernel"]: r for r in rows}
    # the collision kernels are the path's hot kernels: the library must beat the reference there
    for name in ("k17_f32_tgv256", "bgk_f32_tgv256", "k17_f64_tgv256", "bgk_f64_tgv256"):
        assert by[name]["speedup"] > 1.0, by[name]
