"""Benchmark of the LBM time step: D3Q27 K17 cumulant MLUPS on the periodic
Taylor-Green vortex, and its fraction of the HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 512]
                    [--storage fp32|fp64|fp16|bf16] [--impl reference]

One step is one fused collide + stream launch over all n^3 fluid nodes (the
reference's K17CompressibleNavierStokes::runOnIndices on one level).  Inputs
(14.7 GB of FP32 populations at n = 512) are far larger than the 126 MB L2,
so no flush is needed between timed steps.  Multi-GPU runs are independent
replicas (the single-GPU step has no halo exchange); value is the sum of all
ranks' node updates over the slowest rank's time.

Rank 0 prints one JSON line.  ``--impl reference`` times the reference's own
CPU K17 path (oracle/_ref, OpenMP on all host cores) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "D3Q27 cumulant MLUPS & % HBM roofline; FP16-store vs FP32 at stated L2 err"
STORAGE_BYTES = {"fp32": 4, "fp64": 8, "fp16": 2, "bf16": 2, "fx16": 2, "fx16w": 2}
FALLBACK_HBM_GBS = 6650.0


def algorithmic_bytes_per_node(storage: str) -> int:
    """27 population reads + 27 writes, plus the node's fluid-index entry and
    its three neighbour-array entries (the four neighbour-of-neighbour
    lookups are cache hits)."""
    return 54 * STORAGE_BYTES[storage] + 16


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def init_distributed(backend: str = "nccl"):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE); NCCL
    carries only the barriers and the max-over-ranks timing (the replicas
    exchange no data).  The short timeout makes a rank that never arrives end
    the others with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, slowest_ms: float) -> float:
    """Updates per second of all replicas together, over the slowest rank's time
    (weak scaling: every rank processes the same number of units)."""
    return units_per_rank * world / (slowest_ms * 1e-3)


# --------------------------------------------------------------------------- #
# reference arm: the reference's CPU K17 path on the host cores
# --------------------------------------------------------------------------- #
def host_cpu() -> dict:
    """Thread count and CPU model of this host (the cores the CPU legs use)."""
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    model = None
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"threads": threads, "model": model}


def cpu_reference_block(n: int, u0: float):
    """The reference CPU path's EsoSplit block holding the n^3 Taylor-Green
    vortex, or None when oracle/_ref is absent."""
    from oracle.pyoracle import Reference, ref_available
    if not ref_available("f32"):
        return None
    return Reference("f32").cpu_tgv_block(n, u0)


def run_reference(args, world, rank):
    """The reference's CPU K17 loop (EsoSplit storage, FP32, OpenMP on every
    host thread) on the same Taylor-Green n^3 workload: one block created
    once, W untimed passes, then K passes each timed as one step."""
    if rank != 0:
        return 0
    cpu = host_cpu()
    omega = 1.0 / (3.0 * (args.u0 * (args.n / (2 * math.pi)) / 1600.0) + 0.5)
    t0 = time.time()
    block = cpu_reference_block(args.n, args.u0)
    if block is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference tree absent)"}))
        return 0
    setup_s = time.time() - t0
    for _ in range(args.warmup):
        block.run(1, omega)
    secs = [block.run(1, omega) for _ in range(args.steps)]
    block.close()
    nodes = args.n ** 3
    value = nodes * len(secs) / sum(secs) / 1e6
    sample = (f"the whole {args.n}^3 Taylor-Green block in the reference CPU K17 loop (EsoSplit storage, FP32), "
              f"{args.steps} timed passes after {args.warmup} warm-up passes on the same block, OpenMP on "
              f"{cpu['threads']} threads ({cpu['model']})")
    line = {"metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": f"taylor-green {args.n}^3 periodic, K17 cumulant, fp32 storage",
                       "fluid_nodes": nodes, "same_config": True, "setup_s": round(setup_s, 1),
                       "cpu_threads": cpu["threads"], "cpu_model": cpu["model"]},
            "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": cpu["threads"], "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def cpu_baseline(n: int, u0: float, omega: float, seconds_target: float = 12.0):
    """The reference CPU K17 path on the host cores for about
    `seconds_target` seconds (rank 0, one GPU only): the same n^3
    Taylor-Green block as the reference arm, created once, one warm-up pass,
    then whole passes until the target time is reached."""
    cpu = host_cpu()
    try:
        block = cpu_reference_block(n, u0)
    except Exception as e:  # the baseline must not sink the GPU result
        return {"value": None, "unit": "MLUPS", "cores": cpu["threads"], "kind": "reference",
                "sample": f"failed: {e}"}
    if block is None:
        return {"value": None, "unit": "MLUPS", "cores": cpu["threads"], "kind": "reference",
                "sample": "oracle/_ref not built"}
    first = block.run(1, omega)
    passes = int(max(1, min(1000, seconds_target / max(first, 1e-3))))
    sec = block.run(passes, omega)
    block.close()
    return {"value": n ** 3 * passes / sec / 1e6, "unit": "MLUPS", "cores": cpu["threads"], "kind": "reference",
            "sample": f"reference CPU K17 loop (EsoSplit, FP32) on the whole {n}^3 Taylor-Green block, {passes} "
                      f"passes after one warm-up pass, {sec:.1f} s, OpenMP on {cpu['threads']} threads "
                      f"({cpu['model']})"}


def run_gpu(args, world, rank, local):
    import numpy as np
    import torch

    from virtualfluids_b200 import kernels as K
    from virtualfluids_b200.workloads import taylor_green

    dtype = {"fp32": torch.float32, "fp64": torch.float64, "fp16": torch.float16, "bf16": torch.bfloat16,
             "fx16": torch.int16}[
        args.storage]
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    t_setup = time.time()
    w = taylor_green(args.n)
    g = w.grid
    lat = K.DeviceLattice.from_arrays(g, device)
    n_fluid = lat.numberOfFluidNodes
    cd = K.compute_dtype(dtype)
    # host copies of the initial fields in pinned memory (the user's input)
    host_fields = [torch.from_numpy(a.astype(np.float64 if cd == torch.float64 else np.float32)).pin_memory()
                   for a in (w.rho, w.vx, w.vy, w.vz)]
    del w
    dist = K.new_distributions(lat, dtype, device)
    dev_fields = [h.to(device, non_blocking=True) for h in host_fields]
    stream = torch.cuda.current_stream(device)
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *dev_fields, ev)
    del dev_fields
    torch.cuda.synchronize(device)
    setup_s = time.time() - t_setup

    omega = 1.0 / (3.0 * (args.u0 * (args.n / (2 * math.pi)) / 1600.0) + 0.5)
    plan = K.CollisionPlan(dtype, lat, stream=stream) if args.path == "planned" else None
    plan_stats = plan.stats() if plan is not None else None
    even = True
    # the generic (index-chain) kernel, for comparison only
    generic_ms = None
    if plan is not None:
        for _ in range(2):
            K.collision("K17", dist, lat, omega, even, stream=stream)
            even = not even
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(4):
            K.collision("K17", dist, lat, omega, even, stream=stream)
            even = not even
        g1.record(stream)
        torch.cuda.synchronize(device)
        generic_ms = g0.elapsed_time(g1) / 4
    for _ in range(args.warmup):
        K.collision("K17", dist, lat, omega, even, stream=stream, plan=plan)
        even = not even
    torch.cuda.synchronize(device)

    # --- device-resident timing (value) ---------------------------------------
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize(device)
    with ClockSampler(local) as clocks:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for i in range(args.steps):
            starts[i].record(stream)
            K.collision("K17", dist, lat, omega, even, stream=stream, plan=plan)
            stops[i].record(stream)
            even = not even
        t1.record(stream)
        torch.cuda.synchronize(device)
    barrier(world)
    total_ms = max_over_ranks(world, t0.elapsed_time(t1))
    launch_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    avg_launch_ms = sum(launch_ms) / len(launch_ms)
    clk = clocks.summary()

    if plan is not None:
        plan.check(stream)
        lane_nodes = plan_stats["lane_nodes"]
        plan.close()
    else:
        lane_nodes = 0
    del dist, plan
    torch.cuda.empty_cache()

    # --- end to end through the public API with host buffers -------------------
    # Simulation (the C++ schedule behind vfb_sim_*): the timed region holds
    # the H2D of the initial fields from host arrays, the initialisation of
    # both parities, K time steps and the D2H of the resulting fields; the
    # per-step bytes are the totals divided by K
    from virtualfluids_b200.grid import MultipleGridBuilder
    from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation
    b = MultipleGridBuilder()
    d = 2.0 * math.pi / args.n
    b.addCoarseGrid(-math.pi, -math.pi, -math.pi, math.pi, math.pi, math.pi, d)
    b.setPeriodicBoundaryCondition(True, True, True)
    b.buildGrids(True)
    p = Parameter()
    p.set_storage(args.storage)
    p.set_viscosity_LB(args.u0 * (args.n / (2 * math.pi)) / 1600.0)
    sim = Simulation(p, b, BoundaryConditionFactory(), stream=stream.cuda_stream)
    real = np.float64 if cd == torch.float64 else np.float32
    # the user's host buffers are pinned (page-locked), as for any fast copy
    fields_np = [h.numpy().astype(real, copy=False) for h in host_fields]
    out_pinned = [torch.empty(lat.N, dtype=cd).pin_memory() for _ in range(4)]
    out_np = [t.numpy() for t in out_pinned]
    barrier(world)
    torch.cuda.synchronize(device)
    e0, ea, eb, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
    e0.record(stream)
    sim.init_level(0, *fields_np)
    ea.record(stream)
    sim.run(args.steps)
    eb.record(stream)
    out_host = sim.macroscopic(0, out=out_np)
    e1.record(stream)
    torch.cuda.synchronize(device)
    barrier(world)
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1))
    # where the end-to-end time goes (rank 0's events)
    e2e_parts = {"h2d_and_init_ms": e0.elapsed_time(ea), "steps_ms": ea.elapsed_time(eb),
                 "macroscopic_and_d2h_ms": eb.elapsed_time(e1)}
    h2d = sum(a.nbytes for a in fields_np)
    d2h = sum(a.nbytes for a in out_host)
    finite = bool(np.isfinite(out_host[1][g["fluid"][:1000]]).all())
    sim.close()

    if rank != 0:
        return 0
    value = whole_job_rate(n_fluid * args.steps, world, total_ms) / 1e6
    e2e_value = whole_job_rate(n_fluid * args.steps, world, e2e_ms) / 1e6
    bpn = algorithmic_bytes_per_node(args.storage)
    achieved = bpn * n_fluid / (avg_launch_ms * 1e-3) / 1e9
    peak, peak_kind = hbm_peak()
    traffic = None
    prof = ROOT / "profiles" / "traffic.json"
    if prof.exists():
        try:
            traffic = json.loads(prof.read_text()).get(f"k17_{args.storage}_{args.n}")
        except Exception:
            traffic = None
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp32": "f32", "fp64": "f64", "fp16": "f16-store/f32", "bf16": "bf16-store/f32",
                                         "fx16": "fx16-store/f32"}[
            args.storage],
        "data": "synthetic",
        "config": {"workload": f"taylor-green {args.n}^3 periodic, K17 cumulant, {args.storage} storage",
                   "fluid_nodes_per_gpu": n_fluid, "stored_nodes_per_gpu": lat.N, "omega": omega,
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (no flush)",
                   "setup_s": round(setup_s, 1), "finite": finite, "path": args.path, "plan": plan_stats,
                   "generic_kernel_mlups": (n_fluid / (generic_ms * 1e-3) / 1e6) if generic_ms else None},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "bytes_per_node": bpn, "peak_kind": f"of {peak_kind}",
                     "avg_launch_ms": avg_launch_ms},
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps, "breakdown": e2e_parts},
        "gpu_launches": args.steps * (2 if lane_nodes else 1),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.n, args.u0, omega)
    if world == 1 and args.precision_steps > 0 and args.storage == "fp32":
        line["precision_form"] = precision_form_record(args, value, device)
    print(json.dumps(line), flush=True)
    return 0


def precision_form_record(args, fp32_value, device):
    """The precision form beside the FP32 bench value: the FX16 storage's
    throughput on the same K planned steps of the same workload, its ratio to
    the FP32 value of this run, and its L2 velocity error against FP64 storage
    after --precision-steps steps (both run through the Simulation API from
    the same initial field; the FP64 path matches the FP64 oracle to 1e-12 in
    the GPU tests)."""
    import numpy as np
    import torch

    from virtualfluids_b200 import kernels as K
    from virtualfluids_b200.grid import MultipleGridBuilder
    from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation
    from virtualfluids_b200.workloads import taylor_green

    w = taylor_green(args.n)
    g = w.grid
    lat = K.DeviceLattice.from_arrays(g, device)
    dist = K.new_distributions(lat, torch.int16, device)
    fields = [torch.from_numpy(a).to(device, torch.float32) for a in (w.rho, w.vx, w.vy, w.vz)]
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    del fields
    stream = torch.cuda.current_stream(device)
    plan = K.CollisionPlan(torch.int16, lat, stream=stream)
    even = True
    for _ in range(args.warmup):
        K.collision("K17", dist, lat, w.omega, even, stream=stream, plan=plan)
        even = not even
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        K.collision("K17", dist, lat, w.omega, even, stream=stream, plan=plan)
        even = not even
    e1.record(stream)
    torch.cuda.synchronize(device)
    plan.check(stream)
    plan.close()
    ms = e0.elapsed_time(e1)
    value = lat.numberOfFluidNodes * args.steps / (ms * 1e-3) / 1e6
    bpn = algorithmic_bytes_per_node("fx16")
    del dist, plan, lat
    torch.cuda.empty_cache()

    fl = g["fluid"]
    b = MultipleGridBuilder()
    d = 2.0 * math.pi / args.n
    b.addCoarseGrid(-math.pi, -math.pi, -math.pi, math.pi, math.pi, math.pi, d)
    b.setPeriodicBoundaryCondition(True, True, True)
    b.buildGrids(True)
    nu = args.u0 * (args.n / (2 * math.pi)) / 1600.0
    u = {}
    for storage in ("fp64", "fx16"):
        p = Parameter()
        p.set_storage(storage)
        p.set_viscosity_LB(nu)
        sim = Simulation(p, b, BoundaryConditionFactory())
        sim.init_level(0, w.rho, w.vx, w.vy, w.vz)
        sim.run(args.precision_steps)
        _, vx, vy, vz = sim.macroscopic(0)
        u[storage] = [a[fl].astype(np.float64) for a in (vx, vy, vz)]
        sim.close()
    num = math.sqrt(sum(float(np.sum((a - r) ** 2)) for a, r in zip(u["fx16"], u["fp64"])))
    den = math.sqrt(sum(float(np.sum(r ** 2)) for r in u["fp64"]))
    return {"storage": "fx16", "value": value, "unit": "MLUPS", "ratio_vs_fp32": value / fp32_value,
            "bytes_per_node": bpn, "ms_per_step": ms / args.steps,
            "l2_velocity_err_vs_fp64": num / den, "l2_steps": args.precision_steps,
            "format": "int16 q, f_d - w_d = q w_d 2^-17 (FP32 arithmetic)"}


def format_study(args):
    """Which 16-bit storage format reaches the precision target: the
    Taylor-Green case (n^3, --steps steps, default 2000) run by the FP32
    planned kernel with the stored populations rounded to a candidate format
    after every step (what storing in that format does to FP32 arithmetic),
    against FP64 storage.  Formats: IEEE FP16 (x 2^12), fixed point of
    (f - w)/w over +-R (R = 1, 0.5, 0.25: the last is FX16), and floating
    formats of (f - w)/w with p significant bits (FP16C-like 1/4/11 and
    1/3/12).  The real FX16 kernel is run beside its emulation.  One JSON line."""
    import numpy as np
    import torch

    from virtualfluids_b200 import kernels as K
    from virtualfluids_b200.workloads import taylor_green

    steps = args.steps if args.steps != 50 else 2000
    dev = torch.device("cuda", 0)
    w = taylor_green(args.n)
    g = w.grid
    lat = K.DeviceLattice.from_arrays(g, dev)
    N = lat.N
    fl = torch.from_numpy(g["fluid"].astype(np.int64)).to(dev)
    W = torch.tensor(K.WEIGHTS, dtype=torch.float32, device=dev)
    fields = [torch.from_numpy(a).to(dev) for a in (w.rho, w.vx, w.vy, w.vz)]

    def rounder(kind, **kw):
        def rnd(dist):
            d = dist.view(27, N)
            for r in range(27):
                x = d[r]
                if kind == "fp16":
                    x.copy_((x * 4096.0).half().float() / 4096.0)
                    continue
                v = x / W[r]
                if kind == "fixed":
                    R = kw["R"]
                    q = torch.clamp(torch.round(v / R * 32768.0), -32768, 32767)
                    x.copy_(q * (R / 32768.0) * W[r])
                else:
                    p, emin, emax = kw["p"], kw["emin"], kw["emax"]
                    _, e = torch.frexp(v)
                    e = torch.clamp(e - 1, min=emin)
                    step = torch.ldexp(torch.ones_like(v), e - (p - 1))
                    top = (2.0 - 2.0 ** (1 - p)) * 2.0 ** emax
                    x.copy_(torch.clamp(torch.round(v / step) * step, -top, top) * W[r])
        return rnd

    def run(dtype, rnd=None):
        dist = K.new_distributions(lat, dtype, dev)
        cd = K.compute_dtype(dtype)
        f = [a.to(cd) for a in fields]
        for ev in (False, True):
            K.init_equilibrium(dist, lat, *f, ev)
        plan = K.CollisionPlan(dtype, lat)
        if rnd:
            rnd(dist)
        even = True
        for _ in range(steps):
            K.collision("K17", dist, lat, w.omega, even, plan=plan)
            if rnd:
                rnd(dist)
            even = not even
        plan.check()
        plan.close()
        _, vx, vy, vz = K.macroscopic(dist, lat, even)
        u = torch.stack([vx[fl], vy[fl], vz[fl]]).double()
        del dist
        torch.cuda.empty_cache()
        return u

    ref = run(torch.float64)
    nref = float(torch.linalg.norm(ref))
    rows = {}
    cases = [("fp32", torch.float32, None), ("fp16_ieee_x4096", torch.float32, rounder("fp16")),
             ("fixed_R1", torch.float32, rounder("fixed", R=1.0)), ("fixed_R0.5", torch.float32, rounder("fixed", R=0.5)),
             ("fixed_R0.25_emulated", torch.float32, rounder("fixed", R=0.25)),
             ("float_p12_e4", torch.float32, rounder("float", p=12, emin=-14, emax=0)),
             ("float_p13_e3", torch.float32, rounder("float", p=13, emin=-6, emax=0)),
             ("fx16_kernel", torch.int16, None), ("fp16_kernel", torch.float16, None)]
    for name, dt, rnd in cases:
        u = run(dt, rnd)
        rows[name] = float(torch.linalg.norm(u - ref)) / nref
        print(json.dumps({name: rows[name]}), file=sys.stderr, flush=True)
    print(json.dumps({"report": "16-bit format study", "workload": f"taylor-green {args.n}^3, K17, FP32 arithmetic",
                      "steps": steps, "l2_velocity_error_vs_fp64": rows}), flush=True)
    return 0


def precision_report(args):
    """The precision form: the Taylor-Green case run for --steps steps with
    every storage format through the same public API; L2 velocity error and
    kinetic-energy error of FP32 / FP16 / BF16 against the FP64 run (itself
    checked against the FP64 oracle at small sizes by the GPU tests), and the
    MLUPS of each.  One JSON line."""
    import numpy as np
    import torch

    from virtualfluids_b200.grid import MultipleGridBuilder
    from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation
    from virtualfluids_b200.workloads import taylor_green

    w = taylor_green(args.n)
    fl = w.grid["fluid"]
    nu = args.u0 * (args.n / (2 * math.pi)) / 1600.0
    b = MultipleGridBuilder()
    d = 2.0 * math.pi / args.n
    b.addCoarseGrid(-math.pi, -math.pi, -math.pi, math.pi, math.pi, math.pi, d)
    b.setPeriodicBoundaryCondition(True, True, True)
    b.buildGrids(True)
    rows, ref = {}, None
    for storage in ("fp64", "fp32", "fp16", "bf16", "fx16", "fx16w"):
        p = Parameter()
        p.set_storage(storage)
        p.set_viscosity_LB(nu)
        sim = Simulation(p, b, BoundaryConditionFactory())
        sim.init_level(0, w.rho, w.vx, w.vy, w.vz)
        ke0 = sim.mass_and_energy(0)[1]
        sim.run(3)
        sim.init_level(0, w.rho, w.vx, w.vy, w.vz)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        sim.run(args.steps)
        e1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        mass, ke, bad = sim.mass_and_energy(0)
        _, vx, vy, vz = [a[fl].astype(np.float64) for a in sim.macroscopic(0)]
        sim.close()
        row = {"mlups": len(fl) * args.steps / (ms * 1e-3) / 1e6, "bytes_per_node": algorithmic_bytes_per_node(storage),
               "kinetic_energy": ke, "kinetic_energy_initial": ke0, "nonfinite": bad}
        if ref is None:
            ref = (vx, vy, vz, ke, ke0)
        else:
            num = np.sqrt(np.sum((vx - ref[0]) ** 2 + (vy - ref[1]) ** 2 + (vz - ref[2]) ** 2))
            den = np.sqrt(np.sum(ref[0] ** 2 + ref[1] ** 2 + ref[2] ** 2))
            row["l2_velocity_error_vs_fp64"] = float(num / den)
            row["kinetic_energy_error_vs_fp64"] = abs(ke - ref[3]) / ref[3]
            row["kinetic_energy_decay_error_vs_fp64"] = abs((ref[4] - ref[3]) - (ke0 - ke)) / max(ref[4] - ref[3], 1e-300)
        rows[storage] = row
    rows["fp16_over_fp32_mlups"] = rows["fp16"]["mlups"] / rows["fp32"]["mlups"]
    rows["bf16_over_fp32_mlups"] = rows["bf16"]["mlups"] / rows["fp32"]["mlups"]
    rows["fx16_over_fp32_mlups"] = rows["fx16"]["mlups"] / rows["fp32"]["mlups"]
    rows["fx16w_over_fp32_mlups"] = rows["fx16w"]["mlups"] / rows["fp32"]["mlups"]
    print(json.dumps({"report": "precision form", "workload": f"taylor-green {args.n}^3 periodic, K17",
                      "steps": args.steps, "reference": "fp64 storage on the GPU", "results": rows}), flush=True)
    return 0


def cavity_report(args):
    """The lid-driven cavity (64^3, FP64, lid u = 0.05 on +z, q = 1/2 walls,
    nu = 0.0032, 2000 steps): the C++ schedule with and without CUDA-graph
    replay (its parity with the FP64 oracle is checked by
    tests/test_gpu_cavity.py).  One JSON line."""
    import numpy as np
    import torch

    from virtualfluids_b200.grid import MultipleGridBuilder, SideType
    from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, Simulation

    n, nu, steps = 64, 0.0032, 2000

    def builder():
        b = MultipleGridBuilder()
        b.addCoarseGrid(0, 0, 0, n - 1, n - 1, n - 1, 1.0)
        b.buildGrids()
        for side in (SideType.MX, SideType.PX, SideType.MY, SideType.PY, SideType.MZ):
            b.setNoSlipBoundaryCondition(side)
        b.setVelocityBoundaryCondition(SideType.PZ, 0.05, 0.0, 0.0)
        return b

    result = {"report": "lid-driven cavity", "workload": f"cavity {n}^3, K17, fp64, lid 0.05, nu {nu}",
              "steps": steps}
    for graphs in (False, True):
        p = Parameter()
        p.set_storage("fp64")
        p.set_viscosity_LB(nu)
        p.use_graphs = graphs
        p.use_bc_epilogue = bool(args.bc_epilogue)
        sim = Simulation(p, builder(), BoundaryConditionFactory())
        g = sim.levels[0]
        zero = np.zeros(len(g["geo"]))
        sim.init_level(0, zero, zero, zero, zero)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        sim.run(steps)
        e1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        key = "graphs" if graphs else "direct_launches"
        result[key] = {"mlups": len(g["fluid"]) * steps / (ms * 1e-3) / 1e6, "ms_per_step": ms / steps}
        if graphs:
            _, vx, vy, vz = sim.macroscopic(0)
            fl = g["fluid"]
            result["max_speed_after_steps"] = float(np.sqrt(vx[fl] ** 2 + vy[fl] ** 2 + vz[fl] ** 2).max())
        sim.close()
    result["graph_speedup"] = result["graphs"]["mlups"] / result["direct_launches"]["mlups"]
    print(json.dumps(result), flush=True)
    return 0


def cube_report(args):
    """The wall-mounted cube in a channel, two levels (coarse 256 x 96 x 96,
    refined box x 48..128, y 24..72, z 0..40, cube of side 16 on the floor at
    x = 64, inlet 0.04 with +-1% seeded noise, pressure outlet, slip top,
    periodic span, nu = 0.04 * 16 / 2000 on the coarse level), grid built by
    the library's builder, stepped by the C++ schedule with graph replay.
    Per storage: NUPS as the reference counts them (steps x sum over levels
    of nodes x 2^level / s, PerformanceMeasurement.cpp:43,63) and fluid-node
    updates per second; for FP32 / FP16 / BF16 / FX16 the L2 velocity error and the
    kinetic-energy error against the FP64 run after --steps coarse steps
    (both levels).  One JSON line."""
    import numpy as np
    import torch

    from virtualfluids_b200.simulation import (BoundaryConditionFactory, NoSlipBC, Parameter, PressureBC, SlipBC,
                                               Simulation)
    from virtualfluids_b200.workloads import wall_mounted_cube

    t0 = time.time()
    levels = wall_mounted_cube()
    build_s = time.time() - t0
    nu = 0.04 * 16 / 2000
    nodes = [len(g["geo"]) for g in levels]
    fluid = [len(g["fluid"]) for g in levels]
    per_step_nodes = sum(n * 2 ** lvl for lvl, n in enumerate(nodes))
    per_step_fluid = sum(n * 2 ** lvl for lvl, n in enumerate(fluid))
    rows, ref = {}, None
    for storage in ("fp64", "fp32", "fp16", "bf16", "fx16", "fx16w"):
        p = Parameter()
        p.set_storage(storage)
        p.set_viscosity_LB(nu)
        p.use_bc_epilogue = bool(args.bc_epilogue)
        bc = BoundaryConditionFactory()
        bc.set_slip_boundary_condition(SlipBC.SlipCompressible)
        bc.set_geometry_boundary_condition(NoSlipBC.NoSlipInterpolatedCompressible)
        bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
        sim = Simulation(p, levels, bc)
        for lvl, g in enumerate(levels):
            zero = np.zeros(len(g["geo"]))
            sim.init_level(lvl, zero, zero, zero, zero)
        sim.run(4)  # warm-up: graph capture of the two-step pattern
        for lvl, g in enumerate(levels):
            zero = np.zeros(len(g["geo"]))
            sim.init_level(lvl, zero, zero, zero, zero)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        sim.run(args.steps)
        e1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        fields = []
        for lvl, g in enumerate(levels):
            fl = g["fluid"]
            _, vx, vy, vz = [a[fl].astype(np.float64) for a in sim.macroscopic(lvl)]
            fields.append((vx, vy, vz, sim.kinetic_energy(lvl)[0], int(sim.mass_and_energy(lvl)[2])))
        saturated = [sim.saturated_populations(lvl) for lvl in range(len(levels))]
        sim.close()
        row = {"nups": per_step_nodes * args.steps / (ms * 1e-3), "fluid_updates_per_s": per_step_fluid * args.steps /
               (ms * 1e-3), "ms_per_coarse_step": ms / args.steps, "nonfinite": sum(f[4] for f in fields),
               "kinetic_energy": [f[3] for f in fields]}
        if storage in ("fx16", "fx16w"):
            # stored deviations clipped at the end of the format's range, per level
            row["saturated_populations"] = saturated
        if ref is None:
            ref = fields
        else:
            num = sum(np.sum((f[0] - r[0]) ** 2 + (f[1] - r[1]) ** 2 + (f[2] - r[2]) ** 2) for f, r in zip(fields, ref))
            den = sum(np.sum(r[0] ** 2 + r[1] ** 2 + r[2] ** 2) for r in ref)
            row["l2_velocity_error_vs_fp64"] = float(np.sqrt(num / den))
            row["kinetic_energy_error_vs_fp64"] = [abs(f[3] - r[3]) / abs(r[3]) if r[3] != 0 else None
                                                   for f, r in zip(fields, ref)]
        rows[storage] = row
    for s16 in ("fp16", "bf16", "fx16", "fx16w"):
        rows[f"{s16}_over_fp32_nups"] = rows[s16]["nups"] / rows["fp32"]["nups"]
    print(json.dumps({"report": "wall-mounted cube, two levels", "workload":
                      "cube channel 256x96x96 + refined box 48..128 x 24..72 x 0..40, cube 16 at x=64, K17",
                      "nodes_per_level": nodes, "fluid_nodes_per_level": fluid, "grid_build_s": build_s,
                      "steps": args.steps, "bc_epilogue": bool(args.bc_epilogue),
                      "reference": "fp64 storage on the GPU", "results": rows}), flush=True)
    return 0


def kernel_report(args):
    """Achieved bandwidth of the other kernels of the step, event-timed, with
    their algorithmic bytes per unit (s = bytes per stored population):
      BGK (planned, TGV n^3):            27 s read + 27 s write + 16 B per node
      velocity BC (interpolated):        27 s read + 27 q (4 B) + 4 B k + 12 B u + active q writes per BC node
      pressure BC (non-equilibrium):     27 s read at the neighbour + 18 s write + 8 B k/kN + 4 B rho per BC node
      coarse to fine / fine to coarse:   8 * 27 s read + 8 * 27 s (CF) or 27 s (FC) write + 20 B per cell
    One JSON line."""
    import numpy as np
    import torch

    from virtualfluids_b200 import _lib
    from virtualfluids_b200 import kernels as K
    from virtualfluids_b200.grid import MultipleGridBuilder, SideType
    from virtualfluids_b200.workloads import cavity_grid, interface_planes, taylor_green

    peak, peak_kind = hbm_peak()
    out = {"report": "kernels", "peak_gbs": peak, "peak_kind": peak_kind, "storage": "fp32", "kernels": {}}

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def record(name, units, bytes_per_unit, ms, unit_name):
        gbs = units * bytes_per_unit / (ms * 1e-3) / 1e9
        out["kernels"][name] = {unit_name: int(units), "bytes_per_unit": bytes_per_unit, "ms": ms, "gbs": gbs,
                                "frac_of_peak": gbs / peak}

    # BGK, planned, TGV
    w = taylor_green(args.n)
    lat = K.DeviceLattice.from_arrays(w.grid)
    dist = K.new_distributions(lat, torch.float32)
    fields = [torch.from_numpy(a).to("cuda", torch.float32) for a in (w.rho, w.vx, w.vy, w.vz)]
    for ev in (False, True):
        K.init_equilibrium(dist, lat, *fields, ev)
    del fields
    plan = K.CollisionPlan(torch.float32, lat)
    state = {"even": True}

    def bgk():
        K.collision("BGK", dist, lat, w.omega, state["even"], plan=plan)
        state["even"] = not state["even"]
    record("bgk_planned_tgv", lat.numberOfFluidNodes, 54 * 4 + 16, timed(bgk), "nodes")
    plan.close()
    del dist, plan, lat, w
    torch.cuda.empty_cache()

    # BC kernels on a cavity (velocity list on all six walls) and a channel (pressure outlet)
    def grid_of(builder):
        return builder.arrays()[0]
    nb = 256
    g = cavity_grid(nb)
    lat = K.DeviceLattice.from_arrays(g)
    dist = K.new_distributions(lat, torch.float32)
    dist.uniform_(-1e-3, 1e-3)
    k = torch.from_numpy(g["velocity.k"]).cuda()
    q = torch.from_numpy(g["velocity.q"].astype(np.float32)).cuda()
    v = [torch.from_numpy(g[f"velocity.{c}"].astype(np.float32)).cuda() for c in ("vx", "vy", "vz")]
    active = int((g["velocity.q"].reshape(27, -1) >= 0).sum())
    n_bc = len(g["velocity.k"])
    ms = timed(lambda: K.bc_post(_lib.BC_VELOCITY_INTERPOLATED, dist, lat, k, q, 1.9, True, *v))
    record(f"velocity_bc_cavity{nb}", n_bc, (27 * 4 + 27 * 4 + 4 + 12) + active * 4 / n_bc, ms, "bc_nodes")
    # the same with the list's location table (as the simulation runs it): 32 B of
    # locations per node in place of the neighbour chain
    locs = K.bc_locations(lat, k)
    ms = timed(lambda: K.bc_post(_lib.BC_VELOCITY_INTERPOLATED, dist, lat, k, q, 1.9, True, *v, locations=locs))
    record(f"velocity_bc_cavity{nb}_location_table", n_bc, (27 * 4 + 27 * 4 + 32 + 12) + active * 4 / n_bc, ms,
           "bc_nodes")
    # the same list split by wall: x faces (consecutive entries a row apart in
    # memory) against y and z faces (consecutive entries adjacent)
    kk = g["velocity.k"]
    qq = g["velocity.q"].reshape(27, n_bc)
    cx, cy = g["coordX"][kk], g["coordY"][kk]
    on_x = (cx == cx.min()) | (cx == cx.max())
    on_y = ((cy == cy.min()) | (cy == cy.max())) & ~on_x
    for face, sel in (("x", on_x), ("y", on_y), ("z", ~on_x & ~on_y)):
        idx = np.flatnonzero(sel)
        fk = torch.from_numpy(kk[idx].astype(np.int32)).cuda()
        fq = torch.from_numpy(np.ascontiguousarray(qq[:, idx]).astype(np.float32).ravel()).cuda()
        fv = [torch.from_numpy(g[f"velocity.{c}"][idx].astype(np.float32)).cuda() for c in ("vx", "vy", "vz")]
        floc = K.bc_locations(lat, fk)
        fa = int((qq[:, idx] >= 0).sum())
        ms = timed(lambda: K.bc_post(_lib.BC_VELOCITY_INTERPOLATED, dist, lat, fk, fq, 1.9, True, *fv,
                                     locations=floc))
        record(f"velocity_bc_cavity{nb}_{face}_faces", len(idx), (27 * 4 + 27 * 4 + 32 + 12) + fa * 4 / len(idx), ms,
               "bc_nodes")
    del dist, lat
    torch.cuda.empty_cache()
    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 255, 127, 127, 1.0)
    b.setPeriodicBoundaryCondition(False, True, True)
    b.buildGrids()
    b.setVelocityBoundaryCondition(SideType.MX, 0.04, 0.0, 0.0)
    b.setPressureBoundaryCondition(SideType.PX, 0.0)
    g = grid_of(b)
    lat = K.DeviceLattice.from_arrays(g)
    dist = K.new_distributions(lat, torch.float32)
    dist.uniform_(-1e-3, 1e-3)
    pk, pkn = (torch.from_numpy(g[f"pressure0.{x}"]).cuda() for x in ("k", "kN"))
    prho = torch.from_numpy(g["pressure0.rho"].astype(np.float32)).cuda()
    ms = timed(lambda: K.bc_pressure(dist, lat, pk, pkn, prho, int(g["pressure0.dir"][0]), True))
    record("pressure_bc_channel256x128x128", len(g["pressure0.k"]), 27 * 4 + 18 * 4 + 12, ms, "bc_nodes")
    del dist, lat
    torch.cuda.empty_cache()

    # interface interpolation: structured coarse-to-fine / fine-to-coarse planes
    # between a coarse 128^3 and a fine 256^3 periodic box
    gc, gf, cells = interface_planes(128, 256)
    latc, latf = K.DeviceLattice.from_arrays(gc), K.DeviceLattice.from_arrays(gf)
    dc, df = K.new_distributions(latc, torch.float32), K.new_distributions(latf, torch.float32)
    dc.uniform_(-1e-3, 1e-3)
    df.uniform_(-1e-3, 1e-3)
    keep = []

    def dev(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        keep.append(t)
        return t.data_ptr()
    for tag, fn, write in (("cf", _lib.lib().vfb_scale_coarse_to_fine, 8 * 27 * 4),
                           ("fc", _lib.lib().vfb_scale_fine_to_coarse, 27 * 4)):
        coarse, fine = cells[tag]
        n = len(coarse)
        zeros = np.zeros(n, np.float32)
        a = _lib.ScalingArgs()
        a.distributionsCoarse, a.distributionsFine = dc.data_ptr(), df.data_ptr()
        a.neighborXcoarse, a.neighborYcoarse, a.neighborZcoarse = (latc.neighborX.data_ptr(), latc.neighborY.data_ptr(),
                                                                   latc.neighborZ.data_ptr())
        a.neighborXfine, a.neighborYfine, a.neighborZfine = (latf.neighborX.data_ptr(), latf.neighborY.data_ptr(),
                                                             latf.neighborZ.data_ptr())
        a.numberOfLBnodesCoarse, a.numberOfLBnodesFine = latc.N, latf.N
        a.isEvenTimestep = 1
        a.coarseCells, a.fineCells = dev(coarse.view(np.int32)), dev(fine.view(np.int32))
        a.numberOfCells = n
        a.omegaCoarse, a.omegaFine = 1.9, 1.85
        a.offsetX = a.offsetY = a.offsetZ = dev(zeros)
        ms = timed(lambda: _lib.check(fn(_lib.FP32, a, None)))
        name = "coarse_to_fine_cells" if tag == "cf" else "fine_to_coarse_cells"
        record(name, n, 8 * 27 * 4 + write + 20, ms, "cells")
        # the same cells with their node blocks read from tables (vfb_scaling_blocks, as the simulation builds
        # them once at setup) instead of walked through the neighbour arrays: 2 x 27 indices more per cell
        bc = torch.empty(27 * n, dtype=torch.int32, device="cuda")
        bf = torch.empty(27 * n, dtype=torch.int32, device="cuda")
        keep += [bc, bf]
        for cells_ptr, lat_, out_ in ((a.coarseCells, latc, bc), (a.fineCells, latf, bf)):
            _lib.check(_lib.lib().vfb_scaling_blocks(cells_ptr, n, lat_.neighborX.data_ptr(), lat_.neighborY.data_ptr(),
                                                     lat_.neighborZ.data_ptr(), out_.data_ptr(), None))
        a.coarseBlocks, a.fineBlocks = bc.data_ptr(), bf.data_ptr()
        ms = timed(lambda: _lib.check(fn(_lib.FP32, a, None)))
        record(name + "_block_tables", n, 8 * 27 * 4 + write + 20 + 2 * 27 * 4, ms, "cells")
    print(json.dumps(out), flush=True)
    return 0


def adjoint_report(args):
    """The adjoint form: the channel of 128 x 64 x 64 nodes (12^3 cube at x =
    40, parabolic inlet profile with +-2% noise, pressure outlet, no-slip
    walls, g = (1e-6, 0, 0), nu = 0.02), K17, T = --steps (default 1000) time
    steps, objective J = mean u_x over the 16^3 box x in [80, 96).  Per
    storage (FP32, FP64): the plain forward step through the Simulation API
    (graph replay), then for two schedules the adjoint's forward pass and its
    backward pass, all event-timed per step, with the backward / forward
    ratio: "checkpointed" keeps a state every 32 steps and recomputes each
    segment with tapes backwards; "taped" (checkpoint interval = T, when its
    tapes fit in device memory) records the tapes in the forward pass and
    recomputes nothing.  One JSON line."""
    import numpy as np
    import torch

    from virtualfluids_b200.adjoint import FlowProblem
    from virtualfluids_b200.simulation import BoundaryConditionFactory, NoSlipBC, Parameter, PressureBC, Simulation
    from virtualfluids_b200.workloads import adjoint_channel, inlet_entries, inlet_profile, initial_fields, objective_box

    steps = args.steps if args.steps != 50 else 1000
    force = (1e-6, 0.0, 0.0)
    rows = {}
    for storage in ("fp32", "fp64"):
        p = Parameter()
        p.set_storage(storage)
        p.set_viscosity_LB(0.02)
        p.set_forcing(*force)
        bc = BoundaryConditionFactory()
        bc.set_geometry_boundary_condition(NoSlipBC.NoSlipInterpolatedCompressible)
        bc.set_pressure_boundary_condition(PressureBC.PressureNonEquilibriumCompressible)
        sim = Simulation(p, adjoint_channel(), bc)
        g = sim.levels[0]
        nodes, w = objective_box(g, 80, 96, 24, 40, 24, 40)
        prof = inlet_profile(g)
        stream = torch.cuda.current_stream()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        sim.init_level(0, *initial_fields(g))
        sim.run(4)
        torch.cuda.synchronize()
        ev[0].record(stream)
        sim.run(steps)
        ev[1].record(stream)
        torch.cuda.synchronize()
        fwd = ev[0].elapsed_time(ev[1]) / steps
        row = {"forward_ms_per_step": fwd, "fluid_nodes": len(g["fluid"])}
        # tape and BC records of one segment of T steps (27 values per fluid node, BC node and step)
        real = 8 if storage == "fp64" else 4
        bc_nodes = len(g["velocity.k"]) + len(g["geometry.k"]) + int(np.sum(g["pressure.count"]))
        tape_bytes = 27 * real * steps * (len(g["fluid"]) + bc_nodes)
        free = torch.cuda.mem_get_info()[0]
        schedules = [("checkpointed", 32)]
        if tape_bytes < 0.85 * free:
            schedules.append(("taped", steps))
        else:
            row["taped"] = {"skipped": f"tapes of {tape_bytes / 1e9:.1f} GB exceed 85% of the free "
                                       f"{free / 1e9:.1f} GB"}
        for name, interval in schedules:
            pb = FlowProblem(sim, inlet_entries(g), initial_fields(g), steps, interval, nodes, (w, None, None))
            pb.evaluate(prof, force)  # warm-up: allocations, first launches, segment graphs
            pb.gradient(1.0)
            sim.init_level(0, *initial_fields(g))
            torch.cuda.synchronize()
            ev[2].record(stream)
            J = sim.adjoint_forward(steps, interval, nodes, w)
            ev[3].record(stream)
            ev[4].record(stream)
            dv, df = sim.adjoint_backward(1.0)
            ev[5].record(stream)
            torch.cuda.synchronize()
            afwd = ev[2].elapsed_time(ev[3]) / steps
            bwd = ev[4].elapsed_time(ev[5]) / steps
            row[name] = {"checkpoint_interval": interval, "schedule": sim.adjoint_schedule(),
                         "adjoint_forward_ms_per_step": afwd, "adjoint_backward_ms_per_step": bwd,
                         "backward_over_forward": bwd / fwd, "gradient_over_forward": (afwd + bwd) / fwd,
                         "J": J, "dJ_dg": [float(x) for x in df],
                         "dJ_dinlet_norm": float(np.linalg.norm(dv[0][inlet_entries(g)]))}
            if name == "taped":
                row[name]["tape_gb"] = tape_bytes / 1e9
        rows[storage] = row
        sim.close()
        del sim
        torch.cuda.empty_cache()
    print(json.dumps({"report": "adjoint form", "workload": "channel 128x64x64, 12^3 cube at x=40, parabolic inlet "
                      "(peak 0.04, +-2% noise), pressure outlet, no-slip walls, g=(1e-6,0,0), nu=0.02, K17",
                      "steps": steps, "objective": "mean u_x over x in [80,96), 16^3 box",
                      "results": rows}), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--u0", type=float, default=0.05)
    ap.add_argument("--storage", default="fp32", choices=sorted(STORAGE_BYTES))
    ap.add_argument("--path", default="planned", choices=["planned", "generic"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision-steps", type=int, default=2000,
                    help="steps of the FX16-vs-FP64 error in the bench line's precision_form record (0: skip it)")
    ap.add_argument("--kernel-report", action="store_true",
                    help="bandwidth of the BGK, BC and interface kernels (not a bench line)")
    ap.add_argument("--cavity-report", action="store_true",
                    help="lid-driven cavity 64^3 FP64: graph replay vs direct launches (not a bench line)")
    ap.add_argument("--bc-epilogue", type=int, default=0, choices=[0, 1],
                    help="reports: 1 lets the planned collision apply the wall nodes' post-collision BCs, "
                         "0 (default) runs every BC entry in the separate BC launches")
    ap.add_argument("--cube-report", action="store_true",
                    help="wall-mounted cube on two levels: NUPS per storage and errors against FP64 (not a bench line)")
    ap.add_argument("--precision-report", action="store_true",
                    help="run every storage format --steps steps and report errors against FP64 (not a bench line)")
    ap.add_argument("--format-study", action="store_true",
                    help="L2 error of candidate 16-bit storage formats at TGV n^3 (not a bench line)")
    ap.add_argument("--adjoint-report", action="store_true",
                    help="adjoint channel 128x64x64: forward, adjoint forward and backward step times (not a bench line)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.precision_report:
        return precision_report(args)
    if args.cavity_report:
        return cavity_report(args)
    if args.cube_report:
        return cube_report(args)
    if args.kernel_report:
        return kernel_report(args)
    if args.adjoint_report:
        return adjoint_report(args)
    if args.format_study:
        return format_study(args)
    world, rank, local = init_distributed()
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_gpu(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
