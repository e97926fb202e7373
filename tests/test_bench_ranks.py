"""The multi-rank logic of bench.py on CPU: two gloo ranks (one process per
rank, as torchrun launches them) check the max-over-ranks timing, the
whole-job rate and that only rank 0 of the reference arm prints a line."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

WORKER = r"""
import json, os, sys
sys.path.insert(0, os.environ["ROOT"])
import bench
world, rank, local = bench.init_distributed("gloo")
bench.barrier(world)
slowest = bench.max_over_ranks(world, 10.0 + rank)   # rank 1 is slower
rate = bench.whole_job_rate(1000, world, slowest)
print(json.dumps({"rank": rank, "world": world, "slowest": slowest, "rate": rate}))
import torch.distributed as dist
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(code, world=2, extra_env=None, timeout=120):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, ROOT=str(ROOT), RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, err
        outs.append(out)
    return outs


def test_max_over_ranks_and_whole_job_rate_with_two_gloo_ranks():
    outs = _launch(WORKER)
    lines = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert [x["rank"] for x in lines] == [0, 1]
    for x in lines:
        assert x["world"] == 2
        assert x["slowest"] == 11.0                   # the max over ranks, on every rank
        assert x["rate"] == pytest.approx(1000 * 2 / 11e-3)


REFERENCE_ARM = r"""
import os, sys
sys.path.insert(0, os.environ["ROOT"])
import bench
rank = int(os.environ["RANK"])
class A:
    steps, warmup, n, gpus = 1, 3, 512, 2
if rank != 0:
    # the reference arm: ranks other than 0 exit without work or output
    sys.exit(bench.run_reference(A, 2, rank))
print("rank0")
"""


def test_reference_arm_runs_on_rank_zero_only():
    outs = _launch(REFERENCE_ARM)
    assert outs[0].strip().endswith("rank0")
    assert outs[1].strip() == ""


def test_reference_arm_line_on_a_small_block(capsys):
    """The reference arm's JSON line: one block created once, W untimed and K
    timed passes, the same workload name as the GPU arm, the host's threads
    and CPU model recorded."""
    sys.path.insert(0, str(ROOT))
    import bench
    from oracle.pyoracle import ref_available
    if not ref_available("f32"):
        pytest.skip("reference build oracle/_ref absent")

    class A:
        steps, warmup, n, gpus, u0 = 3, 1, 16, 1, 0.05

    assert bench.run_reference(A, 1, 0) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "MLUPS" and line["value"] > 0
    assert line["config"]["workload"] == "taylor-green 16^3 periodic, K17 cumulant, fp32 storage"
    assert line["config"]["same_config"] is True and line["config"]["fluid_nodes"] == 16 ** 3
    assert line["cpu_baseline"]["cores"] == line["config"]["cpu_threads"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
