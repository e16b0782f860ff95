"""The multi-rank path of bench.py on CPU: replicas only (one process per GPU,
no data-path collective), so the ranks meet only at barriers and at the
max-reduction of their timings.  Run with world_size 2 over gloo on
127.0.0.1; no GPU is needed."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


RANK_SCRIPT = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
import bench
world, rank, local = bench.dist_setup()
assert (world, rank, local) == (2, int(os.environ["RANK"]), int(os.environ["LOCAL_RANK"]))
bench.dist_barrier(world)
m = bench.dist_max(1.5 + rank, world)
bench.dist_barrier(world)
import torch.distributed as dist
dist.destroy_process_group()
print(f"rank {rank} max {m}")
"""


def test_timing_max_and_barriers_over_two_gloo_ranks(tmp_path):
    """Each rank reports the maximum of the ranks' timings (dist_max) after the barriers."""
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), FIRESIM_BENCH_BACKEND="gloo")
        procs.append(subprocess.Popen([sys.executable, str(script), str(ROOT)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=180) for p in procs]
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    assert sorted(o.strip() for o, _ in outs) == ["rank 0 max 2.5", "rank 1 max 2.5"]


def test_reference_arm_prints_one_line_from_rank_zero(tmp_path):
    """bench.py --impl reference under torchrun with two ranks: rank 0 alone times
    the CPU restatement and prints the JSON line; the other rank exits 0."""
    port = _free_port()
    env = dict(os.environ, FIRESIM_BENCH_BACKEND="gloo")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "3", "--grid", "24", "--frame", "32", "--reference-steps", "1"]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["steps"] == 1 and line["warmup"] == 3
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_for_config_workloads_is_unavailable(tmp_path):
    """native-firesim has no config physics, so its arm prints an `unavailable`
    line (one, from rank 0) and exits 0."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--physics", "config", "--workload", "c2"],
                         env=env, capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and "config physics" in lines[0]["unavailable"]
