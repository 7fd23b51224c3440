"""bench.py's multi-rank host logic on the CPU, as two gloo ranks.

Multi-GPU runs are independent replicas of the solve: the only collectives are
the barrier around the timed region and the max over ranks of the timed
durations.  These tests run them with world size 2 on gloo, and the reference
arm under torchrun, where rank 0 alone works and prints the one line.
"""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": "2",
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    r, world, local = bench.dist_init(2)
    bench.barrier(world)
    v = bench.max_over_ranks(10.0 + 5.0 * r, world)   # rank 1 is the slower one
    w = bench.max_over_ranks(7.25 - r, world)          # rank 0 is the slower one
    backend = dist.get_backend()
    bench.barrier(world)
    dist.destroy_process_group()
    q.put((r, world, local, v, w, backend))


def test_max_over_ranks_and_barrier_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[:3] for g in got] == [(0, 2, 0), (1, 2, 1)]
    assert all(g[3] == 15.0 and g[4] == 7.25 and g[5] == "gloo" for g in got)


def test_reference_arm_two_ranks_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--gpus", "2", "--impl", "reference", "--workload", "dam2d", "--steps", "1", "--warmup", "0"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["config"]["workload"] == "dam2d" and d["config"]["parallelism"] == "replicas x2"
