"""The bench's multi-rank plumbing on CPU with the gloo backend, world size 2 (the GPU runs use
NCCL with one process per GPU; the path is replicas only, so its collectives are the timing
barrier and the max over ranks):

- every rank gets the maximum of the ranks' step times, after a common barrier;
- the reference arm under two ranks: rank 0 alone times the reference kernels and prints one JSON
  line, rank 1 prints nothing, and both exit 0."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def rank_env(rank, world, port):
    env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(port), HG_BENCH_BACKEND="gloo", CUDA_VISIBLE_DEVICES="")
    return env


MAX_SCRIPT = r"""
import sys, json
sys.path.insert(0, sys.argv[1])
import bench
world, rank, local, pg = bench.dist_setup(None)
bench.barrier(pg)
v = bench.max_over_ranks(1.0 + 2.5 * rank, pg)
bench.barrier(pg)
print(json.dumps({"rank": rank, "world": world, "max": v}), flush=True)
pg.destroy_process_group()
"""


def run_ranks(args, world=2, timeout=300):
    port = free_port()
    procs = [subprocess.Popen(args, cwd=ROOT, env=rank_env(r, world, port), stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True) for r in range(world)]
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        outs.append((p.returncode, o, e))
    return outs


def test_max_over_ranks_and_barrier():
    outs = run_ranks([sys.executable, "-c", MAX_SCRIPT, ROOT])
    for rc, o, e in outs:
        assert rc == 0, e[-2000:]
    res = [json.loads(o.strip().splitlines()[-1]) for _, o, _ in outs]
    assert sorted(r["rank"] for r in res) == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 3.5 for r in res)


def test_reference_arm_runs_on_rank0_only():
    from oracle import oracle
    if oracle.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    outs = run_ranks([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--level", "3", "--steps", "1",
                      "--warmup", "1"])
    for rc, o, e in outs:
        assert rc == 0, e[-2000:]
    lines0 = [l for l in outs[0][1].splitlines() if l.strip().startswith("{")]
    lines1 = [l for l in outs[1][1].splitlines() if l.strip().startswith("{")]
    assert len(lines0) == 1 and lines1 == []
    d = json.loads(lines0[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"
