"""Multi-process (world size 2, gloo, CPU) coverage of the replicas-only N>1 path.

The hot path does not shard: every rank runs its own replica and the only
cross-rank steps are a barrier and the max over ranks of the timed region.
"""
import json
import os
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, port, out):
    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE="2")
    sys.path.insert(0, ROOT)
    import bench
    td.init_process_group("gloo", rank=rank, world_size=2)
    bench.barrier(2)
    m = bench.allreduce_max(1.5 + rank, 2)
    out[rank] = m
    td.destroy_process_group()


def test_max_over_ranks_gloo():
    port = 29611
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(port, out), nprocs=2, join=True)
        assert out[0] == 2.5 and out[1] == 2.5


def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", "29612", "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--workload",
           "gly150_wat2500_9k"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
