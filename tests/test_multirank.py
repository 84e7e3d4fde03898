"""world_size-2 CPU tests (gloo) of the multi-rank logic of bench.py: slices are
sharded per rank with no collective on the data path; the job time is the maximum
over ranks; the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.0 + rank, "cpu", world)
        first = bench.rank_first_seed(rank, 256)
        with open(os.path.join(out, f"r{rank}.json"), "w") as f:
            json.dump({"t": t, "first": first}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_disjoint_shards(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r = [json.load(open(tmp_path / f"r{k}.json")) for k in range(2)]
    assert r[0]["t"] == r[1]["t"] == 2.0       # the slower rank sets the job time
    seeds = [set(range(x["first"], x["first"] + 256)) for x in r]
    assert not (seeds[0] & seeds[1])           # each rank reconstructs its own slices


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun with 2 ranks the reference arm prints one line from rank 0 and
    the other rank exits 0 without work (a tiny 32 x 24 case keeps it quick)."""
    port = _free_port()
    env = dict(os.environ)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--n-det", "32", "--n-ang", "24"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
