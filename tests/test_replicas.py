"""Multi-process plumbing of the multi-GPU runs, on the host with gloo:
two ranks split a batch of meshes by cells (every mesh to exactly one rank,
loads balanced within the largest mesh), agree on the maximum of their
timings, and meet at a barrier -- the same steps bench.py takes under
torchrun with NCCL, without a GPU."""
import json
import os
import socket
import subprocess
import sys

import numpy as np

from fvm_b200.replicas import shard_meshes

SIZES = [int(s) ** 2 for s in np.random.default_rng(2).integers(32, 257, 64)]


def test_shard_meshes_partition():
    for world in (1, 2, 3, 8):
        parts = [shard_meshes(SIZES, world, r) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(SIZES)))
        loads = [sum(SIZES[i] for i in p) for p in parts]
        assert max(loads) - sum(loads) / world <= max(SIZES)
        # deterministic
        assert parts == [shard_meshes(SIZES, world, r) for r in range(world)]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks(tmp_path):
    port = _free_port()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
        out = tmp_path / ("rank%d.json" % rank)
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__), str(out)], env=env,
                                      cwd=root))
    for p in procs:
        assert p.wait(timeout=120) == 0
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(2)]
    mine = [set(r["mine"]) for r in res]
    assert not (mine[0] & mine[1]) and (mine[0] | mine[1]) == set(range(len(SIZES)))
    loads = [sum(SIZES[i] for i in m) for m in mine]
    for r in res:
        assert r["max"] == max(loads)
        assert r["sum"] == sum(SIZES)


if __name__ == "__main__":  # one rank of test_two_gloo_ranks
    from fvm_b200.replicas import Ranks

    ranks = Ranks(backend="gloo", timeout_s=60)
    part = shard_meshes(SIZES, ranks.world, ranks.rank)
    load = float(sum(SIZES[i] for i in part))
    mx = ranks.max(load)
    tot = ranks.sum(load)
    ranks.barrier()
    with open(sys.argv[1], "w") as f:
        json.dump({"rank": ranks.rank, "mine": part, "max": mx, "sum": tot}, f)
    ranks.close()
