"""The multi-process plumbing of bench.py (replicas: one process per GPU, no data-path
collective) on CPU with the gloo backend, world size 2: the barrier, the max-over-ranks time and the
per-rank roles (only rank 0 runs the reference arm and prints)."""
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    d = bench.Dist()
    d.barrier()
    m = d.max(float(10 * (rank + 1)))
    # rank != 0 leaves the reference arm at once, without touching the oracle
    class A:
        gpus, steps, warmup, level, k = world, 1, 0, 2, 1.0
    if rank != 0:
        bench.reference_arm(A(), d)
    d.barrier()
    d.close()
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(repr(m))


def test_replica_plumbing_gloo_two_ranks(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        assert float(open(tmp_path / f"rank{r}.txt").read()) == 20.0
