"""Multi-process (replicas-only) host logic of bench.py on CPU: two gloo ranks on 127.0.0.1.

The CheFSI path has no exchange step, so N GPUs run N independent replicas; the only
collective is the max-over-ranks of the timed region.  Each rank here runs the numpy oracle's
filter on its own seeded start block (the CPU stand-in for one replica) and the ranks reduce a
rank-dependent time."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    import bench
    from oracle import chefsi_oracle as O

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        op = O.Operator(np.eye(3) * 6.0, (8, 8, 8), order=4)
        V = np.zeros(8 * 8 * 8)
        rng = np.random.default_rng(bench.replica_seed(rank))
        X = rng.uniform(-0.5, 0.5, (8 * 8 * 8, 3))
        Y = O.chebyshev_filter(op, X, V, 1.0, -0.1, 20.0, 4)
        t = bench.max_over_ranks(0.5 + rank, world, "cpu")
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), Y=Y, t=t, seed=bench.replica_seed(rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r = [np.load(tmp_path / f"rank{k}.npz") for k in range(world)]
    assert all(float(x["t"]) == 1.5 for x in r)          # every rank sees the slowest replica
    assert int(r[0]["seed"]) != int(r[1]["seed"])         # independent problems
    assert np.all(np.isfinite(r[0]["Y"])) and np.all(np.isfinite(r[1]["Y"]))
    assert not np.allclose(r[0]["Y"], r[1]["Y"])
