"""Multi-process host logic on the CPU (gloo, world size 2): the bench's
weak-scaling sharding gives every rank the same graph and its own queries,
rank 0's share is exactly the single-GPU workload, and the step time is the
max over ranks.  No GPU and no collective on the data path."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from golden_util import csr_digest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nq, outdir):
    import sys
    from pathlib import Path
    import torch
    import torch.distributed as dist
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    import bench
    r, wsize, _ = bench.dist_env()
    assert (r, wsize) == (rank, world)
    w = bench.workload(rank, nq)
    dig = csr_digest(w.row_ptr, w.col, w.len, w.delay)
    digs = [None] * world
    dist.all_gather_object(digs, dig)
    qs = [None] * world
    dist.all_gather_object(qs, (w.src.tolist(), w.dst.tolist(), w.budget.tolist()))
    # per-rank step times: the reported time is the max over ranks
    t = torch.tensor([1.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    np.save(os.path.join(outdir, f"rank{rank}.npy"),
            np.array([dig == digs[0], qs[0] != qs[1], float(t.item())], dtype=object),
            allow_pickle=True)
    dist.destroy_process_group()


def test_two_rank_sharding(tmp_path):
    world, nq = 2, 64
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nq, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    for r in range(world):
        same_graph, distinct_queries, tmax = np.load(tmp_path / f"rank{r}.npy", allow_pickle=True)
        assert same_graph and distinct_queries and tmax == float(world)


def test_rank0_share_is_the_single_gpu_workload():
    import bench
    import vine_b200 as v
    a = bench.workload(0, 64)
    b = v.Workload.generate(5, n_pairs=64)
    assert np.array_equal(a.src, b.src) and np.array_equal(a.dst, b.dst)
    assert np.array_equal(a.budget, b.budget)
    c = bench.workload(1, 64)
    assert not np.array_equal(a.src, c.src)
    assert csr_digest(a.row_ptr, a.col, a.len, a.delay) == csr_digest(c.row_ptr, c.col, c.len, c.delay)
