"""The host side of multi-GPU runs, as two gloo ranks on the CPU: the
bench's process group, its max-over-ranks timing reduction and barrier, and
the weak-scaling tile assignment (each rank its own tile, no data-path
collective).  The GPU path itself runs one process per GPU under torchrun."""
import os

import pytest
import torch
import torch.multiprocessing as mp


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    got_ws, got_rank, _ = bench.dist_init()
    bench.barrier(got_ws)
    m = bench.max_over_ranks(float(10 + 5 * rank), got_ws)
    seeds = [None] * ws
    torch.distributed.all_gather_object(seeds, bench.tile_seed(got_rank))
    torch.distributed.destroy_process_group()
    q.put((rank, got_ws, m, seeds))


@pytest.mark.skipif(not torch.distributed.is_gloo_available(), reason="gloo backend missing")
def test_two_ranks_reduce_and_tiles():
    ws, port = 2, 29500 + (os.getpid() % 2000)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got_ws, m, seeds in res:
        assert got_ws == ws
        assert m == 15.0            # max over ranks of 10 and 15
        assert len(set(seeds)) == ws  # every rank its own tile
