"""Multi-GPU path of the batching form on CPU: two gloo ranks shard the
ensemble (whole realizations per rank, no data exchange during the solves),
gather the per-rank assignments and reduce a per-rank time with MAX, the way
bench.py reports on N GPUs."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from ml_prec_b200 import ensemble
    dims = ensemble.realization_dims(64)
    mine = ensemble.shard(dims, rank, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    import bench
    # bench.py's reduction of the per-rank timings: each is the slowest rank's
    t = bench.max_over_ranks([float(rank + 1), 10.0 - rank])
    if rank == 0:
        out.put((gathered, t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_covers_ensemble_once():
    from ml_prec_b200 import ensemble
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    gathered, tmax = q.get(timeout=180)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    allv = sorted(gathered[0] + gathered[1])
    assert allv == list(range(64))
    assert not set(gathered[0]) & set(gathered[1])
    dims = ensemble.realization_dims(64)
    loads = [sum(int(dims[i][0] * dims[i][1] * dims[i][2]) for i in g) for g in gathered]
    assert max(loads) <= 1.05 * min(loads)
    assert tmax == [2.0, 10.0]


def test_shard_is_deterministic_and_single_rank_takes_all():
    from ml_prec_b200 import ensemble
    dims = ensemble.realization_dims(64)
    assert ensemble.shard(dims, 0, 1) == list(range(64))
    assert ensemble.shard(dims, 1, 4) == ensemble.shard(dims, 1, 4)
