"""Multi-rank path on CPU: two gloo ranks shard the columns, run the step
on their blocks independently, and reduce only timing and checksums. The
result of each block must not depend on how the columns were sharded."""

import os
import socket

import numpy as np
import pytest

from mam4xx_b200.distributed import shard_columns


def test_shard_columns_cover_exactly():
    for total in (0, 1, 7, 64, 65536, 65537):
        for world in (1, 2, 3, 4, 8):
            seen = []
            for r in range(world):
                s, c = shard_columns(total, world, r)
                seen.extend(range(s, s + c))
            assert seen == list(range(total))
            sizes = [shard_columns(total, world, r)[1] for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_columns(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from mam4xx_b200.distributed import max_over_ranks, sum_over_ranks
    from mam4xx_b200.workloads import make_workload, pblh_per_cell
    from oracle.pyoracle import PortOracle
    w = make_workload("c2", ncol=12, nlev=8, seed=11)
    start, count = shard_columns(w["ncol"], world, rank)
    x = w["in_slab"][:, start * 8:(start + count) * 8]
    pb = pblh_per_cell(w)[start * 8:(start + count) * 8]
    import time
    t = time.perf_counter()
    out = PortOracle().step(x, pb, w["dt"], nthreads=1)
    el = time.perf_counter() - t
    tmax = max_over_ranks(el)
    cells = sum_over_ranks(x.shape[1])
    csum = sum_over_ranks(float(np.abs(out).sum()))
    np.save(os.path.join(outdir, "r%d.npy" % rank), out)
    if rank == 0:
        np.save(os.path.join(outdir, "meta.npy"), np.array([tmax, cells, csum]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_match_single_process(tmp_path):
    import torch.multiprocessing as mp
    from mam4xx_b200.workloads import make_workload, pblh_per_cell
    from oracle.pyoracle import PortOracle
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    w = make_workload("c2", ncol=12, nlev=8, seed=11)
    full = PortOracle().step(w["in_slab"], pblh_per_cell(w), w["dt"], nthreads=1)
    parts = [np.load(tmp_path / ("r%d.npy" % r)) for r in range(world)]
    np.testing.assert_array_equal(np.concatenate(parts, axis=1), full)
    tmax, cells, csum = np.load(tmp_path / "meta.npy")
    assert cells == full.shape[1] and tmax > 0
    np.testing.assert_allclose(csum, np.abs(full).sum(), rtol=1e-12)
