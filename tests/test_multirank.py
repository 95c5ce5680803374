"""Multi-rank path: two gloo ranks shard the columns, run the step on their
blocks independently through mam4xx_b200.distributed (the functions
bench.py times its multi-GPU runs with) and reduce only timing and
checksums. The result of each block must not depend on how the columns
were sharded.

The CPU test steps with the CPU restatement; the GPU test runs both ranks'
mam4b_step_slab on one device (the ranks never wait on each other inside a
kernel: each step is an independent launch sequence) and requires the
concatenated blocks to equal one whole-batch call bit for bit."""

import os
import socket

import numpy as np
import pytest

from mam4xx_b200.distributed import shard_columns

NCOL, NLEV = 12, 8


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


def test_timed_steps_without_process_group():
    from mam4xx_b200.distributed import WallClock, sharded_rate, timed_steps
    calls = []
    ms_max, ms, laps = timed_steps(lambda: calls.append(1), 4, 3, WallClock())
    assert len(calls) == 7 and ms_max == ms >= 0 and laps == []
    assert sharded_rate(100, 4, 2.0) == pytest.approx(100 * 4 / 2e-3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outdir, use_gpu):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from mam4xx_b200.distributed import (EventClock, WallClock, sharded_rate, sum_over_ranks,
                                         timed_steps)
    from mam4xx_b200.workloads import make_workload, pblh_per_cell
    w = make_workload("c2", ncol=NCOL, nlev=NLEV, seed=11)
    start, count = shard_columns(w["ncol"], world, rank)
    x = np.ascontiguousarray(w["in_slab"][:, start * NLEV:(start + count) * NLEV])
    n = x.shape[1]
    if use_gpu:
        import torch
        from mam4xx_b200 import native
        dev = torch.device("cuda:0")
        xd = torch.from_numpy(x).to(dev)
        pbd = torch.from_numpy(np.ascontiguousarray(w["pblh"][start:start + count])).to(dev)
        od = torch.empty((native.NOUT, n), dtype=torch.float64, device=dev)
        ctx = native.Context()
        stream = torch.cuda.current_stream(dev)

        def step():
            ctx.step_slab(xd.data_ptr(), pbd.data_ptr(), od.data_ptr(), n, count, NLEV, w["dt"],
                          stream=stream.cuda_stream)
        clock, sync = EventClock(stream), torch.cuda.synchronize
    else:
        from oracle.pyoracle import PortOracle
        orc = PortOracle()
        pb = pblh_per_cell(w)[start * NLEV:(start + count) * NLEV]
        res = {}

        def step():
            res["out"] = orc.step(x, pb, w["dt"], nthreads=1)
        clock, sync = WallClock(), None
    ms_max, ms, laps = timed_steps(step, 3, 3, clock, sync=sync)
    rate = sharded_rate(n, 3, ms_max)
    out = od.cpu().numpy() if use_gpu else res["out"]
    if use_gpu:
        ctx.close()
    csum = sum_over_ranks(float(np.abs(out).sum()))
    np.save(os.path.join(outdir, "r%d.npy" % rank), out)
    if rank == 0:
        np.save(os.path.join(outdir, "meta.npy"), np.array([ms_max, ms, rate, csum, len(laps)]))
    dist.barrier()
    dist.destroy_process_group()


def _run_two_ranks(tmp_path, use_gpu):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), use_gpu),
                       nprocs=world, join=True, start_method="spawn")
    parts = [np.load(tmp_path / ("r%d.npy" % r)) for r in range(world)]
    ms_max, ms, rate, csum, nlaps = np.load(tmp_path / "meta.npy")
    assert ms_max >= ms > 0 and rate > 0
    assert rate == pytest.approx(NCOL * NLEV * 3 / (ms_max * 1e-3))
    return np.concatenate(parts, axis=1), csum, nlaps


def test_two_rank_shards_match_single_process(tmp_path):
    from mam4xx_b200.workloads import make_workload, pblh_per_cell
    from oracle.pyoracle import PortOracle
    got, csum, _ = _run_two_ranks(tmp_path, use_gpu=False)
    w = make_workload("c2", ncol=NCOL, nlev=NLEV, seed=11)
    full = PortOracle().step(w["in_slab"], pblh_per_cell(w), w["dt"], nthreads=1)
    np.testing.assert_array_equal(got, full)
    np.testing.assert_allclose(csum, np.abs(full).sum(), rtol=1e-12)


@pytest.mark.gpu
def test_two_rank_gpu_shards_match_one_call(tmp_path, cuda_device):
    import torch
    from mam4xx_b200 import native
    from mam4xx_b200.workloads import make_workload
    got, csum, nlaps = _run_two_ranks(tmp_path, use_gpu=True)
    assert nlaps == 3
    w = make_workload("c2", ncol=NCOL, nlev=NLEV, seed=11)
    x = torch.from_numpy(w["in_slab"]).to(cuda_device)
    pb = torch.from_numpy(w["pblh"]).to(cuda_device)
    n = x.shape[1]
    out = torch.empty((native.NOUT, n), dtype=torch.float64, device=cuda_device)
    ctx = native.Context()
    ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, NCOL, NLEV, w["dt"])
    torch.cuda.synchronize()
    full = out.cpu().numpy()
    ctx.close()
    assert np.array_equal(got, full), "sharded GPU steps differ from one whole-batch call"
    np.testing.assert_allclose(csum, np.abs(full).sum(), rtol=1e-12)
