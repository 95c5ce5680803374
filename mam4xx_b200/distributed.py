"""Column sharding across GPUs (one process per GPU).

Every cell of the microphysics step is independent, so a multi-GPU step is
N independent single-GPU steps on disjoint column blocks: no collective on
the data path. The only collectives are the barrier around the timed region
and a max-reduction of the per-rank time (and, for checks, sums of scalars).
"""


def shard_columns(total_ncol, world, rank):
    """Contiguous column block of `rank`: (first column, number of columns).
    Blocks differ in size by at most one column."""
    if world <= 0 or not (0 <= rank < world) or total_ncol < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(total_ncol, world)
    count = base + (1 if rank < extra else 0)
    start = rank * base + min(rank, extra)
    return start, count


def max_over_ranks(value, device=None):
    """Max of a float over the default process group (identity when not
    initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
