"""Column sharding across GPUs (one process per GPU).

Every cell of the microphysics step is independent, so a multi-GPU step is
N independent single-GPU steps on disjoint column blocks: no collective on
the data path. The only collectives are the barrier around the timed region
and a max-reduction of the per-rank time (and, for checks, sums of scalars).

  shard_columns   the contiguous column block of a rank
  timed_steps     warm-up, barrier, K timed steps, barrier, max over ranks
  sharded_rate    whole-job units per second from the per-rank units and
                  the max-over-ranks time
  EventClock      CUDA events on the stream the steps are queued on
  WallClock       host wall clock, for CPU steppers

bench.py runs the GPU step through these; tests/test_multirank.py runs them
over two gloo ranks with a CPU stepper and with the GPU step.
"""

import time


def shard_columns(total_ncol, world, rank):
    """Contiguous column block of `rank`: (first column, number of columns).
    Blocks differ in size by at most one column."""
    if world <= 0 or not (0 <= rank < world) or total_ncol < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(total_ncol, world)
    count = base + (1 if rank < extra else 0)
    start = rank * base + min(rank, extra)
    return start, count


def _initialised():
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized()


def barrier():
    """Barrier over the default process group (no-op when not initialised)."""
    if _initialised():
        import torch.distributed as dist
        dist.barrier()


def _reduce(value, op, device):
    import torch
    import torch.distributed as dist
    if not _initialised():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, device=None):
    """Max of a float over the default process group (identity when not
    initialised). device: where the reduction tensor lives (a CUDA device
    for NCCL, None = CPU for gloo)."""
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX if _initialised() else None, device)


def sum_over_ranks(value, device=None):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM if _initialised() else None, device)


class WallClock:
    """Host wall clock around CPU steps (milliseconds)."""

    def start(self):
        self.t0 = time.perf_counter()

    def lap(self):
        pass

    def stop(self):
        return 1e3 * (time.perf_counter() - self.t0)

    def laps_ms(self):
        return []


class EventClock:
    """CUDA events recorded on `stream`, the stream the steps are queued on
    (torch's events see only the stream they are recorded on). lap() after
    each step records the per-step boundaries; stop() synchronises and
    returns the total milliseconds."""

    def __init__(self, stream):
        import torch
        self.torch = torch
        self.stream = stream

    def _ev(self):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        return e

    def start(self):
        self.marks = [self._ev()]

    def lap(self):
        self.marks.append(self._ev())

    def stop(self):
        self.end = self._ev()
        self.torch.cuda.synchronize()
        return self.marks[0].elapsed_time(self.end)

    def laps_ms(self):
        return [a.elapsed_time(b) for a, b in zip(self.marks[:-1], self.marks[1:])]


def timed_steps(step, steps, warmup, clock, sync=None, device=None, on_start=None):
    """Runs `warmup` untimed steps, then `steps` steps timed by `clock`,
    bracketed by a barrier and `sync` (e.g. torch.cuda.synchronize) on both
    sides. Every rank takes the same collective steps in the same order.
    on_start: called after the opening barrier, before the clock starts
    (e.g. to start a clock sampler). Returns (max-over-ranks ms, this
    rank's ms, per-step ms of this rank)."""
    sync = sync or (lambda: None)
    for _ in range(warmup):
        step()
    sync()
    barrier()
    sync()
    if on_start is not None:
        on_start()
    clock.start()
    for _ in range(steps):
        step()
        clock.lap()
    ms = clock.stop()
    sync()
    barrier()
    return max_over_ranks(ms, device), ms, clock.laps_ms()


def sharded_rate(local_units, steps, ms_max, device=None):
    """Whole-job throughput: all ranks' units x steps / max-over-ranks time."""
    total = sum_over_ranks(local_units, device)
    return total * steps / (ms_max * 1e-3)
