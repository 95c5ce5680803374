"""Launch shapes, the autotuner and graph mode of the forward step.

Every launch shape runs the same arithmetic, so each must give the default
shape's results bit for bit; so must graph mode (the step captured once
into a CUDA graph and replayed), also when the arguments change between
calls (recapture and in-place update) and across precisions. The step is
also capturable into a caller's own CUDA graph once its scratch exists."""

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import make_workload

pytestmark = pytest.mark.gpu


def _dev(w):
    x = torch.from_numpy(np.ascontiguousarray(w["in_slab"])).cuda()
    pb = torch.from_numpy(np.ascontiguousarray(w["pblh"])).cuda()
    return x, pb


def _step(ctx, w, x, pb, precision=native.FP64):
    n = x.shape[1]
    out = torch.full((native.NOUT, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"], w["dt"],
                  precision=precision)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _shapes():
    """Shapes covering every compiled variant of every kernel."""
    d = native.default_tuning().as_dict()
    out = []
    for k, vals in (("size_regs", (96,)), ("size_block", (64, 256)), ("mode_block", (64, 256)),
                    ("pair_block", (64, 256)), ("pre_regs", (168, 128)), ("pre_block", (64, 256)),
                    ("post_regs", (255, 168)), ("post_block", (64, 256)),
                    ("soa_regs", (96, 128)), ("soa_block", (128,)), ("soa_blocks_per_sm", (1, 2)),
                    ("cells_per_thread", (2, 4)), ("inline_scale", (1, 4, 16, 64))):
        for v in vals:
            t = dict(d)
            t[k] = v
            if k == "pre_block" and v == 256:
                t["pre_regs"] = 128
            if k == "post_block" and v == 256:
                t["post_regs"] = 128
            out.append(t)
    return out


@pytest.mark.parametrize("name,ncol", [("c4", 96), ("c2", 64)])
def test_every_launch_shape_is_bitwise_equal(cuda_device, name, ncol):
    w = make_workload(name, ncol=ncol, seed=17)
    x, pb = _dev(w)
    ctx = native.Context()
    ctx.set_tuning(native.default_tuning())
    ref = _step(ctx, w, x, pb)
    for shape in _shapes():
        t = native.Tuning(**shape)
        ctx.set_tuning(t)
        got = _step(ctx, w, x, pb)
        assert np.array_equal(got, ref), shape
    # mixed precision through non-default shapes (the last ones finish
    # short SOA loops inside pre)
    ctx.set_tuning(native.default_tuning())
    mref = _step(ctx, w, x, pb, native.MIXED)
    fref = _step(ctx, w, x, pb, native.MIXED_FAST)
    for shape in _shapes()[-3:]:
        ctx.set_tuning(native.Tuning(**shape))
        assert np.array_equal(_step(ctx, w, x, pb, native.MIXED), mref), shape
        assert np.array_equal(_step(ctx, w, x, pb, native.MIXED_FAST), fref), shape
    ctx.close()


def test_invalid_shape_is_rejected(cuda_device):
    ctx = native.Context()
    t = native.default_tuning()
    t.pre_regs = 200
    with pytest.raises(native.MicrophysicsError):
        ctx.set_tuning(t)
    t = native.default_tuning()
    t.soa_block = 96
    with pytest.raises(native.MicrophysicsError):
        ctx.set_tuning(t)
    ctx.close()


def test_autotune_picks_a_valid_shape_with_equal_results(cuda_device):
    w = make_workload("c4", ncol=512, seed=23)
    x, pb = _dev(w)
    n = x.shape[1]
    ctx = native.Context()
    ctx.set_tuning(native.default_tuning())
    ref = _step(ctx, w, x, pb)
    out = torch.empty((native.NOUT, n), dtype=torch.float64, device="cuda")
    t, d_ms, b_ms = ctx.autotune(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"],
                                 w["nlev"], w["dt"], reps=2)
    assert d_ms > 0 and 0 < b_ms <= d_ms
    assert ctx.tuning().as_dict() == t.as_dict()
    native.Context().set_tuning(t)  # valid
    assert np.array_equal(out.cpu().numpy(), ref)
    assert np.array_equal(_step(ctx, w, x, pb), ref)
    ctx.close()


def test_graph_mode_equals_plain_launches_across_argument_changes(cuda_device):
    plain = native.Context()
    ctx = native.Context()
    ctx.set_graph_mode(True)
    cases = [make_workload("c4", ncol=64, seed=31), make_workload("c2", ncol=48, seed=32)]
    devs = [_dev(w) for w in cases]
    refs = [_step(plain, w, x, pb) for w, (x, pb) in zip(cases, devs)]
    mref = _step(plain, cases[0], *devs[0], precision=native.MIXED)
    launches0 = ctx.launch_count()
    # replay, argument change (recapture + update), back, precision change
    for k in (0, 0, 1, 0, 1, 1):
        assert np.array_equal(_step(ctx, cases[k], *devs[k]), refs[k]), k
    assert np.array_equal(_step(ctx, cases[0], *devs[0], precision=native.MIXED), mref)
    # a different launch shape while in graph mode
    t = native.default_tuning()
    t.pre_regs, t.cells_per_thread = 168, 2
    ctx.set_tuning(t)
    assert np.array_equal(_step(ctx, cases[1], *devs[1]), refs[1])
    assert ctx.launch_count() - launches0 == 6 * 8
    ctx.set_graph_mode(False)
    assert np.array_equal(_step(ctx, cases[0], *devs[0]), refs[0])
    ctx.close()
    plain.close()


def test_step_is_capturable_in_a_callers_graph(cuda_device):
    """After one plain call (the context's scratch exists), the step can be
    captured into the caller's own CUDA graph and replayed."""
    w = make_workload("c4", ncol=32, seed=41)
    x, pb = _dev(w)
    n = x.shape[1]
    ctx = native.Context()
    ref = _step(ctx, w, x, pb)
    out = torch.zeros((native.NOUT, n), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"],
                      w["dt"], stream=s.cuda_stream)
    for _ in range(2):
        out.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref)
    del g
    ctx.close()
