"""The step on tracer-layout arrays (mam4b_step_tracers): the E3SM state_q
tracer order in a mam4::TracersView (tracer, column, level) with a padded
tracer stride gives mam4b_step_slab's results bit for bit, written into
the tendency rows of the prognostic tracers only."""

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import IN_AER_C, IN_AER_I, make_workload

pytestmark = pytest.mark.gpu


def to_tracers(x, stride, rng):
    n = x.shape[1]
    q = rng.uniform(1.0, 2.0, (40, stride))      # rows the step must not read
    qqcw = rng.uniform(1.0, 2.0, (40, stride))
    q[0, :n] = x[3]
    q[11, :n] = x[5]
    q[14, :n] = x[6]
    q[15:40, :n] = x[IN_AER_I:IN_AER_I + 25]
    qqcw[15:40, :n] = x[IN_AER_C:IN_AER_C + 25]
    return q, qqcw


@pytest.mark.parametrize("name,ncol,pad", [("c2", 64, 0), ("c4", 128, 13), ("c1", None, 3)])
def test_step_tracers_equals_step_slab(cuda_device, name, ncol, pad):
    w = make_workload(name, ncol=ncol, seed=71)
    x = w["in_slab"]
    n = x.shape[1]
    stride = n + pad
    q, qqcw = to_tracers(x, stride, np.random.default_rng(5))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    qd, cd = d(q), d(qqcw)
    met = [d(x[f]) for f in (0, 1, 2, 4)]
    pb = d(w["pblh"])
    pt_q = torch.full((40, stride), -7.0, dtype=torch.float64, device="cuda")
    pt_c = torch.full((40, stride), -7.0, dtype=torch.float64, device="cuda")
    mode = torch.full((16, stride), -7.0, dtype=torch.float64, device="cuda")
    ctx = native.Context()
    ctx.step_tracers(qd.data_ptr(), cd.data_ptr(), stride, *[m.data_ptr() for m in met],
                     pb.data_ptr(), pt_q.data_ptr(), pt_c.data_ptr(), mode.data_ptr(), stride,
                     w["ncol"], w["nlev"], w["dt"])
    xs = d(x)
    out = torch.full((native.NOUT, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx.step_slab(xs.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"], w["dt"])
    torch.cuda.synchronize()
    ref = out.cpu().numpy()
    pq, pc, md = pt_q.cpu().numpy(), pt_c.cpu().numpy(), mode.cpu().numpy()
    np.testing.assert_array_equal(pq[11, :n], ref[0])
    np.testing.assert_array_equal(pq[14, :n], ref[1])
    np.testing.assert_array_equal(pq[15:40, :n], ref[2:27])
    np.testing.assert_array_equal(pc[15:40, :n], ref[27:52])
    np.testing.assert_array_equal(md[:, :n], ref[52:68])
    written = {11, 14} | set(range(15, 40))
    for r in range(40):
        if r not in written:
            assert (pq[r] == -7.0).all(), r
        if r < 15:
            assert (pc[r] == -7.0).all(), r
    assert (pq[:, n:] == -7.0).all() and (md[:, n:] == -7.0).all()


def test_step_tracers_rejects_short_stride(cuda_device):
    ctx = native.Context()
    t = torch.zeros((40, 10), dtype=torch.float64, device="cuda")
    p = t.data_ptr()
    with pytest.raises(native.MicrophysicsError, match="invalid argument"):
        ctx.step_tracers(p, p, 9, p, p, p, p, p, p, p, p, 10, 1, 10, 1800.0)
