"""Test-only torch.autograd.Function over the C ABI: forward is
mam4b_step_slab, backward is mam4b_adjoint_slab. Used by the tests to take
gradients of objectives of the step with torch; not part of the library."""

import torch

from mam4xx_b200 import native


class MicrophysicsStep(torch.autograd.Function):
    """out = step(in_slab); in_slab (NIN, n) float64 CUDA, pblh (ncol,)."""

    @staticmethod
    def forward(ctx, in_slab, pblh, ncol, nlev, dt, mctx):
        n = in_slab.shape[1]
        x = in_slab.contiguous()
        out = torch.empty((native.NOUT, n), dtype=torch.float64, device=x.device)
        mctx.step_slab(x.data_ptr(), pblh.data_ptr(), out.data_ptr(), n, ncol, nlev, dt,
                       stream=torch.cuda.current_stream().cuda_stream)
        ctx.save_for_backward(x, pblh)
        ctx.shape = (ncol, nlev, dt)
        ctx.mctx = mctx
        return out

    @staticmethod
    def backward(ctx, out_bar):
        x, pblh = ctx.saved_tensors
        ncol, nlev, dt = ctx.shape
        n = x.shape[1]
        ob = out_bar.contiguous()
        in_bar = torch.empty_like(x)
        ctx.mctx.adjoint_slab(x.data_ptr(), pblh.data_ptr(), ob.data_ptr(), in_bar.data_ptr(), n,
                              ncol, nlev, dt, stream=torch.cuda.current_stream().cuda_stream)
        return in_bar, None, None, None, None, None
