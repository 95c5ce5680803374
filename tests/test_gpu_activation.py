"""Aerosol activation on the GPU (mam4b_activate) against the reference's
own ndrop::get_activate_frac compiled unchanged for the host
(oracle/_ref). The two share every arithmetic step and differ only in the
last bits of exp, log, pow, sqrt and erf; the bar is 1e-12 relative (with
an absolute floor of 1e-15 for fractions near zero) on every output of
every cell."""

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import make_activation_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,ncol", [("c2", 512), ("c3", 256), ("c4", 256)])
def test_activation_matches_reference(cuda_device, ref_oracle, name, ncol):
    d = make_activation_inputs(name, ncol=ncol, seed=29)
    x = torch.from_numpy(d["in_slab"]).cuda()
    rho = torch.from_numpy(d["rho"]).cuda()
    w = torch.from_numpy(d["w"]).cuda()
    n = x.shape[1]
    out = torch.full((17, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx = native.Context()
    ctx.activate(x.data_ptr(), n, rho.data_ptr(), w.data_ptr(), out.data_ptr(), d["ncol"],
                 d["nlev"])
    torch.cuda.synchronize()
    g = out.cpu().numpy()
    r = ref_oracle.activate(d["in_slab"], d["rho"], d["w"])
    assert np.isfinite(g).all()
    err = np.abs(g - r) / np.maximum(np.abs(r), 1e-3)
    assert (np.abs(g - r) <= 1e-12 * np.abs(r) + 1e-15).all(), err.max()
    # a real mix: activation happens, not everywhere completely
    fn = g[0:4]
    assert ((fn > 0.01) & (fn < 0.99)).mean() > 0.05
