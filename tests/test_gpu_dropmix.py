"""Droplet activation and vertical mixing on the GPU (mam4b_dropmixnuc)
against the reference's own ndrop::dropmixnuc compiled unchanged for the
host (oracle/_ref), column by column. Both round every sum and product
alike (no FMA contraction); they differ in the last bits of the
activation's exp, log, pow and erf, which the linear mixing carries along.
The bar is 1e-10, relative to each output's scale: the value itself, or
for the tendencies and the mixed aerosol the input amounts they are
differences of (droplet number over dt, interstitial plus cloud-borne
population), the CCN at 1 % supersaturation for every CCN value (the
1 - erf of the low supersaturations cancels), absolute for the activated
fractions.""" 

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import make_dropmix_inputs

pytestmark = pytest.mark.gpu

NIN_AER_I, NIN_AER_C = 7, 32


def run_gpu(w, top_lev, vertical_mix=True, ld_pad=0):
    n = w["in_slab"].shape[1]
    ld = n + ld_pad

    def slab(a):
        t = torch.full((a.shape[0], ld), float("nan"), dtype=torch.float64, device="cuda")
        t[:, :n] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        return t

    x, mix = slab(w["in_slab"]), slab(w["mix"])
    pint = torch.from_numpy(np.ascontiguousarray(w["pint"])).cuda()
    kvh = torch.from_numpy(np.ascontiguousarray(w["kvh"])).cuda()
    out = torch.full((66, ld), float("nan"), dtype=torch.float64, device="cuda")
    ctx = native.Context()
    ctx.dropmixnuc(x.data_ptr(), ld, mix.data_ptr(), pint.data_ptr(), kvh.data_ptr(),
                   out.data_ptr(), w["ncol"], w["nlev"], top_lev, w["dt"], vertical_mix)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    if ld_pad:
        assert np.isnan(o[:, n:]).all()
    return o[:, :n]


def scales(w, r):
    x, mix, dt = w["in_slab"], w["mix"], w["dt"]
    nd = mix[2]
    s = np.abs(r).copy()
    s[0] = np.maximum(s[0], nd)
    for f in (1, 2, 3):
        s[f] = np.maximum(s[f], (nd + np.abs(r[0])) / dt)
    s[6:10] = 1.0
    # CCN sums n (1 - erf) / 2, which cancels at low supersaturation: its
    # scale is the largest CCN value (at 1 %)
    s[10:16] = np.maximum(s[10:16], np.abs(r[15]))
    pops = np.abs(x[NIN_AER_I:NIN_AER_I + 25]) + np.abs(x[NIN_AER_C:NIN_AER_C + 25])
    s[16:41] = np.maximum(s[16:41], pops / dt)
    s[41:66] = np.maximum(s[41:66], pops)
    return np.maximum(s, 1e-300)


@pytest.mark.parametrize("name,ncol,top_lev,mix", [("c2", 128, 6, True), ("c4", 128, 6, True),
                                                   ("c2", 64, 1, True), ("c2", 64, 6, False)])
def test_dropmixnuc_matches_reference(cuda_device, ref_oracle, name, ncol, top_lev, mix):
    w = make_dropmix_inputs(name, ncol=ncol, seed=29)
    g = run_gpu(w, top_lev, mix)
    r = ref_oracle.dropmixnuc(w["ncol"], w["nlev"], top_lev, mix, w["dt"], w["in_slab"],
                              w["mix"], w["pint"], w["kvh"])
    assert np.isfinite(g).all()
    err = np.abs(g - r) / scales(w, r)
    f, c = np.unravel_index(np.argmax(err), err.shape)
    assert err.max() <= 1e-10, (f, c, g[f, c], r[f, c], err.max())
    # above top_lev: droplet number as given, cloud-borne aerosol removed
    above = np.arange(g.shape[1]) % w["nlev"] < top_lev
    np.testing.assert_array_equal(g[0, above], w["mix"][2, above])
    assert (g[41:66, above] == 0).all()
    # activation, sources and mixing all acted somewhere
    below = ~above
    assert (g[6, below] > 0).mean() > 0.2 and (g[2, below] != 0).mean() > 0.2


def test_dropmixnuc_leading_dimension(cuda_device, ref_oracle):
    w = make_dropmix_inputs("c2", ncol=8, seed=31)
    g = run_gpu(w, 6, ld_pad=11)
    r = ref_oracle.dropmixnuc(w["ncol"], w["nlev"], 6, True, w["dt"], w["in_slab"], w["mix"],
                              w["pint"], w["kvh"])
    assert (np.abs(g - r) / scales(w, r)).max() <= 1e-10


def test_dropmixnuc_rejects_bad_arguments(cuda_device):
    ctx = native.Context()
    t = torch.zeros((4,), dtype=torch.float64, device="cuda")
    p = t.data_ptr()
    with pytest.raises(native.MicrophysicsError):
        ctx.dropmixnuc(p, 72, p, p, p, p, 1, 72, 0, 1800.0)  # top_lev < 1
    with pytest.raises(native.MicrophysicsError):
        ctx.dropmixnuc(p, 72, p, p, p, p, 1, 72, 71, 1800.0)  # top_lev > nlev - 2
