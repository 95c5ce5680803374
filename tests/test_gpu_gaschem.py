"""Gas-phase chemistry on the GPU (mam4b_gas_chemistry) against the
reference's own microphysics::gas_phase_chemistry compiled unchanged for
the host (oracle/_ref). Both round every sum and product alike (no FMA
contraction); they differ only in the last bits of exp, pow and log10 in the
reaction rates, so the bar is 1e-12 relative on every tracer of every cell.
The cells given a slightly negative tracer never converge (the iterate is
clipped at zero) and take imp_sol's step-cutting path on both sides."""

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import make_gas_chemistry_inputs

pytestmark = pytest.mark.gpu

KEYS = ("temp", "photo", "extfrc", "inv", "het")


def run_gpu(d, ld_pad=0):
    n = d["qq"].shape[1]
    ld = n + ld_pad

    def g(a):
        a = np.asarray(a, dtype=np.float64)
        if a.ndim == 1:
            return torch.from_numpy(np.ascontiguousarray(a)).cuda()
        t = torch.full((a.shape[0], ld), float("nan"), dtype=torch.float64, device="cuda")
        t[:, :n] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        return t

    dev = {k: g(d[k]) for k in KEYS + ("qq",)}
    ctx = native.Context()
    ctx.gas_chemistry(*[dev[k].data_ptr() for k in KEYS], dev["qq"].data_ptr(), ld, d["ncol"],
                      d["nlev"], d["dt"])
    torch.cuda.synchronize()
    out = dev["qq"].cpu().numpy()
    if ld_pad:
        assert np.isnan(out[:, n:]).all()  # nothing written past the cells
    return out[:, :n]


def close(g, r):
    return np.abs(g - r) <= 1e-12 * np.abs(r) + 1e-300


@pytest.mark.parametrize("name,ncol,neg", [("c2", 512, 0.0), ("c4", 256, 0.02),
                                           ("c5", 128, 0.0)])
def test_gas_chemistry_matches_reference(cuda_device, ref_oracle, name, ncol, neg):
    d = make_gas_chemistry_inputs(name, ncol=ncol, seed=23, negative_frac=neg)
    g = run_gpu(d)
    r = ref_oracle.gas_chemistry(d["dt"], d["temp"], d["photo"], d["extfrc"], d["inv"], d["het"],
                                 d["qq"])
    assert np.isfinite(g).all()
    ok = close(g, r)
    assert ok.all(), (np.argwhere(~ok)[:5], (~ok).sum())
    np.testing.assert_array_equal(g[0], d["qq"][0])  # O3 untouched
    assert (g[1:] >= 0).all()
    # the chemistry did something: H2O2, H2SO4, SO2 and DMS all moved
    for t in (1, 2, 3, 4):
        assert (np.abs(g[t] - d["qq"][t]) > 1e-6 * np.abs(d["qq"][t])).mean() > 0.5


def test_gas_chemistry_leading_dimension(cuda_device, ref_oracle):
    d = make_gas_chemistry_inputs("c2", ncol=8, seed=5)
    g = run_gpu(d, ld_pad=37)
    r = ref_oracle.gas_chemistry(d["dt"], d["temp"], d["photo"], d["extfrc"], d["inv"], d["het"],
                                 d["qq"])
    assert close(g, r).all()


def test_gas_chemistry_rejects_bad_arguments(cuda_device):
    ctx = native.Context()
    t = torch.zeros((31, 4), dtype=torch.float64, device="cuda")
    p = t.data_ptr()
    with pytest.raises(native.MicrophysicsError):
        ctx.gas_chemistry(p, p, p, p, p, p, 3, 1, 4, 1800.0)  # ld < ncell
    with pytest.raises(native.MicrophysicsError):
        ctx.gas_chemistry(p, p, p, p, p, p, 4, 1, 4, 0.0)  # dt <= 0
