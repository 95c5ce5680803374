"""Mixed-precision forms of the step (MAM4B_MIXED, MAM4B_MIXED_FAST) on the
GPU, against the FP64 step and the host oracle.

Errors are per cell and output: tendencies relative to the state they
change, sizes/densities/water relative (mam4xx_b200.precision). The bounds
below are the measured behaviour with margin, not the 1e-12 of the FP64
path: FP32 rounding enters the bulk (water uptake, uptake and coagulation
coefficients), and with MIXED_FAST also the SOA sub-stepping, which
amplifies rounding near equilibrium (the FP64 algorithm does the same to
1-ulp libm differences, at 1e-16 instead of 1e-7 scale). MIXED keeps the
SOA loop in double precision (division-free, fused) and its cells outside
1e-5 are, but for 0.2 %, cells where the FP64 step itself moves by more
than 1e-5 when its inputs are rounded to FP32.
"""

import numpy as np
import pytest

from mam4xx_b200 import native
from mam4xx_b200.precision import error_report
from mam4xx_b200.workloads import POPULATIONS, make_workload, pblh_per_cell

pytestmark = pytest.mark.gpu


def run(w, precision, ctx=None):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(w["in_slab"])).cuda()
    pb = torch.from_numpy(np.ascontiguousarray(w["pblh"])).cuda()
    n = x.shape[1]
    out = torch.full((native.NOUT, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx = ctx or native.Context()
    ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"], w["dt"],
                  precision=precision)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("cfg", ["c2", "c3", "c4"])
def test_mixed_against_fp64(cuda_device, cfg):
    w = make_workload(cfg, ncol=256, seed=300 + int(cfg[1]))
    ref = run(w, native.FP64)
    mix = run(w, native.MIXED)
    assert np.isfinite(mix).all()
    r = error_report(mix, ref, w["in_slab"], w["dt"], tol=1e-5)
    assert r["cells_within_tol"] >= 0.98, r
    assert r["cell_err_quantiles"]["0.5"] <= 2e-6, r
    assert r["cell_err_quantiles"]["0.99"] <= 5e-5, r
    assert max(r["per_output_median"]) <= 1e-6, r


def test_mixed_against_host_oracle(cuda_device):
    from oracle.pyoracle import PortOracle
    w = make_workload("c2", ncol=64, seed=321)
    mix = run(w, native.MIXED)
    orc = PortOracle().step(w["in_slab"], pblh_per_cell(w), w["dt"])
    r = error_report(mix, orc, w["in_slab"], w["dt"], tol=1e-5)
    assert r["cells_within_tol"] >= 0.97, r
    assert max(r["per_output_median"]) <= 1e-6, r


def test_mixed_fast_against_fp64(cuda_device):
    w = make_workload("c4", ncol=256, seed=331)
    ref = run(w, native.FP64)
    fast = run(w, native.MIXED_FAST)
    assert np.isfinite(fast).all()
    r = error_report(fast, ref, w["in_slab"], w["dt"], tol=1e-5)
    assert r["cells_within_tol"] >= 0.5, r
    assert r["cell_err_quantiles"]["0.5"] <= 2e-5, r
    assert r["cell_err_quantiles"]["0.9"] <= 5e-3, r


@pytest.mark.parametrize("precision", [native.MIXED, native.MIXED_FAST])
def test_mixed_conserves_and_is_deterministic(cuda_device, precision):
    """Mass moves between modes in FP64 in every form: per-species totals of
    the non-condensing species are conserved as in FP64; reruns are bitwise
    identical."""
    w = make_workload("c4", ncol=128, seed=341)
    a = run(w, precision)
    b = run(w, precision)
    assert np.array_equal(a, b)
    x = w["in_slab"]
    after = x[5:57] + a[:52] * w["dt"]
    for spec in ("POM", "BC", "DST", "NaCl", "MOM"):
        rows = [2 + s for s, (_, sp) in enumerate(POPULATIONS) if sp == spec]
        rows += [27 + s for s, (_, sp) in enumerate(POPULATIONS) if sp == spec]
        tot0 = np.sum([x[5 + r].sum() for r in rows])
        tot1 = np.sum([after[r].sum() for r in rows])
        assert abs(tot1 - tot0) <= 1e-12 * tot0, spec


def test_mixed_host_entry_matches_device_entry(cuda_device):
    w = make_workload("c4", ncol=64, seed=351)
    dev = run(w, native.MIXED)
    ctx = native.Context()
    x = np.ascontiguousarray(w["in_slab"])
    out = np.zeros((native.NOUT, x.shape[1]))
    ctx.step_host(x.ctypes.data, w["pblh"].ctypes.data, out.ctypes.data, x.shape[1],
                  w["ncol"], w["nlev"], w["dt"], precision=native.MIXED)
    np.testing.assert_array_equal(out, dev)


def test_mixed_precision_arguments(cuda_device):
    import torch
    w = make_workload("c2", ncol=4, seed=361)
    ctx = native.Context()
    x = torch.from_numpy(w["in_slab"]).cuda()
    pb = torch.from_numpy(w["pblh"]).cuda()
    n = x.shape[1]
    out = torch.zeros((native.NOUT, n), dtype=torch.float64, device="cuda")
    dg = torch.zeros((native.NDIAG, n), dtype=torch.float64, device="cuda")
    with pytest.raises(native.MicrophysicsError, match="not supported"):
        ctx.step([x[f].data_ptr() for f in range(native.NIN)], pb.data_ptr(),
                 [out[f].data_ptr() for f in range(native.NOUT)], w["ncol"], w["nlev"], w["dt"],
                 diag_ptrs=[dg[f].data_ptr() for f in range(native.NDIAG)],
                 precision=native.MIXED)
    with pytest.raises(native.MicrophysicsError, match="invalid argument"):
        ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"],
                      w["dt"], precision=7)


@pytest.mark.parametrize("cfg", ["c3", "c4"])
def test_mixed_errors_against_the_steps_own_conditioning(cuda_device, cfg):
    """Where the mixed form misses 1e-5 of the FP64 step, the FP64 step
    itself is that sensitive: per cell, the FP64 step for its inputs rounded
    to single precision (a relative change of at most 6e-8 per input)
    against the FP64 step for the exact inputs. The FP64 algorithm's
    results jump where a decision (an SOA sub-step count, a clip, a
    threshold) changes with its inputs, so no form that rounds any input of
    such a decision to FP32 can meet 1e-5 on those cells; on the others
    (well-conditioned at FP32 rounding) the mixed form does, but for its own
    FP32 rounding in the bulk (a few ulps over tens of operations, more
    than the one rounding of each input): at least 99.5 % of them."""
    from mam4xx_b200.precision import output_errors
    w = make_workload(cfg, ncol=256, seed=310 + int(cfg[1]))
    ref = run(w, native.FP64)
    mix = run(w, native.MIXED)
    w32 = dict(w)
    w32["in_slab"] = w["in_slab"].astype(np.float32).astype(np.float64)
    r32 = run(w32, native.FP64)
    e_mix = output_errors(mix, ref, w["in_slab"], w["dt"]).max(axis=0)
    e_cond = output_errors(r32, ref, w["in_slab"], w["dt"]).max(axis=0)
    well = e_cond <= 1e-5
    frac_well = float((e_mix[well] <= 1e-5).mean())
    print("CONDITIONING %s: cells %d, ill-conditioned %d, mixed outside 1e-5 %d "
          "(well-conditioned %d), well-conditioned within 1e-5 %.6f"
          % (cfg, e_mix.size, int((~well).sum()), int((e_mix > 1e-5).sum()),
             int((e_mix[well] > 1e-5).sum()), frac_well))
    assert frac_well >= 0.995
    assert float((e_mix <= 1e-5).mean()) >= 0.98
