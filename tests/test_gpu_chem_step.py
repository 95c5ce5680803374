"""The step with gas-phase and aqueous chemistry ahead of amicphys
(mam4b_step_chem_slab) against the reference's own functions composed the
same way on the host (oracle/_ref: gas_phase_chemistry, setsox_single_level,
modal_aero_amicphys_intr with distinct pre-chemistry states).

1. Structure: with every chemistry rate, forcing and the cloud water zero
   the chemistry changes nothing, and the step must equal the plain step
   (mam4b_step_slab) bit for bit -- the generalised subarea set-up, renaming
   growth and H2SO4 production reduce exactly to the plain ones.
2. Numbers: with active chemistry the step differs from the host reference
   only through the math libraries, which the SOA loop and the Koehler
   quartic amplify as in the plain step. The bar is the plain step's own
   parity on the same cells: the fraction of cells whose 68 outputs are all
   within 1e-12 (state-relative) may fall short of the plain step's by at
   most 0.02, and each error quantile may exceed the plain step's by at most
   3x unless below 1e-12. The four chemistry-gas tendencies are within 1e-10
   relative of the reference on every cell."""

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import make_chem_step_inputs, pblh_per_cell
from oracle.pyoracle import QUANTILES, TOL, output_errors

pytestmark = pytest.mark.gpu


def run_gpu(w, plain=False, cfg=None):
    x = torch.from_numpy(np.ascontiguousarray(w["in_slab"])).cuda()
    pb = torch.from_numpy(np.ascontiguousarray(w["pblh"])).cuda()
    n = x.shape[1]
    out = torch.full((native.NOUT, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx = native.Context(cfg)
    if plain:
        ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"],
                      w["dt"])
        torch.cuda.synchronize()
        return out.cpu().numpy()
    ch = torch.from_numpy(np.ascontiguousarray(w["chem_in"])).cuda()
    cout = torch.full((native.CHEM_NOUT, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx.step_chem_slab(x.data_ptr(), pb.data_ptr(), ch.data_ptr(), out.data_ptr(),
                       cout.data_ptr(), n, w["ncol"], w["nlev"], w["dt"])
    torch.cuda.synchronize()
    assert ctx.last_status() & 0x5 == 0  # no nonfinite input or output
    return out.cpu().numpy(), cout.cpu().numpy()


@pytest.mark.parametrize("name,ncol,cond", [("c2", 256, 1), ("c4", 256, 1), ("c2", 128, 0)])
def test_inert_chemistry_equals_plain_step(cuda_device, name, ncol, cond):
    """Pipelined (condensation on) and one-thread-per-cell (off) paths."""
    cfg = native.default_config(do_cond=cond)
    w = make_chem_step_inputs(name, ncol=ncol, inert=True)
    out, _ = run_gpu(w, cfg=cfg)
    np.testing.assert_array_equal(out, run_gpu(w, plain=True, cfg=cfg))


def _stats(err):
    ec = err.max(axis=0)
    return (ec <= TOL).mean(), np.quantile(ec, QUANTILES)


def check_against_reference(ref_oracle, w, cfg=None, ocfg=None):
    pb = pblh_per_cell(w)
    out, cout = run_gpu(w, cfg=cfg)
    assert np.isfinite(out).all() and np.isfinite(cout).all()
    r_out, r_cout = ref_oracle.step_chem(w["in_slab"], pb, w["chem_in"], w["dt"], cfg=ocfg)
    frac, q = _stats(output_errors(out, r_out, w["in_slab"], w["dt"]))
    # the plain step's parity on the same cells
    plain = run_gpu(w, plain=True, cfg=cfg)
    p_frac, p_q = _stats(output_errors(plain, ref_oracle.step(w["in_slab"], pb, w["dt"], cfg=ocfg),
                                       w["in_slab"], w["dt"]))
    print(frac, q, p_frac, p_q)
    assert frac >= p_frac - 0.02
    for c, b in zip(q, p_q):
        assert c <= max(TOL, 3.0 * b)
    scale = np.abs(w["chem_in"][:4]) / w["dt"]
    assert (np.abs(cout - r_cout) <= 1e-10 * np.maximum(np.abs(r_cout), scale) + 1e-300).all()
    return out, cout, plain


@pytest.mark.parametrize("name,ncol", [("c2", 512), ("c4", 512), ("c5", 256)])
def test_chem_step_matches_reference(cuda_device, ref_oracle, name, ncol):
    w = make_chem_step_inputs(name, ncol=ncol)
    out, cout, plain = check_against_reference(ref_oracle, w)
    # the chemistry acted: H2O2 and SO2 changed in most cells, and the
    # step's H2SO4 tendency differs from the plain step's
    assert (np.abs(cout[1]) > 0).mean() > 0.5 and (np.abs(cout[2]) > 0).mean() > 0.5
    assert (np.abs(out[0] - plain[0]) > 1e-6 * np.abs(plain[0])).mean() > 0.1


def test_chem_step_without_condensation_matches_reference(cuda_device, ref_oracle):
    """The one-thread-per-cell path (condensation off)."""
    from oracle.pyoracle import default_config
    w = make_chem_step_inputs("c2", ncol=256)
    check_against_reference(ref_oracle, w, cfg=native.default_config(do_cond=0),
                            ocfg=default_config(do_cond=0))


def test_chem_step_rejects_bad_arguments(cuda_device):
    ctx = native.Context()
    t = torch.zeros((4,), dtype=torch.float64, device="cuda")
    p = t.data_ptr()
    with pytest.raises(native.MicrophysicsError):
        ctx.step_chem_slab(p, p, p, p, p, 3, 1, 4, 1800.0)  # ld < ncell
    with pytest.raises(native.MicrophysicsError):
        ctx.step_chem_slab(p, p, 0, p, p, 4, 1, 4, 1800.0)  # no chemistry inputs
