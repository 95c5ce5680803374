"""Host logic of the mixed-precision error reports (mam4xx_b200.precision):
the per-cell errors computed on a torch device agree with the numpy ones,
and the conditioning split counts cells as stated. CPU only."""

import numpy as np
import pytest

from mam4xx_b200.precision import (cell_errors_device, conditioning_split, error_report,
                                   error_report_device, output_errors)
from mam4xx_b200.workloads import NOUT


def _case(n=300, seed=3):
    rng = np.random.default_rng(seed)
    x = np.abs(rng.standard_normal((57, n))) * 1e-9
    ref = rng.standard_normal((NOUT, n)) * 1e-12
    out = ref * (1.0 + 1e-6 * rng.standard_normal((NOUT, n)))
    out[:, 7] = ref[:, 7] * 2.0  # one cell far off
    out[3, 11] = np.nan          # a non-finite output counts as infinitely far
    return x, ref, out


def test_cell_errors_device_matches_numpy():
    torch = pytest.importorskip("torch")
    x, ref, out = _case()
    dt = 1800.0
    e_np = output_errors(out, ref, x, dt)
    e_np = np.where(np.isnan(e_np), np.inf, e_np).max(axis=0)
    e_t = cell_errors_device(torch.from_numpy(out), torch.from_numpy(ref), torch.from_numpy(x),
                             dt, chunk=64).numpy()
    np.testing.assert_allclose(e_t, e_np, rtol=1e-14, atol=0)
    assert np.isinf(e_t[11]) and e_t[7] > 1e-3


def test_error_report_device_agrees_with_host_report():
    torch = pytest.importorskip("torch")
    x, ref, out = _case(seed=4)
    out[3, 11] = ref[3, 11]
    dt = 1800.0
    h = error_report(out, ref, x, dt, tol=1e-5)
    d = error_report_device(torch.from_numpy(out), torch.from_numpy(ref), torch.from_numpy(x), dt,
                            tol=1e-5, chunk=64)
    assert d["cells"] == x.shape[1]
    assert d["cells_within_tol"] == pytest.approx(h["cells_within_tol"])
    assert d["max"] == pytest.approx(h["max"])
    np.testing.assert_allclose(d["per_output_max"], h["per_output_max"], rtol=1e-14)


def test_conditioning_split_counts():
    torch = pytest.importorskip("torch")
    err = torch.tensor([0.0, 2e-5, 3e-5, 1e-6, 5e-5, 1e-7])
    cond = torch.tensor([0.0, 1e-3, 0.0, 1e-3, 1e-6, 0.0])
    s = conditioning_split(err, cond, tol=1e-5)
    assert s["cells"] == 6
    assert s["ill_conditioned_cells"] == 2          # cells 1, 3
    assert s["outside_tol"] == 3                    # cells 1, 2, 4
    assert s["outside_tol_ill_conditioned"] == 1    # cell 1
    assert s["outside_tol_well_conditioned"] == 2   # cells 2, 4
    assert s["well_conditioned_within_tol"] == pytest.approx(1.0 - 2.0 / 4.0)
