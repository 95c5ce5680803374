"""Per-process entries on the GPU (mam4b_calcsize_process,
mam4b_coagulation_process) against the reference's own CalcSize and
Coagulation process classes, compiled unchanged for the host
(oracle/_ref/libmam4ref.so).

The two sides share every arithmetic step; they differ only in the last
bits of a few math-library results (the mode constants' exp and log, the
diameters' cbrt and exp, coagulation's exp/sqrt/pow). Errors: tendencies in
units of the state they change (|g - r| dt / max(|state before|, |state
after|, |starting tendency| dt)), diameters and updated states relative.
Bar: 1e-12 on every entry.
"""

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import make_process_inputs

pytestmark = pytest.mark.gpu

TOL = 1e-12


def tend_err(g, r, state, tend0, dt):
    after = state + (r - tend0) * dt
    scale = np.maximum(np.maximum(np.abs(state), np.abs(after)), np.abs(tend0) * dt)
    return np.abs(g - r) * dt / np.maximum(scale, 1e-30)


def rel_err(g, r):
    return np.abs(g - r) / np.maximum(np.abs(r), 1e-300)


def run_calcsize(d, **cfg):
    n = d["prog"].shape[1]
    prog = torch.from_numpy(d["prog"]).cuda()
    tend = torch.from_numpy(d["tend0"].copy()).cuda()
    dgn = torch.full((8, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx = native.Context()
    pf = native.ProgFields.from_slab(prog.data_ptr(), n)
    tf = native.ProgFields.from_slab(tend.data_ptr(), n)
    ctx.calcsize_process(pf, tf, [dgn[m].data_ptr() for m in range(4)],
                         [dgn[4 + m].data_ptr() for m in range(4)], d["ncol"], d["nlev"], d["dt"],
                         **cfg)
    torch.cuda.synchronize()
    return tend.cpu().numpy(), dgn.cpu().numpy()


def run_coag(d):
    n = d["prog_aero"].shape[1]
    prog = torch.from_numpy(d["prog_aero"].copy()).cuda()
    tend = torch.from_numpy(d["tend0"].copy()).cuda()
    t = torch.from_numpy(d["temp"]).cuda()
    p = torch.from_numpy(d["pmid"]).cuda()
    wet = torch.from_numpy(d["wet"]).cuda()
    ctx = native.Context()
    ctx.coagulation_process(t.data_ptr(), p.data_ptr(), [wet[m].data_ptr() for m in range(4)],
                            [wet[4 + m].data_ptr() for m in range(4)],
                            native.ProgFields.from_slab(prog.data_ptr(), n),
                            native.ProgFields.from_slab(tend.data_ptr(), n), d["ncol"], d["nlev"],
                            d["dt"])
    torch.cuda.synchronize()
    return prog.cpu().numpy(), tend.cpu().numpy()


@pytest.mark.parametrize("cfg", [dict(), dict(do_adjust=False), dict(do_aitacc_transfer=False),
                                 dict(do_aitacc_transfer=False, do_adjust=False)])
@pytest.mark.parametrize("name,ncol", [("c2", 256), ("c3", 256)])
def test_calcsize_process_matches_reference(cuda_device, ref_oracle, name, ncol, cfg):
    d = make_process_inputs(name, ncol=ncol, seed=21)
    g_t, g_d = run_calcsize(d, **cfg)
    r_t, r_d = ref_oracle.calcsize_process(d["ncol"], d["nlev"], d["prog"], d["tend0"], d["dt"],
                                           **cfg)
    assert np.isfinite(g_t).all() and np.isfinite(g_d).all()
    e = tend_err(g_t, r_t, d["prog"], d["tend0"], d["dt"])
    assert e.max() <= TOL, (e.max(), np.unravel_index(e.argmax(), e.shape))
    assert rel_err(g_d, r_d).max() <= TOL
    # untouched tendency arrays keep their bits
    same = np.all(r_t == d["tend0"], axis=1)
    np.testing.assert_array_equal(g_t[same], d["tend0"][same])


@pytest.mark.parametrize("name,ncol", [("c2", 256), ("c4", 256)])
def test_coagulation_process_matches_reference(cuda_device, ref_oracle, name, ncol):
    d = make_process_inputs(name, ncol=ncol, seed=31)
    g_p, g_t = run_coag(d)
    r_p, r_t = ref_oracle.coag_process(d["ncol"], d["nlev"], d["temp"], d["pmid"], d["wet"],
                                       d["prog_aero"], d["tend0"], d["dt"])
    assert np.isfinite(g_p).all() and np.isfinite(g_t).all()
    e = tend_err(g_t[:36], r_t[:36], d["prog_aero"][:36], d["tend0"][:36], d["dt"])
    assert e.max() <= TOL, e.max()
    scale = np.maximum(np.abs(r_p[:36]), np.abs(d["prog_aero"][:36]))
    assert (np.abs(g_p[:36] - r_p[:36]) / np.maximum(scale, 1e-300)).max() <= TOL
    # cloud-borne fields are neither read nor written
    np.testing.assert_array_equal(g_p[36:], d["prog_aero"][36:])
    np.testing.assert_array_equal(g_t[36:], d["tend0"][36:])


@pytest.mark.parametrize("ncol,nlev", [(1, 1), (3, 7), (97, 5)])
def test_process_entries_ragged_sizes(cuda_device, ref_oracle, ncol, nlev):
    d = make_process_inputs("c2", ncol=ncol, nlev=nlev, seed=41)
    g_t, g_d = run_calcsize(d)
    r_t, r_d = ref_oracle.calcsize_process(d["ncol"], d["nlev"], d["prog"], d["tend0"], d["dt"])
    assert tend_err(g_t, r_t, d["prog"], d["tend0"], d["dt"]).max() <= TOL
    assert rel_err(g_d, r_d).max() <= TOL
    g_p, _ = run_coag(d)
    r_p, _ = ref_oracle.coag_process(d["ncol"], d["nlev"], d["temp"], d["pmid"], d["wet"],
                                     d["prog_aero"], d["tend0"], d["dt"])
    scale = np.maximum(np.abs(r_p[:36]), np.abs(d["prog_aero"][:36]))
    assert (np.abs(g_p[:36] - r_p[:36]) / np.maximum(scale, 1e-300)).max() <= TOL


def test_process_null_field_is_rejected(cuda_device):
    d = make_process_inputs("c2", ncol=2, seed=5)
    n = d["prog"].shape[1]
    prog = torch.from_numpy(d["prog"]).cuda()
    tend = torch.from_numpy(d["tend0"]).cuda()
    dgn = torch.zeros((8, n), dtype=torch.float64, device="cuda")
    pf = native.ProgFields.from_slab(prog.data_ptr(), n)
    pf.q_aero_i[1][2] = None  # aitken NaCl is read by CalcSize
    ctx = native.Context()
    with pytest.raises(native.MicrophysicsError, match="null field"):
        ctx.calcsize_process(pf, native.ProgFields.from_slab(tend.data_ptr(), n),
                             [dgn[m].data_ptr() for m in range(4)],
                             [dgn[4 + m].data_ptr() for m in range(4)], d["ncol"], d["nlev"],
                             d["dt"])


def test_process_mirrors_equal_c_abi(cuda_device):
    """CalcSizeProcess / CoagulationProcess (the AeroProcess mirror over
    (ncol, nlev) tensors) give the C-ABI entries' results bit for bit."""
    from mam4xx_b200.process import (Atmosphere, CalcSizeProcess, CoagulationProcess,
                                     Diagnostics, Prognostics)
    d = make_process_inputs("c2", ncol=32, seed=61)
    ncol, nlev = d["ncol"], d["nlev"]
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda().view(ncol, nlev)
    nspec = (7, 4, 7, 3)

    def progs_of(slab, full):
        k = lambda m: 7 if full else nspec[m]
        return Prognostics([g(slab[m]) for m in range(4)], [g(slab[4 + m]) for m in range(4)],
                           [[g(slab[8 + 7 * m + a]) for a in range(k(m))] for m in range(4)],
                           [[g(slab[36 + 7 * m + a]) for a in range(k(m))] for m in range(4)],
                           [])
    atm = Atmosphere(g(d["temp"]), g(d["pmid"]), None, None, None, None)
    diags = Diagnostics.allocate(ncol, nlev, "cuda")
    tends = progs_of(d["tend0"], False)
    CalcSizeProcess().compute_tendencies(0.0, d["dt"], atm, None, progs_of(d["prog"], False),
                                         diags, tends)
    torch.cuda.synchronize()
    r_t, r_d = run_calcsize(d)
    for m in range(4):
        np.testing.assert_array_equal(tends.n_mode_i[m].cpu().numpy().ravel(), r_t[m])
        np.testing.assert_array_equal(diags.dry_geometric_mean_diameter_c[m].cpu().numpy().ravel(),
                                      r_d[4 + m])
    diags.wet_density = [g(d["wet"][m]) for m in range(4)]
    diags.wet_geometric_mean_diameter_i = [g(d["wet"][4 + m]) for m in range(4)]
    progs = progs_of(d["prog_aero"], True)
    tends = progs_of(d["tend0"], True)
    CoagulationProcess().compute_tendencies(0.0, d["dt"], atm, None, progs, diags, tends)
    torch.cuda.synchronize()
    r_p, r_t = run_coag(d)
    for m in range(4):
        for a in range(7):
            np.testing.assert_array_equal(progs.q_aero_i[m][a].cpu().numpy().ravel(),
                                          r_p[8 + 7 * m + a])
            np.testing.assert_array_equal(tends.q_aero_i[m][a].cpu().numpy().ravel(),
                                          r_t[8 + 7 * m + a])
