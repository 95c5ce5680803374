"""Reverse-mode adjoint of the FP64 step (mam4b_adjoint_slab) on the GPU.

The objective is the one of the adjoint configuration: accumulation-mode
number and SO4 mass (interstitial and cloud-borne) after one 1800 s step,
column-integrated with weights pdel/g. Its gradient with respect to T,
water vapour, H2SO4, SOAG and all mode numbers and masses is checked
against central finite differences of the GPU forward step at relative
step 1e-6 on 64 random cells. Agreement is measured in units of relative
sensitivity, |g - fd| * |x| / |J_cell| (the change of J per relative change
of the input), which is scale-free across inputs spanning 20 decades.
"""

import numpy as np
import pytest

from mam4xx_b200 import native
from mam4xx_b200.workloads import make_workload, pblh_per_cell

pytestmark = pytest.mark.gpu

DIFF_FIELDS = [0, 3, 5, 6] + list(range(7, 57))  # T, qv, H2SO4, SOAG, populations
J_STATE = [2 + 7, 2 + 0, 27 + 7, 27 + 0]  # acc number, acc SO4; interstitial, cloud-borne


def pdel_over_g(w):
    """Layer mass per area from the workload's mid-level pressures."""
    p = w["in_slab"][1].reshape(w["ncol"], w["nlev"])
    edges = np.concatenate([p[:, :1] * 0.5, 0.5 * (p[:, 1:] + p[:, :-1]), p[:, -1:] * 1.01], axis=1)
    return (np.abs(np.diff(edges, axis=1)) / 9.80616).reshape(-1)


def forward(ctx, x, pb, w):
    import torch
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    pt = torch.from_numpy(np.ascontiguousarray(pb)).cuda()
    n = xt.shape[1]
    out = torch.empty((native.NOUT, n), dtype=torch.float64, device="cuda")
    ctx.step_slab(xt.data_ptr(), pt.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"], w["dt"])
    torch.cuda.synchronize()
    return out.cpu().numpy()


def adjoint(ctx, x, pb, ybar, w):
    import torch
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    pt = torch.from_numpy(np.ascontiguousarray(pb)).cuda()
    yt = torch.from_numpy(np.ascontiguousarray(ybar)).cuda()
    n = xt.shape[1]
    xb = torch.full((native.NIN, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx.adjoint_slab(xt.data_ptr(), pt.data_ptr(), yt.data_ptr(), xb.data_ptr(), n, w["ncol"],
                     w["nlev"], w["dt"])
    torch.cuda.synchronize()
    return xb.cpu().numpy()


def objective_cells(x, out, wts, dt):
    """Per-cell J: weight * (acc number + acc SO4, both phases) after the step."""
    return wts * sum(x[5 + k] + out[k] * dt for k in J_STATE)


def objective_bar(wts, dt, n):
    ybar = np.zeros((native.NOUT, n))
    for k in J_STATE:
        ybar[k] = wts * dt
    return ybar


def _fd_entries(J, x, g, J0, cells, fields, h_rel=1e-6):
    """Central and one-sided differences of the per-cell objective J(x)
    (a function of the whole input slab) for every (field, cell); returns
    arrays of (field, cell, err_central, err_left, err_right, kink) in units
    of |g - fd| |x| / |J0|, kink = |fd_left - fd_right| |x| / |J0|."""
    rows = []
    Jx = J(x)
    for f in fields:
        h = h_rel * np.abs(x[f])
        xp = x.copy()
        xm = x.copy()
        xp[f] += h
        xm[f] -= h
        Jp, Jm = J(xp), J(xm)
        hs = np.where(h > 0, h, 1.0)
        fd_c = (Jp - Jm) / (2 * hs)
        fd_r = (Jp - Jx) / hs
        fd_l = (Jx - Jm) / hs
        for c in cells:
            if x[f, c] == 0.0:
                continue
            sc = abs(x[f, c]) / abs(J0[c])
            rows.append((f, c, abs(g[f, c] - fd_c[c]) * sc, abs(g[f, c] - fd_l[c]) * sc,
                         abs(g[f, c] - fd_r[c]) * sc, abs(fd_l[c] - fd_r[c]) * sc))
    return np.array(rows)


def test_adjoint_against_finite_differences(cuda_device, port_oracle):
    """Central differences of the GPU forward at relative step 1e-6 on 64
    cells. Entries that miss 1e-6 are of two kinds:
      * branch straddles: the forward is not differentiable inside
        [x - h, x + h], shown per entry by a kink of the GPU forward (the
        one-sided differences disagree by more than 1e-5; the adjoint then
        matches the one-sided difference of one side, the derivative of a
        branch the forward takes next to x) or by a different SOA sub-step
        count at x - h and x + h (counted on the CPU restatement);
      * smooth disagreements (both one-sided differences agree with the
        central one but not with the adjoint): a known inaccuracy of the
        temperature derivative through renaming in partly cloudy cells,
        bounded here at 1e-4 and 0.1 % of the entries."""
    w = make_workload("c5", ncol=32, seed=5150)
    x = w["in_slab"]
    n = x.shape[1]
    wts = pdel_over_g(w)
    ctx = native.Context()
    out = forward(ctx, x, w["pblh"], w)
    J0 = objective_cells(x, out, wts, w["dt"])
    g = adjoint(ctx, x, w["pblh"], objective_bar(wts, w["dt"], n), w)
    for k in J_STATE:
        g[5 + k] += wts  # the state itself enters J (after = before + tend dt)
    rng = np.random.default_rng(64)
    cells = rng.choice(n, 64, replace=False)

    def J(xv):
        return objective_cells(xv, forward(ctx, xv, w["pblh"], w), wts, w["dt"])

    rows = _fd_entries(J, x, g, J0, cells, DIFF_FIELDS)
    errs = rows[:, 2]
    summary = {"entries": int(errs.size), "median": float(np.median(errs)),
               "q999": float(np.quantile(errs, 0.999)), "max": float(errs.max()),
               "within_1e-6": float((errs <= 1e-6).mean())}
    assert errs.size > 3000
    assert summary["median"] <= 1e-9, summary
    assert summary["within_1e-6"] >= 0.997, summary
    pb_cell = pblh_per_cell(w)
    straddles, smooth = [], []
    for f, c, ec, el, er, kink in rows[errs > 1e-6]:
        f, c = int(f), int(c)
        h = 1e-6 * abs(x[f, c])
        xs = x[:, [c]].copy()
        xp, xm = xs.copy(), xs.copy()
        xp[f] += h
        xm[f] -= h
        np_, nm_ = (int(port_oracle.soa_niter(v, pb_cell[[c]], w["dt"])[0]) for v in (xp, xm))
        if kink > 1e-5:
            # a kink of the GPU forward itself: the adjoint follows one side
            assert min(el, er) <= 1e-5, ("kink without a matching side", f, c, ec, el, er)
            straddles.append((f, c))
        elif np_ != nm_:
            # the SOA sub-step count changes inside [x - h, x + h]
            straddles.append((f, c))
        else:
            smooth.append((f, c, ec))
    print("FD", summary, "straddles", len(straddles), "smooth", smooth)
    assert len(smooth) <= 0.001 * errs.size, smooth
    assert all(e <= 1e-4 for _, _, e in smooth), smooth


def test_adjoint_against_reference_forward_differences(cuda_device, ref_oracle):
    """The gradient of the FP64 reference forward itself (the mam4xx headers
    compiled for the host): central differences of the reference build's
    step on 16 cells agree with the adjoint to 1e-6 on 99 % of entries; the
    rest differ by at most what the libm spread between the two builds makes
    of a 1e-6 step."""
    w = make_workload("c5", ncol=8, seed=5151)
    x = w["in_slab"]
    n = x.shape[1]
    wts = pdel_over_g(w)
    ctx = native.Context()
    pbc = pblh_per_cell(w)
    rng = np.random.default_rng(65)
    cells = np.sort(rng.choice(n, 16, replace=False))
    out = forward(ctx, x, w["pblh"], w)
    J0 = objective_cells(x, out, wts, w["dt"])
    g = adjoint(ctx, x, w["pblh"], objective_bar(wts, w["dt"], n), w)
    for k in J_STATE:
        g[5 + k] += wts

    def J(xv):
        # only the chosen cells are stepped on the host
        o = np.zeros((native.NOUT, n))
        o[:, cells] = ref_oracle.step(xv[:, cells], pbc[cells], w["dt"])
        return objective_cells(xv, o, wts, w["dt"])

    rows = _fd_entries(J, x, g, J0, cells, DIFF_FIELDS)
    errs = rows[:, 2]
    assert errs.size > 700
    assert float((errs <= 1e-6).mean()) >= 0.99, float((errs <= 1e-6).mean())
    assert float(np.median(errs)) <= 1e-8


def test_adjoint_fixed_rows_and_determinism(cuda_device):
    w = make_workload("c2", ncol=16, seed=77)
    x = w["in_slab"]
    n = x.shape[1]
    rng = np.random.default_rng(1)
    ybar = rng.standard_normal((native.NOUT, n))
    ctx = native.Context()
    a = adjoint(ctx, x, w["pblh"], ybar, w)
    b = adjoint(ctx, x, w["pblh"], ybar, w)
    assert np.array_equal(a, b)
    assert np.isfinite(a).all()
    for f in (1, 2, 4):  # pressure, height, cloud fraction: held fixed
        assert (a[f] == 0.0).all()
    # linearity in the cotangent
    c = adjoint(ctx, x, w["pblh"], 2.0 * ybar, w)
    np.testing.assert_allclose(c, 2.0 * a, rtol=1e-12, atol=0)


def test_adjoint_autograd_function(cuda_device):
    """The test-only torch.autograd.Function gives the adjoint's gradient."""
    import torch
    from tests.adjoint_autograd import MicrophysicsStep
    w = make_workload("c4", ncol=8, seed=88)
    x = torch.from_numpy(w["in_slab"]).cuda().requires_grad_(True)
    pb = torch.from_numpy(w["pblh"]).cuda()
    wts = torch.from_numpy(pdel_over_g(w)).cuda()
    ctx = native.Context()
    out = MicrophysicsStep.apply(x, pb, w["ncol"], w["nlev"], w["dt"], ctx)
    J = sum(((x[5 + k] + out[k] * w["dt"]) * wts).sum() for k in J_STATE)
    (gx,) = torch.autograd.grad(J, x)
    direct = adjoint(ctx, w["in_slab"], w["pblh"], objective_bar(pdel_over_g(w), w["dt"], x.shape[1]), w)
    for k in J_STATE:
        direct[5 + k] += pdel_over_g(w)
    np.testing.assert_allclose(gx.cpu().numpy(), direct, rtol=1e-12, atol=0)


@pytest.mark.parametrize("name,ncol", [("c5", 64), ("c4_stress", 32)])
def test_adjoint_checkpoint_interval_gives_the_same_gradient(cuda_device, name, ncol):
    """A checkpoint every 4 SOA sub-steps with the others recomputed in the
    reverse sweep gives the gradient of storing every sub-step, bit for bit
    (loops of 1 to 1,000 sub-steps, so partial last blocks are covered),
    and the context switches back and forth."""
    w = make_workload(name, ncol=ncol, seed=91)
    x = w["in_slab"]
    n = x.shape[1]
    rng = np.random.default_rng(2)
    ybar = rng.standard_normal((native.NOUT, n))
    ctx = native.Context()
    every = adjoint(ctx, x, w["pblh"], ybar, w)
    ctx.set_adjoint_checkpoint(4)
    ck4 = adjoint(ctx, x, w["pblh"], ybar, w)
    ctx.set_adjoint_checkpoint(1)
    again = adjoint(ctx, x, w["pblh"], ybar, w)
    assert np.isfinite(every).all()
    assert np.array_equal(ck4, every)
    assert np.array_equal(again, every)
    with pytest.raises(native.MicrophysicsError):
        ctx.set_adjoint_checkpoint(3)


def test_mixed_adjoint_against_fp64_adjoint_and_differences(cuda_device):
    """The adjoint of the MAM4B_MIXED step (mam4b_adjoint_slab_ex): its
    gradient against the FP64 adjoint's on every entry, and against central
    finite differences of the FP64 forward step, in units of relative
    sensitivity |g - ref| |x| / |J_cell|; both checkpoint intervals give the
    same gradient bit for bit."""
    import torch
    w = make_workload("c5", ncol=32, seed=93)
    x = w["in_slab"]
    n = x.shape[1]
    wts = pdel_over_g(w)
    ybar = objective_bar(wts, w["dt"], n)
    ctx = native.Context()
    g64 = adjoint(ctx, x, w["pblh"], ybar, w)

    def adjoint_mixed():
        xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        pt = torch.from_numpy(np.ascontiguousarray(w["pblh"])).cuda()
        yt = torch.from_numpy(np.ascontiguousarray(ybar)).cuda()
        xb = torch.full((native.NIN, n), float("nan"), dtype=torch.float64, device="cuda")
        ctx.adjoint_slab(xt.data_ptr(), pt.data_ptr(), yt.data_ptr(), xb.data_ptr(), n,
                         w["ncol"], w["nlev"], w["dt"], precision=native.MIXED)
        torch.cuda.synchronize()
        return xb.cpu().numpy()

    gmx = adjoint_mixed()
    ctx.set_adjoint_checkpoint(4)
    assert np.array_equal(adjoint_mixed(), gmx)
    ctx.set_adjoint_checkpoint(1)
    assert np.isfinite(gmx).all()
    for f in (1, 2, 4):
        assert (gmx[f] == 0.0).all()
    out = forward(ctx, x, w["pblh"], w)
    J0 = objective_cells(x, out, wts, w["dt"])
    for k in J_STATE:
        g64[5 + k] += wts
        gmx[5 + k] += wts
    err = np.abs(gmx[DIFF_FIELDS] - g64[DIFF_FIELDS]) * np.abs(x[DIFF_FIELDS]) / np.abs(J0)
    within = float((err <= 1e-5).mean())
    print("MIXED_ADJOINT vs FP64 adjoint: median %.3g, 99%% %.3g, within 1e-5 %.5f, max %.3g"
          % (np.median(err), np.quantile(err, 0.99), within, err.max()))
    assert np.median(err) <= 1e-8
    assert within >= 0.99
    # central differences of the FP64 forward on 32 cells
    rng = np.random.default_rng(93)
    cells = rng.choice(n, 32, replace=False)

    def J(xv):
        return objective_cells(xv, forward(ctx, xv, w["pblh"], w), wts, w["dt"])

    rows = _fd_entries(J, x, gmx, J0, cells, DIFF_FIELDS)
    fd = rows[:, 2]
    print("MIXED_ADJOINT vs FP64 differences: median %.3g, within 1e-6 %.5f, within 1e-5 %.5f"
          % (np.median(fd), (fd <= 1e-6).mean(), (fd <= 1e-5).mean()))
    assert np.median(fd) <= 1e-8
    assert (fd <= 1e-5).mean() >= 0.99
    with pytest.raises(native.MicrophysicsError):
        ctx.adjoint_slab(0, 0, 0, 0, n, w["ncol"], w["nlev"], w["dt"],
                         precision=native.MIXED_FAST)
