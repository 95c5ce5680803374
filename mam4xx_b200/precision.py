"""Error report of the mixed-precision step against FP64 results.

Errors are measured per cell and output, as for the FP64 parity tests:
tendencies relative to the state they change (|d tend| * dt divided by the
larger of |q before| and |q after|, floor 1e-30), the 16 size/density/water
outputs relative to their FP64 value.
"""

import numpy as np

from .workloads import NOUT

STATE0 = 5  # first prognostic input field (H2SO4), 52 of them


def output_errors(out, ref, in_slab, dt):
    """(68, n) per-output, per-cell errors of `out` against `ref`."""
    q0 = np.abs(in_slab[STATE0:STATE0 + 52])
    q1 = np.abs(in_slab[STATE0:STATE0 + 52] + ref[:52] * dt)
    e_t = np.abs(out[:52] - ref[:52]) * dt / np.maximum(np.maximum(q0, q1), 1e-30)
    e_d = np.abs(out[52:] - ref[52:]) / np.maximum(np.abs(ref[52:]), 1e-300)
    return np.concatenate([e_t, e_d], axis=0)


def error_report(out, ref, in_slab, dt, tol=1e-5):
    """Max and median error of every output, the overall maximum and median
    and the fraction of cells whose 68 outputs are all within tol."""
    err = output_errors(out, ref, in_slab, dt)
    assert err.shape[0] == NOUT
    per_cell = err.max(axis=0)
    return {
        "max": float(err.max()),
        "median": float(np.median(err)),
        "per_output_max": [float(v) for v in err.max(axis=1)],
        "per_output_median": [float(v) for v in np.median(err, axis=1)],
        "cells_within_tol": float((per_cell <= tol).mean()),
        "cell_err_quantiles": {str(q): float(np.quantile(per_cell, q))
                               for q in (0.5, 0.9, 0.99, 0.999)},
        "tol": tol,
    }


def cell_errors_device(out, ref, in_slab, dt, chunk=1 << 20):
    """Per-cell error (the largest of the cell's 68 output errors, as in
    output_errors) of `out` against `ref`, on the device: torch tensors
    (68, n), (68, n), (57, n) float64; returns a float64 tensor (n,)."""
    import torch
    n = out.shape[1]
    cell_err = torch.empty(n, dtype=torch.float64, device=out.device)
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        q0 = in_slab[STATE0:STATE0 + 52, c0:c1].abs()
        q1 = (in_slab[STATE0:STATE0 + 52, c0:c1] + ref[:52, c0:c1] * dt).abs()
        e_t = (out[:52, c0:c1] - ref[:52, c0:c1]).abs() * dt / torch.clamp(torch.maximum(q0, q1),
                                                                            min=1e-30)
        e_d = (out[52:, c0:c1] - ref[52:, c0:c1]).abs() / torch.clamp(ref[52:, c0:c1].abs(),
                                                                      min=1e-300)
        e = torch.cat([e_t, e_d], dim=0)
        e = torch.where(torch.isnan(e), torch.full_like(e, float("inf")), e)
        cell_err[c0:c1] = e.max(dim=0).values
    return cell_err


def conditioning_split(err, cond_err, tol=1e-5):
    """Classifies the cells a form gets wrong by more than tol (err, per
    cell) by the FP64 step's own sensitivity cond_err (per cell: its
    results for its inputs rounded to single precision against its results
    for the exact inputs): `ill_conditioned` cells, where that rounding
    alone moves the FP64 result by more than tol, and the rest. Tensors (n,)
    on one device; returns a dict of counts and fractions."""
    out = err > tol
    ill = cond_err > tol
    n = int(err.numel())
    n_out = int(out.sum())
    n_ill_out = int((out & ill).sum())
    return {"tol": tol, "cells": n,
            "ill_conditioned_cells": int(ill.sum()),
            "outside_tol": n_out,
            "outside_tol_ill_conditioned": n_ill_out,
            "outside_tol_well_conditioned": n_out - n_ill_out,
            "well_conditioned_within_tol": float(1.0 - (n_out - n_ill_out) / max(1, int((~ill).sum())))}


def error_report_device(out, ref, in_slab, dt, tol=1e-5, chunk=1 << 20):
    """error_report over every cell, computed on the device in chunks of
    cells (torch tensors (68, n), (68, n), (57, n) float64 on one device).
    Per-output medians are taken over a seeded sample of 2^20 cells."""
    import torch
    n = out.shape[1]
    per_out_max = torch.zeros(NOUT, dtype=torch.float64, device=out.device)
    cell_err = torch.empty(n, dtype=torch.float64, device=out.device)
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        q0 = in_slab[STATE0:STATE0 + 52, c0:c1].abs()
        q1 = (in_slab[STATE0:STATE0 + 52, c0:c1] + ref[:52, c0:c1] * dt).abs()
        e_t = (out[:52, c0:c1] - ref[:52, c0:c1]).abs() * dt / torch.clamp(torch.maximum(q0, q1),
                                                                            min=1e-30)
        e_d = (out[52:, c0:c1] - ref[52:, c0:c1]).abs() / torch.clamp(ref[52:, c0:c1].abs(),
                                                                      min=1e-300)
        e = torch.cat([e_t, e_d], dim=0)
        e = torch.where(torch.isnan(e), torch.full_like(e, float("inf")), e)
        per_out_max = torch.maximum(per_out_max, e.max(dim=1).values)
        cell_err[c0:c1] = e.max(dim=0).values
    g = torch.Generator(device="cpu").manual_seed(12345)
    sample = torch.randperm(n, generator=g)[: min(n, 1 << 20)].to(out.device)
    q0 = in_slab[STATE0:STATE0 + 52][:, sample].abs()
    q1 = (in_slab[STATE0:STATE0 + 52][:, sample] + ref[:52][:, sample] * dt).abs()
    e_t = (out[:52][:, sample] - ref[:52][:, sample]).abs() * dt / torch.clamp(
        torch.maximum(q0, q1), min=1e-30)
    e_d = (out[52:][:, sample] - ref[52:][:, sample]).abs() / torch.clamp(
        ref[52:][:, sample].abs(), min=1e-300)
    es = torch.cat([e_t, e_d], dim=0)
    qs = (0.5, 0.9, 0.99, 0.999, 0.9999)
    cq = torch.quantile(cell_err[sample], torch.tensor(qs, dtype=torch.float64,
                                                       device=out.device))
    return {
        "cells": int(n),
        "max": float(per_out_max.max()),
        "median": float(es.median()),
        "per_output_max": [float(v) for v in per_out_max.cpu()],
        "per_output_median": [float(v) for v in es.median(dim=1).values.cpu()],
        "cells_within_tol": float((cell_err <= tol).double().mean()),
        "cells_outside_tol": int((cell_err > tol).sum()),
        "cell_err_quantiles": {str(q): float(v) for q, v in zip(qs, cq.cpu())},
        "tol": tol,
    }
