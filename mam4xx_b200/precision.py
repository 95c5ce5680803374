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
