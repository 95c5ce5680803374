"""SOA condensation sub-step histogram of a workload configuration,
measured on the CPU restatement (test infrastructure).

The SOA gas-particle exchange of amicphys (gasaerexch_soaexch.hpp:80-335)
integrates with an adaptive step dt = 0.05 / max_ll sum_n k_n |phi_n| until
the condensation time step is covered, at most 1000 passes
(gasaerexch_soaexch.hpp:93, 170-173, 240-270). The pass count of each cell's
clear subarea is taken from mam4orc_soa_niter (oracle/mam4_oracle.c), the
restatement that is bit-for-bit equal to the reference build.

Writes baseline/soa_passes_<config>.json: counts of cells per pass number
over the configuration's full seeded workload, with its quantiles.
Usage: python oracle/soa_pass_histogram.py [--config c4] [--ncol N]
"""

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)


def histogram(name="c4", ncol=None, nthreads=0):
    """(counts per pass number, summary) of configuration `name`."""
    from mam4xx_b200.workloads import make_workload, pblh_per_cell
    from oracle.pyoracle import PortOracle
    w = make_workload(name, ncol=ncol)
    it = np.asarray(PortOracle().soa_niter(w["in_slab"], pblh_per_cell(w), w["dt"],
                                           nthreads=nthreads or (os.cpu_count() or 1)))
    counts = np.bincount(it)
    run = it[it > 0]
    summary = {"cells": int(it.size), "ncol": int(w["ncol"]), "nlev": int(w["nlev"]),
               "cells_without_loop": int((it == 0).sum()),
               "min_passes": int(run.min()) if run.size else 0,
               "max_passes": int(it.max()),
               "mean_passes": float(run.mean()) if run.size else 0.0,
               "quantiles": {str(q): float(np.quantile(run, q))
                             for q in (0.5, 0.9, 0.99, 0.999, 0.9999)} if run.size else {},
               "frac_within_1_20": float(((run >= 1) & (run <= 20)).mean()) if run.size else 0.0}
    return counts, summary


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c4")
    ap.add_argument("--ncol", type=int, default=None)
    a = ap.parse_args(argv)
    counts, summary = histogram(a.config, a.ncol)
    doc = {"what": "SOA condensation sub-step (pass) count per cell, clear subarea, counted on "
                   "the CPU restatement (mam4orc_soa_niter); counts[k] = cells with k passes "
                   "(0 = no SOA loop)",
           "config": a.config,
           "generator": "python oracle/soa_pass_histogram.py --config %s%s"
                        % (a.config, "" if a.ncol is None else " --ncol %d" % a.ncol),
           "summary": summary, "counts": [int(c) for c in counts]}
    out = os.path.join(ROOT, "baseline", "soa_passes_%s.json" % a.config)
    with open(out, "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    print(json.dumps(summary, indent=1))


if __name__ == "__main__":
    main()
