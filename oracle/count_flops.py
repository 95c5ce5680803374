"""Algorithmic flops per cell of the microphysics step, per workload
configuration, counted by the operation-counting build of the CPU
restatement (oracle/libmam4oracle_count.so, see oracle/opcount.cpp).

Counting rule: + - * / one flop each (the restatement has no fused
multiply-add); each libm call (exp, log, pow, sqrt, cbrt, erfc, log10,
hypot, atan2, sin, cos) one "special", reported apart and not in `flops`;
min/max/abs/round and compares are not flops. The counts are data-dependent
(SOA sub-step counts, process early-outs), so they are averages over a
sample of each configuration's seeded cells.

Writes baseline/flops_per_cell.json (committed; bench.py reads it for the
FP64 roofline). Usage: python oracle/count_flops.py [--cells N]
"""

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
OUT = os.path.join(ROOT, "baseline", "flops_per_cell.json")


def count(cells=36864):
    from mam4xx_b200.workloads import CONFIGS, make_workload, pblh_per_cell
    from oracle.pyoracle import CountOracle, PortOracle
    co = CountOracle()
    res = {}
    for name in sorted(CONFIGS):
        w = make_workload(name, ncol=min(CONFIGS[name]["ncol"], -(-cells // 72)))
        n = min(cells, w["in_slab"].shape[1])
        x = np.ascontiguousarray(w["in_slab"][:, :n])
        pb = pblh_per_cell(w)[:n]
        out, t = co.step(x, pb, w["dt"])
        ref = PortOracle().step(x, pb, w["dt"])
        if not np.array_equal(out, ref):
            raise RuntimeError("counting build differs from the plain build on %s" % name)
        flops = t["add"] + t["mul"] + t["div"]
        res[name] = {"sample_cells": n, "flops_per_cell": flops / n,
                     "special_per_cell": t["special"] / n,
                     "add_per_cell": t["add"] / n, "mul_per_cell": t["mul"] / n,
                     "div_per_cell": t["div"] / n, "minmax_per_cell": t["minmax"] / n,
                     "cmp_per_cell": t["cmp"] / n}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=36864)
    a = ap.parse_args(argv)
    res = count(a.cells)
    doc = {"what": "algorithmic operations per cell of one microphysics step (calcsize + water "
                   "uptake + amicphys), counted on the CPU restatement with an operation-counting "
                   "real type; flops = add + mul + div (no fma in the restatement); libm calls "
                   "counted apart as specials",
           "sample": "sample_cells cells of each configuration's seeded workload drawn with "
                     "ceil(sample_cells / 72) columns (mam4xx_b200.workloads)",
           "generator": "python oracle/count_flops.py --cells %d" % a.cells,
           "configs": res}
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
