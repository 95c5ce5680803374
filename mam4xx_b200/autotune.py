"""Chooses the launch shape of the step's kernels on this device and writes
it to the tuning file that new contexts load (mam4b_create reads
mam4b_tuning.json next to libmam4b.so when it was chosen on a device of the
same name).

The search is mam4b_autotune (include/mam4b.h): every stage's candidate
block sizes and register caps, the persistent solver's blocks per SM and
the cells each thread steps, timed stage by stage on a full-size batch of
the uneven-batching workload (c4, 65,536 x 72 cells). The reference's only
launch knob is the Kokkos team size (src/validation/validation.hpp:25-30).

Usage (on the GPU): python -m mam4xx_b200.autotune [--ncol N] [--reps R]
                                                   [--out PATH]
"""

import argparse
import json
import os

PKG = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(PKG, "mam4b_tuning.json")


def tune(ncol=65536, workload="c4", reps=5, precision=0):
    """Runs the autotuner on cuda:0; returns the tuning-file document."""
    import torch
    from . import native
    from .workloads import make_workload
    dev = torch.device("cuda:0")
    w = make_workload(workload, ncol=ncol)
    x = torch.from_numpy(w["in_slab"]).to(dev)
    pb = torch.from_numpy(w["pblh"]).to(dev)
    n = x.shape[1]
    out = torch.empty((native.NOUT, n), dtype=torch.float64, device=dev)
    ctx = native.Context()
    ctx.set_tuning(native.default_tuning())
    t, d_ms, b_ms = ctx.autotune(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"],
                                 w["nlev"], w["dt"], precision=precision, reps=reps)
    ctx.close()
    doc = {"device": torch.cuda.get_device_name(dev)}
    doc.update(t.as_dict())
    doc["chosen_on"] = {"workload": "%s, %d columns x %d levels" % (workload, w["ncol"], w["nlev"]),
                        "precision": precision, "reps": reps,
                        "default_ms": d_ms, "tuned_ms": b_ms}
    return doc


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ncol", type=int, default=65536)
    ap.add_argument("--workload", default="c4")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args(argv)
    doc = tune(a.ncol, a.workload, a.reps)
    with open(a.out, "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    print(json.dumps(doc))


if __name__ == "__main__":
    main()
