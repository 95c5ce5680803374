"""Workload calibration (CPU): the uneven-batching configuration c4 must
spread the SOA condensation sub-step count over 1..20 passes per cell, as
measured on the CPU restatement, and the committed histogram must be the
one its generator gives for the full configuration."""

import json
import os

import numpy as np

from mam4xx_b200.workloads import CONFIGS, make_workload

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c4_soa_pass_histogram_matches_committed_and_spans_1_to_20(port_oracle):
    from oracle.soa_pass_histogram import histogram
    with open(os.path.join(ROOT, "baseline", "soa_passes_c4.json")) as f:
        doc = json.load(f)
    counts, summary = histogram("c4")
    assert summary["cells"] == CONFIGS["c4"]["ncol"] * CONFIGS["c4"]["nlev"]
    assert [int(c) for c in counts] == doc["counts"]
    assert summary["min_passes"] == 1
    # every pass count from 1 to 20 occurs, and 1..20 holds 99.99 % of cells
    assert all(c > 0 for c in counts[1:21])
    assert summary["frac_within_1_20"] >= 0.9999
    # a cell without a loop has no SOA uptake at all; they are rare
    assert summary["cells_without_loop"] <= 0.001 * summary["cells"]


def test_c4_stress_keeps_the_heavy_tail(port_oracle):
    """The stress case (common number range) reaches the reference's cap."""
    w = make_workload("c4_stress", ncol=512)
    from mam4xx_b200.workloads import pblh_per_cell
    it = np.asarray(port_oracle.soa_niter(w["in_slab"], pblh_per_cell(w), w["dt"], nthreads=0))
    assert it.max() == 1001 and it.mean() > 50


def test_c4_differs_from_stress_only_in_numbers():
    a = make_workload("c4", ncol=4)["in_slab"]
    b = make_workload("c4_stress", ncol=4)["in_slab"]
    from mam4xx_b200.workloads import IN_AER_C, IN_AER_I, NUMBER_SLOTS
    num_rows = {base + s for base in (IN_AER_I, IN_AER_C) for s in NUMBER_SLOTS}
    for f in range(a.shape[0]):
        if f in num_rows:
            assert a[f].max() <= 1e6 * (1 + 1e-12) and a[f].min() >= 1e5 * (1 - 1e-12)
        else:
            np.testing.assert_array_equal(a[f], b[f])
