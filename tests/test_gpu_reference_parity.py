"""Parity of the CUDA step with the mam4xx reference itself.

1. Bitwise, on the GPU. The reference headers compiled unchanged for the
   GPU (oracle/_ref/libmam4ref_gpu.so: CUDA libm, no FMA contraction, like
   the product) differ from the product only if the product's algorithm
   does. Every output must be equal bit for bit, for every workload
   configuration, process switch and the edge cases.

2. Statistical, at full size, against the host build of the reference
   (oracle/_ref/libmam4ref.so, glibc libm): C2 (4,096 x 72), C3 and C4
   (65,536 x 72). The reference's algorithm amplifies last-bit libm
   differences (SOA sub-stepping, the water-uptake quartic), so the bar is
   the one of oracle.pyoracle.parity: at least as close to the host build
   as the host build is to itself under 1..2-ulp libm perturbations. The
   target metric, error relative per tendency (absolute floor 1e-30
   kg/kg), is reported beside the state-relative one.

3. Conservation on the GPU, per cell and per column (weights pdel/g), in
   amicphys' internal units (mam4_amicphys.hpp:97-154): SO4 + H2SO4, the
   SOA family 0.08 SOA + (12.011/150) SOAG, and POM, BC, DST, NaCl, MOM, to
   1e-13 relative, for FP64 and MIXED at full size.
"""

import json

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import (ADV_MASS, MW_DRY_AIR, POPULATIONS, make_workload,
                                   pblh_per_cell)
from oracle import pyoracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_gpu():
    if not pyoracle.reference_gpu_available():
        pytest.skip("reference headers not compiled for the GPU (mam4xx tree absent at build)")
    return pyoracle.RefGpuOracle()


def run_gpu(w, cfg=None, precision=native.FP64):
    x = torch.from_numpy(np.ascontiguousarray(w["in_slab"])).cuda()
    pb = torch.from_numpy(np.ascontiguousarray(w["pblh"])).cuda()
    n = x.shape[1]
    out = torch.full((native.NOUT, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx = native.Context(cfg)
    ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"], w["dt"],
                  precision=precision)
    torch.cuda.synchronize()
    assert not (ctx.last_status() & (native.FLAG_NONFINITE_INPUT | native.FLAG_NONFINITE_OUTPUT))
    ctx.close()
    return out.cpu().numpy()


def assert_bitwise(got, ref):
    diff = np.argwhere(got != ref)
    assert diff.size == 0, "%d of %d entries differ, first (output, cell) %s: %r vs %r" % (
        len(diff), got.size, diff[0], got[tuple(diff[0])], ref[tuple(diff[0])])


@pytest.mark.parametrize("name,ncol", [("c1", None), ("c2", 512), ("c3", 512), ("c4", 1024),
                                       ("c5", 256), ("c4_stress", 256)])
def test_step_bitwise_equals_reference_headers_on_gpu(cuda_device, ref_gpu, name, ncol):
    w = make_workload(name, ncol=ncol)
    ref = ref_gpu.step(w["in_slab"], pblh_per_cell(w), w["dt"])
    assert_bitwise(run_gpu(w), ref)


@pytest.mark.parametrize("cfg", [
    dict(do_cond=0), dict(do_rename=0), dict(do_newnuc=0), dict(do_coag=0),
    dict(gaexch_h2so4_uptake_optaa=1), dict(n_so4_monolayers_pcage=3),
    dict(do_cond=0, do_newnuc=0)])
def test_process_switches_bitwise_against_reference_headers(cuda_device, ref_gpu, cfg):
    w = make_workload("c2", ncol=64)
    ref = ref_gpu.step(w["in_slab"], pblh_per_cell(w), w["dt"], cfg=pyoracle.default_config(**cfg))
    assert_bitwise(run_gpu(w, cfg=native.default_config(**cfg)), ref)


def test_edge_cases_bitwise_against_reference_headers(cuda_device, ref_gpu):
    from test_gpu_parity import _edge_workload
    w = _edge_workload()
    ref = ref_gpu.step(w["in_slab"], pblh_per_cell(w), w["dt"])
    assert_bitwise(run_gpu(w), ref)


def tendency_rel_err(got, ref, dt, floor=1e-30):
    """The per-tendency error: |d tend| relative to |tend_ref|, where an error
    below the absolute floor (1e-30 kg/kg over the step) counts as zero;
    the 16 size/density/water outputs relative to their value."""
    e_t = np.abs(got[:52] - ref[:52]) / np.maximum(np.abs(ref[:52]), floor / dt)
    e_t = np.where(np.abs(got[:52] - ref[:52]) * dt <= floor, 0.0, e_t)
    e_d = np.abs(got[52:] - ref[52:]) / np.maximum(np.abs(ref[52:]), 1e-300)
    return np.concatenate([e_t, e_d], axis=0)


@pytest.mark.parametrize("name", ["c2", "c3", "c4"])
def test_full_size_against_reference_host_build(cuda_device, ref_oracle, name):
    w = make_workload(name)
    pb = pblh_per_cell(w)
    ref = ref_oracle.step(w["in_slab"], pb, w["dt"])
    got = run_gpu(w)
    assert np.isfinite(got).all()
    summary = pyoracle.parity(got, ref, w["in_slab"], pb, w["dt"])
    et = tendency_rel_err(got, ref, w["dt"])
    ec = et.max(axis=0)
    summary["tendency_rel"] = {
        "cells_within_1e-12": float((ec <= 1e-12).mean()),
        "entries_within_1e-12": float((et <= 1e-12).mean()),
        "cell_quantiles": [float(q) for q in np.quantile(ec, (0.5, 0.9, 0.99, 0.999))],
        "max": float(ec.max())}
    print("PARITY", name, json.dumps(summary))


# ------------------------------------------------------------ conservation
def _families():
    fam = {}
    for s, (_, sp) in enumerate(POPULATIONS):
        if sp != "num":
            fam.setdefault(sp, []).append(s)
    return fam


def family_totals(state52):
    """Per-cell totals of each species family in amicphys' internal units
    (mol/mol scaled by fcvt_aer / fcvt_gas, mam4_amicphys.hpp:127-152) from
    the 52 prognostics in kg/kg (H2SO4, SOAG, 25 interstitial, 25 cloud)."""
    out = {}
    for sp, slots in _families().items():
        f = 0.08 if sp in ("SOA", "POM") else 1.0
        t = 0.0
        for s in slots:
            i31 = 6 + s
            t = t + f * (state52[2 + s] + state52[27 + s]) * (MW_DRY_AIR / ADV_MASS[i31])
        if sp == "SO4":
            t = t + state52[0] * (MW_DRY_AIR / ADV_MASS[2])
        if sp == "SOA":
            t = t + (12.011 / 150.0) * state52[1] * (MW_DRY_AIR / ADV_MASS[5])
        out[sp] = t
    return out


def pdel_weights(w):
    p = w["in_slab"][1].reshape(w["ncol"], w["nlev"])
    edges = np.concatenate([p[:, :1] * 0.5, 0.5 * (p[:, 1:] + p[:, :-1]), p[:, -1:] * 1.01],
                           axis=1)
    return np.abs(np.diff(edges, axis=1)) / 9.80616


@pytest.mark.parametrize("name,precision", [("c2", native.FP64), ("c3", native.FP64),
                                            ("c4", native.FP64), ("c3", native.MIXED),
                                            ("c4", native.MIXED)])
def test_family_conservation_per_cell_and_column(cuda_device, name, precision):
    w = make_workload(name)
    got = run_gpu(w, precision=precision)
    x = w["in_slab"]
    before = family_totals(x[5:57])
    after = family_totals(x[5:57] + got[:52] * w["dt"])
    wts = pdel_weights(w)
    worst = {}
    for sp in before:
        b, a = before[sp], after[sp]
        cell = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
        cb = (b.reshape(w["ncol"], w["nlev"]) * wts).sum(axis=1)
        ca = (a.reshape(w["ncol"], w["nlev"]) * wts).sum(axis=1)
        col = np.abs(ca - cb) / cb
        worst[sp] = (float(cell.max()), float(col.max()))
        assert cell.max() <= 1e-13, (sp, "cell", int(np.argmax(cell)), cell.max())
        assert col.max() <= 1e-13, (sp, "column", int(np.argmax(col)), col.max())
    print("CONSERVATION", name, precision, json.dumps(worst))
