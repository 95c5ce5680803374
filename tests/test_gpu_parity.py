"""Parity of the CUDA step (through the C ABI) with the oracle.

Two layers:

1. Algorithm. The product kernel and the oracle's restatement compiled for
   the GPU (oracle/libmam4oracle_gpu.so: same math library, no FMA
   contraction on either side) must agree bit for bit on every output, for
   every workload configuration, process switch and edge case. The
   restatement itself agrees bit for bit with the mam4xx headers compiled on
   the host (tests/test_oracle.py).

2. Math library. Against the canonical host oracle (glibc) the kernel must
   be as close as the oracle is to itself when every libm result is moved by
   1..2 ulps (oracle.pyoracle.parity): the target tolerance of 1e-12
   (state-relative per tendency, absolute floor 1e-30; relative for the
   diameters, densities and water) holds on the same fraction of cells as in
   that baseline and the error quantiles stay within 3x of it. No tighter
   libm-independent bound exists: the SOA sub-stepping loop and the
   water-uptake quartic amplify last-bit differences (the reference compiled
   with FMA contraction disagrees with itself by up to O(1) in coarse-mode
   SOA on a few cells in a thousand).
"""

import numpy as np
import pytest
import torch

from mam4xx_b200 import native
from mam4xx_b200.workloads import make_workload, pblh_per_cell
from oracle.pyoracle import GpuOracle, parity

pytestmark = pytest.mark.gpu

def run_gpu(w, cfg=None, diag=False, ctx=None):
    x = torch.from_numpy(np.ascontiguousarray(w["in_slab"])).cuda()
    pb = torch.from_numpy(np.ascontiguousarray(w["pblh"])).cuda()
    n = x.shape[1]
    out = torch.full((native.NOUT, n), float("nan"), dtype=torch.float64, device="cuda")
    ctx = ctx or native.Context(cfg)
    if diag:
        dg = torch.full((native.NDIAG, n), float("nan"), dtype=torch.float64, device="cuda")
        ctx.step([x[f].data_ptr() for f in range(native.NIN)], pb.data_ptr(),
                 [out[f].data_ptr() for f in range(native.NOUT)], w["ncol"], w["nlev"], w["dt"],
                 diag_ptrs=[dg[f].data_ptr() for f in range(native.NDIAG)])
    else:
        ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"],
                      w["dt"])
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    return (res, dg.cpu().numpy()) if diag else res


def check(w, gpu, orc, cfg=None):
    assert np.isfinite(gpu).all()
    return parity(gpu, orc, w["in_slab"], pblh_per_cell(w), w["dt"], cfg=cfg)


def check_bitwise(w, gpu, cfg=None, diag=None):
    """Kernel output == restatement on the GPU, bit for bit."""
    g = GpuOracle()
    if diag is None:
        ref = g.step(w["in_slab"], pblh_per_cell(w), w["dt"], cfg=cfg)
        diff = np.argwhere(gpu != ref)
        assert diff.size == 0, "%d entries differ, first %s: %r vs %r" % (
            len(diff), diff[0], gpu[tuple(diff[0])], ref[tuple(diff[0])])
    else:
        ref, rdg = g.step(w["in_slab"], pblh_per_cell(w), w["dt"], cfg=cfg, diag=True)
        np.testing.assert_array_equal(gpu, ref)
        np.testing.assert_array_equal(diag, rdg)


@pytest.mark.parametrize("name,ncol", [("c1", None), ("c2", 512), ("c3", 512), ("c4", 512),
                                       ("c5", 256)])
def test_step_bitwise_equals_restatement_on_gpu(cuda_device, name, ncol):
    w = make_workload(name, ncol=ncol)
    check_bitwise(w, run_gpu(w))


@pytest.mark.parametrize("name,ncol", [("c1", None), ("c2", None), ("c3", 1024), ("c4", 1024),
                                       ("c5", 512)])
def test_step_matches_oracle(cuda_device, port_oracle, name, ncol):
    w = make_workload(name, ncol=ncol)
    orc = port_oracle.step(w["in_slab"], pblh_per_cell(w), w["dt"])
    gpu = run_gpu(w)
    summary = check(w, gpu, orc)
    print(name, summary)


def test_step_matches_reference_build(cuda_device, ref_oracle):
    w = make_workload("c2", ncol=256)
    orc = ref_oracle.step(w["in_slab"], pblh_per_cell(w), w["dt"])
    check(w, run_gpu(w), orc)


def test_process_diagnostics_match_oracle(cuda_device, port_oracle):
    w = make_workload("c2", ncol=256)
    gpu, gdg = run_gpu(w, diag=True)
    assert np.isfinite(gdg).all()
    check_bitwise(w, gpu, diag=gdg)
    orc = port_oracle.step(w["in_slab"], pblh_per_cell(w), w["dt"])
    check(w, gpu, orc)


@pytest.mark.parametrize("cfg", [
    dict(do_cond=0), dict(do_rename=0), dict(do_newnuc=0), dict(do_coag=0),
    dict(gaexch_h2so4_uptake_optaa=1), dict(n_so4_monolayers_pcage=3),
    dict(do_cond=0, do_newnuc=0)])
def test_process_switches(cuda_device, port_oracle, cfg):
    from oracle.pyoracle import default_config
    w = make_workload("c2", ncol=64)
    orc = port_oracle.step(w["in_slab"], pblh_per_cell(w), w["dt"], cfg=default_config(**cfg))
    gpu = run_gpu(w, cfg=native.default_config(**cfg))
    check_bitwise(w, gpu, cfg=default_config(**cfg))
    check(w, gpu, orc, cfg=default_config(**cfg))


def _edge_workload():
    """Cells at the branch boundaries the reference tests: cloud fraction at
    and around the subarea cut-offs, empty modes, zero gases, tiny and large
    numbers, negative inputs (clipped), saturated and dry air."""
    w = make_workload("c2", ncol=6, nlev=12, seed=99)
    x = w["in_slab"]
    x[4, :] = np.array([0.0, 1e-5, 0.99999e-5, 0.999, 0.9990001, 1.0] * 12)[: x.shape[1]]
    x[7:32, 0:6] = 0.0                 # empty interstitial aerosol
    x[32:57, 6:12] = 0.0               # empty cloud-borne aerosol
    x[5:7, 12:18] = 0.0                # no condensing gas
    x[7 + 12, 18:24] = 0.0             # aitken number zero with mass present
    x[7:32, 24:30] *= -1.0             # negative mixing ratios are clipped
    x[3, 30:36] *= 50.0                # supersaturated vapour
    x[3, 36:42] = 0.0                  # dry air
    x[5, 42:48] = 1e-7                 # strong H2SO4 (nucleation, fast uptake)
    x[7 + 7, 48:54] = 1e12             # huge accumulation number
    x[2, 54:60] = 5.0                  # inside the boundary layer
    return w


def test_edge_cases(cuda_device, port_oracle):
    w = _edge_workload()
    gpu = run_gpu(w)
    check_bitwise(w, gpu)
    orc = port_oracle.step(w["in_slab"], pblh_per_cell(w), w["dt"])
    check(w, gpu, orc)


@pytest.mark.parametrize("ncol,nlev", [(1, 1), (3, 7), (1, 129), (97, 5)])
def test_ragged_sizes(cuda_device, port_oracle, ncol, nlev):
    w = make_workload("c2", ncol=ncol, nlev=nlev, seed=5)
    check_bitwise(w, run_gpu(w))


def test_empty_batch(cuda_device):
    ctx = native.Context()
    x = torch.zeros((native.NIN, 1), dtype=torch.float64, device="cuda")
    out = torch.zeros((native.NOUT, 1), dtype=torch.float64, device="cuda")
    pb = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), 1, 0, 72, 1800.0)
    torch.cuda.synchronize()
    assert ctx.last_status() == 0


def test_nonfinite_input_is_flagged(cuda_device):
    w = make_workload("c1", ncol=2)
    w["in_slab"][0, 3] = float("nan")
    ctx = native.Context()
    run_gpu(w, ctx=ctx)
    assert ctx.last_status() & native.FLAG_NONFINITE_INPUT
    assert not (ctx.last_status() & native.FLAG_NONFINITE_INPUT)  # cleared once read


def test_host_entry_matches_device_entry(cuda_device):
    w = make_workload("c2", ncol=32)
    dev = run_gpu(w)
    ctx = native.Context()
    x = np.ascontiguousarray(w["in_slab"])
    out = np.zeros((native.NOUT, x.shape[1]))
    ctx.step_host(x.ctypes.data, w["pblh"].ctypes.data, out.ctypes.data, x.shape[1],
                  w["ncol"], w["nlev"], w["dt"])
    np.testing.assert_array_equal(out, dev)


def test_host_entry_chunked_pipeline(cuda_device):
    """The host entry streams columns in chunks of up to ~2^18 cells over
    copy-in, compute and copy-out streams: 16,000 x 72 cells make 6 chunks,
    the first two smaller, the last one ragged. A padded
    host leading dimension and a second, smaller call on the same context
    (chunk scratch reused) must give the device entry's results bit for bit."""
    ctx = native.Context()
    for ncol, pad in ((16000, 7), (9000, 0)):
        w = make_workload("c4", ncol=ncol, seed=40 + ncol)
        dev = run_gpu(w)
        n = w["in_slab"].shape[1]
        ld = n + pad
        x = np.zeros((native.NIN, ld))
        x[:, :n] = w["in_slab"]
        out = np.full((native.NOUT, ld), -7.0)
        ctx.step_host(x.ctypes.data, w["pblh"].ctypes.data, out.ctypes.data, ld,
                      w["ncol"], w["nlev"], w["dt"])
        np.testing.assert_array_equal(out[:, :n], dev)
        assert (out[:, n:] == -7.0).all()  # padding untouched


def test_full_size_properties(cuda_device):
    """At 65,536 x 72 cells (too many for the oracle): finite outputs,
    bitwise-deterministic reruns, non-negative post-step state, and
    per-species conservation of POM/BC/DST/NaCl/MOM in grid units summed
    over the whole batch (checksum of checksums)."""
    from mam4xx_b200.workloads import POPULATIONS
    w = make_workload("c4")
    a = run_gpu(w)
    b = run_gpu(w)
    assert np.isfinite(a).all()
    assert np.array_equal(a, b)
    x = w["in_slab"]
    after = x[5:57] + a[:52] * w["dt"]
    assert (after >= -1e-14 * np.abs(x[5:57])).all()
    for spec in ("POM", "BC", "DST", "NaCl", "MOM"):
        rows = [2 + s for s, (_, sp) in enumerate(POPULATIONS) if sp == spec]
        rows += [27 + s for s, (_, sp) in enumerate(POPULATIONS) if sp == spec]
        tot0 = np.sum([x[5 + r].sum() for r in rows])
        tot1 = np.sum([after[r].sum() for r in rows])
        assert abs(tot1 - tot0) <= 1e-12 * tot0, spec
