"""The CPU oracle pinned against mam4xx's own known answers and against the
reference headers compiled unchanged (oracle/_ref)."""

import json
import os

import numpy as np
import pytest

from mam4xx_b200.workloads import make_workload, pblh_per_cell

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.mark.parametrize("which", ["port", "ref"])
def test_h2so4_update_known_answers(which, request):
    """30 vectors of src/tests/mam4_gasaerexch_unit_tests.cpp:40-206 at
    dt = 1, 1e-20, 10 (Taylor, no-uptake and exponential branches), with
    the test's own tolerance of 100*FLT_EPSILON."""
    orc = request.getfixturevalue("port_oracle" if which == "port" else "ref_oracle")
    g = _golden("gasaerexch_h2so4.json")
    tol = g["rel_tol"]
    for p in range(3):
        for n in range(10):
            qg, qavg, qa = orc.h2so4_update(g["dts"][p], g["qgas_netprod_otrproc"],
                                            g["uptkaer"][p][n], g["in_qgas_cur"][p][n],
                                            g["in_qaer_cur"][p][n])
            assert qg == pytest.approx(g["out_qgas_cur"][p][n], rel=tol)
            assert qavg == pytest.approx(g["out_qgas_avg"][p][n], rel=tol)
            np.testing.assert_allclose(qa, g["out_qaer_cur"][p][n], rtol=tol, atol=0)


def test_coag_tables_known_answers(port_oracle):
    """Fortran spot values of bm0ij / bm3i (mam4_coagulation_unit_tests.cpp:22-59)."""
    c = _golden("coag_tables.json")
    for cs in c["cases"]:
        f = port_oracle.bm0ij if cs["table"] == "bm0ij" else port_oracle.bm3i
        assert abs(f(cs["n1"], cs["n2a"], cs["n2n"]) - cs["value"]) < c["abs_tol"]


def test_coag_tables_match_reference(port_oracle, ref_oracle):
    for n1 in range(10):
        for a in range(10):
            for n in range(10):
                assert port_oracle.bm0ij(n1, a, n) == ref_oracle.bm0ij(n1, a, n)
                assert port_oracle.bm3i(n1, a, n) == ref_oracle.bm3i(n1, a, n)


@pytest.mark.parametrize("which", ["port", "ref"])
def test_aging_known_answers(which, request):
    """src/tests/mam4_aging_unit_tests.cpp:120-180: all-zero input stays zero."""
    orc = request.getfixturevalue("port_oracle" if which == "port" else "ref_oracle")
    z4, z74, z71 = np.zeros(4), np.zeros((7, 4)), np.zeros((7, 1))
    outs = orc.aging(8, z4, z4, z4, z4, z74, z74, z74, z71)
    for o in outs:
        assert not np.any(o)


def test_aging_transfer_conservation(port_oracle, ref_oracle):
    """Aging moves primary carbon to the accumulation mode; per species the
    sum over modes of the mass and of its cond+coag increments is conserved
    (the invariant of mam4_aging_unit_tests.cpp:45-115)."""
    rng = np.random.default_rng(7)
    for _ in range(20):
        dgn = rng.uniform(1e-8, 1e-7, 4)
        args = [dgn, rng.uniform(1e6, 1e9, 4), rng.uniform(0, 1e5, 4), rng.uniform(0, 1e5, 4),
                rng.uniform(1e-12, 1e-9, (7, 4)), rng.uniform(0, 1e-12, (7, 4)),
                rng.uniform(0, 1e-12, (7, 4)), rng.uniform(0, 1e-12, (7, 1))]
        po = port_oracle.aging(8, *args)
        ro = ref_oracle.aging(8, *args)
        for a, b in zip(po, ro):
            np.testing.assert_array_equal(a, b)
        qnum, dnc, dng, qaer, dac, dag, _ = po
        np.testing.assert_allclose(qnum.sum(), args[1].sum(), rtol=1e-14)
        np.testing.assert_allclose(qaer.sum(axis=1), args[4].sum(axis=1), rtol=1e-14)
        np.testing.assert_allclose((dac + dag).sum(axis=1), (args[5] + args[6]).sum(axis=1),
                                   rtol=1e-12, atol=1e-30)


@pytest.mark.parametrize("name,ncol", [("c1", None), ("c2", 48), ("c3", 48), ("c4", 48), ("c5", 24)])
def test_port_bitwise_equals_reference(port_oracle, ref_oracle, name, ncol):
    """The plain-C restatement reproduces the reference headers bit for bit,
    for all 68 outputs and the 155 per-process diagnostics."""
    w = make_workload(name, ncol=ncol)
    pb = pblh_per_cell(w)
    po, pd = port_oracle.step(w["in_slab"], pb, w["dt"], diag=True)
    ro, rd = ref_oracle.step(w["in_slab"], pb, w["dt"], diag=True)
    np.testing.assert_array_equal(po, ro)
    np.testing.assert_array_equal(pd, rd)


@pytest.mark.parametrize("cfg", [
    dict(do_cond=0), dict(do_rename=0), dict(do_newnuc=0), dict(do_coag=0),
    dict(gaexch_h2so4_uptake_optaa=1), dict(n_so4_monolayers_pcage=3),
    dict(do_cond=0, do_newnuc=0)])
def test_port_equals_reference_process_switches(port_oracle, ref_oracle, cfg):
    from oracle.pyoracle import default_config
    w = make_workload("c2", ncol=16)
    pb = pblh_per_cell(w)
    c = default_config(**cfg)
    po, pd = port_oracle.step(w["in_slab"], pb, w["dt"], cfg=c, diag=True)
    ro, rd = ref_oracle.step(w["in_slab"], pb, w["dt"], cfg=c, diag=True)
    np.testing.assert_array_equal(po, ro)
    np.testing.assert_array_equal(pd, rd)


def test_stages_equal_reference(port_oracle, ref_oracle):
    """calcsize, water uptake and amicphys separately, on the same cells."""
    w = make_workload("c2", ncol=8)
    x = w["in_slab"]
    n = x.shape[1]
    sq = np.zeros((n, 40))
    cw = np.zeros((n, 40))
    sq[:, 0] = x[3]
    sq[:, 11] = x[5]
    sq[:, 14] = x[6]
    sq[:, 15:40] = x[7:32].T
    cw[:, 15:40] = x[32:57].T
    a = port_oracle.calcsize(sq, cw, w["dt"])
    b = ref_oracle.calcsize(sq, cw, w["dt"])
    for u, v in zip(a, b):
        np.testing.assert_array_equal(u, v)
    wu_a = port_oracle.water_uptake(sq, x[0], x[1], x[4], a[0])
    wu_b = ref_oracle.water_uptake(sq, x[0], x[1], x[4], a[0])
    for u, v in zip(wu_a, wu_b):
        np.testing.assert_array_equal(u, v)
    qq = np.abs(np.random.default_rng(1).standard_normal((n, 31))) * 1e-10
    qqcw = qq * 0.5
    pb = pblh_per_cell(w)
    am_a = port_oracle.amicphys(w["dt"], x[0], x[1], x[2], pb, x[3], x[4], qq, qqcw,
                                a[0], wu_a[0], wu_a[2], diag=True)
    am_b = ref_oracle.amicphys(w["dt"], x[0], x[1], x[2], pb, x[3], x[4], qq, qqcw,
                               a[0], wu_a[0], wu_a[2], diag=True)
    for u, v in zip(am_a, am_b):
        np.testing.assert_array_equal(u, v)


def test_oracle_conservation_internal_units(port_oracle):
    """Per-species mass is conserved through the step in amicphys internal
    units (SOA family weighted by 0.08 for particles and 12.011/150 for the
    gas); nucleation adds SO4 from H2SO4. Checked on clear-sky cells."""
    w = make_workload("c1")
    x = w["in_slab"]
    out = port_oracle.step(x, pblh_per_cell(w), w["dt"])
    after = x[5:57] + out[:52] * w["dt"]
    from mam4xx_b200.workloads import ADV_MASS, MW_DRY_AIR, POPULATIONS
    def fam(v, spec):
        tot = np.zeros(v.shape[1])
        for slot, (m, s) in enumerate(POPULATIONS):
            if s == spec:
                i31 = 6 + slot
                vmr = v[2 + slot] * MW_DRY_AIR / ADV_MASS[i31]
                tot += vmr * (0.08 if spec in ("SOA", "POM") else 1.0)
        return tot
    for spec in ("POM", "BC", "DST", "NaCl", "MOM"):
        np.testing.assert_allclose(fam(after, spec), fam(x[5:57], spec), rtol=1e-13)
    so4_before = fam(x[5:57], "SO4") + x[5] * MW_DRY_AIR / ADV_MASS[2]
    so4_after = fam(after, "SO4") + after[0] * MW_DRY_AIR / ADV_MASS[2]
    np.testing.assert_allclose(so4_after, so4_before, rtol=1e-12)
    soa_before = fam(x[5:57], "SOA") + x[6] * MW_DRY_AIR / ADV_MASS[5] * (12.011 / 150)
    soa_after = fam(after, "SOA") + after[1] * MW_DRY_AIR / ADV_MASS[5] * (12.011 / 150)
    np.testing.assert_allclose(soa_after, soa_before, rtol=1e-12)


def test_counting_build_matches_and_counts():
    """The operation-counting build computes the plain build's outputs bit
    for bit, and the committed flop counts are those of the restatement
    (a fresh count on a smaller sample lands within the sampling spread)."""
    import json
    import os
    from oracle.pyoracle import CountOracle, PortOracle
    w = make_workload("c4", ncol=8, seed=17)
    pb = pblh_per_cell(w)
    out, t = CountOracle().step(w["in_slab"], pb, w["dt"])
    np.testing.assert_array_equal(out, PortOracle().step(w["in_slab"], pb, w["dt"]))
    n = w["in_slab"].shape[1]
    assert t["div"] > 0 and t["special"] > 100 * n
    path = os.path.join(os.path.dirname(os.path.dirname(__file__)), "baseline",
                        "flops_per_cell.json")
    committed = json.load(open(path))["configs"]
    from oracle.count_flops import count
    fresh = count(cells=2304)
    for name, v in fresh.items():
        assert abs(v["flops_per_cell"] / committed[name]["flops_per_cell"] - 1) < 0.15, name


def test_reference_device_build_host_path_equals_reference_build(ref_oracle):
    """oracle/_ref/libmam4ref_gpu.so compiles the reference headers with nvcc
    against the shim's device mode; its composition run on the host (glibc
    libm) must equal the g++ build of the same headers bit for bit, which
    checks the shim's device mode and the device driver's composition
    without a GPU."""
    import ctypes
    from oracle import pyoracle
    if not pyoracle.reference_gpu_available():
        pytest.skip("reference headers not compiled for the GPU")
    lib = ctypes.CDLL(pyoracle.REF_GPU_SO)
    f = lib.mam4refgpu_step_on_host
    P = ctypes.c_void_p
    f.argtypes = [ctypes.c_int, P, ctypes.c_size_t, P, P, ctypes.c_size_t, ctypes.c_double,
                  ctypes.POINTER(pyoracle.Config)]
    for name, ncol, cfg in (("c1", None, {}), ("c2", 24, {}), ("c4", 24, {}),
                            ("c2", 8, {"do_cond": 0}), ("c2", 8, {"gaexch_h2so4_uptake_optaa": 1})):
        w = make_workload(name, ncol=ncol)
        x = np.ascontiguousarray(w["in_slab"])
        pb = pblh_per_cell(w)
        n = x.shape[1]
        out = np.zeros((68, n))
        c = pyoracle.default_config(**cfg)
        f(n, x.ctypes.data, n, pb.ctypes.data, out.ctypes.data, n, w["dt"], ctypes.byref(c))
        ref = ref_oracle.step(x, pb, w["dt"], cfg=c)
        np.testing.assert_array_equal(out, ref)
