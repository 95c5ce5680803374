"""Per-process entries on the CPU side: the reference's own CalcSize and
Coagulation process classes (compiled unchanged into oracle/_ref) behave as
the reference documents, and the C ABI rejects bad arguments before any
CUDA call."""

import ctypes
import os

import numpy as np
import pytest

from mam4xx_b200 import native
from mam4xx_b200.workloads import AERO_IDS, make_process_inputs, prog_slab, make_workload


def test_prog_slab_layouts():
    w = make_workload("c2", ncol=2, seed=4)
    p = prog_slab(w["in_slab"])
    q = prog_slab(w["in_slab"], by_aero_id=True)
    # numbers are the same; accumulation SO4 is species 0 of the mode, AeroId 1
    np.testing.assert_array_equal(p[:8], q[:8])
    np.testing.assert_array_equal(p[8 + 0], q[8 + AERO_IDS.index("SO4")])
    # primary carbon has POM, BC, MOM only
    assert (q[8 + 21 + AERO_IDS.index("SO4")] == 0).all()
    assert (p[8 + 21 + 3:8 + 28] == 0).all()


def test_reference_calcsize_process_touches_what_it_documents(ref_oracle):
    d = make_process_inputs("c2", ncol=16, seed=11)
    tend, dgn = ref_oracle.calcsize_process(d["ncol"], d["nlev"], d["prog"], d["tend0"], d["dt"])
    assert np.isfinite(tend).all() and (dgn > 0).all()
    changed = set(np.nonzero(np.abs(tend - d["tend0"]).max(axis=1))[0])
    # numbers of all modes (adjusted or exchanged), and the species the
    # aitken and accumulation modes share, both phases
    common = {8 + s for s in (0, 2, 5, 6)} | {15 + s for s in range(4)}
    common |= {c + 28 for c in common}
    assert changed <= set(range(8)) | common
    # without adjustment the exchange conserves aitken + accumulation number
    t2, _ = ref_oracle.calcsize_process(d["ncol"], d["nlev"], d["prog"], d["tend0"], d["dt"],
                                        do_adjust=False)
    ch = t2 - d["tend0"]
    assert np.abs(ch[0] + ch[1]).max() <= 1e-12 * np.abs(ch[0]).max()
    # no exchange and no adjustment: nothing changes, diameters still written
    t3, dg3 = ref_oracle.calcsize_process(d["ncol"], d["nlev"], d["prog"], d["tend0"], d["dt"],
                                          do_aitacc_transfer=False, do_adjust=False)
    np.testing.assert_array_equal(t3, d["tend0"])
    assert (dg3 > 0).all()


def test_reference_coag_process_conserves_species_mass(ref_oracle):
    d = make_process_inputs("c2", ncol=16, seed=12)
    prog, tend = ref_oracle.coag_process(d["ncol"], d["nlev"], d["temp"], d["pmid"], d["wet"],
                                         d["prog_aero"], d["tend0"], d["dt"])
    for a in range(7):
        before = sum(d["prog_aero"][8 + 7 * m + a] for m in range(4))
        after = sum(prog[8 + 7 * m + a] for m in range(4))
        assert np.abs(after - before).max() <= 1e-14 * np.abs(before).max() + 1e-300
    assert (prog[:4] <= d["prog_aero"][:4] * (1 + 1e-15)).all()  # coagulation removes number
    np.testing.assert_allclose((tend - d["tend0"])[:36] * d["dt"], (prog - d["prog_aero"])[:36],
                               rtol=1e-9, atol=1e-12 * np.abs(d["prog_aero"]).max())


def test_process_entries_reject_bad_arguments_without_a_device():
    L = native.lib()
    pf = native.ProgFields()
    four = (ctypes.c_void_p * 4)()
    assert L.mam4b_calcsize_process(None, None, ctypes.byref(pf), ctypes.byref(pf),
                                    ctypes.byref(four), ctypes.byref(four), 1, 1, 1.0, None) == 1
    assert L.mam4b_coagulation_process(None, None, None, ctypes.byref(four), ctypes.byref(four),
                                       ctypes.byref(pf), ctypes.byref(pf), 1, 1, 1.0,
                                       None) == 1


def test_reference_setsox_conserves_sulfur(ref_oracle):
    """Aqueous chemistry moves sulfur from SO2 and H2SO4 gas into
    cloud-borne SO4 without creating or losing any (to rounding)."""
    from mam4xx_b200.workloads import make_setsox_inputs
    d = make_setsox_inputs("c2", ncol=32, seed=7)
    qi, qc, d1, d2 = ref_oracle.setsox(d["dt"], d["press"], d["temp"], d["lwc"], d["cldfrc"],
                                       d["cldnum"], d["xhnm"], d["qin"], d["qcw"])
    s0 = d["qin"][2] + d["qin"][3] + d["qcw"][6] + d["qcw"][14] + d["qcw"][21]
    s1 = qi[2] + qi[3] + qc[6] + qc[14] + qc[21]
    assert (np.abs(s1 - s0) <= 1e-14 * s0).all()
    active = d["lwc"] * 0 + (np.abs(qc[6] - d["qcw"][6]) > 0)
    assert 0.2 < active.mean() < 0.9  # a mix of cells with and without cloud water
    assert set(np.nonzero(np.abs(d1).max(axis=1))[0]) <= {6, 14, 21}


def test_reference_maxsat_known_answers(ref_oracle):
    """The maximum-supersaturation values of the reference's own unit test
    (src/tests/mam4_ndrop_unit_tests.cpp:210-257)."""
    assert ref_oracle.maxsat(0.0, [0.0] * 4, [1.0] * 4) == pytest.approx(1e-20, rel=1e-15)
    assert ref_oracle.maxsat(0.0, [0.0] * 4, [0.0] * 4) == pytest.approx(1e-10, rel=1e-15)
    assert ref_oracle.maxsat(0.0, [1.0] * 4, [1.0] * 4) == pytest.approx(0.4698982924029698,
                                                                         rel=1e-14)


def test_reference_activation_fractions(ref_oracle):
    from mam4xx_b200.workloads import make_activation_inputs
    d = make_activation_inputs("c2", ncol=16, seed=3)
    out = ref_oracle.activate(d["in_slab"], d["rho"], d["w"])
    fn, fm = out[0:4], out[4:8]
    assert ((fn >= 0) & (fn <= 1) & (fm >= 0) & (fm <= 1)).all()
    assert (fm >= fn - 1e-12).all()  # larger particles activate first
    no_up = d["w"] <= 0
    assert no_up.any() and (out[:, no_up] == 0).all()
    np.testing.assert_array_equal(out[16, ~no_up], d["w"][~no_up])


def test_reference_optics_lw_scales_with_layer_mass(ref_oracle):
    """Longwave absorption optical depth: finite, non-negative, and
    proportional to the layer's dry mass (pdeldry / g)."""
    from mam4xx_b200.workloads import make_optics_lw_tables
    w = make_workload("c2", ncol=8, seed=6)
    tb = make_optics_lw_tables()
    n = w["in_slab"].shape[1]
    pdel = np.full(n, 1000.0)
    t1 = ref_oracle.optics_lw(w["in_slab"], pdel, w["dt"], tb)
    t2 = ref_oracle.optics_lw(w["in_slab"], 2 * pdel, w["dt"], tb)
    assert np.isfinite(t1).all() and (t1 >= 0).all() and (t1 > 0).mean() > 0.9
    np.testing.assert_allclose(t2, 2 * t1, rtol=1e-14)


def test_reference_gas_chemistry_known_answers(ref_oracle):
    """gas_phase_chemistry's implicit Euler step on the reference: a tracer
    with neither forcing nor coupling (tracers 7-12: aerosol species) and
    removal rate h ends at q / (1 + h dt) when the step converges at once;
    one with no removal stays bit for bit; cells given a slightly negative
    tracer end finite and non-negative after the step-cutting path."""
    from mam4xx_b200.workloads import make_gas_chemistry_inputs
    d = make_gas_chemistry_inputs("c2", ncol=16, seed=11, negative_frac=0.1)
    q = ref_oracle.gas_chemistry(d["dt"], d["temp"], d["photo"], d["extfrc"], d["inv"], d["het"],
                                 d["qq"])
    assert np.isfinite(q).all() and (q[1:] >= 0).all()
    np.testing.assert_array_equal(q[0], d["qq"][0])
    clean = (d["qq"] >= 0).all(axis=0)
    assert 0.5 < clean.mean() < 1.0
    for t in range(7, 13):
        h, q0 = d["het"][t][clean], d["qq"][t][clean]
        expect = q0 / (1.0 + h * d["dt"])
        np.testing.assert_allclose(q[t][clean], expect, rtol=1e-13)
        still = h == 0
        np.testing.assert_array_equal(q[t][clean][still], q0[still])


def test_gas_chemistry_rejects_bad_arguments_without_a_device():
    L = native.lib()
    assert L.mam4b_gas_chemistry(None, None, None, None, None, None, None, 1, 1, 1, 1.0,
                                 None) == 1


_GASCHEM_HOST = r'''
#include "mam4b_gaschem.cuh"
extern "C" void run(int n, double dt, const double *temp, const double *photo, const double *ext,
                    const double *inv, const double *het, double *qq) {
  for (int c = 0; c < n; ++c) {
    double e[9], iv[8], q[31];
    for (int k = 0; k < 9; ++k) e[k] = ext[k * n + c];
    for (int k = 0; k < 8; ++k) iv[k] = inv[k * n + c];
    for (int k = 0; k < 31; ++k) q[k] = qq[k * n + c];
    auto h = [&](int t) { return het[t * n + c]; };
    mam4b::gch::gas_chemistry_cell(temp[c], dt, photo[c], e, iv, h, q);
    for (int k = 0; k < 31; ++k) qq[k * n + c] = q[k];
  }
}
'''


def test_gas_chemistry_restatement_bitwise_on_host(ref_oracle, tmp_path):
    """The kernel's gas-chemistry header compiled for the host (no FMA
    contraction, glibc) equals the reference's gas_phase_chemistry bit for
    bit, the step-cutting path of negative tracers included."""
    import shutil
    import subprocess
    from mam4xx_b200.workloads import make_gas_chemistry_inputs
    nvcc = shutil.which("nvcc")
    if not nvcc:
        pytest.skip("nvcc not found")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "gaschem_host.cu"
    src.write_text(_GASCHEM_HOST)
    so = tmp_path / "gaschem_host.so"
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-I",
                    os.path.join(root, "mam4xx_b200", "csrc"), "-Xcompiler",
                    "-fPIC,-ffp-contract=off", "-shared", str(src), "-o", str(so)], check=True)
    L = ctypes.CDLL(str(so))
    for neg in (0.0, 0.05):
        d = make_gas_chemistry_inputs("c4", ncol=32, seed=3, negative_frac=neg)
        r = ref_oracle.gas_chemistry(d["dt"], d["temp"], d["photo"], d["extfrc"], d["inv"],
                                     d["het"], d["qq"])
        q = np.array(d["qq"], order="C")
        args = [np.ascontiguousarray(d[k]) for k in ("temp", "photo", "extfrc", "inv", "het")]
        L.run(ctypes.c_int(q.shape[1]), ctypes.c_double(d["dt"]),
              *[ctypes.c_void_p(a.ctypes.data) for a in args], ctypes.c_void_p(q.ctypes.data))
        np.testing.assert_array_equal(q, r)


_TROP_HOST = r'''
#include "mam4b_optics.cuh"
extern "C" void run(int ncol, int nlev, const double *temp, const double *pmid,
                    const double *pint, int *out) {
  for (int c = 0; c < ncol; ++c) {
    auto T = [&](int k) { return temp[(size_t)c * nlev + k]; };
    auto P = [&](int k) { return pmid[(size_t)c * nlev + k]; };
    auto PI = [&](int k) { return pint[(size_t)c * (nlev + 1) + k]; };
    out[c] = mam4b::rad::tropopause_level(T, P, PI, nlev);
  }
}
'''


def test_tropopause_restatement_equals_reference_on_host(ref_oracle, tmp_path):
    """The kernel's WMO tropopause search compiled for the host finds the
    reference's level (tropopause_twmo) on every column, including the
    columns without a tropopause (level 0)."""
    import shutil
    import subprocess
    from mam4xx_b200.workloads import make_rad_props_inputs
    nvcc = shutil.which("nvcc")
    if not nvcc:
        pytest.skip("nvcc not found")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "trop_host.cu"
    src.write_text(_TROP_HOST)
    so = tmp_path / "trop_host.so"
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-I",
                    os.path.join(root, "mam4xx_b200", "csrc"), "-Xcompiler",
                    "-fPIC,-ffp-contract=off", "-shared", str(src), "-o", str(so)], check=True)
    L = ctypes.CDLL(str(so))
    w = make_rad_props_inputs("c2", ncol=200, seed=5, no_tropopause_frac=0.2)
    nc, nl = w["ncol"], w["nlev"]
    x = w["in_slab"]
    _, rt = ref_oracle.rad_props_volcanic(False, nc, nl, x, w["pint"], w["zi"], w["ext_lw"],
                                          None, None, np.zeros((16, nc * nl)))
    t, p, pi = (np.ascontiguousarray(a) for a in (x[0], x[1], w["pint"]))
    got = np.zeros(nc, dtype=np.int32)
    L.run(nc, nl, *[ctypes.c_void_p(a.ctypes.data) for a in (t, p, pi, got)])
    np.testing.assert_array_equal(got, rt)
    assert (rt == 0).sum() >= 10 and (rt > 20).sum() >= 100


def test_reference_dropmixnuc_properties(ref_oracle):
    """The reference's dropmixnuc on the seeded column inputs: finite,
    non-negative droplet number and cloud-borne aerosol, and above top_lev
    the droplet number passed through and the cloud-borne aerosol removed."""
    from mam4xx_b200.workloads import make_dropmix_inputs
    w = make_dropmix_inputs("c2", ncol=8, seed=2)
    out = ref_oracle.dropmixnuc(w["ncol"], w["nlev"], 6, True, w["dt"], w["in_slab"], w["mix"],
                                w["pint"], w["kvh"])
    assert np.isfinite(out).all()
    assert (out[0] >= 0).all() and (out[41:66] >= 0).all()
    above = np.arange(out.shape[1]) % w["nlev"] < 6
    np.testing.assert_array_equal(out[0, above], w["mix"][2, above])
    assert (out[41:66, above] == 0).all()


def test_dropmixnuc_rejects_bad_arguments_without_a_device():
    L = native.lib()
    assert L.mam4b_dropmixnuc(None, None, 0, None, None, None, None, 1, 72, 6, 1, 1.0,
                              None) == 1


def test_reference_chem_step_reduces_to_the_plain_step(ref_oracle):
    """With every chemistry rate, forcing and the cloud water zero, the
    reference composition of the step with chemistry (gas chemistry,
    setsox, amicphys with the three states) equals the plain step bit for
    bit; with active chemistry the H2SO4 tendency differs."""
    from mam4xx_b200.workloads import make_chem_step_inputs, pblh_per_cell
    for inert in (True, False):
        w = make_chem_step_inputs("c2", ncol=16, inert=inert)
        out, cout = ref_oracle.step_chem(w["in_slab"], pblh_per_cell(w), w["chem_in"], w["dt"])
        plain = ref_oracle.step(w["in_slab"], pblh_per_cell(w), w["dt"])
        assert np.isfinite(out).all() and np.isfinite(cout).all()
        if inert:
            np.testing.assert_array_equal(out, plain)
            # the chemistry gases only pass through the mmr -> vmr -> mmr round trip
            assert (np.abs(cout) <= 1e-12 * np.abs(w["chem_in"][:4]) / w["dt"]).all()
        else:
            assert (np.abs(out[0] - plain[0]) > 1e-6 * np.abs(plain[0])).mean() > 0.1
