"""ctypes bindings of the two CPU oracles (test infrastructure only).

  ReferenceOracle  oracle/_ref/libmam4ref.so -- mam4xx's own headers compiled
                   unchanged against the host shim (exists only where the
                   reference tree was available at build time).
  PortOracle       oracle/libmam4oracle.so -- the plain-C restatement.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module; the product package never imports it.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libmam4ref.so")
REF_TUNED_SO = os.path.join(HERE, "_ref", "libmam4ref_tuned.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libmam4ref_gpu.so")
# compiler flags of the two reference builds (oracle/build_oracle.py)
REF_FLAGS = "g++ -O3 -ffp-contract=off -fopenmp (parity build)"
REF_TUNED_FLAGS = "g++ -O3 -march=x86-64-v3 -ffp-contract=fast -fopenmp (tuned build)"
PORT_SO = os.path.join(HERE, "libmam4oracle.so")
ULP_SO = os.path.join(HERE, "libmam4oracle_ulp.so")
GPU_SO = os.path.join(HERE, "libmam4oracle_gpu.so")
COUNT_SO = os.path.join(HERE, "libmam4oracle_count.so")

NIN, NOUT, NDIAG = 57, 68, 155
CHEM_NIN, CHEM_NOUT = 55, 4  # step-with-chemistry extra inputs and outputs


class Config(ctypes.Structure):
    _fields_ = [("do_cond", ctypes.c_int), ("do_rename", ctypes.c_int),
                ("do_newnuc", ctypes.c_int), ("do_coag", ctypes.c_int),
                ("gaexch_h2so4_uptake_optaa", ctypes.c_int),
                ("newnuc_h2so4_conc_optaa", ctypes.c_int),
                ("n_so4_monolayers_pcage", ctypes.c_uint)]


def default_config(**kw):
    c = dict(do_cond=1, do_rename=1, do_newnuc=1, do_coag=1,
             gaexch_h2so4_uptake_optaa=2, newnuc_h2so4_conc_optaa=2,
             n_so4_monolayers_pcage=8)
    c.update(kw)
    return Config(**c)


_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_S = ctypes.c_size_t


def _ptr(a):
    return None if a is None else a.ctypes.data


class _Oracle:
    prefix = None
    path = None

    def __init__(self):
        if not os.path.exists(self.path):
            raise FileNotFoundError(self.path)
        self.lib = ctypes.CDLL(self.path)
        p = self.prefix
        f = getattr(self.lib, p + "_step")
        f.argtypes = [_I, _P, _S, _P, _P, _S, _P, _S, _D, ctypes.POINTER(Config), _I]
        f.restype = _I
        getattr(self.lib, p + "_calcsize").argtypes = [_I, _P, _P, _D, _P, _P, _P, _P]
        getattr(self.lib, p + "_water_uptake").argtypes = [_I, _P, _P, _P, _P, _P, _P, _P, _P]
        getattr(self.lib, p + "_amicphys").argtypes = [
            _I, ctypes.POINTER(Config), _D, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        getattr(self.lib, p + "_h2so4_update").argtypes = [_D, _D, _P, _P, _P, _P]
        for t in ("_bm0ij", "_bm3i"):
            g = getattr(self.lib, p + t)
            g.argtypes = [_I, _I, _I]
            g.restype = _D
        getattr(self.lib, p + "_aging").argtypes = [ctypes.c_uint] + [_P] * 8

    def step(self, in_slab, pblh_cell, dt, cfg=None, diag=False, nthreads=0):
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        n = x.shape[1]
        pb = np.ascontiguousarray(pblh_cell, dtype=np.float64)
        out = np.zeros((NOUT, n))
        dg = np.zeros((NDIAG, n)) if diag else None
        cfg = cfg or default_config()
        rc = getattr(self.lib, self.prefix + "_step")(
            n, _ptr(x), n, _ptr(pb), _ptr(out), n, _ptr(dg), n, dt, ctypes.byref(cfg), nthreads)
        if rc != 0:
            raise RuntimeError("oracle step failed: %d" % rc)
        return (out, dg) if diag else out

    def calcsize(self, state_q, qqcw, dt):
        sq = np.ascontiguousarray(state_q, dtype=np.float64)
        cw = np.ascontiguousarray(qqcw, dtype=np.float64)
        n = sq.shape[0]
        a, c = np.zeros((n, 4)), np.zeros((n, 4))
        pt, dq = np.zeros((n, 40)), np.zeros((n, 40))
        getattr(self.lib, self.prefix + "_calcsize")(n, _ptr(sq), _ptr(cw), dt, _ptr(a), _ptr(c),
                                                     _ptr(pt), _ptr(dq))
        return a, c, pt, dq

    def water_uptake(self, state_q, temp, pmid, cld, dgncur_a):
        arrs = [np.ascontiguousarray(v, dtype=np.float64) for v in (state_q, temp, pmid, cld, dgncur_a)]
        n = arrs[0].shape[0]
        w, q, d = np.zeros((n, 4)), np.zeros((n, 4)), np.zeros((n, 4))
        getattr(self.lib, self.prefix + "_water_uptake")(n, *[_ptr(a) for a in arrs], _ptr(w), _ptr(q), _ptr(d))
        return w, q, d

    def amicphys(self, dt, temp, pmid, zm, pblh, qv, cld, qq, qqcw, dgncur_a, dgncur_awet,
                 wetdens, cfg=None, diag=False):
        ins = [np.ascontiguousarray(v, dtype=np.float64) for v in (temp, pmid, zm, pblh, qv, cld)]
        q = np.array(qq, dtype=np.float64, order="C", copy=True)
        cw = np.array(qqcw, dtype=np.float64, order="C", copy=True)
        mo = [np.ascontiguousarray(v, dtype=np.float64) for v in (dgncur_a, dgncur_awet, wetdens)]
        n = q.shape[0]
        dg = np.zeros((n, 5, 31)) if diag else None
        cfg = cfg or default_config()
        getattr(self.lib, self.prefix + "_amicphys")(n, ctypes.byref(cfg), dt, *[_ptr(a) for a in ins],
                                                     _ptr(q), _ptr(cw), *[_ptr(a) for a in mo], _ptr(dg))
        return (q, cw, dg) if diag else (q, cw)

    def h2so4_update(self, dt, netprod, uptkaer, qgas_cur, qaer_cur):
        up = np.ascontiguousarray(uptkaer, dtype=np.float64)
        qg = np.array([qgas_cur], dtype=np.float64)
        av = np.zeros(1)
        qa = np.array(qaer_cur, dtype=np.float64)
        getattr(self.lib, self.prefix + "_h2so4_update")(dt, netprod, _ptr(up), _ptr(qg), _ptr(av), _ptr(qa))
        return qg[0], av[0], qa

    def bm0ij(self, n1, n2a, n2n):
        return getattr(self.lib, self.prefix + "_bm0ij")(n1, n2a, n2n)

    def bm3i(self, n1, n2a, n2n):
        return getattr(self.lib, self.prefix + "_bm3i")(n1, n2a, n2n)

    def aging(self, n_mono, dgn_a, qnum_cur, qnum_del_cond, qnum_del_coag, qaer_cur,
              qaer_del_cond, qaer_del_coag, qaer_del_coag_in):
        a = [np.array(v, dtype=np.float64, copy=True) for v in
             (dgn_a, qnum_cur, qnum_del_cond, qnum_del_coag, qaer_cur, qaer_del_cond,
              qaer_del_coag, qaer_del_coag_in)]
        getattr(self.lib, self.prefix + "_aging")(n_mono, *[_ptr(v) for v in a])
        return a[1:]


class ReferenceOracle(_Oracle):
    prefix = "mam4ref"
    path = REF_SO

    def calcsize_process(self, ncol, nlev, prog, tend, dt, do_aitacc_transfer=True,
                         do_adjust=True):
        """mam4::CalcSize::compute_tendencies column by column. prog, tend:
        (64, ncell) field-major (n_mode_i[4], n_mode_c[4], q_aero_i[4][7],
        q_aero_c[4][7]); returns (tend after, dgn (8, ncell): interstitial
        then cloud-borne dry diameters)."""
        prog = np.array(prog, dtype=np.float64, order="C")
        tend = np.array(tend, dtype=np.float64, order="C")
        dgn = np.zeros((8, prog.shape[1]))
        f = self.lib.mam4ref_calcsize_process
        f.argtypes = [_I, _I, _I, _I, _D, _P, _P, _P]
        f.restype = None
        f(ncol, nlev, int(do_aitacc_transfer), int(do_adjust), dt, prog.ctypes.data,
          tend.ctypes.data, dgn.ctypes.data)
        return tend, dgn

    def optics_lw(self, in_slab, pdeldry, dt, tables):
        """modal_aero_opt::modal_aero_lw_k per cell; returns tau (16, ncell)."""
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        n = x.shape[1]
        tau = np.zeros((16, n))
        pd = np.ascontiguousarray(pdeldry, dtype=np.float64)
        t = [np.ascontiguousarray(tables[k], dtype=np.float64)
             for k in ("specrefindex", "water_refindex", "refrtab", "refitab", "absp")]
        f = self.lib.mam4ref_optics_lw
        f.argtypes = [_I, _P, _P, _D] + [_P] * 6
        f.restype = None
        f(n, x.ctypes.data, pd.ctypes.data, dt, *[a.ctypes.data for a in t], tau.ctypes.data)
        return tau

    def optics_sw(self, ncol, nlev, in_slab, pdeldry, dt, tables):
        """modal_aero_sw per cell with its mode and column sums; returns
        (out (4, 14, ncell): tauxar, wa, ga, fa; aod (ncol,))."""
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        n = x.shape[1]
        out = np.zeros((4, 14, n))
        aod = np.zeros(ncol)
        pd = np.ascontiguousarray(pdeldry, dtype=np.float64)
        t = [np.ascontiguousarray(tables[k], dtype=np.float64)
             for k in ("specrefindex", "water_refindex", "refrtab", "refitab", "extp", "absp",
                       "asmp")]
        f = self.lib.mam4ref_optics_sw
        f.argtypes = [_I, _I, _P, _P, _D] + [_P] * 9
        f.restype = None
        f(ncol, nlev, x.ctypes.data, pd.ctypes.data, dt, *[a.ctypes.data for a in t],
          out.ctypes.data, aod.ctypes.data)
        return out, aod

    def rad_props_volcanic(self, sw, ncol, nlev, in_slab, pint, zi, ext, ssa, af, modal):
        """The reference's tropopause_or_quit and volcanic updates of
        aero_rad_props_sw (sw=True) / aero_rad_props_lw on modal optics
        results; returns (updated copy, tropopause level per column)."""
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        out = np.array(modal, dtype=np.float64, order="C")
        trop = np.zeros(ncol, dtype=np.int32)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (pint, zi, ext)]
        if sw:
            arrs += [np.ascontiguousarray(a, dtype=np.float64) for a in (ssa, af)]
        f = self.lib.mam4ref_rad_props_volcanic
        f.argtypes = [_I, _I, _I] + [_P] * 8
        f.restype = None
        f(int(bool(sw)), ncol, nlev, x.ctypes.data, arrs[0].ctypes.data, arrs[1].ctypes.data,
          arrs[2].ctypes.data, arrs[3].ctypes.data if sw else None,
          arrs[4].ctypes.data if sw else None, out.ctypes.data, trop.ctypes.data)
        return out, trop

    def dropmixnuc(self, ncol, nlev, top_lev, vertical_mix, dt, in_slab, mix, pint, kvh):
        """ndrop::dropmixnuc column by column; returns out (66, ncell) in
        the layout of MAM4B_DROPMIX_OUT_*."""
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (mix, pint, kvh)]
        out = np.zeros((66, x.shape[1]))
        f = self.lib.mam4ref_dropmixnuc
        f.argtypes = [_I, _I, _I, _I, _D] + [_P] * 5
        f.restype = None
        f(ncol, nlev, top_lev, int(bool(vertical_mix)), dt, x.ctypes.data,
          *[a.ctypes.data for a in arrs], out.ctypes.data)
        return out

    def maxsat(self, zeta, eta, smc):
        """ndrop::maxsat for 4 modes."""
        f = self.lib.mam4ref_maxsat
        f.argtypes = [_D, _P, _P]
        f.restype = _D
        e = np.ascontiguousarray(eta, dtype=np.float64)
        s = np.ascontiguousarray(smc, dtype=np.float64)
        return f(zeta, e.ctypes.data, s.ctypes.data)

    def activate(self, in_slab, rho, w):
        """ndrop::get_activate_frac per cell; in_slab (NIN, ncell); returns
        (17, ncell): fn[4], fm[4], fluxn[4], fluxm[4], flux_fullact."""
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        n = x.shape[1]
        out = np.zeros((17, n))
        r = np.ascontiguousarray(rho, dtype=np.float64)
        ww = np.ascontiguousarray(w, dtype=np.float64)
        f = self.lib.mam4ref_activate
        f.argtypes = [_I, _P, _P, _P, _P]
        f.restype = None
        f(n, x.ctypes.data, r.ctypes.data, ww.ctypes.data, out.ctypes.data)
        return out

    def setsox(self, dt, press, temp, lwc, cldfrc, cldnum, xhnm, qin, qcw):
        """mam4::mo_setsox::setsox_single_level per cell (qin, qcw: (31,
        ncell) vmr); returns (qin, qcw, dqdt_aqso4, dqdt_aqh2so4), the last
        two (31, ncell)."""
        qin = np.array(qin, dtype=np.float64, order="C")
        qcw = np.array(qcw, dtype=np.float64, order="C")
        n = qin.shape[1]
        d1 = np.zeros((31, n))
        d2 = np.zeros((31, n))
        args = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (press, temp, lwc, cldfrc, cldnum, xhnm)]
        f = self.lib.mam4ref_setsox
        f.argtypes = [_I, _D] + [_P] * 10
        f.restype = None
        f(n, dt, *[a.ctypes.data for a in args], qin.ctypes.data, qcw.ctypes.data,
          d1.ctypes.data, d2.ctypes.data)
        return qin, qcw, d1, d2

    def step_chem(self, in_slab, pblh_cell, chem_in, dt, cfg=None, nthreads=0):
        """The step with gas-phase and aqueous chemistry ahead of amicphys
        (the reference's functions composed per cell); chem_in
        (MAM4B_CHEM_NIN, ncell). Returns (out, chem_out)."""
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        ch = np.ascontiguousarray(chem_in, dtype=np.float64)
        n = x.shape[1]
        assert ch.shape == (CHEM_NIN, n)
        pb = np.ascontiguousarray(pblh_cell, dtype=np.float64)
        out = np.zeros((NOUT, n))
        cout = np.zeros((CHEM_NOUT, n))
        cfg = cfg or default_config()
        f = self.lib.mam4ref_step_chem
        f.argtypes = [_I, _P, _P, _P, _P, _P, _D, ctypes.POINTER(Config), _I]
        f.restype = _I
        rc = f(n, _ptr(x), _ptr(pb), _ptr(ch), _ptr(out), _ptr(cout), dt, ctypes.byref(cfg),
               nthreads)
        if rc != 0:
            raise RuntimeError("reference step_chem failed: %d" % rc)
        return out, cout

    def gas_chemistry(self, dt, temp, photo, extfrc, inv, het, qq):
        """mam4::microphysics::gas_phase_chemistry per cell (extfrc (9,
        ncell), inv (8, ncell), het and qq (31, ncell)); returns qq after."""
        qq = np.array(qq, dtype=np.float64, order="C")
        n = qq.shape[1]
        args = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (temp, photo, extfrc, inv, het)]
        f = self.lib.mam4ref_gas_chemistry
        f.argtypes = [_I, _D] + [_P] * 6
        f.restype = None
        f(n, dt, *[a.ctypes.data for a in args], qq.ctypes.data)
        return qq

    def coag_process(self, ncol, nlev, temp, pmid, wet, prog, tend, dt):
        """mam4::Coagulation::compute_tendencies column by column. wet: (8,
        ncell) wet density [4] then wet diameter [4]; returns (prog after,
        tend after)."""
        prog = np.array(prog, dtype=np.float64, order="C")
        tend = np.array(tend, dtype=np.float64, order="C")
        wet = np.ascontiguousarray(wet, dtype=np.float64)
        t = np.ascontiguousarray(temp, dtype=np.float64)
        p = np.ascontiguousarray(pmid, dtype=np.float64)
        f = self.lib.mam4ref_coag_process
        f.argtypes = [_I, _I, _D, _P, _P, _P, _P, _P]
        f.restype = None
        f(ncol, nlev, dt, t.ctypes.data, p.ctypes.data, wet.ctypes.data, prog.ctypes.data,
          tend.ctypes.data)
        return prog, tend


def _host_has_avx2_fma():
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln for ln in f if ln.startswith("flags")), "").split()
    except OSError:
        return False
    return "avx2" in flags and "fma" in flags


class TunedReferenceOracle(ReferenceOracle):
    """The reference build tuned for speed (AVX2/FMA, FP contraction): the
    timed CPU baseline. Its results differ from the parity build's in the
    last bits (contracted multiply-adds); it is timed, never compared."""
    path = REF_TUNED_SO
    flags = REF_TUNED_FLAGS


ReferenceOracle.flags = REF_FLAGS


def baseline_oracle():
    """(oracle, kind, flags) of the CPU baseline: the tuned reference build
    where it exists and the host has AVX2 and FMA, else the parity build of
    the reference, else the restatement."""
    if os.path.exists(REF_TUNED_SO) and _host_has_avx2_fma():
        return TunedReferenceOracle(), "reference", REF_TUNED_FLAGS
    if reference_available():
        return ReferenceOracle(), "reference", REF_FLAGS
    return PortOracle(), "port", "gcc -O3 -ffp-contract=off -fopenmp (restatement)"


class PortOracle(_Oracle):
    prefix = "mam4orc"
    path = PORT_SO

    def __init__(self):
        super().__init__()
        self.lib.mam4orc_soa_niter.argtypes = [_I, _P, _S, _P, _D, ctypes.POINTER(Config), _P, _I]

    def soa_niter(self, in_slab, pblh_cell, dt, cfg=None, nthreads=0):
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        n = x.shape[1]
        pb = np.ascontiguousarray(pblh_cell, dtype=np.float64)
        it = np.zeros(n, dtype=np.int32)
        cfg = cfg or default_config()
        self.lib.mam4orc_soa_niter(n, _ptr(x), n, _ptr(pb), dt, ctypes.byref(cfg), _ptr(it), nthreads)
        return it


class UlpOracle(PortOracle):
    """The restatement with every libm result moved by 1..2 ulps (1..5 for
    erfc), drawn per call from a stream seeded by (seed, cell)."""
    path = ULP_SO

    def __init__(self, seed=1):
        super().__init__()
        self.lib.mam4orc_set_ulp_noise.argtypes = [ctypes.c_ulonglong]
        self.lib.mam4orc_set_ulp_noise(int(seed))

    def reseed(self, seed):
        self.lib.mam4orc_set_ulp_noise(int(seed))


class GpuOracle:
    """The restatement compiled for the GPU (CUDA libm, no FMA contraction):
    differs from the host build only through the math library."""

    def __init__(self):
        if not os.path.exists(GPU_SO):
            raise FileNotFoundError(GPU_SO)
        self.lib = ctypes.CDLL(GPU_SO)
        self.lib.mam4orcgpu_step.argtypes = [_I, _P, _S, _P, _P, _S, _P, _S, _D, ctypes.POINTER(Config)]
        self.lib.mam4orcgpu_step.restype = _I

    def step(self, in_slab, pblh_cell, dt, cfg=None, diag=False):
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        n = x.shape[1]
        pb = np.ascontiguousarray(pblh_cell, dtype=np.float64)
        out = np.zeros((NOUT, n))
        dg = np.zeros((NDIAG, n)) if diag else None
        cfg = cfg or default_config()
        rc = self.lib.mam4orcgpu_step(n, _ptr(x), n, _ptr(pb), _ptr(out), n, _ptr(dg), n, dt,
                                      ctypes.byref(cfg))
        if rc != 0:
            raise RuntimeError("GPU oracle failed: %d" % rc)
        return (out, dg) if diag else out


class RefGpuOracle:
    """The mam4xx reference headers compiled unchanged for the GPU (CUDA
    libm, no FMA contraction; oracle/ref/ref_step_gpu.cu): the reference
    itself with the product's math library. step() returns the outputs and
    checks that no reference kernel assert failed."""

    def __init__(self):
        if not os.path.exists(REF_GPU_SO):
            raise FileNotFoundError(REF_GPU_SO)
        self.lib = ctypes.CDLL(REF_GPU_SO)
        self.lib.mam4refgpu_step.argtypes = [_I, _P, _S, _P, _P, _S, _D, ctypes.POINTER(Config),
                                             ctypes.POINTER(ctypes.c_ulonglong)]
        self.lib.mam4refgpu_step.restype = _I

    def step(self, in_slab, pblh_cell, dt, cfg=None):
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        n = x.shape[1]
        pb = np.ascontiguousarray(pblh_cell, dtype=np.float64)
        out = np.zeros((NOUT, n))
        cfg = cfg or default_config()
        na = ctypes.c_ulonglong(0)
        rc = self.lib.mam4refgpu_step(n, _ptr(x), n, _ptr(pb), _ptr(out), n, dt,
                                      ctypes.byref(cfg), ctypes.byref(na))
        if rc != 0:
            raise RuntimeError("GPU reference build failed: %d" % rc)
        if na.value:
            raise RuntimeError("%d reference kernel asserts failed" % na.value)
        return out


def reference_gpu_available():
    return os.path.exists(REF_GPU_SO)


def reference_available():
    return os.path.exists(REF_SO)


# ----------------------------------------------------------------------
# Parity against the oracle
# ----------------------------------------------------------------------
TOL = 1e-12        # the FP64 parity tolerance, state-relative
QUANTILES = (0.5, 0.9, 0.99, 0.999)


def state_rel_err(tend_a, tend_b, in_slab, dt):
    """|a - b| * dt / max(|q_before|, |q_after|, 1e-30): the error of a
    tendency in units of the state it changes (shapes (52, n))."""
    q0 = np.abs(in_slab[5:57])
    q1 = np.abs(in_slab[5:57] + tend_b * dt)
    return np.abs(tend_a - tend_b) * dt / np.maximum(np.maximum(q0, q1), 1e-30)


def output_errors(out, ref, in_slab, dt):
    """(68, n) errors: tendencies state-relative, the 16 size/density/water
    outputs relative."""
    e_t = state_rel_err(out[:52], ref[:52], in_slab, dt)
    e_d = np.abs(out[52:] - ref[52:]) / np.maximum(np.abs(ref[52:]), 1e-300)
    return np.concatenate([e_t, e_d], axis=0)


def libm_spread_baseline(in_slab, pblh_cell, dt, ref_out, cfg=None, seeds=(1, 2)):
    """What the reference algorithm does to itself under a different libm:
    per-cell error statistics of the oracle whose libm results are moved by
    1..2 ulps (1..5 for erfc), against the canonical oracle."""
    u = UlpOracle(seeds[0])
    fracs, qs, maxes = [], [], []
    for sd in seeds:
        u.reseed(sd)
        ec = output_errors(u.step(in_slab, pblh_cell, dt, cfg=cfg), ref_out, in_slab, dt).max(axis=0)
        fracs.append(float((ec <= TOL).mean()))
        qs.append(np.quantile(ec, QUANTILES))
        maxes.append(float(ec.max()))
    u.reseed(0)
    return {"frac_within_tol": min(fracs), "quantiles": np.max(qs, axis=0), "max": max(maxes)}


def parity(candidate, ref_out, in_slab, pblh_cell, dt, cfg=None, tol=TOL):
    """Statistical parity of a candidate (the CUDA step) with the canonical
    oracle when the two differ only through their math libraries.

    The reference algorithm amplifies last-bit libm differences (SOA
    sub-stepping, the water-uptake quartic), so no libm-independent bound
    of 1e-12 exists on every cell. The candidate must be at least as close
    to the oracle as the oracle is to itself under 1..2-ulp libm
    perturbations: the fraction of cells whose 68 outputs are all within
    `tol` may fall short of that baseline by at most 0.02, each per-cell
    error quantile (50/90/99/99.9 %) may exceed the baseline's by at most 3x
    (and never matters below `tol`), and the largest error by at most 10x.
    Returns a summary; raises AssertionError."""
    err = output_errors(candidate, ref_out, in_slab, dt)
    ec = err.max(axis=0)
    base = libm_spread_baseline(in_slab, pblh_cell, dt, ref_out, cfg=cfg)
    cq = np.quantile(ec, QUANTILES)
    summary = {"cells": int(ec.size), "frac_within_tol": float((ec <= tol).mean()),
               "baseline_frac_within_tol": base["frac_within_tol"],
               "quantiles": [float(v) for v in cq],
               "baseline_quantiles": [float(v) for v in base["quantiles"]],
               "max_err": float(ec.max()), "baseline_max": base["max"]}
    problems = []
    if summary["frac_within_tol"] < base["frac_within_tol"] - 0.02:
        problems.append("fraction within tol")
    for q, c, b in zip(QUANTILES, cq, base["quantiles"]):
        if c > max(tol, 3.0 * b):
            problems.append("quantile %g" % q)
    if ec.max() > max(tol, 10.0 * base["max"]):
        problems.append("max")
    if problems:
        f, c = np.unravel_index(np.argmax(err), err.shape)
        raise AssertionError("parity: %s; worst output %d cell %d (%r vs %r); %s"
                             % (", ".join(problems), f, c, candidate[f, c], ref_out[f, c], summary))
    return summary


class CountOracle:
    """The restatement built with an operation-counting real type
    (oracle/opcount.cpp): same outputs as PortOracle, plus the tally of
    + - * /, libm calls, min/max and compares of the cells stepped."""

    FIELDS = ("add", "mul", "div", "special", "minmax", "cmp")

    def __init__(self):
        if not os.path.exists(COUNT_SO):
            raise FileNotFoundError(COUNT_SO)
        self.lib = ctypes.CDLL(COUNT_SO)
        self.lib.mam4orc_step.argtypes = [_I, _P, _S, _P, _P, _S, _P, _S, _D, _P, _I]
        self.lib.mam4orc_step.restype = _I
        self.lib.mam4cnt_tally.argtypes = [_P]
        self.lib.mam4cnt_tally.restype = None
        self.tally()

    def tally(self):
        t = np.zeros(6, dtype=np.uint64)
        self.lib.mam4cnt_tally(t.ctypes.data)
        return dict(zip(self.FIELDS, (int(v) for v in t)))

    def step(self, in_slab, pblh_cell, dt, cfg=None):
        """Steps the cells; returns (outputs, tally of this call)."""
        cfg = cfg or default_config()
        x = np.ascontiguousarray(in_slab, dtype=np.float64)
        pb = np.ascontiguousarray(pblh_cell, dtype=np.float64)
        n = x.shape[1]
        out = np.zeros((NOUT, n))
        self.tally()
        st = self.lib.mam4orc_step(n, x.ctypes.data, n, pb.ctypes.data, out.ctypes.data, n, None,
                                   0, dt, ctypes.byref(cfg), 1)
        if st != 0:
            raise RuntimeError("oracle step failed: %d" % st)
        return out, self.tally()
