"""ctypes binding of the C ABI in include/mam4b.h (libmam4b.so).

The library is loaded from the package directory; there is no fallback: if
the shared object is missing, or a call is made without a CUDA device, the
call raises.
"""

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmam4b.so")

NIN, NOUT, NDIAG, NPOP = 57, 68, 155, 25
CHEM_NIN, CHEM_NOUT = 55, 4  # mam4b_step_chem_slab: MAM4B_CHEM_NIN, MAM4B_CHEM_NOUT
FP64, MIXED, MIXED_FAST = 0, 1, 2
STATUS = {0: "ok", 1: "invalid argument", 2: "cuda error", 3: "not supported",
          4: "device flags", 5: "too many cells for the no-alloc scratch"}
NOALLOC_MAX_CELLS = 16384  # MAM4B_NOALLOC_MAX_CELLS
FLAG_NONFINITE_INPUT = 0x1
FLAG_SOA_NITER_LIMIT = 0x2
FLAG_NONFINITE_OUTPUT = 0x4


class Config(ctypes.Structure):
    """mam4b_config: AmicPhysConfig (src/mam4xx/mam4_amicphys.hpp:223-237)
    plus n_so4_monolayers_pcage (src/mam4xx/aging.hpp:31)."""
    _fields_ = [("do_cond", ctypes.c_int), ("do_rename", ctypes.c_int),
                ("do_newnuc", ctypes.c_int), ("do_coag", ctypes.c_int),
                ("gaexch_h2so4_uptake_optaa", ctypes.c_int),
                ("newnuc_h2so4_conc_optaa", ctypes.c_int),
                ("n_so4_monolayers_pcage", ctypes.c_uint)]


class StateView(ctypes.Structure):
    _fields_ = [("field", ctypes.c_void_p * NIN), ("pblh", ctypes.c_void_p)]


class TendView(ctypes.Structure):
    _fields_ = [("field", ctypes.c_void_p * NOUT), ("diag", ctypes.c_void_p * NDIAG)]


NUM_MODES, NUM_AERO = 4, 7
PROG_FIELDS = 64  # n_mode_i[4], n_mode_c[4], q_aero_i[4][7], q_aero_c[4][7]


class ProgFields(ctypes.Structure):
    """mam4b_prog_fields: Prognostics-style device arrays per (mode, index)."""
    _fields_ = [("n_mode_i", ctypes.c_void_p * NUM_MODES),
                ("n_mode_c", ctypes.c_void_p * NUM_MODES),
                ("q_aero_i", (ctypes.c_void_p * NUM_AERO) * NUM_MODES),
                ("q_aero_c", (ctypes.c_void_p * NUM_AERO) * NUM_MODES)]

    @classmethod
    def from_slab(cls, base, n):
        """The 64 fields of one slab of doubles, field f at base + 8 f n:
        n_mode_i[4], n_mode_c[4], q_aero_i[4][7], q_aero_c[4][7]."""
        f = cls()
        for m in range(NUM_MODES):
            f.n_mode_i[m] = base + 8 * m * n
            f.n_mode_c[m] = base + 8 * (4 + m) * n
            for a in range(NUM_AERO):
                f.q_aero_i[m][a] = base + 8 * (8 + 7 * m + a) * n
                f.q_aero_c[m][a] = base + 8 * (36 + 7 * m + a) * n
        return f


class OpticsLwTables(ctypes.Structure):
    """mam4b_optics_lw_tables (host pointers)."""
    _fields_ = [("specrefindex", ctypes.c_void_p), ("water_refindex", ctypes.c_void_p),
                ("refrtab", ctypes.c_void_p), ("refitab", ctypes.c_void_p),
                ("absp", ctypes.c_void_p)]


class OpticsSwTables(ctypes.Structure):
    """mam4b_optics_sw_tables (host pointers)."""
    _fields_ = [(k, ctypes.c_void_p) for k in ("specrefindex", "water_refindex", "refrtab",
                                               "refitab", "extp", "absp", "asmp")]


class Tuning(ctypes.Structure):
    """mam4b_tuning: launch shape of the forward step's kernels."""
    _fields_ = [(k, ctypes.c_int) for k in (
        "size_block", "size_regs", "mode_block", "pair_block", "pre_block", "pre_regs",
        "post_block", "post_regs", "soa_block", "soa_regs", "soa_blocks_per_sm",
        "cells_per_thread", "inline_scale")]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class CalcSizeConfig(ctypes.Structure):
    """mam4b_calcsize_config: CalcSize::Config (src/mam4xx/calcsize.hpp:835-842)."""
    _fields_ = [("do_aitacc_transfer", ctypes.c_int), ("do_adjust", ctypes.c_int)]


_lib = None


def lib():
    """Loads libmam4b.so once; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libmam4b.so not built: run python -m mam4xx_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        P, I, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
        L.mam4b_abi_version.restype = I
        L.mam4b_default_config.argtypes = [ctypes.POINTER(Config)]
        L.mam4b_create.argtypes = [ctypes.POINTER(P), ctypes.POINTER(Config)]
        L.mam4b_create.restype = I
        L.mam4b_destroy.argtypes = [P]
        L.mam4b_destroy.restype = I
        L.mam4b_step.argtypes = [P, ctypes.POINTER(StateView), ctypes.POINTER(TendView), I, I, D, I, P]
        L.mam4b_step.restype = I
        L.mam4b_step_slab.argtypes = [P, P, P, P, S, I, I, D, I, P]
        L.mam4b_step_slab.restype = I
        L.mam4b_step_host.argtypes = [P, P, P, P, S, I, I, D, I, P]
        L.mam4b_step_host.restype = I
        L.mam4b_last_status.argtypes = [P, ctypes.POINTER(ctypes.c_uint32)]
        L.mam4b_last_status.restype = I
        L.mam4b_last_error.argtypes = [P, ctypes.c_char_p, S]
        L.mam4b_step_slab_noalloc.argtypes = [ctypes.POINTER(Config), P, P, P, S, I, I, D, P, P]
        L.mam4b_step_slab_noalloc.restype = I
        L.mam4b_adjoint_slab.argtypes = [P, P, P, P, P, S, I, I, D, P]
        L.mam4b_adjoint_slab.restype = I
        L.mam4b_adjoint_slab_ex.argtypes = [P, P, P, P, P, S, I, I, D, I, P]
        L.mam4b_adjoint_slab_ex.restype = I
        L.mam4b_step_tracers.argtypes = [P, P, P, S, P, P, P, P, P, P, P, P, S, I, I, D, I, P]
        L.mam4b_step_tracers.restype = I
        L.mam4b_optics_lw_set_tables.argtypes = [P, ctypes.POINTER(OpticsLwTables)]
        L.mam4b_optics_lw_set_tables.restype = I
        L.mam4b_optics_lw.argtypes = [P, P, S, P, P, I, I, D, P]
        L.mam4b_optics_lw.restype = I
        L.mam4b_optics_sw_set_tables.argtypes = [P, ctypes.POINTER(OpticsSwTables)]
        L.mam4b_optics_sw_set_tables.restype = I
        L.mam4b_optics_sw.argtypes = [P, P, S, P, P, P, I, I, D, P]
        L.mam4b_optics_sw.restype = I
        L.mam4b_activate.argtypes = [P, P, S, P, P, P, I, I, P]
        L.mam4b_activate.restype = I
        L.mam4b_setsox.argtypes = [P, P, P, P, P, P, P, P, P, S, P, P, I, I, D, P]
        L.mam4b_setsox.restype = I
        L.mam4b_gas_chemistry.argtypes = [P, P, P, P, P, P, P, S, I, I, D, P]
        L.mam4b_gas_chemistry.restype = I
        L.mam4b_step_chem_slab.argtypes = [P, P, P, P, P, P, S, I, I, D, P]
        L.mam4b_step_chem_slab.restype = I
        L.mam4b_aero_rad_props_sw.argtypes = [P, P, S, P, P, P, P, P, P, P, P, P, I, I, D, P]
        L.mam4b_aero_rad_props_sw.restype = I
        L.mam4b_aero_rad_props_lw.argtypes = [P, P, S, P, P, P, P, P, P, I, I, D, P]
        L.mam4b_aero_rad_props_lw.restype = I
        L.mam4b_dropmixnuc.argtypes = [P, P, S, P, P, P, P, I, I, I, I, D, P]
        L.mam4b_dropmixnuc.restype = I
        PF = ctypes.POINTER(ProgFields)
        P4 = ctypes.c_void_p * NUM_MODES
        L.mam4b_calcsize_process.argtypes = [P, ctypes.POINTER(CalcSizeConfig), PF, PF,
                                             ctypes.POINTER(P4), ctypes.POINTER(P4), I, I, D, P]
        L.mam4b_calcsize_process.restype = I
        L.mam4b_coagulation_process.argtypes = [P, P, P, ctypes.POINTER(P4), ctypes.POINTER(P4),
                                                PF, PF, I, I, D, P]
        L.mam4b_coagulation_process.restype = I
        L.mam4b_launch_count.argtypes = [P]
        L.mam4b_launch_count.restype = ctypes.c_uint64
        TP = ctypes.POINTER(Tuning)
        L.mam4b_default_tuning.argtypes = [TP]
        L.mam4b_get_tuning.argtypes = [P, TP]
        L.mam4b_get_tuning.restype = I
        L.mam4b_set_tuning.argtypes = [P, TP]
        L.mam4b_set_tuning.restype = I
        L.mam4b_tuning_from_json.argtypes = [ctypes.c_char_p, TP, ctypes.c_char_p, S]
        L.mam4b_tuning_from_json.restype = I
        FP = ctypes.POINTER(ctypes.c_float)
        L.mam4b_autotune.argtypes = [P, P, P, P, S, I, I, D, I, I, P, TP, FP, FP]
        L.mam4b_autotune.restype = I
        L.mam4b_set_graph_mode.argtypes = [P, I]
        L.mam4b_set_graph_mode.restype = I
        L.mam4b_set_adjoint_checkpoint.argtypes = [P, I]
        L.mam4b_set_adjoint_checkpoint.restype = I
        _lib = L
    return _lib


EXPORTED = ["mam4b_abi_version", "mam4b_default_config", "mam4b_create", "mam4b_destroy",
            "mam4b_step", "mam4b_step_slab", "mam4b_step_host", "mam4b_last_status",
            "mam4b_last_error", "mam4b_launch_count", "mam4b_step_slab_noalloc",
            "mam4b_adjoint_slab", "mam4b_calcsize_process", "mam4b_coagulation_process",
            "mam4b_step_tracers", "mam4b_setsox", "mam4b_gas_chemistry", "mam4b_step_chem_slab",
            "mam4b_activate",
            "mam4b_optics_lw_set_tables", "mam4b_optics_lw", "mam4b_optics_sw_set_tables",
            "mam4b_optics_sw", "mam4b_aero_rad_props_sw", "mam4b_aero_rad_props_lw",
            "mam4b_dropmixnuc", "mam4b_default_tuning", "mam4b_get_tuning", "mam4b_set_tuning",
            "mam4b_tuning_from_json", "mam4b_autotune", "mam4b_set_graph_mode",
            "mam4b_step_columns", "mam4b_synchronize", "mam4b_set_adjoint_checkpoint",
            "mam4b_adjoint_slab_ex"]


def default_tuning():
    t = Tuning()
    lib().mam4b_default_tuning(ctypes.byref(t))
    return t


def tuning_from_json(path):
    """(Tuning, device name) of a tuning file (mam4b_tuning_from_json)."""
    t = Tuning()
    dev = ctypes.create_string_buffer(256)
    st = lib().mam4b_tuning_from_json(path.encode(), ctypes.byref(t), dev, 256)
    if st != 0:
        raise MicrophysicsError("mam4b_tuning_from_json(%s): %s" % (path, STATUS.get(st, st)))
    return t, dev.value.decode()


def default_config(**overrides):
    c = Config()
    lib().mam4b_default_config(ctypes.byref(c))
    for k, v in overrides.items():
        setattr(c, k, int(v))
    return c


class MicrophysicsError(RuntimeError):
    pass


class Context:
    """Owns one mam4b_ctx (bound to the current CUDA device)."""

    def __init__(self, config=None):
        self._lib = lib()
        self.config = config if config is not None else default_config()
        h = ctypes.c_void_p()
        st = self._lib.mam4b_create(ctypes.byref(h), ctypes.byref(self.config))
        if st != 0:
            raise MicrophysicsError("mam4b_create failed: %s" % STATUS.get(st, st))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mam4b_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != 0:
            buf = ctypes.create_string_buffer(256)
            self._lib.mam4b_last_error(self._h, buf, 256)
            raise MicrophysicsError("%s: %s (%s)" % (what, STATUS.get(st, st), buf.value.decode()))

    def step(self, in_ptrs, pblh_ptr, out_ptrs, ncol, nlev, dt, diag_ptrs=None,
             precision=FP64, stream=0):
        iv = StateView()
        for f, p in enumerate(in_ptrs):
            iv.field[f] = p
        iv.pblh = pblh_ptr
        ov = TendView()
        for f, p in enumerate(out_ptrs):
            ov.field[f] = p
        if diag_ptrs is not None:
            for f, p in enumerate(diag_ptrs):
                ov.diag[f] = p
        st = self._lib.mam4b_step(self._h, ctypes.byref(iv), ctypes.byref(ov), int(ncol),
                                  int(nlev), float(dt), int(precision), ctypes.c_void_p(stream))
        self._check(st, "mam4b_step")

    def step_slab(self, in_ptr, pblh_ptr, out_ptr, ld, ncol, nlev, dt, precision=FP64, stream=0):
        st = self._lib.mam4b_step_slab(self._h, in_ptr, pblh_ptr, out_ptr, int(ld), int(ncol),
                                       int(nlev), float(dt), int(precision),
                                       ctypes.c_void_p(stream))
        self._check(st, "mam4b_step_slab")

    def step_host(self, in_ptr, pblh_ptr, out_ptr, ld, ncol, nlev, dt, precision=FP64, stream=0):
        st = self._lib.mam4b_step_host(self._h, in_ptr, pblh_ptr, out_ptr, int(ld), int(ncol),
                                       int(nlev), float(dt), int(precision),
                                       ctypes.c_void_p(stream))
        self._check(st, "mam4b_step_host")

    def adjoint_slab(self, in_ptr, pblh_ptr, out_bar_ptr, in_bar_ptr, ld, ncol, nlev, dt,
                     stream=0, precision=FP64):
        """in_bar = (d out / d in)^T out_bar (mam4b_adjoint_slab; with
        precision=MIXED the adjoint of the mixed-precision step,
        mam4b_adjoint_slab_ex)."""
        if precision == FP64:
            st = self._lib.mam4b_adjoint_slab(self._h, in_ptr, pblh_ptr, out_bar_ptr, in_bar_ptr,
                                              int(ld), int(ncol), int(nlev), float(dt),
                                              ctypes.c_void_p(stream))
        else:
            st = self._lib.mam4b_adjoint_slab_ex(self._h, in_ptr, pblh_ptr, out_bar_ptr,
                                                 in_bar_ptr, int(ld), int(ncol), int(nlev),
                                                 float(dt), int(precision),
                                                 ctypes.c_void_p(stream))
        self._check(st, "mam4b_adjoint_slab")

    def step_tracers(self, q, qqcw, tracer_stride, temperature, pressure, height,
                     cloud_fraction, pblh, ptend_q, ptend_qqcw, mode_out, mode_stride, ncol,
                     nlev, dt, precision=FP64, stream=0):
        """The step on tracer-layout arrays (mam4b_step_tracers); device
        pointers."""
        st = self._lib.mam4b_step_tracers(self._h, q, qqcw, int(tracer_stride), temperature,
                                          pressure, height, cloud_fraction, pblh, ptend_q,
                                          ptend_qqcw, mode_out, int(mode_stride), int(ncol),
                                          int(nlev), float(dt), int(precision),
                                          ctypes.c_void_p(stream))
        self._check(st, "mam4b_step_tracers")

    def optics_lw_set_tables(self, tables):
        """Copies the longwave optics tables (dict of numpy arrays, see
        workloads.make_optics_lw_tables) into the context."""
        import numpy as np
        arrs = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in tables.items()}
        t = OpticsLwTables(*[arrs[k].ctypes.data for k in ("specrefindex", "water_refindex",
                                                           "refrtab", "refitab", "absp")])
        st = self._lib.mam4b_optics_lw_set_tables(self._h, ctypes.byref(t))
        self._check(st, "mam4b_optics_lw_set_tables")

    def optics_lw(self, in_ptr, ld, pdeldry, tauxar, ncol, nlev, dt, stream=0):
        """Longwave absorption optical depth (mam4b_optics_lw); device
        pointers, tauxar [16][ld]."""
        st = self._lib.mam4b_optics_lw(self._h, in_ptr, int(ld), pdeldry, tauxar, int(ncol),
                                       int(nlev), float(dt), ctypes.c_void_p(stream))
        self._check(st, "mam4b_optics_lw")

    def optics_sw_set_tables(self, tables):
        """Copies the shortwave optics tables (dict of numpy arrays, see
        workloads.make_optics_sw_tables) into the context."""
        import numpy as np
        keys = ("specrefindex", "water_refindex", "refrtab", "refitab", "extp", "absp", "asmp")
        arrs = {k: np.ascontiguousarray(tables[k], dtype=np.float64) for k in keys}
        t = OpticsSwTables(*[arrs[k].ctypes.data for k in keys])
        st = self._lib.mam4b_optics_sw_set_tables(self._h, ctypes.byref(t))
        self._check(st, "mam4b_optics_sw_set_tables")

    def optics_sw(self, in_ptr, ld, pdeldry, out, aodvis, ncol, nlev, dt, stream=0):
        """Shortwave optics (mam4b_optics_sw); device pointers, out [4][14][ld],
        aodvis [ncol] or 0."""
        st = self._lib.mam4b_optics_sw(self._h, in_ptr, int(ld), pdeldry, out, aodvis or None,
                                       int(ncol), int(nlev), float(dt),
                                       ctypes.c_void_p(stream))
        self._check(st, "mam4b_optics_sw")

    def activate(self, in_ptr, ld, air_density, updraft, out, ncol, nlev, stream=0):
        """Aerosol activation fractions (mam4b_activate); device pointers,
        out [17][ld]."""
        st = self._lib.mam4b_activate(self._h, in_ptr, int(ld), air_density, updraft, out,
                                      int(ncol), int(nlev), ctypes.c_void_p(stream))
        self._check(st, "mam4b_activate")

    def setsox(self, pressure, temperature, lwc, cloud_fraction, cloud_number, air_density,
               qin, qcw, ld, dqdt_aqso4, dqdt_aqh2so4, ncol, nlev, dt, stream=0):
        """Aqueous sulfate chemistry (mam4b_setsox); device pointers, qin and
        qcw [31][ld] updated in place, the tendency pointers may be 0."""
        st = self._lib.mam4b_setsox(self._h, pressure, temperature, lwc, cloud_fraction,
                                    cloud_number, air_density, qin, qcw, int(ld),
                                    dqdt_aqso4 or None, dqdt_aqh2so4 or None, int(ncol),
                                    int(nlev), float(dt), ctypes.c_void_p(stream))
        self._check(st, "mam4b_setsox")

    def step_chem_slab(self, in_ptr, pblh_ptr, chem_in_ptr, out_ptr, chem_out_ptr, ld, ncol,
                       nlev, dt, stream=0):
        """The step with gas-phase and aqueous chemistry ahead of amicphys
        (mam4b_step_chem_slab); device slabs of ld doubles per field."""
        st = self._lib.mam4b_step_chem_slab(self._h, in_ptr, pblh_ptr, chem_in_ptr, out_ptr,
                                            chem_out_ptr, int(ld), int(ncol), int(nlev),
                                            float(dt), ctypes.c_void_p(stream))
        self._check(st, "mam4b_step_chem_slab")

    def aero_rad_props_sw(self, in_ptr, ld, pdeldry, pint, zi, ext_sw, ssa_sw, af_sw, out,
                          aodvis, trop_level, ncol, nlev, dt, stream=0):
        """aero_rad_props_sw (mam4b_aero_rad_props_sw): shortwave optics
        with the volcanic aerosol over the tropopause; aodvis and
        trop_level may be 0."""
        st = self._lib.mam4b_aero_rad_props_sw(self._h, in_ptr, int(ld), pdeldry, pint, zi,
                                               ext_sw, ssa_sw, af_sw, out, aodvis or None,
                                               trop_level or None, int(ncol), int(nlev),
                                               float(dt), ctypes.c_void_p(stream))
        self._check(st, "mam4b_aero_rad_props_sw")

    def aero_rad_props_lw(self, in_ptr, ld, pdeldry, pint, zi, ext_lw, odap, trop_level, ncol,
                          nlev, dt, stream=0):
        """aero_rad_props_lw (mam4b_aero_rad_props_lw); trop_level may be 0."""
        st = self._lib.mam4b_aero_rad_props_lw(self._h, in_ptr, int(ld), pdeldry, pint, zi,
                                               ext_lw, odap, trop_level or None, int(ncol),
                                               int(nlev), float(dt), ctypes.c_void_p(stream))
        self._check(st, "mam4b_aero_rad_props_lw")

    def dropmixnuc(self, in_ptr, ld, mix_in, pint, kvh, out, ncol, nlev, top_lev, dt,
                   vertical_mix=True, stream=0):
        """ndrop::dropmixnuc over ncol columns (mam4b_dropmixnuc)."""
        st = self._lib.mam4b_dropmixnuc(self._h, in_ptr, int(ld), mix_in, pint, kvh, out,
                                        int(ncol), int(nlev), int(top_lev),
                                        int(bool(vertical_mix)), float(dt),
                                        ctypes.c_void_p(stream))
        self._check(st, "mam4b_dropmixnuc")

    def gas_chemistry(self, temperature, photo_rates, extfrc, invariants, het_rates, qq, ld,
                      ncol, nlev, dt, stream=0):
        """Gas-phase chemistry (mam4b_gas_chemistry); device pointers, qq
        [31][ld] updated in place."""
        st = self._lib.mam4b_gas_chemistry(self._h, temperature, photo_rates, extfrc, invariants,
                                           het_rates, qq, int(ld), int(ncol), int(nlev), float(dt),
                                           ctypes.c_void_p(stream))
        self._check(st, "mam4b_gas_chemistry")

    def calcsize_process(self, progs, tends, dgncur_i, dgncur_c, ncol, nlev, dt,
                         do_aitacc_transfer=True, do_adjust=True, stream=0):
        """CalcSize::compute_tendencies over ncol x nlev cells
        (mam4b_calcsize_process). progs, tends: ProgFields; dgncur_i,
        dgncur_c: 4 device pointers each."""
        cfg = CalcSizeConfig(int(do_aitacc_transfer), int(do_adjust))
        di = (ctypes.c_void_p * NUM_MODES)(*dgncur_i)
        dc = (ctypes.c_void_p * NUM_MODES)(*dgncur_c)
        st = self._lib.mam4b_calcsize_process(self._h, ctypes.byref(cfg), ctypes.byref(progs),
                                              ctypes.byref(tends), ctypes.byref(di),
                                              ctypes.byref(dc), int(ncol), int(nlev), float(dt),
                                              ctypes.c_void_p(stream))
        self._check(st, "mam4b_calcsize_process")

    def coagulation_process(self, temperature, pressure, wet_density, wet_diameter_i, progs,
                            tends, ncol, nlev, dt, stream=0):
        """Coagulation::compute_tendencies over ncol x nlev cells
        (mam4b_coagulation_process); progs are updated in place."""
        wd = (ctypes.c_void_p * NUM_MODES)(*wet_density)
        wg = (ctypes.c_void_p * NUM_MODES)(*wet_diameter_i)
        st = self._lib.mam4b_coagulation_process(self._h, temperature, pressure, ctypes.byref(wd),
                                                 ctypes.byref(wg), ctypes.byref(progs),
                                                 ctypes.byref(tends), int(ncol), int(nlev),
                                                 float(dt), ctypes.c_void_p(stream))
        self._check(st, "mam4b_coagulation_process")

    def tuning(self):
        t = Tuning()
        self._check(self._lib.mam4b_get_tuning(self._h, ctypes.byref(t)), "mam4b_get_tuning")
        return t

    def set_tuning(self, t):
        self._check(self._lib.mam4b_set_tuning(self._h, ctypes.byref(t)), "mam4b_set_tuning")

    def set_adjoint_checkpoint(self, interval):
        """SOA states of the adjoint: 1 = every sub-step, 4 = a checkpoint
        every 4 sub-steps (same gradient, a quarter of the memory)."""
        self._check(self._lib.mam4b_set_adjoint_checkpoint(self._h, int(interval)),
                    "mam4b_set_adjoint_checkpoint")

    def set_graph_mode(self, enable):
        self._check(self._lib.mam4b_set_graph_mode(self._h, int(bool(enable))),
                    "mam4b_set_graph_mode")

    def autotune(self, in_ptr, pblh_ptr, out_ptr, ld, ncol, nlev, dt, precision=FP64, reps=3,
                 stream=0):
        """Runs mam4b_autotune; returns (Tuning, default ms, tuned ms)."""
        t = Tuning()
        d_ms, b_ms = ctypes.c_float(0), ctypes.c_float(0)
        st = self._lib.mam4b_autotune(self._h, in_ptr, pblh_ptr, out_ptr, int(ld), int(ncol),
                                      int(nlev), float(dt), int(precision), int(reps),
                                      ctypes.c_void_p(stream), ctypes.byref(t), ctypes.byref(d_ms),
                                      ctypes.byref(b_ms))
        self._check(st, "mam4b_autotune")
        return t, float(d_ms.value), float(b_ms.value)

    def last_status(self):
        f = ctypes.c_uint32(0)
        st = self._lib.mam4b_last_status(self._h, ctypes.byref(f))
        if st not in (0, 4):
            self._check(st, "mam4b_last_status")
        return int(f.value)

    def launch_count(self):
        return int(self._lib.mam4b_launch_count(self._h))
