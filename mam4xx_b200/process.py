"""Host-side mirror of the AeroProcess plug-in interface for the
microphysics step, over CUDA tensors.

Mirrors src/validation/aero_process.hpp:19-129 (AeroProcess<Impl>) and the
state containers of src/mam4xx/aero_config.hpp (Prognostics :74,
Diagnostics :170, Tendencies = Prognostics) and src/mam4xx/atmosphere.hpp:16.
A ColumnView per column becomes one (ncol, nlev) float64 CUDA tensor per
field; `compute_tendencies` processes every column in one kernel launch,
which is the batched replacement of the host's per-team dispatch
(`parallel_for(team_policy, ... compute_tendencies(team, ...))`).
"""

import torch

from . import native
from .workloads import NIN, NOUT, NDIAG, IN_AER_C, IN_AER_I

NUM_MODES = 4
NUM_AERO = 7
MODE_NSPEC = (7, 4, 7, 3)
SPEC0 = (0, 8, 13, 21)
NUMSLOT = (7, 12, 20, 24)
GAS_NAMES = ("H2SO4", "SOAG")


class AeroConfig:
    """mam4::AeroConfig (src/mam4xx/aero_config.hpp:21-71)."""
    num_modes = NUM_MODES
    num_aerosol_ids = NUM_AERO
    num_gas_ids = 6
    max_agepair = 1


class Atmosphere:
    """Fields the step reads from mam4::Atmosphere: (ncol, nlev) tensors and
    the per-column boundary-layer height (ncol,)."""

    def __init__(self, temperature, pressure, vapor_mixing_ratio, height, cloud_fraction,
                 planetary_boundary_layer_height):
        self.temperature = temperature
        self.pressure = pressure
        self.vapor_mixing_ratio = vapor_mixing_ratio
        self.height = height
        self.cloud_fraction = cloud_fraction
        self.planetary_boundary_layer_height = planetary_boundary_layer_height

    @property
    def shape(self):
        return tuple(self.temperature.shape)


class Prognostics:
    """mam4::Prognostics: mode numbers and species masses, interstitial (_i)
    and cloud-borne (_c); q_aero_*[mode][species] follows the species order of
    each mode (src/mam4xx/aero_modes.hpp:214-243); q_gas holds H2SO4, SOAG.
    Also used for Tendencies."""

    def __init__(self, n_mode_i, n_mode_c, q_aero_i, q_aero_c, q_gas):
        self.n_mode_i = n_mode_i
        self.n_mode_c = n_mode_c
        self.q_aero_i = q_aero_i
        self.q_aero_c = q_aero_c
        self.q_gas = q_gas

    @classmethod
    def empty_like(cls, ref):
        z = lambda t: torch.empty_like(t)
        return cls([z(t) for t in ref.n_mode_i], [z(t) for t in ref.n_mode_c],
                   [[z(t) for t in m] for m in ref.q_aero_i],
                   [[z(t) for t in m] for m in ref.q_aero_c], [z(t) for t in ref.q_gas])

    def population(self, cloudborne, slot):
        """Tensor of aerosol population `slot` (0..24, E3SM state_q order)."""
        n = self.n_mode_c if cloudborne else self.n_mode_i
        q = self.q_aero_c if cloudborne else self.q_aero_i
        for m in range(NUM_MODES):
            if slot == NUMSLOT[m]:
                return n[m]
            if SPEC0[m] <= slot < SPEC0[m] + MODE_NSPEC[m]:
                return q[m][slot - SPEC0[m]]
        raise IndexError(slot)


Tendencies = Prognostics


class Diagnostics:
    """Outputs of the step from mam4::Diagnostics: dry and wet geometric-mean
    diameters and wet density of the interstitial modes, the aerosol water,
    the cloud-borne dry diameters (written by CalcSizeProcess),
    and optionally the amicphys process tendencies
    (gas_aero_exchange_{condensation, renaming, nucleation, coagulation,
    renaming_cloud_borne}, each a list of 31 tracer tensors)."""

    PROCESSES = ("condensation", "renaming", "nucleation", "coagulation",
                 "renaming_cloud_borne")

    def __init__(self, dry_geometric_mean_diameter_i, wet_geometric_mean_diameter_i,
                 wet_density, aerosol_water, gas_aero_exchange=None,
                 dry_geometric_mean_diameter_c=None):
        self.dry_geometric_mean_diameter_i = dry_geometric_mean_diameter_i
        self.dry_geometric_mean_diameter_c = dry_geometric_mean_diameter_c
        self.wet_geometric_mean_diameter_i = wet_geometric_mean_diameter_i
        self.wet_density = wet_density
        self.aerosol_water = aerosol_water
        self.gas_aero_exchange = gas_aero_exchange

    @classmethod
    def allocate(cls, ncol, nlev, device, with_process_tendencies=False):
        e = lambda: torch.empty((ncol, nlev), dtype=torch.float64, device=device)
        gae = None
        if with_process_tendencies:
            gae = {p: [e() for _ in range(31)] for p in cls.PROCESSES}
        return cls([e() for _ in range(4)], [e() for _ in range(4)], [e() for _ in range(4)],
                   [e() for _ in range(4)], gae, [e() for _ in range(4)])


def _ptr(t, shape, what):
    if t is None:
        raise ValueError("%s is missing" % what)
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise ValueError("%s must be a contiguous float64 CUDA tensor" % what)
    if tuple(t.shape) != shape:
        raise ValueError("%s has shape %s, expected %s" % (what, tuple(t.shape), shape))
    return t.data_ptr()


class MicrophysicsProcess:
    """The B200 microphysics step behind the AeroProcess contract
    (name / init / validate / compute_tendencies)."""

    class Config:
        """Process switches (AmicPhysConfig, mam4_amicphys.hpp:223-237)."""

        def __init__(self, do_cond=True, do_rename=True, do_newnuc=True, do_coag=True,
                     gaexch_h2so4_uptake_optaa=2, newnuc_h2so4_conc_optaa=2,
                     n_so4_monolayers_pcage=8):
            self.do_cond = do_cond
            self.do_rename = do_rename
            self.do_newnuc = do_newnuc
            self.do_coag = do_coag
            self.gaexch_h2so4_uptake_optaa = gaexch_h2so4_uptake_optaa
            self.newnuc_h2so4_conc_optaa = newnuc_h2so4_conc_optaa
            self.n_so4_monolayers_pcage = n_so4_monolayers_pcage

        def to_native(self):
            return native.default_config(
                do_cond=self.do_cond, do_rename=self.do_rename, do_newnuc=self.do_newnuc,
                do_coag=self.do_coag, gaexch_h2so4_uptake_optaa=self.gaexch_h2so4_uptake_optaa,
                newnuc_h2so4_conc_optaa=self.newnuc_h2so4_conc_optaa,
                n_so4_monolayers_pcage=self.n_so4_monolayers_pcage)

    def __init__(self, aero_config=None, process_config=None):
        self._ctx = None
        self.init(aero_config or AeroConfig(), process_config or MicrophysicsProcess.Config())

    @staticmethod
    def name():
        return "MAM4 microphysics (calcsize, water uptake, amicphys) on B200"

    def init(self, aero_config, process_config=None):
        self.aero_config = aero_config
        self.process_config = process_config or MicrophysicsProcess.Config()
        if self._ctx is not None:
            self._ctx.close()
        self._ctx = native.Context(self.process_config.to_native())

    def validate(self, atmosphere, prognostics):
        """True when the state is physical: non-negative temperature, pressure
        and vapour, and non-negative mixing ratios (the checks of the
        reference processes' validate(), e.g. gasaerexch.hpp:97-120)."""
        bad = (atmosphere.temperature < 0).any() | (atmosphere.pressure < 0).any() | \
              (atmosphere.vapor_mixing_ratio < 0).any()
        tens = list(prognostics.n_mode_i) + list(prognostics.n_mode_c) + list(prognostics.q_gas)
        for m in range(NUM_MODES):
            tens += list(prognostics.q_aero_i[m]) + list(prognostics.q_aero_c[m])
        for t in tens:
            bad = bad | (t < 0).any()
        return not bool(bad.item())

    def compute_tendencies(self, t, dt, atmosphere, surface, prognostics, diagnostics,
                           tendencies, stream=None):
        """Computes the step's tendencies for every column: writes
        `tendencies` (same layout as `prognostics`, per second) and the
        diagnostics; asynchronous on `stream` (torch current stream by
        default)."""
        ncol, nlev = atmosphere.shape
        shp = (ncol, nlev)
        ins = [None] * NIN
        ins[0] = _ptr(atmosphere.temperature, shp, "temperature")
        ins[1] = _ptr(atmosphere.pressure, shp, "pressure")
        ins[2] = _ptr(atmosphere.height, shp, "height")
        ins[3] = _ptr(atmosphere.vapor_mixing_ratio, shp, "vapor_mixing_ratio")
        ins[4] = _ptr(atmosphere.cloud_fraction, shp, "cloud_fraction")
        ins[5] = _ptr(prognostics.q_gas[0], shp, "q_gas[H2SO4]")
        ins[6] = _ptr(prognostics.q_gas[1], shp, "q_gas[SOAG]")
        outs = [None] * NOUT
        outs[0] = _ptr(tendencies.q_gas[0], shp, "tend q_gas[H2SO4]")
        outs[1] = _ptr(tendencies.q_gas[1], shp, "tend q_gas[SOAG]")
        for slot in range(25):
            ins[IN_AER_I + slot] = _ptr(prognostics.population(False, slot), shp, "aerosol %d" % slot)
            ins[IN_AER_C + slot] = _ptr(prognostics.population(True, slot), shp, "cloud aerosol %d" % slot)
            outs[2 + slot] = _ptr(tendencies.population(False, slot), shp, "tend aerosol %d" % slot)
            outs[27 + slot] = _ptr(tendencies.population(True, slot), shp, "tend cloud %d" % slot)
        for m in range(NUM_MODES):
            outs[52 + m] = _ptr(diagnostics.dry_geometric_mean_diameter_i[m], shp, "dgn_a")
            outs[56 + m] = _ptr(diagnostics.wet_geometric_mean_diameter_i[m], shp, "dgn_awet")
            outs[60 + m] = _ptr(diagnostics.wet_density[m], shp, "wet_density")
            outs[64 + m] = _ptr(diagnostics.aerosol_water[m], shp, "aerosol_water")
        pblh = atmosphere.planetary_boundary_layer_height
        pb = _ptr(pblh, (ncol,), "planetary_boundary_layer_height")
        diag_ptrs = None
        if diagnostics.gas_aero_exchange is not None:
            diag_ptrs = [0] * NDIAG
            for k, p in enumerate(Diagnostics.PROCESSES):
                for i in range(31):
                    diag_ptrs[k * 31 + i] = _ptr(diagnostics.gas_aero_exchange[p][i], shp, p)
        s = stream if stream is not None else torch.cuda.current_stream()
        self._ctx.step(ins, pb, outs, ncol, nlev, dt, diag_ptrs=diag_ptrs,
                       stream=s.cuda_stream)

    def last_status(self):
        return self._ctx.last_status()

    def launch_count(self):
        return self._ctx.launch_count()


def state_from_slab(in_slab, pblh, ncol, nlev):
    """Views a (NIN, ncol*nlev) CUDA slab as Atmosphere + Prognostics."""
    v = lambda f: in_slab[f].view(ncol, nlev)
    atm = Atmosphere(v(0), v(1), v(3), v(2), v(4), pblh)
    ni = [v(IN_AER_I + NUMSLOT[m]) for m in range(NUM_MODES)]
    nc = [v(IN_AER_C + NUMSLOT[m]) for m in range(NUM_MODES)]
    qi = [[v(IN_AER_I + SPEC0[m] + s) for s in range(MODE_NSPEC[m])] for m in range(NUM_MODES)]
    qc = [[v(IN_AER_C + SPEC0[m] + s) for s in range(MODE_NSPEC[m])] for m in range(NUM_MODES)]
    progs = Prognostics(ni, nc, qi, qc, [v(5), v(6)])
    return atm, progs


def outputs_from_slab(out_slab, ncol, nlev, diag_slab=None):
    """Views a (NOUT, ncol*nlev) CUDA slab as Tendencies + Diagnostics."""
    v = lambda f: out_slab[f].view(ncol, nlev)
    ni = [v(2 + NUMSLOT[m]) for m in range(NUM_MODES)]
    nc = [v(27 + NUMSLOT[m]) for m in range(NUM_MODES)]
    qi = [[v(2 + SPEC0[m] + s) for s in range(MODE_NSPEC[m])] for m in range(NUM_MODES)]
    qc = [[v(27 + SPEC0[m] + s) for s in range(MODE_NSPEC[m])] for m in range(NUM_MODES)]
    tends = Prognostics(ni, nc, qi, qc, [v(0), v(1)])
    gae = None
    if diag_slab is not None:
        d = lambda f: diag_slab[f].view(ncol, nlev)
        gae = {p: [d(k * 31 + i) for i in range(31)] for k, p in enumerate(Diagnostics.PROCESSES)}
    diags = Diagnostics([v(52 + m) for m in range(4)], [v(56 + m) for m in range(4)],
                        [v(60 + m) for m in range(4)], [v(64 + m) for m in range(4)], gae)
    return tends, diags


def _prog_fields(p, shp, what, nspec_only):
    """ProgFields of a Prognostics container of (ncol, nlev) tensors; index
    lists shorter than 7 leave the remaining (mode, index) pairs null."""
    f = native.ProgFields()
    for m in range(NUM_MODES):
        f.n_mode_i[m] = _ptr(p.n_mode_i[m], shp, "%s n_mode_i[%d]" % (what, m))
        f.n_mode_c[m] = _ptr(p.n_mode_c[m], shp, "%s n_mode_c[%d]" % (what, m))
        for k, t in enumerate(p.q_aero_i[m]):
            if t is not None:
                f.q_aero_i[m][k] = _ptr(t, shp, "%s q_aero_i[%d][%d]" % (what, m, k))
        for k, t in enumerate(p.q_aero_c[m]):
            if t is not None:
                f.q_aero_c[m][k] = _ptr(t, shp, "%s q_aero_c[%d][%d]" % (what, m, k))
    return f


class CalcSizeProcess:
    """mam4::CalcSize behind the AeroProcess contract, batched over columns
    (mam4b_calcsize_process; src/mam4xx/calcsize.hpp:835-1220). Prognostics
    and Tendencies index q_aero_*[mode] by the species' position within the
    mode, as CalcSize does. Writes the dry diameters of both phases into
    diagnostics.dry_geometric_mean_diameter_i / _c."""

    class Config:
        def __init__(self, do_aitacc_transfer=True, do_adjust=True):
            self.do_aitacc_transfer = do_aitacc_transfer
            self.do_adjust = do_adjust

    def __init__(self, aero_config=None, process_config=None):
        self.init(aero_config or AeroConfig(), process_config)

    @staticmethod
    def name():
        return "MAM4 CalcSize on B200"

    def init(self, aero_config, process_config=None):
        self.aero_config = aero_config
        self.process_config = process_config or CalcSizeProcess.Config()
        self._ctx = native.Context()

    def validate(self, atmosphere, prognostics):
        return True  # calcsize.hpp: no validity checks

    def compute_tendencies(self, t, dt, atmosphere, surface, prognostics, diagnostics,
                           tendencies, stream=None):
        ncol, nlev = atmosphere.shape
        shp = (ncol, nlev)
        pf = _prog_fields(prognostics, shp, "prognostics", True)
        tf = _prog_fields(tendencies, shp, "tendencies", True)
        di = [_ptr(diagnostics.dry_geometric_mean_diameter_i[m], shp, "dgncur_i") for m in range(4)]
        dc = [_ptr(diagnostics.dry_geometric_mean_diameter_c[m], shp, "dgncur_c") for m in range(4)]
        s = stream if stream is not None else torch.cuda.current_stream()
        c = self.process_config
        self._ctx.calcsize_process(pf, tf, di, dc, ncol, nlev, dt,
                                   do_aitacc_transfer=c.do_aitacc_transfer,
                                   do_adjust=c.do_adjust, stream=s.cuda_stream)


class CoagulationProcess:
    """mam4::Coagulation behind the AeroProcess contract, batched over
    columns (mam4b_coagulation_process; src/mam4xx/coagulation.hpp:
    1121-1209). As that routine, q_aero_i[mode] is indexed by mam4::AeroId
    (SOA SO4 POM BC NaCl DST MOM) and needs all 7 entries for every mode;
    reads diagnostics.wet_density and wet_geometric_mean_diameter_i, adds
    to the interstitial tendencies and overwrites the interstitial
    prognostics with the coagulated state."""

    class Config:
        pass

    def __init__(self, aero_config=None, process_config=None):
        self.init(aero_config or AeroConfig(), process_config)

    @staticmethod
    def name():
        return "MAM4 Coagulation on B200"

    def init(self, aero_config, process_config=None):
        self.aero_config = aero_config
        self.process_config = process_config or CoagulationProcess.Config()
        self._ctx = native.Context()

    def validate(self, atmosphere, prognostics):
        return True  # coagulation.hpp:47-52 returns true

    def compute_tendencies(self, t, dt, atmosphere, surface, prognostics, diagnostics,
                           tendencies, stream=None):
        ncol, nlev = atmosphere.shape
        shp = (ncol, nlev)
        for m in range(NUM_MODES):
            if len(prognostics.q_aero_i[m]) != NUM_AERO or len(tendencies.q_aero_i[m]) != NUM_AERO:
                raise ValueError("Coagulation needs q_aero_i[mode] for all %d AeroIds" % NUM_AERO)
        pf = _prog_fields(prognostics, shp, "prognostics", False)
        tf = _prog_fields(tendencies, shp, "tendencies", False)
        wd = [_ptr(diagnostics.wet_density[m], shp, "wet_density") for m in range(4)]
        wg = [_ptr(diagnostics.wet_geometric_mean_diameter_i[m], shp, "wet diameter")
              for m in range(4)]
        s = stream if stream is not None else torch.cuda.current_stream()
        self._ctx.coagulation_process(_ptr(atmosphere.temperature, shp, "temperature"),
                                      _ptr(atmosphere.pressure, shp, "pressure"), wd, wg, pf, tf,
                                      ncol, nlev, dt, stream=s.cuda_stream)
