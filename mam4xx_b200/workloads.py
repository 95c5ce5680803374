"""Seeded synthetic workloads for the microphysics step.

No public dataset exists for this path, so each named configuration is a
seeded draw (NumPy PCG64, seed = 20261203 + configuration index) with the
shapes and value distributions of the step's benchmark configurations:

  c1  8 x 72 columns x levels, clear sky, no cloud-borne aerosol
  c2  4096 x 72, cloud fraction U(0, 1), cloud-borne aerosol drawn like the
      interstitial aerosol
  c3  65536 x 72, like c2 but 30% of cells get an Aitken number that puts the
      Aitken dry diameter within +-10% of the renaming cut-off diameter
  c4  65536 x 72, H2SO4 log-uniform 1e-15..1e-8 mol/mol, cloud fraction 0 for
      60% of cells and U(0.2, 1) for 40%, mode numbers log-uniform
      1e5..1e6 #/kg: the SOA condensation sub-step count then ranges over
      1..20 per cell (uneven sub-stepping; the histogram measured on the
      CPU oracle is baseline/soa_passes_c4.json, oracle/soa_pass_histogram.py)
  c5  16384 x 72, like c2 (adjoint configuration)
  c4_stress  c4 with the common number range 1e5..1e10 #/kg: 1..1000
      sub-steps per cell (mean about 80, a few cells at the cap of 1000)

The sub-step count of the SOA loop (gasaerexch_soaexch.hpp:170-173) grows
with the uptake rate times the time step, i.e. with the mode numbers; the
H2SO4 range does not drive it.

Common distributions (per cell): T ~ U(200, 310) K; RH ~ U(0.05, 0.99)
converted to a vapour mixing ratio with the Magnus saturation formula used
by amicphys (src/mam4xx/conversions.hpp:148-180, mam4_amicphys.hpp:2199-2205);
H2SO4 ~ logU(1e-14, 1e-10) and SOAG ~ logU(1e-12, 1e-9) mol/mol; mode numbers
~ logU(1e5, 1e10) #/kg; species masses ~ logU(1e-14, 1e-8) kg/kg for the
species present in each mode. Pressure is geometric from 10 to 1000 hPa over
the levels (level 0 at the top), heights follow the hypsometric equation with
the drawn temperatures, and the boundary-layer height is 1000 m.

The arrays use the field-major layout of include/mam4b.h: in_slab has shape
(MAM4B_NIN, ncell) with cell = col*nlev + lev.
"""

import numpy as np

NIN = 57
NOUT = 68
NDIAG = 155
IN_T, IN_P, IN_ZM, IN_QV, IN_CLD, IN_H2SO4, IN_SOAG = range(7)
IN_AER_I = 7
IN_AER_C = 32
OUT_DGN_A, OUT_DGN_AWET, OUT_WETDENS, OUT_QAERWAT = 52, 56, 60, 64

# Population layout of the 25 aerosol entries (E3SM state_q 15..39):
# (mode, species name) or (mode, "num").
POPULATIONS = (
    [(0, s) for s in ("SO4", "POM", "SOA", "BC", "DST", "NaCl", "MOM")] + [(0, "num")]
    + [(1, s) for s in ("SO4", "SOA", "NaCl", "MOM")] + [(1, "num")]
    + [(2, s) for s in ("DST", "NaCl", "SO4", "BC", "POM", "SOA", "MOM")] + [(2, "num")]
    + [(3, s) for s in ("POM", "BC", "MOM")] + [(3, "num")]
)
NUMBER_SLOTS = tuple(i for i, (_, s) in enumerate(POPULATIONS) if s == "num")
MODE_SPECIES_SLOTS = {m: tuple(i for i, (mm, s) in enumerate(POPULATIONS)
                               if mm == m and s != "num") for m in range(4)}

# Chemistry-mechanism molecular weights [g/mol] of the 31 amicphys tracers
# (src/mam4xx/gas_chem_mechanism.hpp:31-38).
ADV_MASS = np.array([
    47.998200, 34.013600, 98.078400, 64.064800, 62.132400, 12.011000,
    115.107340, 12.011000, 12.011000, 12.011000, 135.064039, 58.442468,
    250092.672000, 1.007400, 115.107340, 12.011000, 58.442468, 250092.672000,
    1.007400, 135.064039, 58.442468, 115.107340, 12.011000, 12.011000,
    12.011000, 250092.672000, 1.007400, 12.011000, 12.011000, 250092.672000,
    1.007400])
MW_DRY_AIR = 28.966  # kg/kmol

# Aitken-mode constants used to place cells near the renaming cut-off
# (src/mam4xx/aero_modes.hpp:76-123, rename.hpp:452-465).
_SIG = [1.8, 1.6, 1.8, 1.60000002384186]
_DGN_NOM = [1.1e-7, 2.6e-8, 2e-6, 5e-8]
_DENS = {"SOA": 1000.0, "SO4": 1770.0, "POM": 1000.0, "BC": 1700.0,
         "NaCl": 1900.0, "DST": 2600.0, "MOM": 1601.0}

CONFIGS = {
    "c1": dict(index=0, ncol=8, nlev=72, clouds="none"),
    "c2": dict(index=1, ncol=4096, nlev=72, clouds="uniform"),
    "c3": dict(index=2, ncol=65536, nlev=72, clouds="uniform", near_cutoff=0.3),
    "c4": dict(index=3, ncol=65536, nlev=72, clouds="bimodal",
               h2so4_range=(1e-15, 1e-8), number_range=(1e5, 1e6)),
    "c5": dict(index=4, ncol=16384, nlev=72, clouds="uniform"),
    "c4_stress": dict(index=3, ncol=65536, nlev=72, clouds="bimodal",
                      h2so4_range=(1e-15, 1e-8)),
}

DT = 1800.0


def rename_cutoff_diameter():
    """Aitken->accumulation cut-off diameter (rename.hpp:462-465)."""
    la, lc = np.log(_SIG[1]), np.log(_SIG[0])
    return np.sqrt(_DGN_NOM[1] * np.exp(1.5 * la * la) * _DGN_NOM[0] * np.exp(1.5 * lc * lc))


def magnus_qv_sat(temp, pmid):
    """Saturation specific humidity of the amicphys RH diagnosis."""
    eps = 0.018016 / 0.028966
    tc = temp - 273.15
    ew = 610.94 * np.exp(17.625 * tc / (234.04 + tc))
    es = 1.00071 * np.exp(4.5e-8 * pmid) * ew
    return eps * es / (pmid - (1.0 - eps) * es)


def _logu(rng, lo, hi, n):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


def make_workload(name="c1", ncol=None, nlev=None, seed=None):
    """Draws configuration `name`; ncol/nlev/seed override its defaults.

    Returns a dict with in_slab (NIN, ncell) float64, pblh (ncol,),
    ncol, nlev, dt and the configuration name."""
    cfg = dict(CONFIGS[name])
    ncol = cfg["ncol"] if ncol is None else int(ncol)
    nlev = cfg["nlev"] if nlev is None else int(nlev)
    seed = 20261203 + cfg["index"] if seed is None else int(seed)
    rng = np.random.Generator(np.random.PCG64(seed))
    n = ncol * nlev
    x = np.zeros((NIN, n), dtype=np.float64)

    temp = rng.uniform(200.0, 310.0, n)
    plev = np.geomspace(1000.0, 100000.0, nlev)  # Pa, level 0 at the top
    pmid = np.tile(plev, ncol)
    # hypsometric heights, integrating from the bottom level upward
    tcol = temp.reshape(ncol, nlev)
    zm = np.zeros((ncol, nlev))
    rd_over_g = 287.04 / 9.80616
    zm[:, -1] = rd_over_g * tcol[:, -1] * np.log(101325.0 / plev[-1])
    for k in range(nlev - 2, -1, -1):
        tbar = 0.5 * (tcol[:, k] + tcol[:, k + 1])
        zm[:, k] = zm[:, k + 1] + rd_over_g * tbar * np.log(plev[k + 1] / plev[k])
    rh = rng.uniform(0.05, 0.99, n)
    qv = rh * magnus_qv_sat(temp, pmid)

    if cfg["clouds"] == "none":
        cld = np.zeros(n)
    elif cfg["clouds"] == "uniform":
        cld = rng.uniform(0.0, 1.0, n)
    else:  # bimodal
        cld = np.where(rng.uniform(0.0, 1.0, n) < 0.6, 0.0, rng.uniform(0.2, 1.0, n))

    h2lo, h2hi = cfg.get("h2so4_range", (1e-14, 1e-10))
    h2so4_vmr = _logu(rng, h2lo, h2hi, n)
    soag_vmr = _logu(rng, 1e-12, 1e-9, n)

    x[IN_T] = temp
    x[IN_P] = pmid
    x[IN_ZM] = zm.reshape(-1)
    x[IN_QV] = qv
    x[IN_CLD] = cld
    x[IN_H2SO4] = h2so4_vmr * ADV_MASS[2] / MW_DRY_AIR
    x[IN_SOAG] = soag_vmr * ADV_MASS[5] / MW_DRY_AIR

    nlo, nhi = cfg.get("number_range", (1e5, 1e10))
    for base, cloudy in ((IN_AER_I, False), (IN_AER_C, True)):
        for slot, (mode, spec) in enumerate(POPULATIONS):
            if spec == "num":
                v = _logu(rng, nlo, nhi, n)
            else:
                v = _logu(rng, 1e-14, 1e-8, n)
            if cloudy and cfg["clouds"] == "none":
                v = np.zeros(n)
            x[base + slot] = v

    frac = cfg.get("near_cutoff")
    if frac:
        # For a fraction of cells choose the Aitken number so that the dry
        # number-median diameter from volume/number is within +-10% of the
        # renaming cut-off (mean_particle_diameter_from_volume inverted).
        pick = rng.uniform(0.0, 1.0, n) < frac
        dtarget = rename_cutoff_diameter() * rng.uniform(0.9, 1.1, n)
        vol = np.zeros(n)
        for slot in MODE_SPECIES_SLOTS[1]:
            vol += x[IN_AER_I + slot] / _DENS[POPULATIONS[slot][1]]
        lsg = np.log(_SIG[1])
        vpart = (np.pi / 6.0) * dtarget ** 3 * np.exp(4.5 * lsg * lsg)
        num_ait = vol / vpart
        x[IN_AER_I + NUMBER_SLOTS[1]] = np.where(pick, num_ait, x[IN_AER_I + NUMBER_SLOTS[1]])

    pblh = np.full(ncol, 1000.0)
    return {"name": name, "in_slab": x, "pblh": pblh, "ncol": ncol,
            "nlev": nlev, "dt": DT}


def pblh_per_cell(w):
    return np.repeat(w["pblh"], w["nlev"])


# ------------------------------------------------------ per-process inputs
AERO_IDS = ("SOA", "SO4", "POM", "BC", "NaCl", "DST", "MOM")  # mam4::AeroId order


def prog_slab(in_slab, by_aero_id=False):
    """The 64 Prognostics-style fields (n_mode_i[4], n_mode_c[4],
    q_aero_i[4][7], q_aero_c[4][7]) of a step input slab. The second index
    of q_aero_* is the species' position within its mode (CalcSize's
    indexing), or its mam4::AeroId with by_aero_id (Coagulation's), where
    the (mode, AeroId) pairs that are not species of the mode are zero."""
    n = in_slab.shape[1]
    out = np.zeros((64, n))
    for slot, (m, sp) in enumerate(POPULATIONS):
        for phase, base in ((0, IN_AER_I), (1, IN_AER_C)):
            row = in_slab[base + slot]
            if sp == "num":
                out[4 * phase + m] = row
            else:
                k = AERO_IDS.index(sp) if by_aero_id else MODE_SPECIES_SLOTS[m].index(slot)
                out[8 + 28 * phase + 7 * m + k] = row
    return out


def make_process_inputs(name="c2", ncol=None, nlev=None, seed=None):
    """Inputs of the per-process entries from a workload configuration:
    the step's populations as Prognostics fields (both index conventions),
    T and p, wet diameters of each mode drawn around its nominal size
    (0.5..4 x, log-uniform) and wet densities U(1000, 2000) kg/m3, and
    non-zero starting tendencies (the processes add to them)."""
    w = make_workload(name, ncol=ncol, nlev=nlev, seed=seed)
    x = w["in_slab"]
    n = x.shape[1]
    rng = np.random.default_rng(77 + (seed or 0))
    wet = np.zeros((8, n))
    for m in range(4):
        wet[m] = rng.uniform(1000.0, 2000.0, n)
        wet[4 + m] = _DGN_NOM[m] * _logu(rng, 0.5, 4.0, n)
    prog = prog_slab(x)
    tend0 = rng.standard_normal((64, n)) * (np.abs(prog) / 86400.0 + 1e-30)
    return {"ncol": w["ncol"], "nlev": w["nlev"], "dt": w["dt"], "temp": x[0].copy(),
            "pmid": x[1].copy(), "wet": wet, "prog": prog, "prog_aero": prog_slab(x, True),
            "tend0": tend0}


def make_setsox_inputs(name="c2", ncol=None, nlev=None, seed=None, w=None):
    """Inputs of the aqueous-chemistry entry from a workload configuration:
    T, p and cloud fraction of the workload; the 31 amicphys tracers in
    mol/mol (#/kmol for numbers) from its H2SO4, SOAG and populations, plus
    O3 log-uniform 1e-8..1e-7, H2O2 1e-11..1e-9 and SO2 1e-12..1e-8 mol/mol;
    cloud liquid water log-uniform 1e-6..1e-3 kg/kg in 80 % of the cloudy
    cells (0 elsewhere), droplet number 1e7..1e9 #/kg, and the air number
    density p / (k T) in #/cm3. w: the workload, if already made."""
    w = w or make_workload(name, ncol=ncol, nlev=nlev, seed=seed)
    x = w["in_slab"]
    n = x.shape[1]
    rng = np.random.default_rng(991 + (seed or 0))
    to_vmr = np.array([MW_DRY_AIR if i in (13, 18, 26, 30) else MW_DRY_AIR / ADV_MASS[i]
                       for i in range(31)])
    qin = np.zeros((31, n))
    qcw = np.zeros((31, n))
    qin[0] = _logu(rng, 1e-8, 1e-7, n)
    qin[1] = _logu(rng, 1e-11, 1e-9, n)
    qin[2] = x[5] * to_vmr[2]
    qin[3] = _logu(rng, 1e-12, 1e-8, n)
    qin[5] = x[6] * to_vmr[5]
    qin[6:31] = x[IN_AER_I:IN_AER_I + 25] * to_vmr[6:31, None]
    qcw[6:31] = x[IN_AER_C:IN_AER_C + 25] * to_vmr[6:31, None]
    cld = x[4].copy()
    lwc = np.where((cld > 0) & (rng.uniform(0, 1, n) < 0.8), _logu(rng, 1e-6, 1e-3, n), 0.0)
    cldnum = _logu(rng, 1e7, 1e9, n)
    xhnm = x[1] / (1.380649e-23 * x[0]) * 1e-6
    return {"ncol": w["ncol"], "nlev": w["nlev"], "dt": w["dt"], "press": x[1].copy(),
            "temp": x[0].copy(), "lwc": lwc, "cldfrc": cld, "cldnum": cldnum, "xhnm": xhnm,
            "qin": qin, "qcw": qcw}


def make_gas_chemistry_inputs(name="c2", ncol=None, nlev=None, seed=None, negative_frac=0.0,
                              w=None):
    """Inputs of the gas-phase chemistry entry from a workload configuration:
    its temperature; invariant densities as mo_setinv sets them (total air
    10 p / (k_cgs T), N2 0.79 and O2 0.21 of it, H2O from the workload's qv,
    (clipped at zero), OH, NO3, HO2 and O3 from offline mixing ratios log-uniform 1e-15..1e-12,
    1e-14..1e-10, 1e-13..1e-10 and 1e-8..1e-6); the H2O2 photolysis rate
    log-uniform 1e-7..1e-5 /s, zero (night) in 30 % of the cells; external
    forcing log-uniform 1e-3..1e2 molecules/cm3/s, zero in half the entries;
    wet-removal rates log-uniform 1e-8..1e-3 /s, zero in half the entries;
    the 31 tracers from the workload's H2SO4, SOAG and populations (mol/mol,
    #/kmol) plus O3 1e-8..1e-6, H2O2 1e-12..1e-9, SO2 1e-12..1e-8 and DMS
    1e-12..1e-9 mol/mol. With negative_frac > 0 that fraction of the cells
    gets one tracer slightly negative (-1e-20), which the Newton iteration
    never meets (clipping), so those cells take the step-cutting path.
    w: the workload, if already made."""
    w = w or make_workload(name, ncol=ncol, nlev=nlev, seed=seed)
    x = w["in_slab"]
    n = x.shape[1]
    rng = np.random.default_rng(2718 + (seed or 0))
    to_vmr = np.array([MW_DRY_AIR if i in (13, 18, 26, 30) else MW_DRY_AIR / ADV_MASS[i]
                       for i in range(31)])
    temp = x[0].copy()
    m = 10.0 * x[1] / (0.13806500000000001e-15 * temp)
    # water vapour as a mixing ratio, clipped at zero: the workload's qv is
    # drawn through the Magnus saturation formula, which goes negative where
    # the saturation pressure exceeds the pressure (hot cells near the top)
    h2ovmr = np.maximum(x[3], 0.0) * (MW_DRY_AIR / 18.015)
    inv = np.zeros((8, n))
    inv[0] = m
    inv[1] = 0.79 * m
    inv[2] = 0.21 * m
    inv[3] = h2ovmr * m
    inv[4] = _logu(rng, 1e-15, 1e-12, n) * m
    inv[5] = _logu(rng, 1e-14, 1e-10, n) * m
    inv[6] = _logu(rng, 1e-13, 1e-10, n) * m
    inv[7] = _logu(rng, 1e-8, 1e-6, n) * m
    photo = np.where(rng.uniform(0, 1, n) < 0.3, 0.0, _logu(rng, 1e-7, 1e-5, n))
    extfrc = np.where(rng.uniform(0, 1, (9, n)) < 0.5, 0.0,
                      _logu(rng, 1e-3, 1e2, 9 * n).reshape(9, n))
    het = np.where(rng.uniform(0, 1, (31, n)) < 0.5, 0.0,
                   _logu(rng, 1e-8, 1e-3, 31 * n).reshape(31, n))
    qq = np.zeros((31, n))
    qq[0] = _logu(rng, 1e-8, 1e-6, n)
    qq[1] = _logu(rng, 1e-12, 1e-9, n)
    qq[2] = x[5] * to_vmr[2]
    qq[3] = _logu(rng, 1e-12, 1e-8, n)
    qq[4] = _logu(rng, 1e-12, 1e-9, n)
    qq[5] = x[6] * to_vmr[5]
    qq[6:31] = x[IN_AER_I:IN_AER_I + 25] * to_vmr[6:31, None]
    if negative_frac > 0:
        pick = np.nonzero(rng.uniform(0, 1, n) < negative_frac)[0]
        qq[rng.integers(1, 31, pick.size), pick] = -1e-20
    return {"ncol": w["ncol"], "nlev": w["nlev"], "dt": w["dt"], "temp": temp, "photo": photo,
            "extfrc": extfrc, "inv": inv, "het": het, "qq": qq}


CHEM_NIN, CHEM_NOUT = 55, 4
CHEM_IN_PHOTO, CHEM_IN_EXTFRC, CHEM_IN_INV, CHEM_IN_HET, CHEM_IN_LWC, CHEM_IN_CLDNUM = (
    4, 5, 14, 22, 53, 54)


def make_chem_step_inputs(name="c2", ncol=None, nlev=None, seed=None, inert=False):
    """Inputs of the step with chemistry: the workload (make_workload) and
    its chemistry slab (CHEM_NIN fields): O3, H2O2, SO2, DMS as mass mixing
    ratios and the gas-phase chemistry inputs of make_gas_chemistry_inputs,
    cloud water and droplet number of make_setsox_inputs, for the same
    cells. inert=True zeroes every rate, forcing and the cloud water, so
    that neither chemistry changes anything."""
    w = make_workload(name, ncol=ncol, nlev=nlev, seed=seed)
    g = make_gas_chemistry_inputs(name, seed=seed, w=w)
    sx = make_setsox_inputs(name, seed=seed, w=w)
    n = w["in_slab"].shape[1]
    ch = np.zeros((CHEM_NIN, n))
    for k, i31 in enumerate((0, 1, 3, 4)):
        ch[k] = g["qq"][i31] * (ADV_MASS[i31] / MW_DRY_AIR)
    if not inert:
        ch[CHEM_IN_PHOTO] = g["photo"]
        ch[CHEM_IN_EXTFRC:CHEM_IN_EXTFRC + 9] = g["extfrc"]
        ch[CHEM_IN_HET:CHEM_IN_HET + 31] = g["het"]
        ch[CHEM_IN_LWC] = sx["lwc"]
    ch[CHEM_IN_INV:CHEM_IN_INV + 8] = g["inv"]
    if inert:
        ch[CHEM_IN_INV + 4:CHEM_IN_INV + 7] = 0.0  # no OH, NO3, HO2: no reactions
    ch[CHEM_IN_CLDNUM] = sx["cldnum"]
    w = dict(w)
    w["chem_in"] = ch
    return w


def make_rad_props_inputs(name="c2", ncol=None, nlev=None, seed=None, no_tropopause_frac=0.1):
    """Inputs of the radiation-facing optics entries (aero_rad_props): the
    workload's aerosol with an atmosphere that has a tropopause. Per column:
    surface temperature U(280, 305) K falling 6.5 K/km up to a tropopause at
    U(9, 17) km and rising 1.5 K/km above it, with 0.2 K of noise per level;
    a fraction no_tropopause_frac of the columns falls 8 K/km up to 60 hPa
    and is isothermal above (no tropopause: the reference's level 0). Heights are hypsometric on
    the workload's pressure levels; interfaces at the geometric means of
    adjacent levels, 101325 Pa at the surface; water vapour redrawn at
    relative humidity U(0.05, 0.99). Volcanic inputs per cell: shortwave
    extinction log-uniform 1e-8..1e-5 /m, albedo U(0.9, 1), asymmetry
    U(0.6, 0.8); longwave extinction 1e-9..1e-6 /m."""
    w = dict(make_workload(name, ncol=ncol, nlev=nlev, seed=seed))
    ncol, nlev = w["ncol"], w["nlev"]
    x = w["in_slab"].copy()
    n = ncol * nlev
    rng = np.random.default_rng(4711 + (seed or 0))
    plev = x[1][:nlev].copy()
    pint = np.empty(nlev + 1)
    pint[1:nlev] = np.sqrt(plev[:-1] * plev[1:])
    pint[0] = plev[0] * np.sqrt(plev[0] / plev[1])
    pint[nlev] = 101325.0
    rd_over_g = 287.04 / 9.80616
    z_approx = 7500.0 * np.log(101325.0 / plev)  # first guess of the heights
    t0 = rng.uniform(280.0, 305.0, ncol)[:, None]
    zt = rng.uniform(9000.0, 17000.0, ncol)[:, None]
    none = (rng.uniform(0, 1, ncol) < no_tropopause_frac)[:, None]
    tt = t0 - 6.5e-3 * zt
    temp = np.where(z_approx[None, :] <= zt, t0 - 6.5e-3 * z_approx[None, :],
                    tt + 1.5e-3 * (z_approx[None, :] - zt))
    # no tropopause: unstable up to 60 hPa, isothermal above (stable only
    # above the search's 75 hPa limit)
    z60 = 7500.0 * np.log(101325.0 / 6000.0)
    temp = np.where(none, t0 - 8.0e-3 * np.minimum(z_approx[None, :], z60), temp)
    temp = temp + rng.normal(0.0, 0.2, (ncol, nlev))
    zi = np.zeros((ncol, nlev + 1))
    for k in range(nlev - 1, -1, -1):
        zi[:, k] = zi[:, k + 1] + rd_over_g * temp[:, k] * np.log(pint[k + 1] / pint[k])
    zm = 0.5 * (zi[:, :-1] + zi[:, 1:])
    x[0] = temp.reshape(-1)
    x[2] = zm.reshape(-1)
    x[3] = rng.uniform(0.05, 0.99, n) * np.maximum(magnus_qv_sat(x[0], x[1]), 0.0)
    w["in_slab"] = x
    w["pint"] = np.tile(pint, ncol)
    w["zi"] = zi.reshape(-1)
    w["pdeldry"] = np.tile(np.diff(pint), ncol)
    w["ext_sw"] = _logu(rng, 1e-8, 1e-5, 14 * n).reshape(14, n)
    w["ssa_sw"] = rng.uniform(0.9, 1.0, (14, n))
    w["af_sw"] = rng.uniform(0.6, 0.8, (14, n))
    w["ext_lw"] = _logu(rng, 1e-9, 1e-6, 16 * n).reshape(16, n)
    return w


DROPMIX_NIN, DROPMIX_NOUT = 4, 66


def make_dropmix_inputs(name="c2", ncol=None, nlev=None, seed=None):
    """Inputs of the droplet activation and mixing entry (dropmixnuc): the
    atmosphere and aerosol of make_rad_props_inputs (hypsometric heights,
    interfaces) with the workload's cloud fraction as the new one; the
    previous cloud fraction differs from it by U(-0.3, 0.3) in 70 % of the
    cells (clipped to [0, 1]); droplet number log-uniform 1e6..1e9 #/kg
    where there was cloud; subgrid updraft U(0.02, 2) m/s; vertical
    diffusivity log-uniform 1e-3..200 m2/s at the interfaces."""
    w = dict(make_rad_props_inputs(name, ncol=ncol, nlev=nlev, seed=seed))
    n = w["in_slab"].shape[1]
    rng = np.random.default_rng(8191 + (seed or 0))
    cldn = w["in_slab"][4]
    cldo = np.where(rng.uniform(0, 1, n) < 0.7,
                    np.clip(cldn + rng.uniform(-0.3, 0.3, n), 0.0, 1.0), cldn)
    mix = np.zeros((DROPMIX_NIN, n))
    mix[0] = w["pdeldry"]
    mix[1] = cldo
    mix[2] = np.where(cldo > 0, _logu(rng, 1e6, 1e9, n), 0.0)
    mix[3] = rng.uniform(0.02, 2.0, n)
    w["mix"] = mix
    w["kvh"] = _logu(rng, 1e-3, 200.0, w["ncol"] * (w["nlev"] + 1))
    return w


def make_activation_inputs(name="c2", ncol=None, nlev=None, seed=None):
    """Inputs of the activation entry: a workload's input slab, the air
    density p / (R_air T) and an updraft log-uniform 0.01..3 m/s, zero or
    negative in 10 % of the cells (no activation there)."""
    w = make_workload(name, ncol=ncol, nlev=nlev, seed=seed)
    x = w["in_slab"]
    n = x.shape[1]
    rng = np.random.default_rng(313 + (seed or 0))
    r_air = 6.022214076e23 * 1.380649e-23 / 0.028966
    rho = x[1] / (r_air * x[0])
    wup = _logu(rng, 0.01, 3.0, n)
    cut = rng.uniform(0, 1, n)
    wup = np.where(cut < 0.05, 0.0, np.where(cut < 0.1, -wup, wup))
    return {"ncol": w["ncol"], "nlev": w["nlev"], "in_slab": x, "rho": rho, "w": wup}


def make_optics_lw_tables(seed=0):
    """Seeded stand-ins for the longwave optics tables the host model reads
    from its optics files (same shapes and value ranges, not the data):
    species-type refractive indices (real 1.4..1.9, imaginary 1e-4..0.5),
    water (1.2..1.4, 1e-3..0.5), per-(mode, band) refractive-index grids
    (7 real values over 1.2..2.0, 10 imaginary values over 1e-4..1) and
    Chebyshev absorption coefficients (5 per grid point)."""
    rng = np.random.default_rng(4242 + seed)
    nb, nt = 16, 14
    spec = np.empty((nb, nt, 2))
    spec[..., 0] = rng.uniform(1.4, 1.9, (nb, nt))
    spec[..., 1] = _logu(rng, 1e-4, 0.5, nb * nt).reshape(nb, nt)
    water = np.empty((nb, 2))
    water[:, 0] = rng.uniform(1.2, 1.4, nb)
    water[:, 1] = _logu(rng, 1e-3, 0.5, nb)
    refr = np.sort(rng.uniform(1.2, 2.0, (4, nb, 7)), axis=2)
    refr[..., 0], refr[..., -1] = 1.2, 2.0
    refi = np.sort(_logu(rng, 1e-4, 1.0, 4 * nb * 10).reshape(4, nb, 10), axis=2)
    absp = rng.normal(0.0, 300.0, (4, nb, 5, 7, 10))
    absp[:, :, 0] = rng.uniform(500.0, 2000.0, (4, nb, 7, 10))
    return {"specrefindex": np.ascontiguousarray(spec), "water_refindex": water,
            "refrtab": refr, "refitab": refi, "absp": absp}


def make_optics_sw_tables(seed=0):
    """Seeded stand-ins for the shortwave optics tables (shapes and value
    ranges of the host model's files, not their data): refractive indices
    (real 1.3..1.8, imaginary 1e-8..0.1), water (1.33, 1e-9..1e-6), grids
    as for the longwave, and Chebyshev coefficients of log specific
    extinction (first one 2..10), absorption and asymmetry."""
    rng = np.random.default_rng(5151 + seed)
    nb, nt = 14, 14
    spec = np.empty((nb, nt, 2))
    spec[..., 0] = rng.uniform(1.3, 1.8, (nb, nt))
    spec[..., 1] = _logu(rng, 1e-8, 0.1, nb * nt).reshape(nb, nt)
    water = np.empty((nb, 2))
    water[:, 0] = 1.33
    water[:, 1] = _logu(rng, 1e-9, 1e-6, nb)
    refr = np.sort(rng.uniform(1.2, 2.0, (4, nb, 7)), axis=2)
    refr[..., 0], refr[..., -1] = 1.2, 2.0
    refi = np.sort(_logu(rng, 1e-9, 1.0, 4 * nb * 10).reshape(4, nb, 10), axis=2)
    extp = rng.normal(0.0, 0.5, (4, nb, 5, 7, 10))
    extp[:, :, 0] = rng.uniform(2.0, 10.0, (4, nb, 7, 10))
    absp = rng.normal(0.0, 50.0, (4, nb, 5, 7, 10))
    absp[:, :, 0] = rng.uniform(10.0, 500.0, (4, nb, 7, 10))
    asmp = rng.normal(0.0, 0.1, (4, nb, 5, 7, 10))
    asmp[:, :, 0] = rng.uniform(0.8, 1.6, (4, nb, 7, 10))
    return {"specrefindex": np.ascontiguousarray(spec), "water_refindex": water,
            "refrtab": refr, "refitab": refi, "extp": extp, "absp": absp, "asmp": asmp}
