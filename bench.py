"""Benchmark of the MAM4 microphysics step on B200.

Workload: the uneven-batching configuration, 65,536 columns x 72 levels per
GPU (4,718,592 cells), FP64, seeded synthetic inputs (mam4xx_b200.workloads
'c4': H2SO4 1e-15..1e-8 mol/mol, cloud fraction 60% clear / 40% U(0.2, 1),
mode numbers 1e5..1e6 #/kg so that the SOA condensation sub-step count
ranges over 1..20 per cell). One step = calcsize + water uptake + amicphys
over every cell, dt = 1800 s.

  value  cells/s with inputs resident in HBM (one step = the pipeline
         behind mam4b_step_slab), whole job = all ranks' cells /
         max-over-ranks time (mam4xx_b200.distributed.timed_steps)
  e2e    cells/s through the C ABI host entry (mam4b_step_host): pinned host
         slabs copied in, step, results copied out, every step
  roofline_fp64  algorithmic flops per cell (baseline/flops_per_cell.json,
         counted on the CPU restatement) x cells / step time, against the
         FP64 FMA peak measured in the same run (libmam4b_peaks.so)
  roofline  algorithmic HBM bytes (57 input + 68 output doubles per cell plus
         the per-column boundary-layer height) / measured step time (the
         unit is one step), against the measured copy bandwidth of
         MEASURED_PEAKS.json; traffic = DRAM bytes per cell of the step's
         kernels measured by ncu (baseline/dram_traffic.json) times the cells
  cpu_baseline  the mam4xx reference headers compiled for the host
         (oracle/_ref, the tuned build, OpenMP) on a bounded sample of the
         same cells; the compiler flags are stated in its "sample"

  precisions  the mixed-precision forms on their configuration c3
         (65,536 x 72, 30 % of cells near the renaming cut-off): cells/s,
         speed-up over the FP64 step on the same cells, and every cell's
         error against the FP64 result
  adjoint  forward and adjoint time on c5 (16,384 x 72) and a central
         finite-difference check of the gradient
  processes  the per-process and downstream entries (CalcSize, Coagulation,
         setsox, gas chemistry, the step with chemistry, activation, optics,
         aero_rad_props, dropmixnuc) and the step through
         mam4b_step_tracers: cells/s, the HBM roofline of their algorithmic
         bytes, and the reference's own process classes on the host as their
         CPU baseline

--impl reference times that CPU implementation alone, as the reference arm.
Multi-GPU: one process per GPU (torchrun); each rank owns its own 65,536
columns, no data exchange (cells are independent); timing is max over ranks.
"""

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NCOL_PER_GPU = 65536
NLEV = 72
WORKLOAD = "c4"
REF_SAMPLE_NCOL = 1024  # columns of the reference arm's per-step sample
BYTES_PER_CELL = (57 + 68) * 8  # + 8 bytes of boundary-layer height per column
METRIC = "cells/s per amicphys step, FP64 vs mixed @ stated err; adjoint/forward time"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _flops_per_cell(workload):
    """Algorithmic flops per cell (+ - * /; libm calls apart) of the
    workload, counted on the CPU restatement by oracle/count_flops.py."""
    p = os.path.join(ROOT, "baseline", "flops_per_cell.json")
    if not os.path.exists(p):
        return None, None
    with open(p) as f:
        d = json.load(f)["configs"][workload]
    return float(d["flops_per_cell"]), float(d["special_per_cell"])


def _fp_peaks():
    """FP64 and FP32 vector FMA peaks (GFLOP/s), measured now on this device
    by libmam4b_peaks.so (8 independent FMA chains per thread)."""
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "mam4xx_b200", "libmam4b_peaks.so"))
    lib.mam4b_peak_gflops.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    res = {}
    for name, fp64 in (("fp64", 1), ("fp32", 0)):
        g, ms = ctypes.c_double(), ctypes.c_double()
        if lib.mam4b_peak_gflops(fp64, ctypes.byref(g), ctypes.byref(ms)) != 0:
            raise RuntimeError("peak measurement failed")
        res[name] = g.value
    return res


def _traffic_per_launch(workload, ncell):
    """DRAM bytes (read + write) of one step, from the per-cell traffic of
    the step's kernels measured by ncu (baseline/dram_traffic.json), scaled
    by the cells; None where no capture of this workload is recorded."""
    p = os.path.join(ROOT, "baseline", "dram_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f).get("configs", {}).get(workload)
    return None if not d else float(d["bytes_per_cell"]) * ncell


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for k, n in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(x, pblh_cell, dt, target_s=12.0):
    """Times the reference headers built for the host (the tuned build where
    the host has AVX2/FMA, else the parity build, else the restatement) on a
    bounded sample of the workload, OpenMP over cells on every host core."""
    from oracle import pyoracle
    orc, kind, flags = pyoracle.baseline_oracle()
    cores = os.cpu_count() or 1
    n0 = min(x.shape[1], 8 * 1024)
    t = time.perf_counter()
    orc.step(x[:, :n0], pblh_cell[:n0], dt, nthreads=cores)
    rate0 = n0 / max(time.perf_counter() - t, 1e-6)
    n = int(min(x.shape[1], max(n0, rate0 * target_s)))
    t = time.perf_counter()
    orc.step(x[:, :n], pblh_cell[:n], dt, nthreads=cores)
    el = time.perf_counter() - t
    return {"value": n / el, "unit": "cells/s", "cores": cores, "kind": kind,
            "sample": "first %d cells of the %s workload (%.1f s, OpenMP over cells); %s"
                      % (n, WORKLOAD, el, flags)}


# algorithmic bytes per cell of the per-process entries (FP64): CalcSize
# reads 50 state fields and 20 tendencies it adds to (4 numbers, 16 common
# species) and writes 24 tendencies and 8 diameters; Coagulation reads T,
# p, 8 wet sizes, 32 interstitial states and their 32 tendencies and writes
# both back
# ; setsox reads 6 met fields, 4 gas and 7 cloud-borne tracers and writes 3
# gas tracers, 3 cloud-borne SO4 and 6 tendencies
PROCESS_BYTES_PER_CELL = {"calcsize": (50 + 20 + 24 + 8) * 8, "coagulation": (42 + 32 + 64) * 8,
                          "setsox": (6 + 4 + 7 + 3 + 3 + 6) * 8,
                          "gas_chemistry": (2 + 9 + 8 + 30 + 30 + 30) * 8,
                          "step_chem": (57 + 55 + 68 + 4) * 8,
                          "aero_rad_props_sw": (55 + 1 + 42 + 2 + 56) * 8,
                          "aero_rad_props_lw": (55 + 1 + 16 + 2 + 16) * 8,
                          "dropmixnuc": (54 + 4 + 2 + 66) * 8,
                          "activation": (28 + 17) * 8, "optics_lw": (55 + 16) * 8,
                          "optics_sw": (55 + 56) * 8}


def processes_leg(native, torch, dev, stream, args, ws, hbm_peak):
    """Per-process entries (mam4b_calcsize_process, mam4b_coagulation_process)
    on the forward workload's columns, inputs resident, CUDA events; the
    reference's own process classes (oracle/_ref, OpenMP over columns) timed
    on 256 of those columns for the CPU baseline."""
    from mam4xx_b200.workloads import make_process_inputs
    ncol = args.ncol
    d = make_process_inputs(WORKLOAD, ncol=ncol, seed=20261203 + 3 + 1000 * int(os.environ.get("RANK", "0")))
    n = d["prog"].shape[1]
    prog = torch.from_numpy(d["prog"]).to(dev)
    prog_a0 = torch.from_numpy(d["prog_aero"]).to(dev)
    prog_a = prog_a0.clone()
    tend0 = torch.from_numpy(d["tend0"]).to(dev)
    tend = tend0.clone()
    dgn = torch.empty((8, n), dtype=torch.float64, device=dev)
    t = torch.from_numpy(d["temp"]).to(dev)
    p = torch.from_numpy(d["pmid"]).to(dev)
    wet = torch.from_numpy(d["wet"]).to(dev)
    ctx = native.Context()
    pf = native.ProgFields.from_slab(prog.data_ptr(), n)
    pa = native.ProgFields.from_slab(prog_a.data_ptr(), n)
    tf = native.ProgFields.from_slab(tend.data_ptr(), n)
    di = [dgn[m].data_ptr() for m in range(4)]
    dc = [dgn[4 + m].data_ptr() for m in range(4)]
    wd = [wet[m].data_ptr() for m in range(4)]
    wg = [wet[4 + m].data_ptr() for m in range(4)]

    def calcsize():
        ctx.calcsize_process(pf, tf, di, dc, ncol, NLEV, d["dt"], stream=stream.cuda_stream)

    def coag():
        ctx.coagulation_process(t.data_ptr(), p.data_ptr(), wd, wg, pa, tf, ncol, NLEV, d["dt"],
                                stream=stream.cuda_stream)

    from mam4xx_b200.workloads import make_setsox_inputs
    sx = make_setsox_inputs(WORKLOAD, ncol=ncol, seed=20261203 + 5)
    sx_met = [torch.from_numpy(sx[k]).to(dev) for k in ("press", "temp", "lwc", "cldfrc",
                                                      "cldnum", "xhnm")]
    sx_qin = torch.from_numpy(sx["qin"]).to(dev)
    sx_qcw = torch.from_numpy(sx["qcw"]).to(dev)
    sx_d = torch.empty((6, n), dtype=torch.float64, device=dev)

    def setsox():
        # repeated calls keep reacting the same cells' state (fine for timing)
        ctx.setsox(*[m.data_ptr() for m in sx_met], sx_qin.data_ptr(), sx_qcw.data_ptr(), n,
                   sx_d[0].data_ptr(), sx_d[3].data_ptr(), ncol, NLEV, d["dt"],
                   stream=stream.cuda_stream)

    from mam4xx_b200.workloads import make_gas_chemistry_inputs
    gc = make_gas_chemistry_inputs(WORKLOAD, ncol=ncol, seed=20261203 + 9)
    gc_dev = {k: torch.from_numpy(np.ascontiguousarray(gc[k])).to(dev)
              for k in ("temp", "photo", "extfrc", "inv", "het", "qq")}

    def gas_chemistry():
        # repeated calls keep reacting the same cells' state (fine for timing)
        ctx.gas_chemistry(*[gc_dev[k].data_ptr() for k in ("temp", "photo", "extfrc", "inv",
                                                            "het", "qq")],
                          n, ncol, NLEV, gc["dt"], stream=stream.cuda_stream)

    from mam4xx_b200.workloads import make_chem_step_inputs
    cw = make_chem_step_inputs(WORKLOAD, ncol=ncol, seed=20261203 + 10)
    cw_x = torch.from_numpy(cw["in_slab"]).to(dev)
    cw_pb = torch.from_numpy(cw["pblh"]).to(dev)
    cw_ch = torch.from_numpy(cw["chem_in"]).to(dev)
    cw_out = torch.empty((native.NOUT, n), dtype=torch.float64, device=dev)
    cw_cout = torch.empty((native.CHEM_NOUT, n), dtype=torch.float64, device=dev)

    def step_chem():
        ctx.step_chem_slab(cw_x.data_ptr(), cw_pb.data_ptr(), cw_ch.data_ptr(), cw_out.data_ptr(),
                           cw_cout.data_ptr(), n, ncol, NLEV, cw["dt"], stream=stream.cuda_stream)

    from mam4xx_b200.workloads import make_activation_inputs
    ac = make_activation_inputs(WORKLOAD, ncol=ncol, seed=20261203 + 6)
    ac_x = torch.from_numpy(ac["in_slab"]).to(dev)
    ac_rho = torch.from_numpy(ac["rho"]).to(dev)
    ac_w = torch.from_numpy(ac["w"]).to(dev)
    ac_out = torch.empty((17, n), dtype=torch.float64, device=dev)

    def activation():
        ctx.activate(ac_x.data_ptr(), n, ac_rho.data_ptr(), ac_w.data_ptr(), ac_out.data_ptr(),
                     ncol, NLEV, stream=stream.cuda_stream)

    from mam4xx_b200.workloads import make_optics_lw_tables, make_workload
    ow = make_workload(WORKLOAD, ncol=ncol, seed=20261203 + 7)
    ox = torch.from_numpy(ow["in_slab"]).to(dev)
    opd = torch.from_numpy(np.random.default_rng(8).uniform(100.0, 3000.0, n)).to(dev)
    otau = torch.empty((16, n), dtype=torch.float64, device=dev)
    otables = make_optics_lw_tables(seed=1)
    ctx.optics_lw_set_tables(otables)

    def optics_lw():
        ctx.optics_lw(ox.data_ptr(), n, opd.data_ptr(), otau.data_ptr(), ncol, NLEV, d["dt"],
                      stream=stream.cuda_stream)

    from mam4xx_b200.workloads import make_optics_sw_tables
    sw_tables = make_optics_sw_tables(seed=2)
    ctx.optics_sw_set_tables(sw_tables)
    sw_out = torch.empty((4, 14, n), dtype=torch.float64, device=dev)
    sw_aod = torch.empty((ncol,), dtype=torch.float64, device=dev)

    def optics_sw():
        ctx.optics_sw(ox.data_ptr(), n, opd.data_ptr(), sw_out.data_ptr(), sw_aod.data_ptr(),
                      ncol, NLEV, d["dt"], stream=stream.cuda_stream)

    from mam4xx_b200.workloads import make_rad_props_inputs
    rw = make_rad_props_inputs(WORKLOAD, ncol=ncol, seed=20261203 + 11)
    rd = {k: torch.from_numpy(np.ascontiguousarray(rw[k])).to(dev)
          for k in ("in_slab", "pdeldry", "pint", "zi", "ext_sw", "ssa_sw", "af_sw", "ext_lw")}

    def rad_sw():
        ctx.aero_rad_props_sw(rd["in_slab"].data_ptr(), n, rd["pdeldry"].data_ptr(),
                              rd["pint"].data_ptr(), rd["zi"].data_ptr(), rd["ext_sw"].data_ptr(),
                              rd["ssa_sw"].data_ptr(), rd["af_sw"].data_ptr(), sw_out.data_ptr(),
                              sw_aod.data_ptr(), 0, ncol, NLEV, d["dt"], stream=stream.cuda_stream)

    def rad_lw():
        ctx.aero_rad_props_lw(rd["in_slab"].data_ptr(), n, rd["pdeldry"].data_ptr(),
                              rd["pint"].data_ptr(), rd["zi"].data_ptr(), rd["ext_lw"].data_ptr(),
                              otau.data_ptr(), 0, ncol, NLEV, d["dt"], stream=stream.cuda_stream)

    from mam4xx_b200.workloads import make_dropmix_inputs
    dw = make_dropmix_inputs(WORKLOAD, ncol=ncol, seed=20261203 + 12)
    dd = {k: torch.from_numpy(np.ascontiguousarray(dw[k])).to(dev)
          for k in ("in_slab", "mix", "pint", "kvh")}
    d_out = torch.empty((66, n), dtype=torch.float64, device=dev)

    def dropmix():
        ctx.dropmixnuc(dd["in_slab"].data_ptr(), n, dd["mix"].data_ptr(), dd["pint"].data_ptr(),
                       dd["kvh"].data_ptr(), d_out.data_ptr(), ncol, NLEV, 6, dw["dt"],
                       stream=stream.cuda_stream)

    res = {}
    for name, f in (("calcsize", calcsize), ("coagulation", coag), ("setsox", setsox),
                    ("gas_chemistry", gas_chemistry), ("step_chem", step_chem),
                    ("activation", activation),
                    ("optics_lw", optics_lw), ("optics_sw", optics_sw),
                    ("aero_rad_props_sw", rad_sw), ("aero_rad_props_lw", rad_lw),
                    ("dropmixnuc", dropmix)):
        for _ in range(args.warmup):
            f()
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        k = max(3, args.steps)
        e0.record(stream)
        for _ in range(k):
            f()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / k
        if ws > 1:
            tt = torch.tensor([ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        gbs = PROCESS_BYTES_PER_CELL[name] * n / (ms * 1e-3) / 1e9
        res[name] = {"value": ws * n / (ms * 1e-3), "unit": "cells/s", "ms_per_call": ms,
                     "cells_per_gpu": n,
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm_peak,
                                  "unit": "GB/s", "frac": gbs / hbm_peak,
                                  "algorithmic_bytes_per_cell": PROCESS_BYTES_PER_CELL[name]}}
    # (the timed calls above keep adding to the same tendencies and, for
    # coagulation, keep coagulating the same state: fine for timing)
    if not args.no_cpu_baseline and int(os.environ.get("RANK", "0")) == 0:
        try:
            from oracle.pyoracle import ReferenceOracle
            r = ReferenceOracle()  # the process classes exist in the parity build
            nc = min(ncol, 256)
            m = nc * NLEV
            sl = slice(0, m)
            r.calcsize_process(nc, NLEV, d["prog"][:, sl], d["tend0"][:, sl], d["dt"])
            t0 = time.perf_counter()
            r.calcsize_process(nc, NLEV, d["prog"][:, sl], d["tend0"][:, sl], d["dt"])
            t1 = time.perf_counter()
            r.coag_process(nc, NLEV, d["temp"][sl], d["pmid"][sl], d["wet"][:, sl],
                           d["prog_aero"][:, sl], d["tend0"][:, sl], d["dt"])
            t2 = time.perf_counter()
            r.setsox(d["dt"], *[sx[k][sl] for k in ("press", "temp", "lwc", "cldfrc", "cldnum",
                                                    "xhnm")], sx["qin"][:, sl], sx["qcw"][:, sl])
            t3 = time.perf_counter()
            r.activate(ac["in_slab"][:, sl], ac["rho"][sl], ac["w"][sl])
            t4 = time.perf_counter()
            r.optics_lw(ow["in_slab"][:, sl], opd.cpu().numpy()[sl], d["dt"], otables)
            t5 = time.perf_counter()
            r.optics_sw(nc, NLEV, ow["in_slab"][:, sl], opd.cpu().numpy()[sl], d["dt"], sw_tables)
            t6 = time.perf_counter()
            r.gas_chemistry(gc["dt"], *[gc[k][..., sl] for k in ("temp", "photo", "extfrc", "inv",
                                                                  "het", "qq")])
            t7 = time.perf_counter()
            from mam4xx_b200.workloads import pblh_per_cell
            r.step_chem(cw["in_slab"][:, sl], pblh_per_cell(cw)[sl], cw["chem_in"][:, sl], cw["dt"])
            t8 = time.perf_counter()
            r.dropmixnuc(nc, NLEV, 6, True, dw["dt"], dw["in_slab"][:, sl], dw["mix"][:, sl],
                         dw["pint"][:nc * (NLEV + 1)], dw["kvh"][:nc * (NLEV + 1)])
            t9 = time.perf_counter()
            import multiprocessing
            for name, el in (("calcsize", t1 - t0), ("coagulation", t2 - t1),
                             ("setsox", t3 - t2), ("activation", t4 - t3),
                             ("optics_lw", t5 - t4), ("optics_sw", t6 - t5),
                             ("gas_chemistry", t7 - t6), ("step_chem", t8 - t7),
                             ("dropmixnuc", t9 - t8)):
                res[name]["cpu_baseline"] = {
                    "value": m / el, "unit": "cells/s", "kind": "reference",
                    "cores": multiprocessing.cpu_count(),
                    "sample": "%d columns x %d levels, the reference's process class "
                              "(OpenMP over columns)" % (nc, NLEV)}
        except Exception as e:  # reported, never silently replaced
            res["cpu_baseline_error"] = str(e)
    ctx.close()
    return res


def tracers_leg(native, torch, dev, stream, args, ws, x, pb, ncol, dt, step_ms):
    """The step through mam4b_step_tracers on TracersView-layout arrays
    (state_q tracer order, 40 tracers, tracer stride = cells) built from
    the forward workload's inputs: same kernels, read and written in place."""
    n = x.shape[1]
    q = torch.zeros((40, n), dtype=torch.float64, device=dev)
    qc = torch.zeros((40, n), dtype=torch.float64, device=dev)
    q[0] = x[3]
    q[11] = x[5]
    q[14] = x[6]
    q[15:40] = x[7:32]
    qc[15:40] = x[32:57]
    pt_q = torch.zeros_like(q)
    pt_c = torch.zeros_like(q)
    mode = torch.empty((16, n), dtype=torch.float64, device=dev)
    ctx = native.Context()

    def f():
        ctx.step_tracers(q.data_ptr(), qc.data_ptr(), n, x[0].data_ptr(), x[1].data_ptr(),
                         x[2].data_ptr(), x[4].data_ptr(), pb.data_ptr(), pt_q.data_ptr(),
                         pt_c.data_ptr(), mode.data_ptr(), n, ncol, NLEV, dt,
                         stream=stream.cuda_stream)

    for _ in range(args.warmup):
        f()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    k = max(2, min(args.steps, 5))
    e0.record(stream)
    for _ in range(k):
        f()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / k
    if ws > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    ctx.close()
    return {"value": ws * n / (ms * 1e-3), "unit": "cells/s", "ms_per_step": ms,
            "vs_step_slab": step_ms / ms,
            "layout": "mam4::TracersView (tracer, column, level), E3SM state_q order"}


def adjoint_leg(native, torch, dev, stream, args, ws):
    """Adjoint configuration: 16,384 columns x 72 levels (c5). Forward and
    adjoint (mam4b_adjoint_slab) timed with CUDA events on the same inputs;
    the cotangent is that of accumulation-mode number and SO4 mass after the
    step (both phases), column-integrated with weights pdel/g. A central
    finite-difference check (relative step 1e-6) of that gradient on 64
    cells reports the agreement in units of relative sensitivity."""
    from mam4xx_b200.workloads import make_workload
    wa = make_workload("c5", ncol=args.adjoint_ncol,
                       seed=20261203 + 4 + 1000 * int(os.environ.get("RANK", "0")))
    xa = torch.from_numpy(wa["in_slab"]).to(dev)
    pba = torch.from_numpy(wa["pblh"]).to(dev)
    na = xa.shape[1]
    p = wa["in_slab"][1].reshape(wa["ncol"], wa["nlev"])
    edges = np.concatenate([p[:, :1] * 0.5, 0.5 * (p[:, 1:] + p[:, :-1]), p[:, -1:] * 1.01], axis=1)
    wts = (np.abs(np.diff(edges, axis=1)) / 9.80616).reshape(-1)
    jstate = [2 + 7, 2 + 0, 27 + 7, 27 + 0]
    ybar_h = np.zeros((native.NOUT, na))
    for k in jstate:
        ybar_h[k] = wts * wa["dt"]
    ybar = torch.from_numpy(ybar_h).to(dev)
    outa = torch.empty((native.NOUT, na), dtype=torch.float64, device=dev)
    xbar = torch.empty((native.NIN, na), dtype=torch.float64, device=dev)
    actx = native.Context()

    def fwd():
        actx.step_slab(xa.data_ptr(), pba.data_ptr(), outa.data_ptr(), na, wa["ncol"], wa["nlev"],
                       wa["dt"], stream=stream.cuda_stream)

    def adj():
        actx.adjoint_slab(xa.data_ptr(), pba.data_ptr(), ybar.data_ptr(), xbar.data_ptr(), na,
                          wa["ncol"], wa["nlev"], wa["dt"], stream=stream.cuda_stream)

    def adj_ck4():
        actx.set_adjoint_checkpoint(4)
        adj()

    xbar_mx = torch.empty_like(xbar)

    def fwd_mixed():
        actx.step_slab(xa.data_ptr(), pba.data_ptr(), outa.data_ptr(), na, wa["ncol"], wa["nlev"],
                       wa["dt"], precision=native.MIXED, stream=stream.cuda_stream)

    def adj_mixed():
        actx.adjoint_slab(xa.data_ptr(), pba.data_ptr(), ybar.data_ptr(), xbar_mx.data_ptr(), na,
                          wa["ncol"], wa["nlev"], wa["dt"], stream=stream.cuda_stream,
                          precision=native.MIXED)

    times = {}
    ka = max(5, min(args.steps, 10))
    for name, f in (("forward", fwd), ("forward_mixed", fwd_mixed), ("adjoint_mixed", adj_mixed),
                    ("adjoint_ck4", adj_ck4), ("adjoint", adj)):
        actx.set_adjoint_checkpoint(1)
        for _ in range(args.warmup):
            f()
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ka):
            f()
        e1.record(stream)
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1) / ka
    # the mixed-precision adjoint's gradient against the FP64 one, per
    # entry in units of relative sensitivity |g_mixed - g| |x| / |J_cell|
    fwd()
    torch.cuda.synchronize()
    jcell = torch.from_numpy(wts).to(dev) * sum(xa[5 + k] + outa[k] * wa["dt"] for k in jstate)
    gfull = xbar.clone()
    gmix = xbar_mx.clone()
    for k in jstate:
        gfull[5 + k] += torch.from_numpy(wts).to(dev)
        gmix[5 + k] += torch.from_numpy(wts).to(dev)
    rows = [0, 3, 5, 6] + list(range(7, 57))
    emx = ((gmix[rows] - gfull[rows]).abs() * xa[rows].abs() / jcell.abs().clamp(min=1e-300))
    # cells whose mixed forward step itself departs from the FP64 one by
    # more than 1e-5 (a different sub-step count or branch): the gradients
    # there are of different branches
    from mam4xx_b200.precision import cell_errors_device
    out64 = outa.clone()
    fwd_mixed()
    torch.cuda.synchronize()
    fwd_err = cell_errors_device(outa, out64, xa, wa["dt"])
    bad_entry = emx > 1e-5
    bad_cells = bad_entry.any(dim=0)
    departs = fwd_err > 1e-5
    branch = {"cells_with_entries_above_1e-5": int(bad_cells.sum()),
              "of_which_forward_departs": int((bad_cells & departs).sum()),
              "cells_where_forward_departs": int(departs.sum()),
              "entries_above_1e-5_in_cells_where_forward_departs":
                  float(bad_entry[:, departs].sum()) / max(1.0, float(bad_entry.sum()))}
    del out64, fwd_err
    emx = emx.flatten()
    samp = emx[torch.randperm(emx.numel(), generator=torch.Generator().manual_seed(7))[:1 << 20]
               .to(dev)]
    qs = torch.quantile(samp, torch.tensor([0.999, 0.9999], dtype=samp.dtype, device=dev))
    mixed_vs_fp64 = {"entries": int(emx.numel()), "units": "|g_mixed - g_fp64| |x| / |J_cell|",
                     "median": float(samp.median()), "q999": float(qs[0]),
                     "q9999": float(qs[1]), "entries_above_1": int((emx > 1.0).sum()),
                     "max": float(emx.max()),
                     "within_1e-6": float((emx <= 1e-6).double().mean()),
                     "within_1e-5": float((emx <= 1e-5).double().mean()),
                     "branches": branch}
    del gfull, gmix, emx, samp
    # finite-difference check on 64 cells (first 8 columns x 8 levels)
    g = xbar.cpu().numpy()
    x_h = wa["in_slab"]
    fwd()
    torch.cuda.synchronize()
    out_h = outa.cpu().numpy()
    # 64 cells: 8 levels spread through each of the first 8 columns
    sub = np.concatenate([c * wa["nlev"] + np.arange(0, wa["nlev"], wa["nlev"] // 8)[:8]
                          for c in range(8)])
    ncs = 8
    xs = x_h[:, :ncs * wa["nlev"]]
    j0 = wts[:ncs * wa["nlev"]] * sum(xs[5 + k] + out_h[k, :ncs * wa["nlev"]] * wa["dt"] for k in jstate)
    gs = g[:, :ncs * wa["nlev"]].copy()
    for k in jstate:
        gs[5 + k] += wts[:ncs * wa["nlev"]]
    tx = torch.empty((native.NIN, ncs * wa["nlev"]), dtype=torch.float64, device=dev)
    to = torch.empty((native.NOUT, ncs * wa["nlev"]), dtype=torch.float64, device=dev)
    tp = pba[:ncs].contiguous()
    fctx = native.Context()

    def jcells(xv):
        tx.copy_(torch.from_numpy(xv))
        fctx.step_slab(tx.data_ptr(), tp.data_ptr(), to.data_ptr(), xv.shape[1], ncs, wa["nlev"],
                       wa["dt"], stream=stream.cuda_stream)
        torch.cuda.synchronize()
        o = to.cpu().numpy()
        return wts[:ncs * wa["nlev"]] * sum(xv[5 + k] + o[k] * wa["dt"] for k in jstate)

    errs = []
    for f in [0, 3, 5, 6] + list(range(7, 57)):
        h = 1e-6 * np.abs(xs[f])
        xp = xs.copy()
        xm = xs.copy()
        xp[f] += h
        xm[f] -= h
        fd = (jcells(xp) - jcells(xm)) / np.where(h > 0, 2 * h, 1.0)
        for c in sub:
            if xs[f, c] != 0.0:
                errs.append(abs(gs[f, c] - fd[c]) * abs(xs[f, c]) / abs(j0[c]))
    errs = np.array(errs)
    fctx.close()
    actx.close()
    return {"workload": "c5: 16384 columns x 72 levels, FP64, dt=1800 s",
            "objective": "accumulation-mode number + SO4 (interstitial + cloud-borne) after the step, "
                         "weights pdel/g; gradient w.r.t. T, qv, H2SO4, SOAG, 50 populations",
            "forward_ms": times["forward"], "adjoint_ms": times["adjoint"],
            "adjoint_over_forward": times["adjoint"] / times["forward"],
            "adjoint_ck4_ms": times["adjoint_ck4"],
            "mixed": {"forward_ms": times["forward_mixed"], "adjoint_ms": times["adjoint_mixed"],
                      "adjoint_over_forward": times["adjoint_mixed"] / times["forward_mixed"],
                      "adjoint_vs_fp64_adjoint": times["adjoint_mixed"] / times["adjoint"],
                      "gradient_vs_fp64": mixed_vs_fp64},
            "adjoint_ck4_over_forward": times["adjoint_ck4"] / times["forward"],
            "soa_states": "stored before every sub-step (adjoint_ms; 3.64 GB on 148 SMs) or a "
                          "checkpoint every 4 sub-steps with the others recomputed "
                          "(adjoint_ck4_ms; 0.93 GB); same gradient",
            "fd_check": {"cells": 64, "entries": int(errs.size), "rel_step": 1e-6,
                         "units": "|g - fd| |x| / |J_cell|",
                         "median": float(np.median(errs)), "max": float(errs.max()),
                         "within_1e-6": float((errs <= 1e-6).mean())}}


def run_reference_arm(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from mam4xx_b200.workloads import make_workload, pblh_per_cell
    from oracle import pyoracle
    orc, kind, flags = pyoracle.baseline_oracle()
    cores = os.cpu_count() or 1
    # a bounded sample per step: 1024 columns x 72 levels of the same workload
    w = make_workload(WORKLOAD, ncol=REF_SAMPLE_NCOL)
    x, pb, dt = w["in_slab"], pblh_per_cell(w), w["dt"]
    n = x.shape[1]
    for _ in range(args.warmup):
        orc.step(x, pb, dt, nthreads=cores)
    t = time.perf_counter()
    for _ in range(args.steps):
        orc.step(x, pb, dt, nthreads=cores)
    el = time.perf_counter() - t
    v = n * args.steps / el
    line = {"metric": METRIC, "value": v, "unit": "cells/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": _workload_name(NCOL_PER_GPU),
                       "sample_per_step": "first %d columns x %d levels" % (REF_SAMPLE_NCOL, NLEV),
                       "ncol": REF_SAMPLE_NCOL, "nlev": NLEV, "dt_s": dt},
            "cpu_baseline": {"value": v, "unit": "cells/s", "cores": cores, "kind": kind,
                             "sample": "%d columns x 72 levels of %s per step, OpenMP over cells; %s"
                                       % (REF_SAMPLE_NCOL, WORKLOAD, flags)},
            "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _workload_name(ncol):
    what = {"c4": "uneven batching (SOA sub-steps 1..20 per cell)",
            "c4_stress": "uneven batching stress case (SOA sub-steps 1..1000 per cell)"}
    return ("%s: %s, %d columns x %d levels per GPU, FP64, dt=1800 s"
            % (WORKLOAD, what.get(WORKLOAD, "workload configuration"), ncol, NLEV))


def _r(v, digits=4):
    """Rounds floats (recursively) to `digits` significant digits so the
    JSON line stays short."""
    if isinstance(v, float):
        return float("%.*g" % (digits, v)) if np.isfinite(v) else v
    if isinstance(v, dict):
        return {k: _r(x, digits) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [_r(x, digits) for x in v]
    return v


def mixed_leg(native, torch, dev, stream, args, ws, rank):
    """Mixed precision on its configuration c3 (65,536 x 72, 30 % of cells
    near the renaming cut-off): the FP64 step and both mixed forms timed on
    the same resident inputs; every cell's error against this run's FP64
    result (mam4xx_b200.precision.error_report_device)."""
    from mam4xx_b200.distributed import EventClock, max_over_ranks, timed_steps
    from mam4xx_b200.precision import cell_errors_device, conditioning_split, error_report_device
    from mam4xx_b200.workloads import make_workload
    wm = make_workload("c3", ncol=args.ncol, seed=20261203 + 2 + 1000 * rank)
    xm = torch.from_numpy(wm["in_slab"]).to(dev)
    pbm = torch.from_numpy(wm["pblh"]).to(dev)
    nm = xm.shape[1]
    ref = torch.empty((native.NOUT, nm), dtype=torch.float64, device=dev)
    got = torch.empty_like(ref)
    ctx = native.Context()
    res = {"workload": "c3: %d columns x %d levels, 30%% of cells near the renaming cut-off"
                       % (wm["ncol"], NLEV)}
    times = {}
    for name, prec, o in (("fp64", native.FP64, ref), ("mixed", native.MIXED, got),
                          ("mixed_fast", native.MIXED_FAST, got)):
        def f(prec=prec, o=o):
            ctx.step_slab(xm.data_ptr(), pbm.data_ptr(), o.data_ptr(), nm, wm["ncol"], NLEV,
                          wm["dt"], precision=prec, stream=stream.cuda_stream)
        ms, _, _ = timed_steps(f, args.steps, args.warmup, EventClock(stream),
                               sync=torch.cuda.synchronize, device=dev)
        times[name] = ms / args.steps
        if name == "fp64":
            res["fp64"] = {"value": ws * nm / (times[name] * 1e-3), "ms_per_step": times[name]}
            continue
        r = error_report_device(got, ref, xm, wm["dt"], tol=1e-5)
        if name == "mixed":
            # the FP64 step's own sensitivity: its results for inputs moved
            # by one ulp and by 1e-7 (the size of FP32 rounding), against
            # its results for the unperturbed inputs
            pert = {}
            for lab, eps in (("1ulp", 2.0 ** -52), ("1e-7", 1e-7)):
                xq = xm * (1.0 + eps)
                ctx.step_slab(xq.data_ptr(), pbm.data_ptr(), got.data_ptr(), nm, wm["ncol"], NLEV,
                              wm["dt"], precision=native.FP64, stream=stream.cuda_stream)
                torch.cuda.synchronize()
                rq = error_report_device(got, ref, xm, wm["dt"], tol=1e-5)
                pert[lab] = {"cells_within_1e-5": rq["cells_within_tol"], "max": rq["max"],
                             "cell_err_quantiles": rq["cell_err_quantiles"]}
                del xq
            # per cell: the FP64 step for its inputs rounded to single
            # precision against the FP64 step for the exact inputs
            xq = xm.float().double()
            ctx.step_slab(xq.data_ptr(), pbm.data_ptr(), got.data_ptr(), nm, wm["ncol"], NLEV,
                          wm["dt"], precision=native.FP64, stream=stream.cuda_stream)
            torch.cuda.synchronize()
            del xq
            cond = cell_errors_device(got, ref, xm, wm["dt"])
            rq = error_report_device(got, ref, xm, wm["dt"], tol=1e-5)
            pert["fp32_rounded_inputs"] = {"cells_within_1e-5": rq["cells_within_tol"],
                                           "max": rq["max"],
                                           "cell_err_quantiles": rq["cell_err_quantiles"]}
            res["fp64_input_perturbation"] = pert
            f()  # the mixed results again, for the report below
            torch.cuda.synchronize()
        split = conditioning_split(cell_errors_device(got, ref, xm, wm["dt"]), cond, tol=1e-5)
        worst = sorted(range(native.NOUT), key=lambda k: -r["per_output_max"][k])[:6]
        res[name] = {"value": ws * nm / (times[name] * 1e-3), "unit": "cells/s",
                     "ms_per_step": times[name],
                     "speedup_vs_fp64": max_over_ranks(times["fp64"] / times[name], dev),
                     "err_vs_fp64": {"cells": r["cells"], "max": r["max"], "median": r["median"],
                                     "cells_within_1e-5": r["cells_within_tol"],
                                     "cells_outside_1e-5": r["cells_outside_tol"],
                                     "cell_err_quantiles": r["cell_err_quantiles"],
                                     "conditioning": split,
                                     "worst_outputs": {str(k): r["per_output_max"][k] for k in worst},
                                     "per_output_max": r["per_output_max"],
                                     "per_output_median": r["per_output_median"]}}
    # the uneven-batching configuration c4 in FP64 and MIXED (speed and
    # error; the full reports above are on c3)
    del xm, pbm, ref, got
    w4 = make_workload("c4", ncol=args.ncol, seed=20261203 + 1000 * rank)
    x4 = torch.from_numpy(w4["in_slab"]).to(dev)
    pb4 = torch.from_numpy(w4["pblh"]).to(dev)
    n4 = x4.shape[1]
    r64 = torch.empty((native.NOUT, n4), dtype=torch.float64, device=dev)
    rmx = torch.empty_like(r64)
    t4 = {}
    for name, prec, o in (("fp64", native.FP64, r64), ("mixed", native.MIXED, rmx)):
        def f4(prec=prec, o=o):
            ctx4.step_slab(x4.data_ptr(), pb4.data_ptr(), o.data_ptr(), n4, w4["ncol"], NLEV,
                           w4["dt"], precision=prec, stream=stream.cuda_stream)
        ctx4 = ctx
        ms, _, _ = timed_steps(f4, args.steps, args.warmup, EventClock(stream),
                               sync=torch.cuda.synchronize, device=dev)
        t4[name] = ms / args.steps
    r4 = error_report_device(rmx, r64, x4, w4["dt"], tol=1e-5)
    res["c4"] = {"workload": "c4: %d columns x %d levels (uneven batching)" % (w4["ncol"], NLEV),
                 "fp64_ms_per_step": t4["fp64"], "mixed_ms_per_step": t4["mixed"],
                 "mixed_speedup_vs_fp64": max_over_ranks(t4["fp64"] / t4["mixed"], dev),
                 "mixed_err_vs_fp64": {"cells_within_1e-5": r4["cells_within_tol"],
                                       "median": r4["median"], "max": r4["max"],
                                       "cell_err_quantiles": r4["cell_err_quantiles"]}}
    ctx.close()
    return res


def main():
    global WORKLOAD
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=25)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ncol", type=int, default=NCOL_PER_GPU, help="columns per GPU")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision legs")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint leg")
    ap.add_argument("--no-processes", action="store_true",
                    help="skip the per-process entries (CalcSize, Coagulation) leg")
    ap.add_argument("--workload", default=WORKLOAD,
                    help="workload configuration of the headline step (c4 is the benchmark "
                         "configuration; c4_stress has 1..1000 SOA sub-steps per cell)")
    ap.add_argument("--adjoint-ncol", type=int, default=16384,
                    help="columns of the adjoint leg (16,384 is its configuration; smaller "
                         "only for profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    WORKLOAD = args.workload
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist
    from mam4xx_b200 import native
    from mam4xx_b200.distributed import EventClock, sharded_rate, timed_steps
    from mam4xx_b200.workloads import make_workload, pblh_per_cell

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    ncol = args.ncol
    # weak scaling: rank r owns its own ncol columns (seeded by rank), the
    # columns [r*ncol, (r+1)*ncol) of the whole job's batch
    w = make_workload(WORKLOAD, ncol=ncol, seed=20261203 + 3 + 1000 * rank)
    x_host = w["in_slab"]
    n = x_host.shape[1]
    dt = w["dt"]
    x = torch.from_numpy(x_host).to(dev)
    pb = torch.from_numpy(w["pblh"]).to(dev)
    out = torch.empty((native.NOUT, n), dtype=torch.float64, device=dev)
    # the context starts with the launch shape chosen by the autotuner for
    # this device (mam4xx_b200/mam4b_tuning.json, loaded by mam4b_create)
    # and replays the step as one CUDA graph
    ctx = native.Context()
    ctx.set_graph_mode(True)
    stream = torch.cuda.current_stream(dev)

    def step(precision=native.FP64):
        ctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, ncol, NLEV, dt,
                      precision=precision, stream=stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    flags = ctx.last_status()

    # device-resident timing: CUDA events on the launching stream, per step
    sampler = ClockSampler(local)

    def start_sampler():
        sampler.start()
        time.sleep(0.5)  # nvidia-smi's first sample lands inside the timed region

    launches0 = ctx.launch_count()
    ms_max, _, laps = timed_steps(step, args.steps, 0, EventClock(stream),
                                  sync=torch.cuda.synchronize, device=dev, on_start=start_sampler)
    clocks = sampler.stop()
    launches = ctx.launch_count() - launches0
    kernel_ms = float(np.mean(laps))
    ms_per_step = ms_max / args.steps
    value = sharded_rate(n, args.steps, ms_max, device=dev)

    # the same step with the built-in launch shape and plain launches
    tuned_shape = ctx.tuning().as_dict()
    tfile = os.path.join(ROOT, "mam4xx_b200", "mam4b_tuning.json")
    dctx = native.Context()
    dctx.set_tuning(native.default_tuning())

    def default_step():
        dctx.step_slab(x.data_ptr(), pb.data_ptr(), out.data_ptr(), n, ncol, NLEV, dt,
                       stream=stream.cuda_stream)
    d_ms, _, _ = timed_steps(default_step, args.steps, args.warmup, EventClock(stream),
                             sync=torch.cuda.synchronize, device=dev)
    dctx.close()
    tuning = {"shape": tuned_shape,
              "source": ("mam4xx_b200/mam4b_tuning.json" if tuned_shape
                         != native.default_tuning().as_dict() else "built-in defaults"),
              "file_present": os.path.exists(tfile),
              "graph": True,
              "tuned_graph_ms_per_step": ms_per_step,
              "default_plain_ms_per_step": d_ms / args.steps}

    # end-to-end through the host entry of the C ABI
    e2e = None
    if not args.no_e2e:
        xin = torch.from_numpy(x_host).pin_memory()
        pbh = torch.from_numpy(w["pblh"]).pin_memory()
        oh = torch.empty((native.NOUT, n), dtype=torch.float64).pin_memory()
        ectx = native.Context()

        def host_step():
            ectx.step_host(xin.data_ptr(), pbh.data_ptr(), oh.data_ptr(), n, ncol, NLEV, dt,
                           stream=stream.cuda_stream)
        ke = max(2, min(args.steps, 5))
        e_ms, _, _ = timed_steps(host_step, ke, 2, EventClock(stream),
                                 sync=torch.cuda.synchronize, device=dev)
        e2e = {"value": sharded_rate(n, ke, e_ms, device=dev), "unit": "cells/s",
               "h2d_bytes_per_step": int(native.NIN * n * 8 + ncol * 8),
               "d2h_bytes_per_step": int(native.NOUT * n * 8),
               "steps": ke, "entry": "mam4b_step_host (pinned host slabs)"}
        ectx.close()
        del xin, oh

    precisions = None
    if not args.no_mixed:
        precisions = mixed_leg(native, torch, dev, stream, args, ws, rank)

    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_leg(native, torch, dev, stream, args, ws)

    peak, peak_kind = _peaks()
    processes = None
    if not args.no_processes:
        processes = processes_leg(native, torch, dev, stream, args, ws, peak)
        processes["tracers"] = tracers_leg(native, torch, dev, stream, args, ws, x, pb, ncol,
                                           dt, ms_per_step)
    fpeaks = _fp_peaks()
    flops_cell, special_cell = _flops_per_cell(WORKLOAD)
    roof64 = None
    if flops_cell is not None:
        g = flops_cell * n / (kernel_ms * 1e-3) / 1e9
        roof64 = {"bound": "fp64", "achieved": g, "peak": fpeaks["fp64"], "unit": "GFLOP/s",
                  "frac": g / fpeaks["fp64"],
                  "flops_per_cell": flops_cell, "libm_calls_per_cell": special_cell,
                  "peak_source": "measured now: FP64 FMA chains (libmam4b_peaks.so)",
                  "fp32_peak": fpeaks["fp32"],
                  "flops_source": "baseline/flops_per_cell.json (operation-counting build of "
                                  "the CPU restatement; + - * / one flop each, libm calls apart)"}
    alg_bytes = n * BYTES_PER_CELL + ncol * 8
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    traffic = _traffic_per_launch(WORKLOAD, n)
    # the other legs' key figures, first in the line (the full reports go last)
    legs = {}
    if precisions:
        for k in ("mixed", "mixed_fast"):
            if k in precisions:
                e = precisions[k]["err_vs_fp64"]
                legs[k] = {"speedup_vs_fp64": round(precisions[k]["speedup_vs_fp64"], 3),
                           "cells_within_1e-5": round(e["cells_within_1e-5"], 5),
                           "well_conditioned_within_1e-5":
                               round(e["conditioning"]["well_conditioned_within_tol"], 6)}
        if "c4" in precisions:
            legs["mixed_c4"] = {
                "speedup_vs_fp64": round(precisions["c4"]["mixed_speedup_vs_fp64"], 3),
                "cells_within_1e-5": round(precisions["c4"]["mixed_err_vs_fp64"]["cells_within_1e-5"], 5)}
    if adjoint:
        legs["adjoint"] = {k: round(adjoint[k], 3) for k in
                           ("adjoint_over_forward", "adjoint_ck4_over_forward") if k in adjoint}
        legs["adjoint"]["fd_within_1e-6"] = round(adjoint["fd_check"]["within_1e-6"], 5)
        if "mixed" in adjoint:
            legs["adjoint"]["mixed_over_fp64_adjoint"] = round(
                adjoint["mixed"]["adjoint_vs_fp64_adjoint"], 3)
            legs["adjoint"]["mixed_gradient_within_1e-5"] = round(
                adjoint["mixed"]["gradient_vs_fp64"]["within_1e-5"], 5)
    line = {
        "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "legs": legs, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded draws with the configuration's distributions)",
        "config": {"workload": _workload_name(ncol),
                   "ncol_per_gpu": ncol, "nlev": NLEV, "cells_per_gpu": n,
                   "parallelism": "column shards, one per GPU" if ws > 1 else "single GPU",
                   "l2": "inputs (%.2f GB) larger than L2, no flush" % (native.NIN * n * 8 / 1e9)},
        "gpu_launches": int(launches),
        "tuning": tuning,
        "clocks": clocks,
        "device_flags": flags,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": "%s copy bandwidth" % peak_kind,
                     "kernel_ms": kernel_ms, "algorithmic_bytes_per_launch": alg_bytes,
                     "unit_of_launch": "one step (the pipeline behind mam4b_step_slab)"},
        "roofline_fp64": roof64,
        "e2e": e2e,
    }
    if rank == 0 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(x_host, pblh_per_cell(w), dt)
        except Exception as e:  # reported, never silently replaced
            line["cpu_baseline"] = {"error": str(e)}
    # the long per-entry reports go last, rounded
    line["processes"] = _r(processes, 3)
    line["precisions"] = _r(precisions, 3)
    line["adjoint"] = _r(adjoint, 4)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
