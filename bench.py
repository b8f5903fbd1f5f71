#!/usr/bin/env python
"""Benchmark of the FP64 fluid advance (advection sweeps + TRBDF2 diffusion) on B200.

Workload: the dipole grid 384 x 192 x 192 x 7 species (L-shells 1.2-3.0, MLON span 10 deg,
seeded +-20 % lognormal perturbations), one step = dt_calc at CFL 0.5 followed by the fused
fluid advance (v12rhov1 ... T2rhoe without compression / sources).  Metric: cell-species
updates per second, lx1*lx2*lx3*7*steps / time / 1e9.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1 runs under torchrun, one replica per GPU (the path has no data exchange:
weak scaling); the time is the max over ranks.  --impl reference times the reference's
algorithm on the host CPU (the C++ restatement of the Fortran, all host threads).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(kind="dipole", lx1=384, lx2=192, lx3=192, Lmin=1.2, Lmax=3.0, mlon_span_deg=10.0,
                perturb=0.2, seed=1)
METRIC = "fluid Gcell-species-steps/s"
UNIT = "Gcell-species-steps/s"
LSP = 7
PHASES = ["dt_calc", "ghost_fill", "sweep_x3", "sweep_x1", "sweep_x2_epilogue", "ghost_epilogue", "diffusion"]


def algorithmic_doubles_per_cell(unit_metrics: bool) -> dict:
    """Algorithmic HBM traffic of each phase per interior cell, in 8-byte words: every input
    read once and every output written once.  A sweep moves the 19 advected fields in and out
    and reads 7 face velocities (45 words) plus 3 cell and 3 face metric factors; the x2 sweep
    also writes the derived v1 and n_e; the diffusion reads T and n of 7 species, three
    neutral densities and J1, writes T of 7 species (25 words) and reads h1, h2, h3.  The step
    sums to 162 words per cell, 183 with metric factors (1296 / 1464 bytes).  dt_calc is timed
    in the step but not part of that sum; its own count (T, v1, v2, v3 of 7 species and three
    metric factors) is kept for its phase fraction."""
    ms = 0 if unit_metrics else 6
    md = 0 if unit_metrics else 3
    return {
        "dt_calc": 28 + md,
        "ghost_fill": 0,
        "sweep_x3": 45 + ms,
        "sweep_x1": 45 + ms,
        "sweep_x2_epilogue": 45 + ms + 2,
        "ghost_epilogue": 0,
        "diffusion": 25 + md,
    }


STEP_PHASES = ("sweep_x3", "sweep_x1", "sweep_x2_epilogue", "diffusion")  # the 162 (183) words


def measured_traffic():
    """DRAM bytes per interior cell and launch of each phase's kernels, from an ncu capture
    (dram__bytes_read.sum + dram__bytes_write.sum), kept beside the profile summaries in
    profiles/dram_bytes_per_cell.json; None when absent."""
    p = os.path.join(ROOT, "profiles", "dram_bytes_per_cell.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:  # noqa: BLE001
        return None


def build_problem(lx1, lx2, lx3, seed, perturb, kind="dipole"):
    from gemini_b200 import grid as G
    from gemini_b200 import state as S
    if kind == "dipole":
        g = G.dipole_grid(lx1, lx2, lx3, Lmin=WORKLOAD["Lmin"], Lmax=WORKLOAD["Lmax"],
                          mlon_span_deg=WORKLOAD["mlon_span_deg"])
    else:
        g = G.cartesian_grid(lx1, lx2, lx3)
    st = S.init_state(g, seed=seed, perturb=perturb)
    return g, st


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, path: str | None = None):
        self.idx = gpu_index
        self.proc = None
        self.path = path or os.path.join(tempfile.gettempdir(), f"gemini_b200_clocks_{os.getpid()}_{gpu_index}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001 -- no nvidia-smi
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:  # noqa: BLE001
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


class CpuSample:
    """The oracle (C++ restatement of the reference Fortran) on the host cores (all threads
    unless `threads` is given), on an x3 slab of the workload grid sized so one step takes
    about `step_seconds`."""

    def __init__(self, lx1, lx2, lx3, step_seconds=4.0, threads=None):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O  # checker / CPU baseline only
        self.O = O
        self.threads = threads or os.cpu_count() or 1
        O.set_num_threads(self.threads)
        self.lx1, self.lx2, self.lx3 = lx1, lx2, lx3
        slab, el = 2, None
        while True:
            g, st = build_problem(lx1, lx2, slab, WORKLOAD["seed"], WORKLOAD["perturb"])
            el = self._one(g, st)
            if el * 1.5 > step_seconds or slab >= lx3:
                break
            slab = min(lx3, max(slab * 2, int(slab * step_seconds / max(el, 1e-3))))
        self.g, self.st, self.slab = g, st, slab

    def _one(self, g, st):
        self.O.set_num_threads(self.threads)
        t0 = time.perf_counter()
        dt, _ = self.O.dt_calc(g, st, 0.5)
        self.O.fluid_adv(g, st, dt)
        return time.perf_counter() - t0

    def step(self) -> float:
        """One timed oracle step; returns cell-species-steps/s."""
        el = self._one(self.g, self.st)
        return self.lx1 * self.lx2 * self.slab * LSP / el / 1e9

    def describe(self, nsteps, seconds):
        return (f"{nsteps} step(s) of dt_calc + fluid advance on a {self.lx1}x{self.lx2}x{self.slab} x3-slab "
                f"of the {self.lx1}x{self.lx2}x{self.lx3} dipole workload, {self.threads} OpenMP thread{'s' if self.threads > 1 else ''}, "
                f"{seconds:.1f} s")


def cpu_baseline(lx1, lx2, lx3, target_seconds=15.0):
    """All host threads, then one thread on a smaller slab (about a fifth of the time)."""
    cs = CpuSample(lx1, lx2, lx3, step_seconds=target_seconds / 4)
    t0 = time.perf_counter()
    vals = [cs.step() for _ in range(3)]
    el = time.perf_counter() - t0
    one = CpuSample(lx1, lx2, lx3, step_seconds=target_seconds / 20, threads=1)
    t0 = time.perf_counter()
    vals1 = [one.step() for _ in range(3)]
    el1 = time.perf_counter() - t0
    single = {"value": float(np.median(vals1)), "unit": UNIT, "cores": 1, "sample": one.describe(3, el1)}
    return float(np.median(vals)), cs.threads, cs.describe(3, el), single


def dist_setup(n):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def run_reference(args, world, rank):
    """--impl reference: the reference algorithm on the host CPU (rank 0 only).  Each step is
    one oracle step on a bounded x3-slab of the workload grid."""
    if rank != 0:
        return None
    w = WORKLOAD
    per_step = min(args.cpu_seconds / 3, 150.0 / max(args.steps + args.warmup, 1))
    cs = CpuSample(w["lx1"], w["lx2"], w["lx3"], step_seconds=per_step)
    for _ in range(args.warmup):
        cs.step()
    t0 = time.perf_counter()
    vals = [cs.step() for _ in range(args.steps)]
    el = time.perf_counter() - t0
    value = float(np.median(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * w["lx1"] * w["lx2"] * w["lx3"] * LSP / (value * 1e9),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cs.threads, "kind": "port",
                         "sample": cs.describe(args.steps, el)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def config_dict(world):
    w = WORKLOAD
    return {"workload": f"plain FP64 dipole {w['lx1']}x{w['lx2']}x{w['lx3']} x 7 species, "
                        "dt_calc (CFL 0.5) + fused fluid advance (advection sweeps x3,x1,x2 + TRBDF2 diffusion)",
            "lx1": w["lx1"], "lx2": w["lx2"], "lx3": w["lx3"], "species": LSP, "grid": "closed dipole",
            "L_shells": [w["Lmin"], w["Lmax"]], "mlon_span_deg": w["mlon_span_deg"], "perturb": w["perturb"],
            "diffsolvetype": 2, "tcfl": 0.5, "parallelism": f"replicas x{world}",
            "l2": "state ~7 GB per replica, larger than L2 (no flush between steps)"}


def run_b200(args, world, rank, local):
    import torch
    import torch.distributed as dist

    from gemini_b200 import _lib
    from gemini_b200 import fluid as F

    w = WORKLOAD
    g, st = build_problem(w["lx1"], w["lx2"], w["lx3"], w["seed"] + rank, w["perturb"])
    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st.copy())
    cfg = F.FluidCfg(st.Teinf, 2, 0.5)
    stream = torch.cuda.current_stream()
    L = _lib.lib()
    ccfg = cfg.c()
    import ctypes
    sptr = ctypes.c_void_p(stream.cuda_stream)
    gh = dg.handle
    Fp, Ap, Ep = (ctypes.c_void_p(t.data_ptr()) for t in (ds.fluidvars, ds.fluidauxvars, ds.electrovars))
    dtp = ctypes.c_void_p(ds.dt.data_ptr())

    def step():
        _lib.check(L.gem_dt_calc_dev(gh, 0.5, Fp, ds.work, dtp, sptr))
        _lib.check(L.gem_fluid_adv_dev(ctypes.byref(ccfg), gh, Fp, Ap, Ep, ds.work, dtp, sptr))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    _lib.check(L.gem_work_phase_timing(ds.work, args.steps))
    sampler = ClockSampler(local, args.clocks_csv.format(rank=rank) if args.clocks_csv else None)
    sampler.start()
    time.sleep(0.3)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        step()
    end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = start.elapsed_time(end)
    phase = np.zeros(8)
    nph, nst = ctypes.c_int(0), ctypes.c_int(0)
    _lib.check(L.gem_work_phase_times(ds.work, phase.ctypes.data_as(_lib._D), 8, ctypes.byref(nph),
                                      ctypes.byref(nst)))
    _lib.check(L.gem_work_phase_timing(ds.work, 0))
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    nonfinite = F.check_finite(ds)
    cells = w["lx1"] * w["lx2"] * w["lx3"]
    value = world * cells * LSP * args.steps / (ms_max / 1e3) / 1e9

    # roofline of the dominant phase (algorithmic bytes / mean duration)
    unit = g.unit_metrics
    alg = algorithmic_doubles_per_cell(unit)
    phase_ms = {PHASES[i]: float(phase[i]) for i in range(len(PHASES))}
    dom = max(STEP_PHASES, key=lambda p: phase_ms[p])
    alg_bytes = alg[dom] * 8 * cells
    achieved = alg_bytes / (phase_ms[dom] / 1e3) / 1e9
    peak, peak_src = measured_hbm_peak()
    step_bytes = sum(alg[p] for p in STEP_PHASES) * 8 * cells
    step_achieved = step_bytes / (ms_max / args.steps / 1e3) / 1e9
    tr = measured_traffic()
    traffic = None
    if tr and not unit and dom in tr.get("phases", {}):
        traffic = tr["phases"][dom] * cells
    phase_frac = {p: alg[p] * 8 * cells / (phase_ms[p] / 1e3) / 1e9 / peak for p in PHASES
                  if alg[p] > 0 and phase_ms[p] > 0}

    # end to end through the host-buffer entry point (state copied in and out each step)
    e2e = None
    if args.e2e_steps > 0:
        h = st.copy()
        pin = {}
        for name in ("fluidvars", "fluidauxvars", "electrovars"):
            a = getattr(h, name)
            tpin = torch.from_numpy(a.ravel(order="K")).pin_memory()
            pin[name] = tpin
        dtv = ctypes.c_double(-1.0)
        ptrs = [ctypes.c_void_p(pin[n].data_ptr()) for n in ("fluidvars", "fluidauxvars", "electrovars")]
        for _ in range(1):
            dtv.value = -1.0
            _lib.check(L.gem_fluid_adv_host(ctypes.byref(ccfg), gh, *ptrs, ds.work, ctypes.byref(dtv), sptr))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_start.record(stream)
        for _ in range(args.e2e_steps):
            dtv.value = -1.0
            _lib.check(L.gem_fluid_adv_host(ctypes.byref(ccfg), gh, *ptrs, ds.work, ctypes.byref(dtv), sptr))
        e_end.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        ems = e_start.elapsed_time(e_end)
        te = torch.tensor([ems], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        ems = float(te.item())
        ng = (w["lx1"] + 4) * (w["lx2"] + 4) * (w["lx3"] + 4)
        h2d = ng * 8 * (5 * LSP + 1)        # fluidvars + J1
        # ns, vs1, Ts + the ghost shell of vs2, vs3 (their interior is not written) + rhovs1|rhoes + dt
        s2, s3, nb = w["lx1"] + 4, (w["lx1"] + 4) * (w["lx2"] + 4), 2 * LSP
        shell = 8 * nb * (4 * s3 + 4 * s2 * (w["lx3"] + 4) + 4 * (w["lx2"] + 4) * (w["lx3"] + 4))
        d2h = ng * 8 * (3 * LSP) + shell + ng * 8 * (2 * LSP) + 8
        e2e = {"value": world * cells * LSP * args.e2e_steps / (ems / 1e3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "api": "gem_fluid_adv_host (host blocks, pinned)", "steps": args.e2e_steps,
               "wall_s": wall}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, threads, sample, single = cpu_baseline(w["lx1"], w["lx2"], w["lx3"], args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
               "single_thread": single}

    launches_per_step = 2 + 3 + 3 + 1 + (1 if g.lnull > 0 else 0) + 1
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(world),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_source": (tr or {}).get("source"),
                     "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "step_algorithmic_bytes": step_bytes,
                     "step_achieved_GBs": step_achieved, "step_frac": step_achieved / peak,
                     "phase_frac": phase_frac},
        "phases_ms": phase_ms,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        "gpu_launches": launches_per_step * args.steps,
        "nonfinite": nonfinite,
    }
    ds.close()
    dg.close()
    return line


def run_full_step(args):
    """fluid_adv in full (app/main.f90:280-381) on the workload grid: dt_calc, the step with
    compression (VNRicht_artvisc, RK2 boundary, compression), the diffusion, and the
    source/loss sub-step (rates and ETD solves of energy, momentum, mass), through
    gem_fluid_adv_full_dev.  The neutral atmosphere and ionization rates are seeded
    synthetic inputs (the reference computes them outside this path), made on the device."""
    import torch

    from gemini_b200 import fluid as F

    w = WORKLOAD
    g, st = build_problem(w["lx1"], w["lx2"], w["lx3"], w["seed"], w["perturb"])
    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st.copy())
    cfg = F.FluidCfg(st.Teinf, 2, 0.5)
    nc = g.lx1 * g.lx2 * g.lx3
    gen = torch.Generator(device="cuda").manual_seed(w["seed"])
    U = lambda lo, hi, *shape: torch.rand(*shape, dtype=torch.float64, device="cuda", generator=gen) * (hi - lo) + lo
    # an exponential neutral atmosphere above 80 km and an ionization layer near 150 km, +-10%
    alt = torch.from_numpy(np.ascontiguousarray(g.alt[2:-2, 2:-2, 2:-2].ravel(order="F"))).cuda()
    z = torch.clamp(alt, min=80e3)
    n100 = (4e17, 1e19, 2.6e18, 1e13, 1e14, 1e14)  # O, N2, O2, H, N, NO at 100 km [m^-3]
    scale = (60e3, 40e3, 40e3, 600e3, 60e3, 40e3)
    nn = torch.cat([n100[i] * torch.exp(-(z - 100e3) / scale[i]) * (1 + 0.1 * U(-1, 1, nc)) for i in range(6)])
    layer = torch.exp(-((z - 150e3) / 60e3) ** 2)
    inp = dict(nn=nn, vn1=U(-100, 100, nc), vn2=U(-100, 100, nc), vn3=U(-100, 100, nc),
               Tn=torch.from_numpy(np.ascontiguousarray(st.Tn.ravel(order="F"))).cuda(), alt=alt,
               g1=U(-9.8, -8.0, nc), Prionize=torch.cat([1e9 * layer * U(0.5, 1, nc) for _ in range(6)]),
               Qeionize=1e-13 * layer * U(0.5, 1, nc))
    inputs = F.SourceInputs.of(**inp)
    scratch = torch.empty(F._lib.lib().gem_fluid_adv_full_scratch_doubles(ds.g), dtype=torch.float64, device="cuda")

    def step():
        dt = F.dt_calc(ds, 0.5, out=ds.dt)
        F.fluid_adv_full(cfg, ds, dt, inputs, scratch)

    for _ in range(2):
        step()
    K = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(K):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    nonfinite = F.check_finite(ds)
    ds.close()
    dg.close()
    return {"workload": f"fluid_adv in full on the {g.lx1}x{g.lx2}x{g.lx3} dipole grid: dt_calc, advection, "
                        "compression, diffusion, "
                        "source/loss (seeded synthetic exponential neutral atmosphere and ionization layer)",
            "ms_per_step": ms, "value": nc * LSP / (ms / 1e3) / 1e9, "unit": UNIT, "steps": K,
            "nonfinite": nonfinite,
            "api": "gem_dt_calc_dev + gem_fluid_adv_full_dev"}


BATCHED = dict(instances=64, seed=2024, perturb=0.2)


def run_batched(args, world, rank):
    """The uneven-instance batch: instances sharded across ranks by cost, each rank's shard
    advanced by gem_batch_step (graph replay), timed over args.batch_steps steps; then the
    same instances as sequential plain solves (dt_calc + fluid_adv one after another)."""
    import torch
    import torch.distributed as dist

    from gemini_b200 import batch as BT
    from gemini_b200 import fluid as F
    from gemini_b200 import workloads as WL

    specs = WL.batched_specs(BATCHED["instances"], BATCHED["seed"])
    mine = WL.shard(specs, world, rank)
    insts = []
    for i in mine:
        g = WL.make_grid(specs[i])
        dg = F.DeviceGrid(g)
        ds = WL.device_state(dg, g, specs[i].seed, BATCHED["perturb"])
        insts.append((dg, ds, F.FluidCfg(ds.Teinf)))
    torch.cuda.synchronize()
    b = BT.Batch(insts)
    stream = torch.cuda.current_stream()
    from gemini_b200 import autotune as AT
    tuned = AT.tune(b, steps=2)

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ms_b = timed(b.step, args.batch_steps)

    def sequential():
        for dg, ds, cfg in insts:
            BT.plain_step(dg, ds, cfg)

    ms_s = timed(sequential, max(1, args.batch_steps // 2))
    seq_steps = max(1, args.batch_steps // 2)
    total_cells = sum(s.cells for s in specs)
    my_cells = sum(specs[i].cells for i in mine)
    cells_t = torch.tensor([float(my_cells)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(cells_t)
    launches, items = b.info()
    fin = [F.check_finite(ds) for _, ds, _ in insts]
    out = {
        "workload": f"{len(specs)} instances, lx1~U{{64..512}}, lx2,lx3~U{{16..128}}, Cartesian/dipole 50/50, "
                    f"seeded per instance, {total_cells} cells in total",
        "value": float(cells_t.item()) * LSP * args.batch_steps / (ms_b / 1e3) / 1e9,
        "unit": UNIT, "ms_per_step": ms_b / args.batch_steps, "steps": args.batch_steps,
        "sequential_plain_value": float(cells_t.item()) * LSP * seq_steps / (ms_s / 1e3) / 1e9,
        "sequential_plain_ms_per_step": ms_s / seq_steps,
        "launches_per_step": launches, "work_items_per_step": items,
        "graph": "one CUDA graph per step (replayed)", "instances_on_rank0": len(mine),
        "autotune": {"params": {("grid_pct" if k == 2 else "diff_blocks" if k == 1 else str(k)): v
                                for k, v in tuned["params"].items()},
                     "cached": tuned["cached"],
                     "trials_ms": [round(t["ms_per_step"], 3) for t in tuned["trials"]]},
        "sharding": "longest-processing-time over cells x species, no collective on the data path",
        "nonfinite_cells": int(sum(fin)),
    }
    b.close()
    for dg, ds, _ in insts:
        ds.close()
        dg.close()
    return out


# every step's state kept (20 states of this grid: 2 GB of HBM); the recompute variant keeps
# one state in checkpoint_every_recompute and recomputes the others in the backward
ADJOINT = dict(lx1=128, lx2=64, lx3=64, steps=20, checkpoint_every=1, checkpoint_every_recompute=5, seed=11)


def run_adjoint(args, checkpoint_every=None):
    """Adjoint workload: Cartesian 128x64x64 x 7 species, 20 steps, L2 misfit of the final Te
    and n_O+ against a seeded target; gradient w.r.t. the initial ion densities and the
    per-column top temperature.  Reports forward time, forward+backward time and the ratio
    (device time, CUDA events), and the same with checkpoint recomputation."""
    import torch

    from gemini_b200 import adjoint as AD
    from gemini_b200 import grid as G
    from gemini_b200 import state as S

    a = ADJOINT
    k = a["checkpoint_every"] if checkpoint_every is None else checkpoint_every
    g = G.cartesian_grid(a["lx1"], a["lx2"], a["lx3"])
    st = S.init_state(g, seed=a["seed"], perturb=0.1)
    P = AD.DiffProblem(g, st, a["steps"], checkpoint_every=k)
    I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
    n0 = P.base[(slice(0, 6),) + I].clone()
    rng = np.random.default_rng(a["seed"])
    Ttop = torch.from_numpy(st.Teinf * (1 + 0.05 * rng.uniform(-1, 1, (g.lx3, g.lx2)))).cuda()
    tT = torch.from_numpy(rng.uniform(1500, 3000, (g.lx3, g.lx2, g.lx1))).cuda()
    tn = torch.from_numpy(rng.uniform(0.5e10, 5e10, (g.lx3, g.lx2, g.lx1))).cuda()
    s = torch.cuda.current_stream()

    def fwd():
        (ns, _, Ts, _, _), _ = P.run(n0, Ttop)
        return AD.misfit(ns, Ts, tT, tn, g)

    def fwd_bwd():
        x = n0.clone().requires_grad_(True)
        t = Ttop.clone().requires_grad_(True)
        ns, Ts = AD.FluidAdvance.apply(x, t, P)
        L = AD.misfit(ns, Ts, tT, tn, g)
        L.backward()
        return x.grad, t.grad

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_f = timed(fwd, 3)
    ms_fb = timed(fwd_bwd, 2)
    out = {"workload": f"Cartesian {a['lx1']}x{a['lx2']}x{a['lx3']} x 7 species, {a['steps']} steps, "
                       f"checkpoint every {k}; loss = L2 misfit of final Te and n_O+",
           "forward_ms": ms_f, "forward_backward_ms": ms_fb, "adjoint_over_forward": (ms_fb - ms_f) / ms_f,
           "gradient_wrt": "initial ion densities (6 x cells) and per-column top temperature",
           "backward": "per step: gem_step_vjp_dev, the whole step's adjoint in CUDA (device replay of the "
                       "conversions, ghost fill and nine sweeps; hand-written VJPs of the sweeps, the TRBDF2 "
                       "diffusion, the floors/conversions, the ghost copies and the x1 boundary); the replay of "
                       "step j-1 runs on a side stream during step j's backward"}
    P.close()
    if checkpoint_every is None and a.get("checkpoint_every_recompute"):
        r = run_adjoint(args, a["checkpoint_every_recompute"])
        out["recompute"] = {kk: r[kk] for kk in ("workload", "forward_ms", "forward_backward_ms",
                                                  "adjoint_over_forward")}
    return out


BATCHED_ADJOINT = dict(instances=32, steps=200, checkpoint_every=10, group=8, seed=77)


def run_batched_adjoint(args):
    """Batched + adjoint workload: 32 uneven Cartesian instances (lx1 128-256, lx2, lx3
    32-128), 200 steps, checkpoint every 10; per-instance gradients of the L2 misfit of the
    final Te and n_O+ w.r.t. the initial ion densities and the per-column top temperature.
    Forward: one batched step per time step (graph replay, prescribed time steps)."""
    import torch

    from gemini_b200 import adjoint as AD
    from gemini_b200 import grid as G
    from gemini_b200 import state as S

    a = BATCHED_ADJOINT
    rng = np.random.default_rng(a["seed"])
    inst = []
    for i in range(a["instances"]):
        g = G.cartesian_grid(int(rng.integers(128, 257)), int(rng.integers(32, 129)), int(rng.integers(32, 129)))
        inst.append((g, S.init_state(g, seed=a["seed"] * 100 + i, perturb=0.1)))
    BA = AD.BatchedAdjoint(inst, a["steps"], checkpoint_every=a["checkpoint_every"], group=a["group"])
    controls, targets = [], []
    for (g, st), P in zip(inst, BA.problems):
        I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
        controls.append((P.base[(slice(0, 6),) + I].clone(),
                         torch.from_numpy(st.Teinf * (1 + 0.05 * rng.uniform(-1, 1, (g.lx3, g.lx2)))).cuda()))
        targets.append((torch.from_numpy(rng.uniform(1500, 3000, (g.lx3, g.lx2, g.lx1))).cuda(),
                        torch.from_numpy(rng.uniform(0.5e10, 5e10, (g.lx3, g.lx2, g.lx1))).cuda()))

    def loss(i, ns, Ts):
        return AD.misfit(ns, Ts, targets[i][0], targets[i][1], inst[i][0])

    s = torch.cuda.current_stream()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    e[0].record(s)
    for g0 in range(0, len(inst), a["group"]):
        idx = list(range(g0, min(g0 + a["group"], len(inst))))
        BA.forward_group(idx, [controls[i] for i in idx], keep=False)
    e[1].record(s)
    e[2].record(s)
    res = BA.gradients(controls, loss)
    e[3].record(s)
    torch.cuda.synchronize()
    fwd = e[0].elapsed_time(e[1])
    fb = e[2].elapsed_time(e[3])
    cells = sum(g.lx1 * g.lx2 * g.lx3 for g, _ in inst)
    return {"workload": f"{a['instances']} uneven Cartesian instances (lx1 128-256, lx2,lx3 32-128, {cells} cells), "
                        f"{a['steps']} steps, checkpoint every {a['checkpoint_every']}",
            "forward_ms": fwd, "forward_backward_ms": fb, "adjoint_over_forward": (fb - fwd) / fwd,
            "forward_value": cells * 7 * a["steps"] / (fwd / 1e3) / 1e9, "unit": UNIT,
            "gradients_finite": bool(all(torch.isfinite(gn).all() and torch.isfinite(gt).all() for _, gn, gt in res)),
            "forward": "groups of 8 instances, one batched step (captured graph, prescribed time steps) per time step"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--clocks-csv", default=None,
                    help="keep the nvidia-smi samples of the timed region in this file ({rank} is replaced)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=10, help="timed steps of the batched instances")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-instance measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint measurement")
    ap.add_argument("--no-full-step", action="store_true", help="skip the full fluid_adv measurement")
    ap.add_argument("--full-step", action="store_true",
                    help="run the full fluid_adv measurement on the --lx grid too (profiling a small case)")
    ap.add_argument("--no-batched-adjoint", action="store_true",
                    help="skip the batched adjoint workload (32 instances x 200 steps, about a minute)")
    ap.add_argument("--lx", type=int, nargs=3, default=None, metavar=("LX1", "LX2", "LX3"),
                    help="override the grid size (profiling runs on a smaller case)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the adjoint measurement (profiling of the adjoint kernels)")
    ap.add_argument("--adjoint-steps", type=int, default=None, help="time steps of the adjoint workload")
    args = ap.parse_args()
    if args.adjoint_steps:
        ADJOINT["steps"] = args.adjoint_steps
    if args.adjoint_only:
        print(json.dumps({"adjoint": run_adjoint(args)}))
        return
    if args.lx:
        WORKLOAD.update(lx1=args.lx[0], lx2=args.lx[1], lx3=args.lx[2])
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, world, rank)
        if line is not None:
            print(json.dumps(line))
        return
    world, rank, local = dist_setup(args.gpus)
    line = run_b200(args, world, rank, local)
    if not args.no_batched and not args.lx:
        import torch
        torch.cuda.empty_cache()
        line["batched"] = run_batched(args, world, rank)
    if not args.no_adjoint and not args.lx and world == 1:  # single-GPU figures, taken at N = 1
        import torch
        torch.cuda.empty_cache()
        line["adjoint"] = run_adjoint(args)
    if not args.no_full_step and (not args.lx or args.full_step) and world == 1:  # single-GPU, N = 1
        import torch
        torch.cuda.empty_cache()
        line["full_step"] = run_full_step(args)
    if not args.no_batched_adjoint and not args.lx and world == 1:  # single-GPU figures, taken at N = 1
        import torch
        torch.cuda.empty_cache()
        line["batched_adjoint"] = run_batched_adjoint(args)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
