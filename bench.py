#!/usr/bin/env python
"""Benchmark: zone-updates/s of the explicit FV step on B200 (and the CPU reference arm).

Default workload: 3D magnetised stratified box (Helmholtz EoS, well-balanced LHLLD + PLM + RK3,
constrained transport, uniform horizontal B at plasma beta 1e4), 256^3 cells: the 3D Helmholtz
MHD configuration the headline target is quoted on; --config stratified runs the hydro box.
A "step" is one full hydro step (3 RK stages) plus the CFL dt reduction, i.e. one iteration of
time_loop without output; zone-updates/s = steps * cells / time (the reference's own "updated
cells/s", source/source.F90:6834-6835).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--n SIZE] [--impl ours|reference]

One process per GPU; for N > 1 (torchrun) every rank advances an independent replica of the
workload (the single-GPU path has no data-path collective) and rank 0 prints the aggregate.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s on 1 B200: FP32+learned-EoS vs FP64 plain vs CPU, at stated L1 err"
_T0 = time.perf_counter()


def log(msg):
    """Progress on stderr (the JSON line is the only stdout output)."""
    print("[bench %7.1fs] %s" % (time.perf_counter() - _T0, msg), file=sys.stderr, flush=True)
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
MLP_NPARAMS = 4 * 64 + 64 + 64 * 64 + 64 + 64 + 1  # PHL_MLP_NPARAMS


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return dict(PEAKS_FALLBACK), "fallback"


def table_workers():
    """Host processes for the Fermi-gas table: the cores shared among the ranks of this node."""
    return max(1, (os.cpu_count() or 1) // max(1, int(os.environ.get("LOCAL_WORLD_SIZE", "1"))))


def build_problem(name, n, fasteos=True, eos_table="fermi"):
    from phlegethon_b200 import helm_table, problems
    table = None
    if name == "stratified":
        cfg, h = problems.stratified_3d(n, fasteos=fasteos, eos_model=eos_table)
        table = helm_table.make(eos_table, workers=table_workers())
    elif name == "stratified_mhd":
        cfg, h = problems.stratified_3d(n, mhd=True, fasteos=fasteos, eos_model=eos_table)
        table = helm_table.make(eos_table, workers=table_workers())
    elif name == "hot_bubble":
        cfg, h = problems.hot_bubble_2d(n)
    elif name == "orszag_tang":
        cfg, h = problems.orszag_tang_2d(n)
    else:
        raise SystemExit("unknown config " + name)
    return cfg, h, table


def default_size(name):
    return {"stratified": 256, "stratified_mhd": 256, "hot_bubble": 256, "orszag_tang": 1024}[name]


def stage_kernels(cfg, form, guess="warm"):
    """Name of what the per-stage timing covers, and the kernel launches of one step (the stage
    kernels plus k_pre_step and k_post_step; the learned rescue adds its queue kernel to every
    stage)."""
    s = cfg.rk_stages
    if cfg.mhd:
        nax = 3 if cfg.sdims == 3 else 1
        if form == "fp32_split":
            per = cfg.sdims + nax + cfg.sdims + 1 + (1 if guess == "mlp_rescue" else 0)
            names = "k_face_split_mhd + k_corner_split + k_bface_split + k_c2p_mhd_split"
        else:
            per = cfg.sdims + nax + cfg.sdims + 1
            names = "k_face + k_corner + k_bface + k_c2p"
        return names + " (one MHD stage)", s * per + 2
    if form == "fp32_split":
        tiled = cfg.sdims == 3 and cfg.nx1 % 32 == 0 and cfg.nx2 % 8 == 0 and cfg.nx3 % 16 == 0
        return ("k_stage_split_tiled" if tiled else "k_stage_split") + " (FP32 fluxes, FP64 state/EoS)", s + 2
    return "k_face + k_c2p (FP64)", s * (cfg.sdims + 1) + 2


# DRAM bytes per cell of one stage-kernel launch, from ncu captures of the 128^3 stratified box
# (dram__bytes_read.sum + dram__bytes_write.sum over 2,097,152 cells); the kernel streams the
# domain once per launch, so the per-launch traffic scales with the cell count
TRAFFIC_PER_CELL = {("stratified", "fp32_split"): 499.604224e6 / 2097152,
                    ("stratified", "fp64"): 557.258496e6 / 2097152,
                    # one split MHD stage at 128^3 (a middle stage: U0 read): x1 tile faces
                    # 216.9 MB, walking x2/x3 faces 186.1 + 190.0 MB, corners 3 x 42.2 MB,
                    # face-B 3 x 50.9 MB, cons->prim 755.2 MB
                    ("stratified_mhd", "fp32_split"): (216.9e6 + 186.1e6 + 190.0e6 + 3 * 42.2e6 + 3 * 50.9e6
                                                       + 755.2e6) / 2097152}


# Algorithmic HBM bytes per zone-update of the workloads (minimum traffic of one step of a fused
# stage: every field the step needs read once and every field it produces written once, per
# stage; no intermediate such as face fluxes or EMFs counted).  FP64 plain / FP32 split:
#   2D hot bubble, ideal gas, nv = 4                          448 B  (FP64)
#   2D Orszag-Tang, nv = 4 + 2 face-B components               576 B  (FP64)
#   3D Helmholtz box, nv = 7 + T + (gamma_e, gamma_c)          928 B / 712 B
#   3D Helmholtz MHD box, adds 3 face-B (r+w) and B^n reads   1120 B / 904 B
# The split form stores W' and the gammas in FP32; U, U0, T and the face B stay FP64.
ALGORITHMIC_BYTES = {("hot_bubble", "fp64"): 448, ("orszag_tang", "fp64"): 576,
                     ("stratified", "fp64"): 928, ("stratified", "fp32_split"): 712,
                     ("stratified_mhd", "fp64"): 1120, ("stratified_mhd", "fp32_split"): 904}


def algorithmic_bytes_per_cell(name, form):
    """Roofline numerator: algorithmic HBM bytes per zone-update (ALGORITHMIC_BYTES)."""
    return ALGORITHMIC_BYTES[(name, form)]


def step_bytes_per_cell(cfg):
    """Traffic model of the implementation: HBM bytes per zone-update with every intermediate
    the kernels materialise (FP32 face fluxes, face EMFs, CT signs, corner EMFs) counted.  Kept
    beside the algorithmic bytes as `roofline.traffic_model`; the excess over the algorithmic
    figure is the traffic a fused stage would not need.

    Stage 1 reads W (nv) and eint and writes U0, U, W; middle stages read W, U0, U and write U,
    W; the last stage reads W, U0, U and writes W and eint.  Helmholtz adds temp (read+write per
    stage) and the two gamma fields (read+write per stage).  MHD adds the face fields: per stage
    b read, b0 read (b0 written in stage 1), b written, plus the face EMFs and signs written and
    read once (2D: 1 EMF + 1 sign per face direction; 3D: 2 + 1).
    """
    nv = cfg.nvars
    s = cfg.rk_stages
    if cfg.precision == "fp32_split":
        # per stage: FP32 deviations W' read + written (nv), FP64 U read + written, U0 written in
        # stage 1 and read in later stages; temp read + written, eint written in the last stage
        b = s * (4 * nv + 4 * nv + 8 * nv + 8 * nv) + 8 * nv + (s - 1) * 8 * nv + 8
        if cfg.helmholtz:
            b += s * (16 + 16)  # temp (r+w, FP64) and the two FP32 gammas (r+w)
        if cfg.mhd:
            # per stage and cell, nd face directions: face kernel reads the normal face B (FP64)
            # and b_cc (FP32), writes 2 EMF components + 1 sign per face (FP32; 1 + 1 in 2D);
            # corner kernel reads those, the FP32 velocities and b_cc, writes one corner EMF per
            # axis; face update reads corner EMFs, B and B0, writes B; cons->prim reads B and
            # writes b_cc
            nd = cfg.sdims
            ne = 2 if nd == 3 else 1
            nax = 3 if nd == 3 else 1
            # the flux divergence moves into cons->prim: face fluxes (FP32, nv per face) are
            # written once and read once per cell-face direction
            flux = 8 * nd + 4 * nd + 4 * nd * (ne + 1) + 4 * nv * nd
            corner = 4 * nd * (ne + 1) + 4 * nd + 4 * nd + 4 * nax
            face = 4 * nax + 8 * nd * 3
            c2p = 8 * nd + 4 * nv * nd + 4 * nd
            b += s * (flux + corner + face + c2p)
        return b
    doubles = (nv + 1 + 3 * nv) + (s - 2) * (5 * nv) + (3 * nv + nv + 1)
    if cfg.helmholtz:
        doubles += s * (2 + 4)
    # face fluxes (FP64, nv per face) written once and read back per direction
    doubles += s * 2 * nv * cfg.sdims
    if cfg.mhd:
        nd = cfg.sdims
        emf = 1 if nd == 2 else 2
        doubles += s * nd * (3 + 2 * (emf + 1)) + nd
        doubles += s * nd  # b_cc write
    return 8 * doubles


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region: NVML read every 10 ms
    from a thread (the GPU found by the PCI bus id of the CUDA device), else nvidia-smi every
    200 ms.  Reads only; no setting is changed."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop_flag = threading.Event()

            def loop():
                while not self.stop_flag.is_set():
                    try:
                        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                          int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except Exception:
                        pass
                    self.stop_flag.wait(0.01)
            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            rows = self.rows
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"], "source": "nvml"}
            reasons = [nm for nm, bit in self.REASONS if any(r[1] & bit for r in rows)]
            return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(rows), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = []
        for k, nm in enumerate(names):
            if any(r[5 + k].lower().startswith("active") for r in rows):
                reasons.append(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi"}


def cpu_rate(name, steps, nthreads=0, slab=None, fasteos=True, eos_table="fermi"):
    """Oracle (CPU restatement) zone-updates/s on a bounded slab of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from phlegethon_b200 import helm_table, problems
    if name in ("stratified", "stratified_mhd"):
        n = default_size(name)
        nz = slab or 32
        cfg, h = problems.stratified_3d(n, nz=nz, mhd=(name == "stratified_mhd"), fasteos=fasteos,
                                        eos_model=eos_table)
        tab, dpdr = helm_table.make(eos_table, workers=table_workers())
        helm = pyoracle.Helm.for_config(cfg, tab, dpdr)
        sample = "%dx%dx%d slab of the %d^3 workload" % (cfg.nx1, cfg.nx2, cfg.nx3, n)
    else:
        n = default_size(name)
        cfg, h, _ = build_problem(name, n)
        helm = None
        sample = "%dx%d full workload" % (cfg.nx1, cfg.nx2)
    o = pyoracle.OracleGrid(h, helm, nthreads=nthreads)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(1)  # warm-up: first-touch allocations
    t0 = time.perf_counter()
    o.time_loop(steps)
    dt = time.perf_counter() - t0
    cores = nthreads or os.cpu_count()
    return steps * cfg.n_cells / dt, cores, sample + ", %d steps" % steps


def eos_reference_line(args):
    """The EoS batch's reference arm: the oracle's bracket-guess inversion (helm_rhoe_given) of a
    bounded slice of the same 2^24-sample batch, on all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from phlegethon_b200 import helm_table, problems
    n = args.n or (1 << 24)
    k = min(n, 1 << 16)
    rho, T, abar, zbar = problems.eos_samples(n, seed=99)
    rho, T, abar, zbar = rho[:k], T[:k], abar[:k], zbar[:k]
    cfg, _ = problems.stratified_3d(8)
    helm = pyoracle.Helm.for_config(cfg, *helm_table.make(args.eos_table, workers=table_workers()))
    e = np.array([helm.given2(*a, deriv=False)[0] for a in zip(rho, T, abar, zbar)])
    cpu = eos_cpu_rate(rho, e, abar, zbar, seconds=max(5.0, 2.0 * max(1, args.steps)), eos_table=args.eos_table)
    return {"impl": "reference", "metric": EOS_METRIC, "value": cpu["value"], "unit": "inversions/s",
            "n_gpus": args.gpus, "steps": max(1, args.steps), "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "eos_batch", "n": n, "eos_table": args.eos_table},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "inversions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "CPU restatement of the reference routines (oracle/), OpenMP over all host cores; "
                    "the reference's Fortran build is unavailable (no gfortran/mpifort)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.config == "eos":
        print(json.dumps(eos_reference_line(args)), flush=True)
        return
    steps = max(1, args.steps)
    rate, cores, sample = cpu_rate(args.config, steps, fasteos=not args.no_fasteos, eos_table=args.eos_table)
    cfgname = args.config
    n = args.n or default_size(cfgname)
    # the same workload keys as the GPU arm's line (its name, size, cells and table); the
    # oracle times a bounded slab of it, named in cpu_baseline.sample
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "zone-updates/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfgname + ("_no_fasteos" if args.no_fasteos else ""), "n": n,
                       "cells": n ** 3 if cfgname.startswith("stratified") else n ** 2,
                       "eos_table": args.eos_table, "form": "fp64 (CPU oracle)",
                       "parallelism": "single"},
            "cpu_baseline": {"value": rate, "unit": "zone-updates/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": rate, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "CPU restatement of the reference routines (oracle/), OpenMP over all host cores; "
                    "the reference's Fortran build is unavailable (no gfortran/mpifort)"}
    print(json.dumps(line), flush=True)


def max_over_ranks(ms, dist, device="cuda"):
    """Largest elapsed time over all ranks (the job is as slow as its slowest replica)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, steps, cells, ms):
    """Whole-job zone-updates/s of `world` replicas that each advanced `steps` steps."""
    return world * steps * cells / (ms * 1e-3)


def pinned_like(a):
    import torch
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    v = t.numpy().reshape(a.shape, order="F")
    v[...] = a
    return t, v


def measure_form(args, name, cfg, h, table, form, local, dist, want_e2e, guess="warm", mlp_params=None,
                 kernel_timing=True):
    """Time one arithmetic form on the workload; returns timings and the final host state.
    guess: the temperature guess of the step's Newton -- "warm" (previous stage), "mlp_rescue"
    (warm, and the learned guess where the warm start is poor) or "mlp" (learned guess for every
    cell).  A learned guess needs the network: trained on the device first (untimed) unless
    mlp_params (a previous run's parameters) is given."""
    import ctypes as C

    import torch
    from phlegethon_b200 import abi
    from phlegethon_b200.grid import HostGrid, helm_state_range

    c = cfg.replace(precision=form, device=local, eos_guess=guess)
    log("measure %s %s (%d cells)" % (form, guess, cfg.n_cells))
    sim = abi.Simulation(c, table)
    train = None
    sim.upload(h)
    sim.init_thermo()
    if guess != "warm" and mlp_params is not None:
        assert sim.lib.phl_mlp_set_params(sim.ctx, mlp_params.ctypes.data_as(C.POINTER(C.c_float))) == 0
    elif guess != "warm":
        # the network is fitted over the states of the run: log10 rho and log10 T of the initial
        # state widened by 0.1 dex, its Abar and Zbar
        h0 = h.copy()
        sim.download(h0)
        lo, hi = helm_state_range(h0, cfg)
        sim.set_mlp_sample_range(lo, hi)
        loss = C.c_double()
        t0 = time.perf_counter()
        rc = sim.lib.phl_mlp_train(sim.ctx, 1 << 22, 12345, args.train_epochs, 8192, C.c_double(3e-3), C.byref(loss))
        if rc != 0:
            raise RuntimeError("phl_mlp_train failed: %d" % rc)
        train = {"samples": 1 << 22, "epochs": args.train_epochs, "seconds": time.perf_counter() - t0,
                 "loss": loss.value, "range_lo": lo, "range_hi": hi}
        mlp_params = np.zeros(MLP_NPARAMS, dtype=np.float32)
        assert sim.lib.phl_mlp_get_params(sim.ctx, mlp_params.ctypes.data_as(C.POINTER(C.c_float))) == 0
    sim.compute_hyperbolic_dt()
    stream = torch.cuda.ExternalStream(sim.stream(), device=torch.device("cuda", local))
    sim.time_loop(args.warmup)
    sim.reset_status()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    done, _ = sim.time_loop(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    status = sim.status()
    out = h.copy()
    sim.download(out)
    res = {"form": form, "guess": guess, "ms": ms, "done": done, "clocks": clocks, "status": status, "state": out,
           "train": train, "mlp_params": mlp_params}
    if not kernel_timing:
        sim.close()
        return res

    # dominant kernel: hydro_step launches the RK stage kernels back to back (no graph); their
    # average duration is measured with events on the library's stream
    reps = max(2, min(args.steps, 5))
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for _ in range(reps):
        sim.hydro_step()
    k1.record(stream)
    torch.cuda.synchronize()
    res["launch_ms"] = k0.elapsed_time(k1) / (reps * c.rk_stages)

    if want_e2e:
        # host-owned state in pinned memory: every step uploads the dynamic state, advances one
        # step and downloads it again (prim, temp, eint [, gammaf, b_cc, b faces])
        dyn = HostGrid.__new__(HostGrid)
        dyn.__dict__.update(h.__dict__)
        keep = []
        for nm in ("prim", "temp", "eint", "gammaf", "b_cc"):
            a = getattr(h, nm)
            if a is not None:
                t_, v_ = pinned_like(a)
                keep.append(t_)
                setattr(dyn, nm, v_)
        bx = []
        for d in range(3):
            a = h.b_x[d]
            if a is not None:
                t_, v_ = pinned_like(a)
                keep.append(t_)
                bx.append(v_)
            else:
                bx.append(None)
        dyn.b_x = bx
        for nm in ("grav", "phi_cc", "eq_prim_cc", "eq_gammae_cc"):
            setattr(dyn, nm, None)
        dyn.phi_x = [None] * 3
        dyn.eq_prim_x = [None] * 3
        dyn.eq_gammae_x = [None] * 3
        sim.download(dyn)
        e2e_steps = max(1, min(args.steps, 10))
        # bytes per step: each call uploads the whole host arrays (ghost layers included:
        # contiguous copies) and downloads their interiors
        h2d = sum(a.nbytes for a in [dyn.prim, dyn.temp, dyn.eint, dyn.gammaf, dyn.b_cc] + bx if a is not None)
        cells = cfg.n_cells
        d2h = 8 * sum(x for x in [cfg.nvars * cells, cells, cells,
                                  2 * cells if (cfg.helmholtz and cfg.fasteos) else 0,
                                  cfg.sdims * cells if cfg.mhd else 0] if x)
        if cfg.mhd:
            n3 = [cfg.nx1, cfg.nx2, cfg.nx3]
            for d in range(cfg.sdims):
                d2h += 8 * int(np.prod([n3[a] + (a == d) for a in range(3)]))
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        x0 = torch.cuda.Event(enable_timing=True)
        x1 = torch.cuda.Event(enable_timing=True)
        x0.record(stream)
        # the public host-state call: upload, one step, download, queued per step; a step's
        # uploads wait for the previous step's downloads of the same host planes
        for _ in range(e2e_steps):
            sim.time_loop_host_async(dyn, 1)
        sim.wait_host()
        x1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(x0.elapsed_time(x1), dist)
        res["e2e_ms_per_step"] = e2e_ms / e2e_steps
        res["h2d"] = int(h2d)
        res["d2h"] = int(d2h)
    sim.close()
    return res


def long_run_errors(cfg, h, table, form, steps, local, guess="warm", mlp_params=None):
    """Per-field relative L1 of `form` (with its EoS guess) against the FP64 form after `steps`
    steps from h."""
    import ctypes as C

    from phlegethon_b200 import abi
    from util import field_errors
    out = {}
    log("long run: %d steps of %s and fp64" % (steps, form))
    for f, gs in ((form, guess), ("fp64", "warm")):
        hh = h.copy()
        with abi.Simulation(cfg.replace(precision=f, device=local, eos_guess=gs), table) as sim:
            sim.upload(hh)
            sim.init_thermo()
            if gs != "warm":
                assert sim.lib.phl_mlp_set_params(sim.ctx, mlp_params.ctypes.data_as(C.POINTER(C.c_float))) == 0
            sim.compute_hyperbolic_dt()
            done, _ = sim.time_loop(steps)
            assert done == steps
            sim.download(hh)
        out[f] = hh
    return field_errors(out[form], out["fp64"])


def run_case(cfg, h, table, local, nsteps, tmax=float("inf"), warmup=3, guess="warm", mlp_params=None):
    """Advance h by `nsteps` steps (or until tmax) on a fresh context, timed on the device after
    `warmup` untimed steps from the same start (the state is re-uploaded and the clock reset, so
    the graphs are captured before the timed region).  Returns (ms, steps, time, final state,
    status)."""
    import ctypes as C

    import torch
    from phlegethon_b200 import abi
    c = cfg.replace(device=local, eos_guess=guess)
    log("case %dx%dx%d %s %s" % (cfg.nx1, cfg.nx2, cfg.nx3, cfg.precision, guess))
    sim = abi.Simulation(c, table if cfg.helmholtz else None)
    sim.upload(h)
    sim.init_thermo()
    if guess != "warm":
        assert sim.lib.phl_mlp_set_params(sim.ctx, mlp_params.ctypes.data_as(C.POINTER(C.c_float))) == 0
    dt0, smax0 = sim.compute_hyperbolic_dt()
    start = h.dynamic_copy()
    sim.download(start)
    sim.time_loop(warmup, tmax)
    sim.upload(start)
    sim.set_time(0.0, dt0, smax0)
    sim.reset_status()
    stream = torch.cuda.ExternalStream(sim.stream(), device=torch.device("cuda", local))
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if tmax == float("inf"):
        done, t = sim.time_loop(nsteps, tmax)
    else:
        # to a final time: batches of steps until the device stops at tmax (the host learns the
        # time once per batch)
        done, t = 0, 0.0
        while done < nsteps and t < tmax:
            d, t = sim.time_loop(min(256, nsteps - done), tmax)
            done += d
            if d == 0:
                break
    e1.record(stream)
    torch.cuda.synchronize()
    out = h.copy()
    sim.download(out)
    st = sim.status()
    sim.close()
    return e0.elapsed_time(e1), done, t, out, st


def run_suite(args, local, mlp_params):
    """The other workloads, each at its stated size: zone-updates/s of the FP64 and split forms,
    the split form's per-field L1 against FP64, div B where there is a magnetic field, and a
    bounded CPU oracle sample (same zone-update metric)."""
    from util import div_b_max, field_errors
    suite = {}

    def rate(cfg, ms, done):
        return done * cfg.n_cells / (ms * 1e-3)

    # 2D hot bubble 256^2, 100 steps
    cfg, h, _ = build_problem("hot_bubble", 256)
    r = {}
    for form in ("fp64", "fp32_split"):
        ms, done, t, out, st = run_case(cfg.replace(precision=form), h, None, local, 100)
        r[form] = (ms, done, out)
    cpu = cpu_rate("hot_bubble", 5) if not args.no_cpu else None
    suite["hot_bubble_256"] = {
        "steps": r["fp64"][1], "fp64": {"value": rate(cfg, r["fp64"][0], r["fp64"][1]),
                                        "ms_per_step": r["fp64"][0] / r["fp64"][1]},
        "fp32_split": {"value": rate(cfg, r["fp32_split"][0], r["fp32_split"][1]),
                       "ms_per_step": r["fp32_split"][0] / r["fp32_split"][1],
                       "l1_vs_fp64": field_errors(r["fp32_split"][2], r["fp64"][2])},
        "cpu_oracle": {"value": cpu[0], "cores": cpu[1], "sample": cpu[2]} if cpu else None}
    # Orszag-Tang 1024^2 (HLLD, CT) to t = 0.5
    cfg, h, _ = build_problem("orszag_tang", 1024)
    r = {}
    for form in ("fp64", "fp32_split"):
        ms, done, t, out, st = run_case(cfg.replace(precision=form), h, None, local, 1 << 20, tmax=0.5)
        r[form] = (ms, done, out, t)
    cpu = cpu_rate("orszag_tang", 2) if not args.no_cpu else None
    suite["orszag_tang_1024"] = {
        "t_end": r["fp64"][3], "steps": r["fp64"][1],
        "fp64": {"value": rate(cfg, r["fp64"][0], r["fp64"][1]), "ms_per_step": r["fp64"][0] / r["fp64"][1],
                 "div_b_max": div_b_max(r["fp64"][2])},
        "fp32_split": {"value": rate(cfg, r["fp32_split"][0], r["fp32_split"][1]), "steps": r["fp32_split"][1],
                       "ms_per_step": r["fp32_split"][0] / r["fp32_split"][1],
                       "div_b_max": div_b_max(r["fp32_split"][2]),
                       "l1_vs_fp64": field_errors(r["fp32_split"][2], r["fp64"][2])},
        "cpu_oracle": {"value": cpu[0], "cores": cpu[1], "sample": cpu[2]} if cpu else None}
    # EoS inversion batch of 2^24 samples, learned vs bracket guess
    ea = argparse.Namespace(**vars(args))
    ea.n, ea.steps, ea.warmup = 0, 5, 3
    el = eos_line(ea, with_cpu=False)
    suite["eos_batch_2^24"] = {k: el[k] for k in ("value", "unit", "ms_per_step", "bracket", "mlp", "agreement", "e2e")}
    # the Helmholtz hydro box 256^3 (no B), split and FP64 rates, and the split form's
    # per-field L1 against FP64 after 1000 steps
    cfg, h, table = build_problem("stratified", 256, eos_table=args.eos_table)
    r = {}
    for form in ("fp32_split", "fp64"):
        ms, done, t, out, st = run_case(cfg.replace(precision=form), h, table, local, 10)
        r[form] = (ms, done, out)
    suite["stratified_hydro_256"] = {
        "steps": r["fp32_split"][1],
        "fp32_split": {"value": rate(cfg, r["fp32_split"][0], r["fp32_split"][1]),
                       "ms_per_step": r["fp32_split"][0] / r["fp32_split"][1], "eos_guess": "warm",
                       "l1_vs_fp64": field_errors(r["fp32_split"][2], r["fp64"][2])},
        "fp64": {"value": rate(cfg, r["fp64"][0], r["fp64"][1]), "ms_per_step": r["fp64"][0] / r["fp64"][1]},
        "l1_vs_fp64_1000_steps": long_run_errors(cfg, h, table, "fp32_split", 1000, local)}
    if not args.no_cpu:
        cpu = cpu_rate("stratified", 2, eos_table=args.eos_table)
        suite["stratified_hydro_256"]["cpu_oracle"] = {"value": cpu[0], "cores": cpu[1], "sample": cpu[2]}
    # magnetised box 384^3, the headline form and FP64, a few steps each
    cfg, h, table = build_problem("stratified_mhd", 384, eos_table=args.eos_table)
    r = {}
    for form, guess in (("fp32_split", "mlp_rescue" if mlp_params is not None else "warm"), ("fp64", "warm")):
        ms, done, t, out, st = run_case(cfg.replace(precision=form), h, table, local, 5, guess=guess,
                                        mlp_params=mlp_params)
        r[form] = (ms, done, out, st)
    suite["stratified_mhd_384"] = {
        "steps": r["fp32_split"][1],
        "fp32_split": {"value": rate(cfg, r["fp32_split"][0], r["fp32_split"][1]),
                       "ms_per_step": r["fp32_split"][0] / r["fp32_split"][1],
                       "eos_guess": "mlp_rescue" if mlp_params is not None else "warm",
                       "l1_vs_fp64": field_errors(r["fp32_split"][2], r["fp64"][2])},
        "fp64": {"value": rate(cfg, r["fp64"][0], r["fp64"][1]), "ms_per_step": r["fp64"][0] / r["fp64"][1]},
        "div_b_max_split": div_b_max(r["fp32_split"][2])}
    return suite


def run_ours(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    sys.path.insert(0, os.path.join(ROOT, "tests"))

    name = args.config
    n = args.n or default_size(name)
    log("building %s at %d" % (name, n))
    cfg, h, table = build_problem(name, n, fasteos=not args.no_fasteos, eos_table=args.eos_table)
    log("built")
    peaks, peak_kind = load_peaks()
    cells = cfg.n_cells
    head_form = args.form
    # the metric's form: FP32 split fluxes with the learned EoS guess in the step (the warm start,
    # and the network's judged guess for every cell whose warm start is poor); the learned guess
    # in the step is built for the Helmholtz MHD box
    learned_ok = head_form == "fp32_split" and name == "stratified_mhd" and not args.no_learned
    head_guess = "mlp_rescue" if learned_ok else "warm"
    from util import field_errors
    head = measure_form(args, name, cfg, h, table, head_form, local, dist, want_e2e=True, guess=head_guess)
    results = {head_form: head}
    if head_form != "fp64":
        results["fp64"] = measure_form(args, name, cfg, h, table, "fp64", local, dist, want_e2e=False)
    side = {}
    if learned_ok:
        def summary(r, ref):
            st = r["status"]
            return {"value": aggregate_rate(world, r["done"], cells, r["ms"]),
                    "ms_per_step": r["ms"] / max(r["done"], 1),
                    "newton_iters_per_call": st["newton_iterations"] / max(st["newton_calls"], 1),
                    "learned_guesses": st["mlp_accepted"] + st["mlp_rejected"],
                    "learned_accepted": st["mlp_accepted"],
                    "l1_vs_headline": field_errors(r["state"], ref["state"])}
        # the same split form with the reference's warm start alone, and with the learned guess
        # for every cell, timed the same way (network parameters shared with the headline run)
        for key, guess in (("warm_guess_step", "warm"), ("learned_every_cell_step", "mlp")):
            r = measure_form(args, name, cfg, h, table, head_form, local, dist, want_e2e=False, guess=guess,
                             mlp_params=head["mlp_params"], kernel_timing=False)
            side[key] = summary(r, head)
    hst = head["status"]
    learned_info = None
    if learned_ok:
        learned_info = {"mode": "mlp_rescue: warm start; cells whose first warm Newton correction exceeds 2% "
                                "of T take the network's judged guess",
                        "learned_guesses": hst["mlp_accepted"] + hst["mlp_rejected"],
                        "learned_accepted": hst["mlp_accepted"],
                        "newton_iters_per_call": hst["newton_iterations"] / max(hst["newton_calls"], 1),
                        "train": head["train"]}
    l1_long = None
    l1_steps = args.l1_steps if args.l1_steps >= 0 else (1000 if cfg.helmholtz else 0)
    if l1_steps and head_form != "fp64":
        l1_long = {"steps": l1_steps, "form": head_form, "eos_guess": head_guess,
                   "errors": long_run_errors(cfg, h, table, head_form, l1_steps, local, guess=head_guess,
                                             mlp_params=head["mlp_params"])}
    value = aggregate_rate(world, head["done"], cells, head["ms"])
    fp64 = results["fp64"]
    fp64_value = aggregate_rate(world, fp64["done"], cells, fp64["ms"])
    errors = None
    if head_form != "fp64":
        from util import field_errors
        errors = field_errors(head["state"], fp64["state"])

    # roofline of one RK stage (all kernels of the stage, CUDA events on the library's stream):
    # algorithmic bytes of a stage = the per-zone-update figure / stages x cells
    bytes_per_cell = algorithmic_bytes_per_cell(name, head_form)
    model_bytes = step_bytes_per_cell(cfg.replace(precision=head_form))
    launch_ms = head["launch_ms"]
    achieved = bytes_per_cell * cells / cfg.rk_stages / (launch_ms * 1e-3) / 1e9
    kname, launches_per_step = stage_kernels(cfg, head_form, head_guess)
    tpc = TRAFFIC_PER_CELL.get((name, head_form))
    roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": tpc * cells if tpc else None,
            "traffic_source": ("ncu DRAM bytes of one stage at 128^3, scaled by cells" if name == "stratified_mhd"
                               else "ncu DRAM bytes of one launch at 128^3, scaled by cells") if tpc else None,
            "kernel": kname, "peak_kind": peak_kind,
            "launch_ms": launch_ms, "bytes_per_zone_update": bytes_per_cell,
            "traffic_model": {"bytes_per_zone_update": model_bytes,
                              "note": "every materialised intermediate counted (face fluxes, EMFs, signs)"}}

    suite = None
    if rank == 0 and world == 1 and not args.no_suite and name == "stratified_mhd" and not args.n:
        try:
            suite = run_suite(args, local, head["mlp_params"])
        except Exception as exc:  # the headline line is printed even if a side workload fails
            log("suite failed: %r" % (exc,))
            suite = {"error": repr(exc)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        log("cpu baseline")
        rate, cores, sample = cpu_rate(name, steps=5, fasteos=not args.no_fasteos, eos_table=args.eos_table)
        cpu = {"value": rate, "unit": "zone-updates/s", "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        e2e_value = world * cells / (head["e2e_ms_per_step"] * 1e-3)
        status = head["status"]
        line = {"metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms"] / max(head["done"], 1), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 fluxes / f64 state+EoS" if head_form == "fp32_split" else "f64",
                "data": "synthetic",
                "config": {"workload": name + ("_no_fasteos" if args.no_fasteos else ""), "n": n, "cells": cells,
                           "eos_table": args.eos_table,
                           "form": head_form,
                           "eos_guess": head_guess,
                           "parallelism": "replicas" if world > 1 else "single",
                           "l2": "inputs larger than L2 (%.0f MB dynamic state)" % (h.state_bytes() / 1e6)},
                "fp64_plain": {"value": fp64_value, "ms_per_step": fp64["ms"] / max(fp64["done"], 1),
                               "speedup_of_form": value / fp64_value},
                "l1_vs_fp64": errors, "l1_vs_fp64_long": l1_long, "learned_eos": learned_info, **side,
                "suite": suite,
                "roofline": roof, "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": "zone-updates/s", "h2d_bytes_per_step": head["h2d"],
                        "d2h_bytes_per_step": head["d2h"], "ms_per_step": head["e2e_ms_per_step"],
                        "api": "phl_run_steps_host_async (pinned host arrays; upload, step, download per step)"},
                "gpu_launches": int(head["done"] * launches_per_step), "clocks": head["clocks"],
                "newton": {k: status[k] for k in ("newton_calls", "newton_iterations", "newton_nonconverged")},
                "nonfinite": status["nonfinite"]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


EOS_METRIC = "(rho,e)->T inversions/s on 1 B200: learned vs bracket guess, T identical to 1e-10"
EOS_BYTES_PER_SAMPLE = 44  # rho, e, Abar, Zbar in (FP64), T out (FP64), iteration count out (int32)


def run_eos(args):
    print(json.dumps(eos_line(args)), flush=True)


def eos_line(args, with_cpu=True):
    """EoS inversion batch: 2^24 samples over the full table range, bracket vs learned guess.

    A step is one inversion of the whole batch (inputs resident in HBM, 2^24 x 44 B > L2).
    """
    import torch
    from phlegethon_b200 import helm_table, problems
    from phlegethon_b200.abi import Simulation
    n = args.n or (1 << 24)
    cfg, _ = problems.stratified_3d(8)
    table = helm_table.make(args.eos_table, workers=table_workers())
    peaks, peak_kind = load_peaks()
    import ctypes as C
    with Simulation(cfg, table) as sim:
        lib = sim.lib
        stream = torch.cuda.ExternalStream(sim.stream())
        t0 = time.perf_counter()
        loss = C.c_double()
        rc = lib.phl_mlp_train(sim.ctx, 1 << 22, 12345, args.train_epochs, 8192, C.c_double(3e-3), C.byref(loss))
        train_s = time.perf_counter() - t0
        assert rc == 0, rc
        rho, T, abar, zbar = problems.eos_samples(n, seed=99)
        d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
             dict(rho=rho, T=T, abar=abar, zbar=zbar).items()}
        e = torch.zeros(n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert lib.phl_eos_energy_device(sim.ctx, n, d["rho"].data_ptr(), d["T"].data_ptr(), d["abar"].data_ptr(),
                                         d["zbar"].data_ptr(), e.data_ptr()) == 0
        out = {}
        for guess, gname in ((2, "bracket"), (1, "mlp")):
            Tout = torch.zeros(n, dtype=torch.float64, device="cuda")
            its = torch.zeros(n, dtype=torch.int32, device="cuda")

            def step():
                return lib.phl_eos_invert_batch_device(sim.ctx, n, d["rho"].data_ptr(), e.data_ptr(),
                                                       d["abar"].data_ptr(), d["zbar"].data_ptr(), Tout.data_ptr(),
                                                       None, None, its.data_ptr(), guess)
            for _ in range(args.warmup):
                assert step() == 0
            sim.reset_status()
            torch.cuda.synchronize()
            clk = ClockSampler(0)
            clk.start()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                assert step() == 0
            e1.record(stream)
            torch.cuda.synchronize()
            clocks = clk.stop()
            ms = e0.elapsed_time(e1) / args.steps
            st = sim.status()
            out[gname] = dict(ms=ms, rate=n / (ms * 1e-3), T=Tout.clone(), iters=its.double().mean().item(),
                              evals=(st["guess_evaluations"] + st["newton_iterations"]) / (n * args.steps),
                              accepted=st["mlp_accepted"] / (n * args.steps), clocks=clocks,
                              nonconv=st["newton_nonconverged"])
        # host-buffer end to end through the public host-pointer entry point
        e_host = e.cpu().numpy()
        h_in = [torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for v in (rho, e_host, abar, zbar)]
        h_T = torch.zeros(n, dtype=torch.float64).pin_memory()
        h_it = torch.zeros(n, dtype=torch.int32).pin_memory()
        x0 = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 3))
        for _ in range(e2e_steps):
            assert lib.phl_eos_invert_batch(sim.ctx, n, *[a.data_ptr() for a in h_in], h_T.data_ptr(), None, None,
                                            h_it.data_ptr(), 1) == 0
        e2e_ms = (time.perf_counter() - x0) * 1e3 / e2e_steps
        # agreement of the two answers, judged by the conditioning kappa = |E / (T dE/dT)|
        Tb = out["bracket"]["T"]
        hh = 1e-6
        ep = torch.zeros_like(e)
        em = torch.zeros_like(e)
        tp = Tb * (1 + hh)
        tm = Tb * (1 - hh)
        lib.phl_eos_energy_device(sim.ctx, n, d["rho"].data_ptr(), tp.data_ptr(), d["abar"].data_ptr(),
                                  d["zbar"].data_ptr(), ep.data_ptr())
        lib.phl_eos_energy_device(sim.ctx, n, d["rho"].data_ptr(), tm.data_ptr(), d["abar"].data_ptr(),
                                  d["zbar"].data_ptr(), em.data_ptr())
        kappa = (e / ((ep - em) / (2 * hh))).abs()
        rel = (out["mlp"]["T"] - Tb).abs() / Tb
        good = kappa < 10
        agree = {"frac_kappa_lt_10": good.double().mean().item(),
                 "max_rel_T_diff_kappa_lt_10": rel[good].max().item(),
                 "frac_within_1e-10_plus_4e-11_kappa": (rel <= 1e-10 + 4e-11 * kappa).double().mean().item()}
    m, b = out["mlp"], out["bracket"]
    cpu = None
    if with_cpu and not args.no_cpu:
        k = min(n, 1 << 20)
        cpu = eos_cpu_rate(rho[:k], e_host[:k], abar[:k], zbar[:k], eos_table=args.eos_table)
    achieved = EOS_BYTES_PER_SAMPLE * m["rate"] / 1e9
    line = {"metric": EOS_METRIC, "value": m["rate"], "unit": "inversions/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (EoS/Newton), bf16/f32 (MLP)", "data": "synthetic",
            "config": {"workload": "eos_batch", "n": n, "eos_table": args.eos_table, "l2": "inputs larger than L2 (%.0f MB)" % (n * 44 / 1e6),
                       "train": {"samples": 1 << 22, "epochs": args.train_epochs, "seconds": train_s,
                                 "loss": loss.value}},
            "bracket": {"value": b["rate"], "ms_per_step": b["ms"], "newton_iters_per_sample": b["iters"],
                        "eos_evals_per_sample": b["evals"]},
            "mlp": {"newton_iters_per_sample": m["iters"], "eos_evals_per_sample": m["evals"],
                    "accepted": m["accepted"], "speedup_vs_bracket": m["rate"] / b["rate"]},
            "agreement": agree,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": None, "peak_kind": peak_kind,
                         "kernel": "k_eos_invert + k_eos_fallback",
                         "note": "FP64-compute bound (EoS evaluations); HBM fraction stated for completeness"},
            "cpu_baseline": cpu,
            "e2e": {"value": n / (e2e_ms * 1e-3), "unit": "inversions/s", "h2d_bytes_per_step": 40 * n,
                    "d2h_bytes_per_step": 12 * n},
            "gpu_launches": 2 * args.steps, "clocks": m["clocks"]}
    return line


def eos_cpu_rate(rho, e, abar, zbar, seconds=10.0, eos_table="fermi"):
    """Oracle bracket-guess inversions/s on all host cores, repeating a bounded slice of the batch."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from phlegethon_b200 import helm_table, problems
    cfg, _ = problems.stratified_3d(8)
    helm = pyoracle.Helm.for_config(cfg, *helm_table.make(eos_table, workers=table_workers()))
    done = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        helm.invert_batch(rho, e, abar, zbar, guess=2)
        done += rho.size
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "inversions/s", "cores": os.cpu_count(), "kind": "port",
            "sample": "%d inversions (first %d samples of the batch, repeated; oracle bracket guess + "
                      "helm_rhoe_given Newton, OpenMP)" % (done, rho.size)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="stratified_mhd",
                    choices=["stratified", "stratified_mhd", "hot_bubble", "orszag_tang", "eos"])
    ap.add_argument("--l1-steps", type=int, default=-1,
                    help="also run both forms this many steps from the initial state and report the "
                         "per-field relative L1 difference (untimed); default 1000 for the Helmholtz boxes")
    ap.add_argument("--no-suite", action="store_true",
                    help="skip the other workloads (hot bubble 256^2, Orszag-Tang 1024^2 to t = 0.5, EoS "
                         "batch 2^24, Helmholtz hydro box 256^3, MHD box 384^3) reported under `suite`")
    ap.add_argument("--n", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--train-epochs", type=int, default=256, help="MLP training epochs (eos workload)")
    ap.add_argument("--no-fasteos", action="store_true",
                    help="Helmholtz boxes without USE_FASTEOS (helm_rhoP_given per Riemann side)")
    ap.add_argument("--form", default="fp32_split", choices=["fp32_split", "fp64"])
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the split MHD form with the learned temperature guess in the step")
    ap.add_argument("--eos-table", default="fermi", choices=["fermi", "synthetic"],
                    help="electron free-energy table of the Helmholtz workloads: the electron-positron "
                         "Fermi gas (helm_fermi) or the closed-form synthetic model (helm_table.generate)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "eos":
        run_eos(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
