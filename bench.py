#!/usr/bin/env python
"""Throughput of AFiD's RK3 flow + temperature step on a B200.

Workload (default ``rbc3d``): 3-D Rayleigh-Benard convection, FP64, Ra=1e9, Pr=1, aspect ratio
1, 384 x 384 periodic horizontal x 256 tanh-clustered (STR3=2) wall-normal cells, no-slip walls
at T = +0.5 / -0.5, fluid at rest plus a seeded +-1e-3 perturbation, CFL-limited dt (CFLMAX 1.2,
DT 1e-4 for the first two steps as main.F90:288-296 does).  A step is one main-loop iteration
(CalcMaxCFL -> dt rule -> TimeMarcher, three substeps) of the whole 37.7 M-cell domain.

value : Mcell-RK3-steps/s with the state resident in HBM (CUDA events on the solver stream,
        max over ranks; ranks are independent replicas).
e2e   : the same metric through the C ABI from pinned host buffers: upload of the five state
        fields, K steps each reading back the CFL and the Nusselt/kinetic-energy metrics, and
        download of the five fields, all inside the timed region.
--impl reference : the CPU restatement of the same path (C + OpenMP, oracle/afid_cpu.c) on all
        host cores, a bounded number of steps of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "afid-murphfi_b200"))

WORKLOADS = {
    "rbc3d": dict(nxm=256, nym=384, nzm=384, rayt=1e9, prat=1.0, ylen=1.0, zlen=1.0, precision=0,
                  idtv=1, dt=1e-4, cflmax=1.2, dtmax=1e-2,
                  name="rbc3d_384x384x256_fp64_ra1e9"),
    "rbc3d_mixed": dict(nxm=384, nym=512, nzm=512, rayt=1e10, prat=1.0, ylen=1.0, zlen=1.0, precision=1,
                        idtv=1, dt=1e-4, cflmax=1.2, dtmax=1e-2,
                        name="rbc3d_512x512x384_mixed_ra1e10"),
    # same kernels at 1/9 of the cells (4.2 M, ~0.6 GB per K1 launch > L2) for ncu captures
    "rbc3d_small": dict(nxm=256, nym=128, nzm=128, rayt=1e9, prat=1.0, ylen=1.0, zlen=1.0, precision=0,
                        idtv=1, dt=1e-4, cflmax=1.2, dtmax=1e-2,
                        name="rbc3d_128x128x256_fp64_ra1e9"),
    # 16.8 M cells (2.3 GB): state and spectrum larger than L2, small enough for multi-pass ncu
    "rbc3d_medium": dict(nxm=256, nym=256, nzm=256, rayt=1e9, prat=1.0, ylen=1.0, zlen=1.0, precision=0,
                         idtv=1, dt=1e-4, cflmax=1.2, dtmax=1e-2,
                         name="rbc3d_256x256x256_fp64_ra1e9"),
    "rbc2d": dict(nxm=128, nym=256, nzm=1, rayt=1e8, prat=1.0, ylen=2.0, zlen=0.01, precision=0,
                  idtv=0, dt=5e-4, cflmax=1.2, dtmax=5e-4,
                  name="rbc2d_256x128_fp64_ra1e8"),
}

# Algorithmic HBM bytes per cell of the fused explicit + RHS + CN kernel: read vx, vy, vz, T, p
# and the RK3 histories rux, ruy, ruz, rutemp, write vx, vy, vz, T and the histories.  FP64:
# 17 x 8 B; mixed (FP32 histories): 9 x 8 + 8 x 4 B.
K1_BYTES_PER_CELL = {0: 136, 1: 104}
# Algorithmic HBM bytes per cell per RK3 step of the whole path (one compulsory pass per
# operator): 3 x 328 B per substep + 24 B for CalcMaxCFL.
STEP_BYTES_PER_CELL = 1008
# Algorithmic HBM bytes per cell of each kernel class of the profile (one launch), FP64 and mixed
# (FP32 spectrum and phi): K2 reads vx, vy, vz and writes the half spectrum (nym/2+1 of nym rows
# of complex values, counted as half a complex a cell); K3, K4, K5 read and write the spectrum;
# K6 reads it and writes phi; K7 reads the intermediate velocities, pr and phi and writes the
# velocities and pr; the CFL reduction reads vx, vy, vz.
KERNEL_BYTES_PER_CELL = {
    0: {"explicit_implicit": 136, "div_fft_y": 32, "fft_z_fwd": 16, "tridiag_pressure": 16, "fft_z_inv": 16,
        "ifft_y": 16, "correct": 72, "reductions": 24},
    1: {"explicit_implicit": 104, "div_fft_y": 28, "fft_z_fwd": 8, "tridiag_pressure": 8, "fft_z_inv": 8,
        "ifft_y": 8, "correct": 68, "reductions": 24},
}


def kernels_roofline(prof: dict, cells: int, precision: int, peak: float) -> dict:
    """Achieved GB/s and fraction of the copy peak of every kernel class, from its CUDA-event
    time per launch and its algorithmic bytes per launch."""
    out = {}
    for k, b in KERNEL_BYTES_PER_CELL[precision].items():
        ms, n = prof.get(k, (0.0, 0))
        if n:
            gbs = b * cells / (ms / n * 1e-3) / 1e9
            out[k] = {"bytes_per_cell": b, "ms_per_launch": round(ms / n, 4), "gbs": round(gbs, 1),
                      "frac": round(gbs / peak, 3)}
    return out


def bou_text(w: dict, ntst: int) -> str:
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import bou_text as _bt  # noqa: E402  (shared bou.in template)
    return _bt(w["nxm"], w["nym"], w["nzm"], rayt=w["rayt"], prat=w["prat"], ylen=w["ylen"],
               zlen=w["zlen"], istr3=4, str3=2.0, idtv=w["idtv"], dt=w["dt"], cflmax=w["cflmax"],
               dtmax=w["dtmax"], ntst=ntst, resid=1e-3)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic_kernel(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary that covers this workload
    (profiles/<kernel>_<workload>.md, or a summary of a smaller capture whose `covers:` line names
    the workload and whose traffic is scaled to it)."""
    import glob
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", f"{kernel}_*.md"))):
        lines = open(p).read().splitlines()
        named = os.path.basename(p) == f"{kernel}_{workload}.md"
        covers = any(line.strip() == f"covers: {workload}" for line in lines)
        if named or covers:
            for line in lines:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":")[1])
    return None


def committed_traffic(workload: str):
    """DRAM bytes per launch of the fused explicit/implicit kernel from the committed ncu
    summary for this workload (profiles/), or None."""
    p = os.path.join(ROOT, "profiles", f"k_explicit_implicit_{workload}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def reduce_max(x: float, world: int) -> float:
    """Max over the ranks (timing is the slowest replica's); NCCL on GPUs, gloo on CPU."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_gpu(args):
    import numpy as np
    import torch
    import afid_gpu as ag

    world, rank, local = dist_setup()
    w = WORKLOADS[args.config]
    cells = w["nxm"] * w["nym"] * w["nzm"]
    inp = ag.parse_bou_in(bou_text(w, args.steps + args.warmup))
    tables = ag.Tables(inp, w["precision"])
    stream = torch.cuda.Stream()
    solver = ag.Solver(tables.grid, tables.params)
    solver.set_stream(stream.cuda_stream)
    if args.k1_shape >= 0:  # a saved autotuner pick (profiling runs use the bench's pick)
        solver.set_k1_shape(args.k1_shape)
        if args.k4_form >= 0:
            solver.set_k4_form(args.k4_form)
        if args.fftz_form >= 0:
            solver.set_fftz_form(args.fftz_form)
        if args.ify_form >= 0:
            solver.set_ify_form(args.ify_form)
        if args.div_form >= 0:
            solver.set_div_form(args.div_form)
    temp0 = tables.initial_temperature(20261203)
    nx, nym, nzm = w["nxm"] + 1, w["nym"], w["nzm"]
    zeros = np.zeros((nzm, nym, nx))
    solver.upload(zeros, zeros, zeros, temp0, zeros)
    ra_pr = w["prat"] * abs(w["rayt"])

    dt_box = [inp.dt]
    dtc = ctypes.c_double()
    dts = []  # dt of every step before the end-to-end run (replayed by the FP64 accuracy check)

    def step(ntime: int):
        cflm = solver.calc_max_cfl()
        dtc.value = dt_box[0]
        err = ag.lib().afid_next_dt(ctypes.byref(inp), ntime, ctypes.byref(dtc), cflm, None)
        dt_box[0] = dtc.value
        solver.time_marcher(dt_box[0], ntime)
        dts.append(dt_box[0])
        return err

    # ---- device-resident throughput ---------------------------------------------------------
    ntime = 0
    for _ in range(args.warmup):
        step(ntime)
        ntime += 1
    solver.synchronize()
    tune = solver.autotune()  # the shape the autotuner picked during the first step
    solver.profile_report()  # drop warm-up records
    solver.profile(True)
    launches0 = solver.launch_count()
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(ntime)
        ntime += 1
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    prof = solver.profile_report()
    solver.profile(False)
    launches = solver.launch_count() - launches0
    ms_max = reduce_max(ms, world)
    value = world * cells * args.steps / (ms_max * 1e-3) / 1e6

    nusselt = nusselt_numbers(solver, tables, w, ra_pr)
    k1_ms, k1_n = prof["explicit_implicit"]
    k1_avg_s = (k1_ms / k1_n) * 1e-3 if k1_n else float("nan")
    peak, peak_kind = measured_peak()
    k1_bytes = K1_BYTES_PER_CELL[w["precision"]] * cells
    achieved = k1_bytes / k1_avg_s / 1e9
    traffic = committed_traffic(w["name"])

    # ---- mixed precision: fields and Nu against an FP64 run with the same dt sequence --------
    accuracy = None
    if w["precision"] == 1 and not args.no_nu_check:
        # the run continues (untimed) to the workload's full length before the comparison
        while len(dts) < args.accuracy_steps:
            step(ntime)
            ntime += 1
        accuracy = mixed_vs_fp64(ag, w, inp, solver, temp0, list(dts), ra_pr)

    # ---- end to end through the C ABI with host buffers -----------------------------------
    pin = lambda: torch.empty((nzm, nym, nx), dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    h_in = {k: pin() for k in ("vx", "vy", "vz", "temp", "pr")}
    for k in ("vx", "vy", "vz", "pr"):
        h_in[k][...] = 0.0
    h_in["temp"][...] = temp0
    h_out = {k: pin() for k in ("vx", "vy", "vz", "temp", "pr")}
    dp = ctypes.POINTER(ctypes.c_double)
    ptr = lambda a: a.ctypes.data_as(dp)  # noqa: E731
    lib = ag.lib()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rc = lib.afid_gpu_upload(solver._h, *(ptr(h_in[k]) for k in ("vx", "vy", "vz", "temp", "pr")), nx, nym)
    assert rc == 0, rc
    dt_box[0] = inp.dt
    nu = ke = None
    for n in range(args.steps):
        step(n)
        nu, ke, _ = solver.global_quantities(ra_pr)
    rc = lib.afid_gpu_download(solver._h, *(ptr(h_out[k]) for k in ("vx", "vy", "vz", "temp", "pr")), nx, nym)
    assert rc == 0, rc
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_max(e0.elapsed_time(e1), world)
    e2e_value = world * cells * args.steps / (e2e_ms * 1e-3) / 1e6
    field_bytes = 5 * nx * nym * nzm * 8
    h2d = field_bytes / args.steps
    d2h = field_bytes / args.steps + 8 + 3 * 8

    restart = restart_io(ag, solver, inp) if (args.restart_io and rank == 0) else None

    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, args.cpu_steps, budget_s=args.cpu_budget, keep_state=w["precision"] == 0)
        if "_state" in cpu:
            solver.close()  # room for the replay
            parity = parity_vs_cpu(ag, w, inp, temp0, cpu)

    solver.close()
    tables.close()
    if rank == 0:
        line = {
            "metric": "Mcell-RK3-steps/s",
            "value": round(value, 3),
            "unit": "Mcell-RK3-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if w["precision"] == 0 else "f32+f64",
            "data": "synthetic: conductive RBC state + Philox-seeded +-1e-3 temperature perturbation",
            "config": {"workload": w["name"], "grid_xyz": [w["nxm"], w["nym"], w["nzm"]],
                       "cells": cells, "Ra": w["rayt"], "Pr": w["prat"],
                       "dt": "CFL-limited (CFLMAX 1.2, DTMAX 1e-2)" if w["idtv"] else f"fixed {w['dt']}",
                       "l2": "inputs larger than L2 (~%.1f GB resident state)" % (cells * 8 * 17 / 1e9),
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "kernel": "k_explicit_implicit",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                         "algorithmic_bytes_per_launch": k1_bytes,
                         "avg_launch_ms": round(k1_avg_s * 1e3, 4),
                         "traffic": traffic,
                         "step_frac": round(value * 1e6 * STEP_BYTES_PER_CELL / (peak * 1e9 * world), 4)},
            "kernels_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in prof.items() if v[1]},
            "kernels_roofline": kernels_roofline(prof, cells, w["precision"], peak),
            "e2e": {"value": round(e2e_value, 3), "unit": "Mcell-RK3-steps/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "note": "upload 5 fields, K steps with CFL + Nu/KE read back, download 5 fields"},
            "gpu_launches": int(launches),
            "k1_autotune": tune,
            "clocks": clk,
            "nu_vol_end": nu,
            "nusselt_after_timed_steps": nusselt,
            "cpu_baseline": cpu,
        }
        if accuracy is not None:
            line["accuracy_vs_fp64"] = accuracy
        if parity is not None:
            line["parity_vs_cpu_port"] = parity
        if restart is not None:
            line["restart_io"] = restart
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def nusselt_numbers(solver, tables, w, ra_pr):
    """Nusselt numbers of the resident state as the reference's post-processing defines them
    (tools/afidtools/boundary_layers.py:41-62): the plate values from the first and last Tbar
    rows, the dissipation value Pe * sum(chiT dx), and the volume value of GlobalQuantities."""
    import numpy as np
    prof = solver.mean_profiles()
    xm, xc = tables.array("xm"), tables.array("xc")
    nxm = w["nxm"]
    tup, tlo = (-0.5, 0.5) if w["rayt"] > 0 else (0.5, -0.5)
    lo = (prof["Tbar"][0] - tlo) / xm[0]
    up = (tup - prof["Tbar"][nxm - 1]) / (1.0 - xm[nxm - 1])
    if w["rayt"] > 0:
        lo, up = -lo, -up
    pect = np.sqrt(abs(w["rayt"]) / w["prat"]) * w["prat"]
    diss = pect * float(np.sum(prof["chiT"] * (xc[1:nxm + 1] - xc[:nxm])))
    nu_vol, ke, _ = solver.global_quantities(ra_pr)
    return {"nu_plate_lower": float(lo), "nu_plate_upper": float(up), "nu_dissipation": diss,
            "nu_volume": nu_vol, "kinetic_energy": ke}


def mixed_vs_fp64(ag, w, inp, solver, temp0, dts, ra_pr):
    """Per-field relative L2 (pressure modulo its mean) and the Nusselt-number error of the
    mixed-precision state after len(dts) steps against an FP64 solver advanced from the same
    initial state with the same dt sequence (the mixed-precision accuracy gate: Nu within 0.5%)."""
    import numpy as np
    got = solver.download()
    nu_mx, ke_mx, _ = solver.global_quantities(ra_pr)
    t64 = ag.Tables(inp, ag.PREC_FP64)
    ref = ag.Solver(t64.grid, t64.params)
    nx, nym, nzm = w["nxm"] + 1, w["nym"], w["nzm"]
    zeros = np.zeros((nzm, nym, nx))
    ref.upload(zeros, zeros, zeros, temp0, zeros)
    for n, dt in enumerate(dts):
        ref.time_marcher(dt, n)
    exp = ref.download()
    nu_64, ke_64, _ = ref.global_quantities(ra_pr)
    ref.close()
    t64.close()
    nxm = w["nxm"]

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    out = {f: rel(got[f], exp[f]) for f in ("vx", "vy", "vz", "temp")}
    pa, pb = got["pr"][..., :nxm], exp["pr"][..., :nxm]
    out["pr_mod_mean"] = rel(pa - pa.mean(), pb - pb.mean())
    return {"steps": len(dts), "rel_l2": out, "nu_vol_mixed": nu_mx, "nu_vol_fp64": nu_64,
            "nu_rel_err": abs(nu_mx - nu_64) / abs(nu_64), "ke_mixed": ke_mx, "ke_fp64": ke_64,
            "ke_rel_err": abs(ke_mx - ke_64) / max(abs(ke_64), 1e-300), "nu_within_half_pct": abs(nu_mx - nu_64) <= 0.005 * abs(nu_64),
            "note": "Nu - 1 is the signal while the flow is still near conduction: see nu_minus_1_rel_err",
            "nu_minus_1_rel_err": abs(nu_mx - nu_64) / max(abs(nu_64 - 1.0), 1e-300)}


# ---- batched sweep: independent 2-D instances of four size classes ------------------------
BATCH_SEED = 20261203
BATCH_SIZES = [(128, 64), (256, 128), (512, 256), (1024, 512)]  # (horizontal nym, wall-normal nxm)
BATCH_PR = [0.7, 1.0, 4.4]
BATCH_ASPECT = [1.0, 2.0, 4.0]


def batch_instances(n: int = 256, seed: int = BATCH_SEED):
    """Instance b draws size class, log10 Ra ~ U[6, 10], Pr and aspect ratio from the Philox
    stream keyed by ``seed`` at counters 4b .. 4b+3."""
    import afid_gpu as ag
    u = lambda b, d: ag.lib().afid_philox_uniform(seed, 4 * b + d)  # noqa: E731
    out = []
    for b in range(n):
        nym, nxm = BATCH_SIZES[min(int(u(b, 0) * 4), 3)]
        out.append(dict(index=b, nxm=nxm, nym=nym, rayt=10.0 ** (6.0 + 4.0 * u(b, 1)),
                        prat=BATCH_PR[min(int(u(b, 2) * 3), 2)], ylen=BATCH_ASPECT[min(int(u(b, 3) * 3), 2)]))
    return out


def diffusive_dtmax(nym: int, ylen: float, rayt: float, prat: float, cap: float = 1e-2) -> float:
    """DTMAX of an instance: AFiD integrates the horizontal diffusion explicitly (ExplicitTerms*),
    so RK3 needs dt < 0.63 dy^2 min(Re, Pe) (the real-axis stability bound 2.51 over the largest
    eigenvalue 4 / (dy^2 Re)); the main-loop dt rule has only the CFL bound.  Half of it, capped
    at 1e-2."""
    dy = ylen / nym
    re, pe = math.sqrt(rayt / prat), math.sqrt(rayt * prat)
    return min(cap, 0.5 * dy * dy * min(re, pe))


def batch_bou(inst: dict) -> str:
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import bou_text as _bt  # noqa: E402
    dtmax = diffusive_dtmax(inst["nym"], inst["ylen"], inst["rayt"], inst["prat"])
    return _bt(inst["nxm"], inst["nym"], 1, rayt=inst["rayt"], prat=inst["prat"], ylen=inst["ylen"],
               zlen=1.0, istr3=4, str3=2.0, idtv=1, dt=min(1e-4, dtmax), cflmax=1.2, dtmax=dtmax,
               ntst=1000000, resid=1e-3)


class BatchSet:
    """One ag.Batch per size class, each on its own stream; a step forks from and joins to a
    master stream so the classes overlap on the device.

    With ``group_bytes`` > 0 each class is split into groups whose device state stays under that
    many bytes (so that a group fits the L2 cache), one ag.Batch per group, and a step of ``n``
    runs group after group, each group ``n`` steps in a row, consecutive groups alternating
    between ``lanes`` streams: the state of a group stays in L2 across its steps instead of
    streaming through HBM every step.  Instances are independent, so the grouping changes the
    schedule only."""

    def __init__(self, instances, precision: int, group_bytes: int = 0, lanes: int = 2):
        import torch
        import afid_gpu as ag
        self.classes = {}
        for inst in instances:
            self.classes.setdefault((inst["nxm"], inst["nym"]), []).append(inst)
        self.master = torch.cuda.Stream()
        self.batches, self.class_of = [], []
        grouped = group_bytes > 0
        for key in sorted(self.classes):
            members = self.classes[key]
            if grouped:
                # device bytes of one slot, from a batch of one of this class
                with ag.Batch(ag.parse_bou_in(batch_bou(members[0])), 1, precision) as probe:
                    per = max(1, probe.device_bytes())
                size = max(1, int(group_bytes // per))
                parts = [members[i:i + size] for i in range(0, len(members), size)]
            else:
                parts = [members]
            for part in parts:
                b = ag.Batch(ag.parse_bou_in(batch_bou(part[0])), len(part), precision)
                for slot, inst in enumerate(part):
                    b.configure(slot, ag.parse_bou_in(batch_bou(inst)))
                    b.seed(slot, BATCH_SEED + 1 + inst["index"])
                b.set_active([1] * len(part))
                self.batches.append(b)
                self.class_of.append(key)
        nstreams = lanes if grouped else len(self.batches)
        self.streams = [torch.cuda.Stream() for _ in range(nstreams)]
        for q, b in enumerate(self.batches):
            b.set_stream(self.streams[q % nstreams].cuda_stream)
        self.cells = sum(i["nxm"] * i["nym"] for i in instances)

    def step(self, n: int = 1):
        import torch
        fork = torch.cuda.Event()
        fork.record(self.master)
        for s in self.streams:
            s.wait_event(fork)
        for b in self.batches:
            b.step(n)
        for s in self.streams:
            e = torch.cuda.Event()
            e.record(s)
            self.master.wait_event(e)

    def autotune(self):
        out = {}
        for key, b in zip(self.class_of, self.batches):
            name = f"{key[1]}x{key[0]}"
            if name not in out:
                out[name] = b.autotune()
        return out

    def stats(self):
        return [b.stats() for b in self.batches]

    def launches(self):
        return sum(b.launch_count() for b in self.batches)

    def device_bytes(self):
        return sum(b.device_bytes() for b in self.batches)

    def close(self):
        for b in self.batches:
            b.close()


def run_batched(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup()
    insts = batch_instances(args.instances)
    precision = 1 if args.config == "batched" else 0
    group_bytes = int(args.l2_group_mb * 1e6)
    chunk = max(1, args.group_steps) if group_bytes else 1
    if args.steps % chunk:
        args.steps += chunk - args.steps % chunk  # whole visits of every group
    bs = BatchSet(insts, precision, group_bytes)
    for _ in range(args.warmup):
        bs.step()
    torch.cuda.synchronize()
    tune = bs.autotune()
    l0 = bs.launches()
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(bs.master)
    for _ in range(args.steps // chunk):
        bs.step(chunk)
    ev1.record(bs.master)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = reduce_max(ev0.elapsed_time(ev1), world)
    launches = bs.launches() - l0
    value = world * bs.cells * args.steps / (ms * 1e-3) / 1e6
    st = bs.stats()
    nsteps_done = int(min(int(s["ntime"].min()) for s in st))
    errors = int(sum(int((s["errorcode"] != 0).sum()) for s in st))
    nu = np.concatenate([s["nu_vol"] for s in st])
    bs_bytes = bs.device_bytes()
    bs.close()

    # Nusselt of the same instances and steps on the FP64 path (untimed) for the error gate
    nu_err = None
    if precision == 1 and not args.no_nu_check:
        ref = BatchSet(insts, 0)
        for _ in range(args.warmup + args.steps):
            ref.step()
        torch.cuda.synchronize()
        nu64 = np.concatenate([s["nu_vol"] for s in ref.stats()])
        ref.close()
        ok = np.isfinite(nu) & np.isfinite(nu64)
        rel = np.abs(nu[ok] - nu64[ok]) / np.abs(nu64[ok])
        nu_err = {"max": float(rel.max()), "median": float(np.median(rel)),
                  "within_0.5pct": int((rel <= 5e-3).sum()), "compared": int(ok.sum()),
                  "note": "instantaneous Nu_vol after the timed steps, mixed vs FP64 batch"}

    if rank == 0:
        counts = {f"{k[1]}x{k[0]}": len(v) for k, v in sorted(bs.classes.items())}
        line = {
            "metric": "Mcell-RK3-steps/s",
            "value": round(value, 3),
            "unit": "Mcell-RK3-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64" if precision else "f64",
            "data": "synthetic: 256 Philox-drawn 2-D RBC instances, conductive state + seeded +-1e-3 perturbation",
            "config": {"workload": f"batched_{len(insts)}x2d_" + ("mixed" if precision else "fp64"),
                       "instances": len(insts), "cells": bs.cells, "classes_nymxnxm": counts,
                       "schedule": (f"L2 groups of <= {args.l2_group_mb:g} MB, {chunk} steps per group visit, "
                                    f"{len(bs.batches)} groups" if group_bytes else "one batch per class, stepped together"),
                       "dt": "CFL-limited per instance (CFLMAX 1.2; DTMAX = min(1e-2, 0.5 dy^2 min(Re, Pe)))",
                       "l2": "inputs larger than L2 (%.1f GB resident)" % (bs_bytes / 1e9),
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "gpu_launches": int(launches),
            "k1_autotune": tune,
            "clocks": clk,
            "steps_done_min": nsteps_done,
            "instances_with_error": errors,
            "instances_nonfinite": int((~np.isfinite(nu)).sum()),
            "nu_rel_err_max_vs_fp64": nu_err,
            "device_bytes": int(bs_bytes),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---- served stream: Poisson arrivals of 2-D and 3-D jobs -----------------------------------
SERVE_SEED = BATCH_SEED + 1


def serve_jobs(n: int, rate: float = 50.0, seed: int = SERVE_SEED):
    """Job j draws from the Philox stream keyed by ``seed`` at counters 8j .. 8j+7: exponential
    inter-arrival at ``rate``/s, 2-D (90%, sizes/Ra/Pr/aspect as the batched sweep) or 3-D
    (96 x 128 x 128 wall-normal x horizontal, log10 Ra ~ U[6, 8], Pr 1), steps ~ U[500, 5000]."""
    import afid_gpu as ag
    u = lambda j, d: ag.lib().afid_philox_uniform(seed, 8 * j + d)  # noqa: E731
    jobs, t = [], 0.0
    for j in range(n):
        t += -math.log(1.0 - u(j, 0)) / rate
        nsteps = 500 + min(int(u(j, 1) * 4501), 4500)
        if u(j, 2) < 0.9:
            nym, nxm = BATCH_SIZES[min(int(u(j, 3) * 4), 3)]
            job = dict(nxm=nxm, nym=nym, nzm=1, rayt=10.0 ** (6.0 + 4.0 * u(j, 4)),
                       prat=BATCH_PR[min(int(u(j, 5) * 3), 2)], ylen=BATCH_ASPECT[min(int(u(j, 6) * 3), 2)],
                       zlen=1.0)
        else:
            job = dict(nxm=96, nym=128, nzm=128, rayt=10.0 ** (6.0 + 2.0 * u(j, 4)), prat=1.0, ylen=1.0, zlen=1.0)
        job.update(index=j, arrival=t, nsteps=nsteps, seed=SERVE_SEED + 1 + j)
        jobs.append(job)
    return jobs


def serve_bou(job: dict) -> str:
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import bou_text as _bt  # noqa: E402
    dtmax = diffusive_dtmax(job["nym"], job["ylen"], job["rayt"], job["prat"])
    if job["nzm"] > 1:
        dtmax = min(dtmax, diffusive_dtmax(job["nzm"], job["zlen"], job["rayt"], job["prat"]))
    return _bt(job["nxm"], job["nym"], job["nzm"], rayt=job["rayt"], prat=job["prat"], ylen=job["ylen"],
               zlen=job["zlen"], istr3=4, str3=2.0, idtv=1, dt=min(1e-4, dtmax), cflmax=1.2, dtmax=dtmax,
               ntst=1000000, resid=1e-3)


def run_served(args):
    import numpy as np
    import torch
    import afid_gpu as ag

    world, rank, local = dist_setup()
    jobs = serve_jobs(args.jobs, rate=args.rate)
    inputs = [ag.parse_bou_in(serve_bou(j)) for j in jobs]
    policy = ag.SERVE_SHORTEST_FIRST if args.policy == "shortest" else ag.SERVE_FIFO
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(free * 0.8, 120e9))
    srv = ag.Server(ag.PREC_MIXED, hbm_budget_bytes=budget, slots_per_pool=args.slots, chunk_steps=args.chunk,
                    max_cells_in_flight=args.max_cells, policy=policy)
    # warm-up: a few 3-step jobs (device context, allocator, first captures)
    for k, inp in enumerate(inputs[: min(4, len(inputs))]):
        srv.submit(inp, 1, 3, 10_000_000 + k)
    while True:
        srv.pump()
        srv.poll()
        st = srv.status()
        if st["running"] + st["queued"] == 0:
            break
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t0 = srv.now()
    nxt, results = 0, {}
    while len(results) < len(jobs):
        now = srv.now() - t0
        while nxt < len(jobs) and jobs[nxt]["arrival"] <= now:
            srv.submit(inputs[nxt], jobs[nxt]["seed"], jobs[nxt]["nsteps"], nxt)
            nxt += 1
        st = srv.status()
        if st["running"] == 0 and st["queued"] == 0 and nxt < len(jobs):
            time.sleep(max(0.0, jobs[nxt]["arrival"] - (srv.now() - t0)))
            continue
        srv.pump()
        for r in srv.poll():
            results[r["tag"]] = r
    t_end = srv.now() - t0
    torch.cuda.synchronize()
    clk = clocks.stop()
    status = srv.status()
    srv.close()
    lat = np.array([results[j["index"]]["t_done"] - t0 - j["arrival"] for j in jobs])
    wait = np.array([results[j["index"]]["t_admit"] - t0 - j["arrival"] for j in jobs])
    cell_steps = sum(j["nxm"] * j["nym"] * j["nzm"] * results[j["index"]]["steps_done"] for j in jobs)
    value = cell_steps / t_end / 1e6
    errors = sum(1 for r in results.values() if r["errorcode"] != 0)
    error_codes = {}
    for j in jobs:
        c = int(results[j["index"]]["errorcode"])
        if c:
            key = f"{c} ({j['nym']}x{j['nxm']}x{j['nzm']})"
            error_codes[key] = error_codes.get(key, 0) + 1
    offered = sum(j["nxm"] * j["nym"] * j["nzm"] * j["nsteps"] for j in jobs) / jobs[-1]["arrival"] / 1e6
    if rank == 0:
        line = {
            "metric": "Mcell-RK3-steps/s; p50/p99 job latency",
            "value": round(value, 3),
            "unit": "Mcell-RK3-steps/s",
            "n_gpus": world,
            "steps": len(jobs),
            "warmup": 4,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64",
            "data": f"synthetic: Poisson arrivals ({args.rate:g}/s), Philox-drawn 2-D/3-D RBC jobs, seeded conductive IC",
            "config": {"workload": f"served_{len(jobs)}jobs_poisson{args.rate:g}", "jobs": len(jobs),
                       "arrival_rate_per_s": args.rate,
                       "mix": {"2d": sum(1 for j in jobs if j["nzm"] == 1), "3d_96x128x128": sum(1 for j in jobs if j["nzm"] > 1)},
                       "policy": args.policy, "chunk_steps": args.chunk, "slots_per_pool": args.slots,
                       "max_cells_in_flight": args.max_cells, "hbm_budget_bytes": budget,
                       "offered_load_mcell_steps_per_s": round(offered, 1),
                       "l2": "resident state larger than L2",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "latency_s": {"p50": round(float(np.percentile(lat, 50)), 3), "p99": round(float(np.percentile(lat, 99)), 3),
                          "mean": round(float(lat.mean()), 3), "max": round(float(lat.max()), 3)},
            "queue_wait_s": {"p50": round(float(np.percentile(wait, 50)), 3), "p99": round(float(np.percentile(wait, 99)), 3)},
            "horizon_s": round(t_end, 3),
            "e2e": {"value": round(value, 3), "unit": "Mcell-RK3-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0,
                    "note": "served loop: host submission -> result on host; initial states built on the host and uploaded per job"},
            "jobs_with_error": errors,
            "error_codes": error_codes,
            "pool_failures": status["pool_failures"],
            "last_cuda_error": status["last_cuda_error"],
            "peak_device_bytes": status["device_bytes"],
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---- double-diffusive convection with the multi-resolution salinity scalar ------------------
# Coarse flow + temperature grid as rbc3d, salinity on a grid refined 2x in every direction
# (MULTIRES = FLAGSAL = 1), both scalars active along x, salinity free-fall scaling (FFscaleS = 1),
# Le = PraS / Pr = 10; the reference's bounded double-diffusive initial salinity
# 0.5 (2 (xmr - 0.5))^7 (salinity.F90:148-157) and the conductive temperature + noise.
DDC_WORKLOADS = {
    "ddc3d": dict(nxm=256, nym=384, nzm=384, nxmr=512, nymr=768, nzmr=768, rayt=1e8, prat=7.0, rays=1e9,
                  pras=70.0, name="ddc3d_384x384x256_refined_768x768x512_fp64"),
    # 1/8 of the refined cells (33.6 M, 2.2 GB of refined fields) for ncu captures
    "ddc3d_small": dict(nxm=256, nym=128, nzm=128, nxmr=512, nymr=256, nzmr=256, rayt=1e8, prat=7.0, rays=1e9,
                        pras=70.0, name="ddc3d_128x128x256_refined_256x256x512_fp64"),
}
# Algorithmic HBM bytes per refined cell of k_sal_step: read sal, vxr, vyr, vzr, rusal, write
# sal_o, rusal (7 x 8 B).
SAL_STEP_BYTES_PER_CELL = 56


def ddc_bou_text(w: dict, ntst: int) -> str:
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import bou_text as _bt  # noqa: E402
    return _bt(w["nxm"], w["nym"], w["nzm"], rayt=w["rayt"], prat=w["prat"], ylen=1.0, zlen=1.0, istr3=4,
               str3=2.0, idtv=1, dt=1e-4, cflmax=1.2, dtmax=1e-2, ntst=ntst, resid=1e-3, multires=1,
               nxmr=w["nxmr"], nymr=w["nymr"], nzmr=w["nzmr"], flagsal=1, istr3r=4, rays=w["rays"],
               pras=w["pras"], ffscales=1, active_s=1)


def ddc_cpu_baseline(budget_s: float = 30.0):
    """The C + OpenMP restatement with the salinity scalar (oracle/afid_cpu.c) on all host cores,
    main-loop steps of the ddc3d_small workload (same kernels, 1/9 of the cells) until
    ``budget_s`` seconds are spent."""
    try:
        from oracle import cpu_port
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"CPU port not importable: {e}"}
    w = DDC_WORKLOADS["ddc3d_small"]
    res = cpu_port.time_steps_sal(ddc_bou_text(w, 10), 10, seed=20261203, budget_s=budget_s)
    return {"value": round(res["mcells_per_s"], 4), "unit": "Mcell-RK3-steps/s", "cores": res["threads"],
            "kind": "port", "sample": f"{res['steps']} full steps of {w['name']} (C+OpenMP restatement)",
            "steps": res["steps"], "seconds": round(res["seconds"], 2)}


def run_ddc(args):
    import numpy as np
    import torch
    import afid_gpu as ag

    world, rank, local = dist_setup()
    w = DDC_WORKLOADS[args.config]
    cells = w["nxm"] * w["nym"] * w["nzm"]
    rcells = w["nxmr"] * w["nymr"] * w["nzmr"]
    inp = ag.parse_bou_in(ddc_bou_text(w, args.steps + args.warmup))
    tables = ag.Tables(inp, ag.PREC_FP64)
    mgrd = ag.Mgrd(tables)
    stream = torch.cuda.Stream()
    solver = ag.Solver(tables.grid, tables.params)
    solver.set_stream(stream.cuda_stream)
    if args.k1_shape >= 0:
        solver.set_k1_shape(args.k1_shape)
    solver.sal_create(mgrd)
    temp0 = tables.initial_temperature(20261203)
    sal0 = mgrd.initial_salinity(20261204)
    nx, nym, nzm = w["nxm"] + 1, w["nym"], w["nzm"]
    zeros = np.zeros((nzm, nym, nx))
    solver.upload(zeros, zeros, zeros, temp0, zeros)
    solver.sal_upload(sal0)
    dt_box = [inp.dt]
    dtc = ctypes.c_double()

    def step(ntime: int):
        cflmr = solver.sal_cfl()  # main.F90:285-293: the dt rule takes CFLmr with salinity on
        dtc.value = dt_box[0]
        err = ag.lib().afid_next_dt(ctypes.byref(inp), ntime, ctypes.byref(dtc), cflmr, None)
        dt_box[0] = dtc.value
        solver.time_marcher(dt_box[0], ntime)
        return err

    ntime = 0
    for _ in range(args.warmup):
        step(ntime)
        ntime += 1
    solver.synchronize()
    tune = solver.autotune()
    solver.profile_report()
    solver.profile(True)
    launches0 = solver.launch_count()
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(ntime)
        ntime += 1
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms_max = reduce_max(ev0.elapsed_time(ev1), world)
    prof = solver.profile_report()
    solver.profile(False)
    launches = solver.launch_count() - launches0
    value = world * cells * args.steps / (ms_max * 1e-3) / 1e6
    s_ms, s_n = prof["sal_step"]
    s_avg = (s_ms / s_n) * 1e-3 if s_n else float("nan")
    peak, peak_kind = measured_peak()
    s_bytes = SAL_STEP_BYTES_PER_CELL * rcells
    achieved = s_bytes / s_avg / 1e9
    prof_s = solver.sal_profiles()
    # solutal Nusselt numbers as tools/afidtools/boundary_layers.py:64-81 defines them
    xmr, xcr = mgrd.array("xmr"), mgrd.array("xcr")
    sup, slo = (0.5, -0.5) if w["rays"] > 0 else (-0.5, 0.5)
    nus_lo = (prof_s["Sbar"][0] - slo) / xmr[0]
    nus_up = (sup - prof_s["Sbar"][-1]) / (1.0 - xmr[-1])
    if w["rays"] < 0:
        nus_lo, nus_up = -nus_lo, -nus_up
    ren = (abs(w["rays"]) / w["pras"]) ** 0.5  # FFscaleS = 1
    nus = {"nu_s_plate_lower": float(nus_lo), "nu_s_plate_upper": float(nus_up),
           "nu_s_dissipation": float(ren * w["pras"] * (prof_s["chiS"] * (xcr[1:] - xcr[:-1])).sum())}

    # ---- end to end through the C ABI with host buffers -----------------------------------
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    h_in = {k: pin((nzm, nym, nx)) for k in ("vx", "vy", "vz", "temp", "pr")}
    for k in ("vx", "vy", "vz", "pr"):
        h_in[k][...] = 0.0
    h_in["temp"][...] = temp0
    h_out = {k: pin((nzm, nym, nx)) for k in ("vx", "vy", "vz", "temp", "pr")}
    rshape = (w["nzmr"], w["nymr"], w["nxmr"])
    h_sal, h_sal_out = pin(rshape), pin(rshape)
    h_sal[...] = sal0
    dp = ctypes.POINTER(ctypes.c_double)
    ptr = lambda a: a.ctypes.data_as(dp)  # noqa: E731
    lib = ag.lib()
    ra_pr = w["prat"] * abs(w["rayt"])
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    assert lib.afid_gpu_upload(solver._h, *(ptr(h_in[k]) for k in ("vx", "vy", "vz", "temp", "pr")), nx, nym) == 0
    assert lib.afid_gpu_sal_upload(solver._h, ptr(h_sal), w["nxmr"], w["nymr"]) == 0
    dt_box[0] = inp.dt
    nu = None
    for n in range(args.steps):
        step(n)
        nu, _, _ = solver.global_quantities(ra_pr)
    assert lib.afid_gpu_download(solver._h, *(ptr(h_out[k]) for k in ("vx", "vy", "vz", "temp", "pr")), nx, nym) == 0
    assert lib.afid_gpu_sal_download(solver._h, ptr(h_sal_out), w["nxmr"], w["nymr"]) == 0
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_max(e0.elapsed_time(e1), world)
    e2e_value = world * cells * args.steps / (e2e_ms * 1e-3) / 1e6
    io_bytes = 5 * nx * nym * nzm * 8 + rcells * 8
    finite = bool(np.isfinite(h_sal_out).all() and np.isfinite(h_out["vx"]).all())

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = ddc_cpu_baseline()
    solver.close()
    mgrd.close()
    tables.close()
    if rank == 0:
        line = {
            "metric": "Mcell-RK3-steps/s",
            "value": round(value, 3),
            "unit": "Mcell-RK3-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic: conductive temperature + Philox noise, double-diffusive salinity profile",
            "config": {"workload": w["name"], "grid_xyz": [w["nxm"], w["nym"], w["nzm"]],
                       "refined_xyz": [w["nxmr"], w["nymr"], w["nzmr"]], "cells": cells, "refined_cells": rcells,
                       "refined_value": round(world * rcells * args.steps / (ms_max * 1e-3) / 1e6, 3),
                       "RaT": w["rayt"], "Pr": w["prat"], "RaS": w["rays"], "PraS": w["pras"],
                       "dt": "CFL-limited on the refined grid (CFLMAX 1.2, DTMAX 1e-2)",
                       "l2": "inputs larger than L2 (~%.1f GB resident)" % ((cells * 21 + rcells * 8) * 8 / 1e9),
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "kernel": "k_sal_step", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                         "algorithmic_bytes_per_launch": s_bytes, "avg_launch_ms": round(s_avg * 1e3, 4),
                         "traffic": committed_traffic_kernel("k_sal_step", w["name"])},
            "kernels_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in prof.items() if v[1]},
            "e2e": {"value": round(e2e_value, 3), "unit": "Mcell-RK3-steps/s",
                    "h2d_bytes_per_step": int(io_bytes / args.steps),
                    "d2h_bytes_per_step": int(io_bytes / args.steps + 8 + 3 * 8),
                    "note": "upload 5 fields + salinity, K steps with CFLmr + Nu/KE read back, download all"},
            "gpu_launches": int(launches),
            "k1_autotune": tune,
            "clocks": clk,
            "nu_vol_end": nu,
            "sbar_range": [float(prof_s["Sbar"].min()), float(prof_s["Sbar"].max())],
            "solutal_nusselt_after_timed_steps": nus,
            "finite": finite,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---- the reference's published Rayleigh-Benard example -------------------------------------
# docs/examples/rbc.md: Ra = 1e8, Pr = 10, 128^3 cells for the velocity and 384^3 refined cells for
# the scalar that plays the temperature (the salinity field, active_S = 1, with the temperature
# switched off as a buoyancy source, active_T = 0), free-fall units of the scalar (FFscaleS = 1);
# grids and time stepping of examples/RayleighBenardConvection/bou.in (clipped Chebyshev
# wall-normal coarse grid ISTR3 = 6, STR3 = 12, uniform refined grid ISTR3R = 0, CFLMAX 1,
# DTMAX 1e-2).  The reference publishes the five Nusselt numbers of tools/plot_time_series.py over
# t = 0 .. 200 (docs/figures/Nusselt.svg, digitised in tests/golden/).
PUBLISHED = dict(nxm=128, nym=128, nzm=128, nxmr=384, nymr=384, nzmr=384, rays=1e8, pras=10.0,
                 name="rbc3d_sal_128cubed_refined_384cubed_ra1e8_pr10")


def published_bou_text(t_end: float) -> str:
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import bou_text as _bt  # noqa: E402
    w = PUBLISHED
    return _bt(w["nxm"], w["nym"], w["nzm"], rayt=1e8, prat=1.0, ylen=1.0, zlen=1.0, istr3=6, str3=12.0,
               idtv=1, dt=1e-2, cflmax=1.0, dtmax=1e-2, ntst=10_000_000, tmax=t_end, resid=1e-3, multires=1,
               nxmr=w["nxmr"], nymr=w["nymr"], nzmr=w["nzmr"], flagsal=1, istr3r=0, rays=w["rays"],
               pras=w["pras"], ffscales=1, active_s=1, active_t=0, tout=0.2, tframe=1.0)


def run_published(args):
    """The published example on the device from a seeded start to t = args.t_end: the main loop
    (CFLmr -> dt rule -> TimeMarcher) with the Nusselt and Reynolds numbers of
    tools/plot_time_series.py sampled every args.sample_dt, their averages from t = 75 against the
    digitised figures."""
    import numpy as np
    import torch
    import afid_gpu as ag

    world, rank, local = dist_setup()
    w = PUBLISHED
    inp = ag.parse_bou_in(published_bou_text(args.t_end))
    tables = ag.Tables(inp, ag.PREC_FP64)
    mgrd = ag.Mgrd(tables)
    solver = ag.Solver(tables.grid, tables.params)
    solver.sal_create(mgrd)
    nx, nym, nzm = w["nxm"] + 1, w["nym"], w["nzm"]
    zeros = np.zeros((nzm, nym, nx))
    solver.upload(zeros, zeros, zeros, tables.initial_temperature(args.seed), zeros)
    solver.sal_upload(mgrd.initial_salinity(args.seed + 1))
    xmr, xcr, xc = mgrd.array("xmr"), mgrd.array("xcr"), tables.array("xc")
    dxr, dxc = xcr[1:] - xcr[:-1], xc[1:w["nxm"] + 1] - xc[:w["nxm"]]
    pec = (w["rays"] * w["pras"]) ** 0.5

    inu = (w["rays"] / w["pras"]) ** 0.5

    def sample():  # tools/plot_time_series.py:17-35 (Nusselt), :50-61 (Reynolds)
        ps, pf = solver.sal_profiles(), solver.mean_profiles()
        re_v = float((pf["vxrms"] ** 2 * dxc).sum()) ** 0.5 * inu
        re_h = float(((pf["vyrms"] ** 2 + pf["vzrms"] ** 2) * dxc).sum()) ** 0.5 * inu
        return {"nu_pl": (0.5 + ps["Sbar"][0]) / xmr[0], "nu_pu": (0.5 - ps["Sbar"][-1]) / (1.0 - xmr[-1]),
                "nu_chi": float((ps["chiS"] * dxr).sum()) * pec,
                "nu_eps": 1.0 + float((pf["epsilon"] * dxc).sum()) * pec,
                "nu_vol": 1.0 - float((ps["vxS"] * dxr).sum()) * pec,
                "re_v": re_v, "re_h": re_h, "re_t": (re_v ** 2 + re_h ** 2) ** 0.5}

    dtc = ctypes.c_double(inp.dt)
    t, n, err = 0.0, 0, 0
    times, series = [], {k: [] for k in ("nu_pl", "nu_pu", "nu_chi", "nu_eps", "nu_vol", "re_v", "re_h", "re_t")}
    next_sample = args.sample_dt
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while t < args.t_end and err == 0:
        err = ag.lib().afid_next_dt(ctypes.byref(inp), n, ctypes.byref(dtc), solver.sal_cfl(), None)
        solver.time_marcher(dtc.value, n)
        t += dtc.value
        n += 1
        if t >= next_sample - 1e-12:
            for k, v in sample().items():
                series[k].append(float(v))
            times.append(t)
            next_sample += args.sample_dt
    solver.synchronize()
    wall = time.perf_counter() - t0
    solver.close()
    tables.close()
    with open(os.path.join(ROOT, "tests", "golden", "published_rbc_ra1e8_pr10.json")) as f:
        pub = json.load(f)
    tt = np.array(times)
    ours = {}
    for k, v in series.items():
        v = np.array(v)
        m = tt >= 75.0
        ours[k] = float(np.trapezoid(v[m], tt[m]) / (tt[m][-1] - tt[m][0])) if m.sum() > 1 else float("nan")
    ref = dict(pub["nusselt"]["mean_from_75"], **pub["reynolds"]["mean_from_75"])
    line = {"metric": "Nusselt and Reynolds numbers of the reference's published RBC example, averaged over t >= 75",
            "config": {"workload": w["name"], "t_end": args.t_end, "steps": n, "sample_dt": args.sample_dt,
                       "data": "synthetic seeded start (the statistically steady state is what is compared)"},
            "errorcode": err, "wall_s": round(wall, 1), "mean_from_75": {k: round(v, 3) for k, v in ours.items()},
            "published_mean_from_75": ref,
            "rel_diff": {k: round(abs(ours[k] - ref[k]) / ref[k], 4) for k in ref},
            "series_every": args.sample_dt,
            "series": {"t": [round(x, 3) for x in times], **{k: [round(x, 3) for x in v] for k, v in series.items()}}}
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_baseline(w: dict, steps: int, budget_s: float = 60.0, keep_state: bool = False, warmup: int = 0):
    """The CPU restatement (C + OpenMP, oracle/afid_cpu.c) on the same workload: ``warmup``
    untimed main-loop steps, then up to ``steps`` timed ones, stopping once ``budget_s`` seconds
    have been spent.  With ``keep_state`` the final fields and dt sequence come back under
    "_state" / "_dts"."""
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import cpu_port
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"CPU port not importable: {e}"}
    text = bou_text(w, steps + warmup)
    res = cpu_port.time_steps(text, steps, seed=20261203, mixed=False, budget_s=budget_s, keep_state=keep_state,
                              warmup=warmup)
    out = {"value": round(res["mcells_per_s"], 4), "unit": "Mcell-RK3-steps/s",
           "cores": res["threads"], "kind": "port",
           "sample": f"{res['steps']} full steps of {w['name']} (C+OpenMP restatement)",
           "steps": res["steps"], "seconds": round(res["seconds"], 2)}
    if keep_state:
        out["_state"], out["_dts"], out["_stats"] = res["state"], res["dts"], res["stats"]
    return out


def restart_io(ag, solver, inp):
    """The restart files of the resident state: WriteFlowField (download + HDF5 write of the five
    continua files and the master file) and ReadFlowInterp's same-grid branch (HDF5 read +
    upload), host wall clock; the state read back must equal the state written."""
    import shutil
    import tempfile

    import numpy as np
    d = tempfile.mkdtemp(prefix="afid_continua_")
    try:
        before = solver.download()
        master = ag.continua_master(inp, 0.0)
        t0 = time.perf_counter()
        solver.write_flow_field(d, master, final=True)
        t1 = time.perf_counter()
        _, interpolated = solver.read_flow_interp(d, inp)
        solver.synchronize()
        t2 = time.perf_counter()
        after = solver.download()
        exact = all(np.array_equal(before[k], after[k]) for k in before)
        nbytes = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return {"bytes": nbytes, "write_s": round(t1 - t0, 3), "read_s": round(t2 - t1, 3),
            "write_GBps": round(nbytes / (t1 - t0) / 1e9, 2), "read_GBps": round(nbytes / (t2 - t1) / 1e9, 2),
            "interpolated": interpolated, "roundtrip_exact": exact,
            "note": "continua_{vx,vy,vz,temp,pr}.h5 + continua_master.h5 in a temporary directory on the "
                    "host's local disk (page cache), via afid_gpu_write_flow_field / afid_gpu_read_flow_interp"}


def parity_vs_cpu(ag, w, inp, temp0, cpu):
    """The default workload at full size against the C restatement: the GPU path replays its dt
    sequence from the same initial state.  Fields after the last step: relative L2 per field
    (pressure modulo its mean).  Over the run: Nu_vol, the plate Nusselt numbers and the kinetic
    energy after every step (GlobalQuantities; boundary_layers.py:41-54 from the Tbar rows), their
    largest relative difference and the relative difference of their run averages (gate 1%)."""
    import numpy as np
    from oracle.cpu_port import plate_and_volume_stats
    from oracle import afid_oracle as o
    state, dts, cstats = cpu.pop("_state"), cpu.pop("_dts"), cpu.pop("_stats")
    p = o.parse_bou_in(bou_text(w, len(dts)))
    xm = o.create_grid(p).xm
    ra_pr = w["prat"] * abs(w["rayt"])
    t = ag.Tables(inp, w["precision"])
    sv = ag.Solver(t.grid, t.params)
    nx, nym, nzm = w["nxm"] + 1, w["nym"], w["nzm"]
    zeros = np.zeros((nzm, nym, nx))
    sv.upload(zeros, zeros, zeros, temp0, zeros)
    gstats = []
    for n, dt in enumerate(dts):
        sv.time_marcher(dt, n)
        nu, ke, _ = sv.global_quantities(ra_pr)
        tbar = sv.mean_profiles()["Tbar"]
        gstats.append(plate_and_volume_stats(p, xm, nu, ke, tbar[0], tbar[w["nxm"] - 1]))
    got = sv.download()
    sv.close()
    t.close()
    series = {}
    for k in ("nu_vol", "nu_plate_lower", "nu_plate_upper", "ke"):
        a = np.array([g[k] for g in gstats])
        b = np.array([c[k] for c in cstats])
        series[k] = {"gpu_mean": float(a.mean()), "cpu_mean": float(b.mean()),
                     "mean_rel_diff": float(abs(a.mean() - b.mean()) / abs(b.mean())),
                     "max_rel_diff": float(np.max(np.abs(a - b) / np.abs(b))),
                     "cpu_last": float(b[-1])}
    series["within_1pct"] = all(v["mean_rel_diff"] <= 0.01 for v in series.values())

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    nxm = w["nxm"]
    out = {f: rel(got[f], state[f]) for f in ("vx", "vy", "vz", "temp")}
    pa, pb = got["pr"][..., :nxm], state["pr"][..., :nxm]
    out["pr_mod_mean"] = rel(pa - pa.mean(), pb - pb.mean())
    return {"steps": len(dts), "rel_l2": out, "tolerance": 1e-10, "nu_ke_over_run": series,
            "against": "C + OpenMP restatement (oracle/afid_cpu.c), same initial state and dt sequence"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.config in DDC_WORKLOADS:
        w = DDC_WORKLOADS[args.config]
        cpu = ddc_cpu_baseline(budget_s=120.0)
    elif args.config in WORKLOADS:
        w = WORKLOADS[args.config]
        cpu = cpu_baseline(w, args.steps, budget_s=120.0, warmup=args.warmup)
    else:
        print(json.dumps({"impl": "reference", "unavailable": f"no CPU arm for the {args.config} workload"}),
              flush=True)
        return
    if "unavailable" in cpu:
        print(json.dumps({"impl": "reference", "unavailable": cpu["unavailable"]}), flush=True)
        return
    line = {
        "impl": "reference",
        "metric": "Mcell-RK3-steps/s",
        "value": cpu["value"],
        "unit": "Mcell-RK3-steps/s",
        "n_gpus": world,
        "steps": cpu.get("steps"),
        "steps_requested": args.steps if args.config in WORKLOADS else None,
        "warmup": args.warmup if args.config in WORKLOADS else 0,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: conductive RBC state + Philox-seeded +-1e-3 temperature perturbation",
        "config": {"workload": w["name"], "grid_xyz": [w["nxm"], w["nym"], w["nzm"]]},
        "cpu_baseline": cpu,
        "e2e": {"value": cpu["value"], "unit": "Mcell-RK3-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="afid", choices=["afid", "reference"])
    ap.add_argument("--config", default="rbc3d",
                    choices=sorted(WORKLOADS) + sorted(DDC_WORKLOADS) + ["batched", "batched_fp64", "served",
                                                                         "published_rbc"])
    ap.add_argument("--t-end", type=float, default=200.0, help="published_rbc: simulated time to reach")
    ap.add_argument("--sample-dt", type=float, default=0.5, help="published_rbc: time between Nusselt samples")
    ap.add_argument("--seed", type=int, default=20261203, help="published_rbc: seed of the initial perturbations")
    ap.add_argument("--no-nu-check", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=500,
                    help="rbc3d_mixed: steps of the mixed run compared with the FP64 replay (500 = the full run)")
    ap.add_argument("--k1-shape", type=int, default=-1, help="fixed K1 thread shape instead of autotuning")
    ap.add_argument("--k4-form", type=int, default=-1, help="with --k1-shape: fixed Poisson tridiagonal form")
    ap.add_argument("--fftz-form", type=int, default=-1, help="with --k1-shape: fixed z-transform form")
    ap.add_argument("--ify-form", type=int, default=-1, help="with --k1-shape: fixed inverse-y-transform form")
    ap.add_argument("--div-form", type=int, default=-1, help="with --k1-shape: fixed divergence + y-transform form")
    ap.add_argument("--jobs", type=int, default=100, help="served: number of jobs")
    ap.add_argument("--rate", type=float, default=50.0,
                    help="served: Poisson arrival rate per second (50 = the benchmark's stream, ~16x capacity; "
                         "2 offers ~0.6 of capacity)")
    ap.add_argument("--chunk", type=int, default=25, help="served: steps per pump")
    ap.add_argument("--slots", type=int, default=32, help="served: 2-D slots per pool")
    ap.add_argument("--max-cells", type=int, default=16_000_000, help="served: cells-in-flight cap (0 = memory only)")
    ap.add_argument("--policy", default="shortest", choices=["fifo", "shortest"])
    ap.add_argument("--cpu-steps", type=int, default=10,
                    help="steps of the CPU baseline (and of the GPU replay compared with it)")
    ap.add_argument("--cpu-budget", type=float, default=60.0, help="seconds of CPU-baseline steps at most")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--restart-io", action="store_true", help="rbc3d: time writing and reading the restart files")
    ap.add_argument("--l2-group-mb", type=float, default=0.0,
                    help="batched: split each class into groups of at most this many MB of device state, stepped "
                         "group after group (0 = one batch per class)")
    ap.add_argument("--group-steps", type=int, default=10, help="batched: steps per group visit with --l2-group-mb")
    ap.add_argument("--instances", type=int, default=256,
                    help="batched: the first N instances of the 256-instance draw (profiling a smaller set)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.config.startswith("batched"):
        run_batched(args)
    elif args.config == "served":
        run_served(args)
    elif args.config in DDC_WORKLOADS:
        run_ddc(args)
    elif args.config == "published_rbc":
        run_published(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
