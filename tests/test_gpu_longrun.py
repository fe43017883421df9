"""Long-run accuracy gate: the FP64 GPU path against the FP64 CPU restatement of the reference
(oracle/afid_cpu.c, itself checked against the NumPy oracle) over hundreds to thousands of
main-loop steps from the same seeded state.

Each run advances both from the seeded initial condition (fluid at rest, conductive T plus a
+-1e-3 Philox perturbation), samples the volume Nusselt number and kinetic energy
(GlobalQuantities.F90:35-79), and the plate Nusselt numbers from the first and last Tbar rows
(CalcMeanProfiles.F90 Tbar; tools/afidtools/boundary_layers.py:41-54) every few steps, and
compares their time averages over the second half of the run.  Gate: within 1%.  The series
are also compared sample by sample, since both paths compute in FP64 and agree far below the
gate.

* the 2-D benchmark case: 256 (periodic, aspect 2) x 128 (tanh-clustered, STR3 = 2) cells,
  Ra = 1e8, Pr = 1, fixed dt = 5e-4, 1000 steps (main.F90:281-385 with NTST = 999).  At t = 0.5
  the perturbation is still growing in the conductive state (KE ~ 1e-9), so Nu_vol - 1 and KE
  carry the comparison;
* a convecting 2-D case: 128 x 64 cells, Ra = 1e6, aspect 2, CFL-limited dt, 8000 steps, which
  reaches periodic convection rolls (Nu_vol between ~4 and ~10, plate Nu ~ 8).
"""
import ctypes

import numpy as np
import pytest

import afid_gpu as ag
from helpers import bou_text
from oracle import afid_oracle as o
from oracle.cpu_port import CpuSolver, plate_and_volume_stats

pytestmark = pytest.mark.gpu

SEED = 20261203
KEYS = ("nu_vol", "nu_plate_lower", "nu_plate_upper", "ke")


def _gpu_stats(gpu, p, xm, ra_pr):
    nu, ke, _ = gpu.global_quantities(ra_pr)
    tbar = gpu.mean_profiles()["Tbar"]
    return plate_and_volume_stats(p, xm, nu, ke, tbar[0], tbar[p.nxm - 1])


def _run_both(text: str, steps: int, every: int):
    p = o.parse_bou_in(text)
    g = o.create_grid(p)
    s = o.initial_state(g, SEED)
    inp = ag.parse_bou_in(text)
    tables = ag.Tables(inp)
    ra_pr = p.prat * abs(p.rayt)
    cpu = CpuSolver(g, s)
    series = {"step": [], "gpu": {k: [] for k in KEYS}, "cpu": {k: [] for k in KEYS}}
    dt_c = dt_g = p.dt
    with ag.Solver(tables.grid, tables.params) as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        for n in range(steps):
            dt_c, err_c, _ = o.next_dt(p, n, dt_c, cpu.cfl())
            dtc = ctypes.c_double(dt_g)
            err_g = ag.lib().afid_next_dt(ctypes.byref(inp), n, ctypes.byref(dtc), gpu.calc_max_cfl(), None)
            dt_g = dtc.value
            assert err_c == 0 and err_g == 0, (n, err_c, err_g)
            assert dt_g == pytest.approx(dt_c, rel=1e-9), n
            cpu.time_marcher(dt_c)
            gpu.time_marcher(dt_g, n)
            if (n + 1) % every == 0:
                series["step"].append(n + 1)
                for k, v in _gpu_stats(gpu, p, g.xm, ra_pr).items():
                    series["gpu"][k].append(v)
                for k, v in cpu.stats().items():
                    series["cpu"][k].append(v)
        assert gpu.check_divergence() < 1e-10
    cpu.close()
    tables.close()
    return {side: {k: np.array(v) for k, v in series[side].items()} for side in ("gpu", "cpu")}


def _compare(name, series, series_rtol):
    gpu, cpu = series["gpu"], series["cpu"]
    half = len(gpu["nu_vol"]) // 2
    report = {}
    for k in KEYS:
        a, b = gpu[k][half:].mean(), cpu[k][half:].mean()
        report[k] = (a, b, abs(a - b) / abs(b))
    a, b = gpu["nu_vol"][half:].mean() - 1.0, cpu["nu_vol"][half:].mean() - 1.0
    report["nu_vol-1"] = (a, b, abs(a - b) / abs(b))
    print(f"\n{name}: time averages over the second half (GPU FP64, CPU FP64, relative difference)")
    for k, (a, b, r) in report.items():
        print(f"  {k:15s} {a: .12e} {b: .12e} {r:.2e}")
    for k, (a, b, r) in report.items():
        assert r <= 0.01, (k, a, b, r)                       # the long-run gate: 1%
    for k in KEYS:                                           # and sample by sample
        np.testing.assert_allclose(gpu[k], cpu[k], rtol=series_rtol, atol=0.0, err_msg=k)


def test_rbc2d_ra1e8_1000_steps_nu_ke_within_one_percent():
    text = bou_text(128, 256, 1, rayt=1e8, prat=1.0, ylen=2.0, zlen=0.01, istr3=4, str3=2.0, idtv=0, dt=5e-4,
                    cflmax=1.2, dtmax=5e-4, ntst=999, resid=1e-3)
    series = _run_both(text, 1000, every=10)
    _compare("rbc2d 256x128 Ra=1e8 dt=5e-4 1000 steps", series, series_rtol=1e-8)


def test_rbc2d_ra1e6_convecting_8000_steps_nu_ke_within_one_percent():
    text = bou_text(64, 128, 1, rayt=1e6, prat=1.0, ylen=2.0, zlen=0.01, istr3=4, str3=2.0, idtv=1, dt=1e-3,
                    cflmax=1.2, dtmax=2e-2, ntst=7999, resid=1e-3)
    series = _run_both(text, 8000, every=20)
    assert series["cpu"]["nu_plate_lower"][len(series["cpu"]["nu_vol"]) // 2:].mean() > 5.0   # convecting
    _compare("rbc2d 128x64 Ra=1e6 CFL dt 8000 steps", series, series_rtol=1e-4)
