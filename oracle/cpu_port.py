"""ctypes driver of the C + OpenMP restatement (oracle/afid_cpu.c).  TEST INFRASTRUCTURE ONLY:
used by tests/ as a second oracle and by bench.py as the timed CPU baseline."""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from oracle import afid_oracle as o

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        from oracle import build_oracle
        path = build_oracle.build()
        _lib = C.CDLL(path)
        _lib.afid_cpu_create.restype = C.c_void_p
        _lib.afid_cpu_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                         C.POINTER(C.c_void_p), C.POINTER(C.c_double), C.POINTER(C.c_int)]
        _lib.afid_cpu_destroy.argtypes = [C.c_void_p]
        _lib.afid_cpu_set.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib.afid_cpu_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib.afid_cpu_timemarcher.argtypes = [C.c_void_p, C.c_double]
        _lib.afid_cpu_cfl.restype = C.c_double
        _lib.afid_cpu_cfl.argtypes = [C.c_void_p]
        _lib.afid_cpu_threads.restype = C.c_int
        _lib.afid_cpu_stats.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_double)]
    return _lib


class CpuSolver:
    NAMES = ("vx", "vy", "vz", "temp", "pr")

    def __init__(self, g: o.Grid, s: o.State):
        p = g.p
        self.g = g
        nx = g.nx
        tempbp, temptp = s.tempbp, s.temptp

        def pad(a, n):
            b = np.zeros(max(n, 1))
            b[:min(a.size, n)] = a[:min(a.size, n)]
            return b
        self._keep = [pad(g.udx3c, nx), pad(g.udx3m, nx), pad(g.ap3ck, nx), pad(g.ac3ck, nx), pad(g.am3ck, nx),
                      pad(g.ap3sk, nx), pad(g.ac3sk, nx), pad(g.am3sk, nx), pad(g.ap3ssk, nx), pad(g.ac3ssk, nx),
                      pad(g.am3ssk, nx), pad(g.amphk, nx), pad(g.acphk, nx), pad(g.apphk, nx),
                      np.ascontiguousarray(g.ak1), np.ascontiguousarray(g.ak2),
                      np.ascontiguousarray(tempbp).ravel(), np.ascontiguousarray(temptp).ravel(),
                      pad(g.g3rc, nx)]
        tabs = (C.c_void_p * 19)(*[a.ctypes.data for a in self._keep])
        prm = (C.c_double * 6)(g.ren, g.pect, g.byct, p.xplusu, p.xminusu, p.dpdy)
        ipr = (C.c_int * 7)(p.active_t, p.gaxis, p.inslws, p.inslwn, p.tfixs, p.tfixn, p.nsst)
        self._h = lib().afid_cpu_create(p.nxm, p.nym, p.nzm, p.ylen, p.zlen, tabs, prm, ipr)
        if not self._h:
            raise ValueError("unsupported FFT size")
        for w, n in enumerate(self.NAMES):
            a = np.ascontiguousarray(getattr(s, n))
            lib().afid_cpu_set(self._h, w, a.ctypes.data)

    def time_marcher(self, dt):
        lib().afid_cpu_timemarcher(self._h, dt)

    def cfl(self):
        return lib().afid_cpu_cfl(self._h)

    def stats(self) -> dict:
        """Volume Nusselt number and kinetic energy (GlobalQuantities) and the plate Nusselt
        numbers from the first and last Tbar rows, as the reference's post-processing forms
        them (tools/afidtools/boundary_layers.py:41-54)."""
        p, g = self.g.p, self.g
        out = (C.c_double * 4)()
        lib().afid_cpu_stats(self._h, p.prat * abs(p.rayt), out)
        return plate_and_volume_stats(p, g.xm, out[0], out[1], out[2], out[3])

    def get(self):
        p = self.g.p
        out = {}
        for w, n in enumerate(self.NAMES):
            a = np.zeros((p.nzm, p.nym, self.g.nx))
            lib().afid_cpu_get(self._h, w, a.ctypes.data)
            out[n] = a
        return out

    def close(self):
        if self._h:
            lib().afid_cpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plate_and_volume_stats(p, xm, nu_vol: float, ke: float, tbar_lo: float, tbar_up: float) -> dict:
    """Nu_vol and KE as given; the plate Nusselt numbers of boundary_layers.py:41-54 from the
    first and last Tbar rows (plates at T = +-0.5, the sign flipped for Ra > 0; a zero-flux
    plate gives 0)."""
    nxm = p.nxm
    tup, tlo = (-0.5, 0.5) if p.rayt > 0 else (0.5, -0.5)
    lo = (tbar_lo - tlo) / xm[0] if p.tfixs else 0.0
    up = (tup - tbar_up) / (1.0 - xm[nxm - 1]) if p.tfixn else 0.0
    if p.rayt > 0:
        lo, up = -lo, -up
    return {"nu_vol": float(nu_vol), "ke": float(ke), "nu_plate_lower": float(lo), "nu_plate_upper": float(up)}


def time_steps(bou_text: str, steps: int, seed: int = 20261203, mixed: bool = False,
               budget_s: float = 1e30, keep_state: bool = False, warmup: int = 0) -> dict:
    """Main-loop steps (CFL -> dt rule -> TimeMarcher) of the C restatement on all host cores,
    from the seeded initial state: ``warmup`` untimed steps, then up to ``steps`` timed ones,
    stopping early once ``budget_s`` seconds of timed steps have been spent; returns the
    throughput in Mcell-RK3-steps/s and the steps actually timed (with ``keep_state``, also the
    final fields, the dt of every step and the Nusselt numbers and kinetic energy after every
    step, warm-up steps included; the statistics are taken outside the timed interval)."""
    p = o.parse_bou_in(bou_text)
    g = o.create_grid(p)
    s = o.initial_state(g, seed)
    cpu = CpuSolver(g, s)
    dt = p.dt
    dts, stats = [], []
    for n in range(warmup):
        cflm = cpu.cfl()
        dt, _, _ = o.next_dt(p, n, dt, cflm)
        cpu.time_marcher(dt)
        dts.append(dt)
        if keep_state:
            stats.append(cpu.stats())
    sec = 0.0
    done = 0
    for n in range(warmup, warmup + steps):
        t0 = time.perf_counter()
        cflm = cpu.cfl()
        dt, _, _ = o.next_dt(p, n, dt, cflm)
        cpu.time_marcher(dt)
        sec += time.perf_counter() - t0
        dts.append(dt)
        done += 1
        if keep_state:
            stats.append(cpu.stats())
        if sec > budget_s:
            break
    cells = p.nxm * p.nym * p.nzm
    res = {"seconds": sec, "steps": done, "mcells_per_s": cells * done / sec / 1e6,
           "threads": lib().afid_cpu_threads()}
    if keep_state:
        res["state"] = cpu.get()
        res["dts"] = dts
        res["stats"] = stats
    cpu.close()
    return res


def _sal_lib():
    L = lib()
    if not hasattr(L, "_sal_ready"):
        L.afid_cpu_sal_create.restype = C.c_void_p
        L.afid_cpu_sal_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_double),
                                          C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.afid_cpu_sal_destroy.argtypes = [C.c_void_p]
        L.afid_cpu_sal_set.argtypes = [C.c_void_p, C.c_void_p]
        L.afid_cpu_sal_get.argtypes = [C.c_void_p, C.c_void_p]
        L.afid_cpu_timemarcher_sal.argtypes = [C.c_void_p, C.c_double]
        L.afid_cpu_sal_cfl.restype = C.c_double
        L.afid_cpu_sal_cfl.argtypes = [C.c_void_p]
        L._sal_ready = True
    return L


class CpuSalSolver:
    """The C restatement with the multi-resolution salinity scalar, on the oracle's refined grid
    and per-target stencils (``oracle.afid_salinity.Mgrd``)."""

    def __init__(self, g: o.Grid, s: o.State, m, sal: np.ndarray):
        self.flow = CpuSolver(g, s)
        self.m = m
        nxr = m.nxmr + 1
        planes = np.full((m.nzmr, m.nymr), 1.0)
        self._keep = [np.ascontiguousarray(m.xcr), np.ascontiguousarray(m.udx3mr), np.ascontiguousarray(m.g3rmr),
                      np.ascontiguousarray(m.ap3sskr), np.ascontiguousarray(m.ac3sskr),
                      np.ascontiguousarray(m.am3sskr), (planes * m.salbp).ravel(), (planes * m.saltp).ravel()]
        tabs = (C.c_void_p * 8)(*[a.ctypes.data for a in self._keep])
        dprm = (C.c_double * 5)(m.dxr, m.dyr, m.dzr, m.pecs, m.bycs)
        iprm = (C.c_int * 6)(m.nxmr, m.nymr, m.nzmr, m.active_s, m.sfixs, m.sfixn)
        sts = list(m.to_ref) + list(m.to_coarse)
        self._st = [np.ascontiguousarray(t.start, dtype=np.int32) for t in sts]
        self._w = [np.ascontiguousarray(t.w.T) for t in sts]  # [target][4]
        stp = (C.c_void_p * 6)(*[a.ctypes.data for a in self._st])
        wp = (C.c_void_p * 6)(*[a.ctypes.data for a in self._w])
        self._h = _sal_lib().afid_cpu_sal_create(self.flow._h, tabs, dprm, iprm, stp, wp)
        full = np.zeros((m.nzmr, m.nymr, nxr))
        full[..., :m.nxmr] = sal
        _sal_lib().afid_cpu_sal_set(self._h, full.ctypes.data)

    def time_marcher(self, dt):
        _sal_lib().afid_cpu_timemarcher_sal(self._h, dt)

    def cfl(self):
        return _sal_lib().afid_cpu_sal_cfl(self._h)

    def sal(self):
        m = self.m
        a = np.zeros((m.nzmr, m.nymr, m.nxmr + 1))
        _sal_lib().afid_cpu_sal_get(self._h, a.ctypes.data)
        return a[..., :m.nxmr]

    def get(self):
        return self.flow.get()

    def close(self):
        if self._h:
            _sal_lib().afid_cpu_sal_destroy(self._h)
            self._h = None
        self.flow.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def time_steps_sal(bou_text: str, steps: int, seed: int = 20261203, budget_s: float = 1e30) -> dict:
    """Main-loop steps with salinity (CFLmr -> dt rule -> TimeMarcher) of the C restatement on all
    host cores from the seeded temperature and the reference's initial salinity."""
    from oracle import afid_salinity as sa
    p = o.parse_bou_in(bou_text)
    g = o.create_grid(p)
    m = sa.create_mgrd(g)
    s = o.initial_state(g, seed)
    cpu = CpuSalSolver(g, s, m, sa.initial_salinity(m, g, seed + 1))
    dt = p.dt
    t0 = time.perf_counter()
    done = 0
    for n in range(steps):
        dt, _, _ = o.next_dt(p, n, dt, cpu.cfl())
        cpu.time_marcher(dt)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    sec = time.perf_counter() - t0
    cells = p.nxm * p.nym * p.nzm
    cpu.close()
    return {"seconds": sec, "steps": done, "mcells_per_s": cells * done / sec / 1e6,
            "threads": lib().afid_cpu_threads()}
