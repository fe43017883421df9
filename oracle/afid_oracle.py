"""CPU oracle for the AFiD RK3 flow + temperature substep.  TEST INFRASTRUCTURE ONLY.

This module is test infrastructure, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py`` (its CPU-baseline / reference arm) may import it.  The product path is the
sm_100a CUDA library behind ``include/afid_gpu.h`` and fails loudly without it.

It is an FP64 NumPy restatement of the reference Fortran routines (``-fdefault-real-8``, so
every ``real`` is a double), following the reference loop bodies expression by expression so
that rounding differences stay at the 1e-16 level:

* grid and metrics        ``src/flow_solver/CreateGrid.F90:11-179``, ``src/grid.F90:12-307``
* RK3 coefficients        ``src/flow_solver/InitTimeMarchScheme.F90:16-49``
* input derivations       ``src/flow_solver/ReadInputFile.F90:109-123``
* temperature plates      ``src/flow_solver/SetTempBCs.F90:18-41``
* explicit terms          ``src/flow_solver/ExplicitTerms{VX,VY,VZ,Temp}.F90``
* RHS assembly            ``src/flow_solver/ImplicitAndUpdate{VX,VY,VZ,Temp}.F90``
* CN solves               ``src/flow_solver/SolveImpEqnUpdate_{X,YZ,Temp}.F90`` with the same
                          LAPACK ``dgttrf``/``dgttrs`` (scipy's OpenBLAS LAPACK)
* Poisson solve           ``src/pressure.F90:61-301``: y r2c / z c2c FFT (numpy pocketfft in
                          place of FFTW, same normalisation), ``zgttrf``/``zgttrs`` per mode
* projection              ``src/flow_solver/CorrectVelocity.F90:24`` → ``pressure.F90:240-267``
* CFL / divergence        ``src/flow_solver/CalcMaxCFL.F90:30-43``, ``CheckDivergence.F90:30-42``
* substep loop            ``src/flow_solver/TimeMarcher.F90:28-133``
* step control            ``src/main.F90:281-304``

Parity pins (the reference has no tests and cannot be compiled in this container — no Fortran
compiler, MPI, FFTW or HDF5): (1) the published 1-D pure-diffusion convergence errors of
``docs/convergence.md:3-31`` / ``docs/figures/spatial_convergence.svg`` (the temperature CN
path), (2) the discrete divergence-free invariant after projection (the modified wavenumbers of
``pressure.F90:78-97`` make the FFT solve exact for the discrete operator), (3) FFT and
tridiagonal kernels against direct dense solves.  Field-level parity against a reference run
is otherwise unpinned.

Array layout: C-order ``a[i, j, k]`` = Fortran ``a(k, j, i)`` with 0-based indices, i.e. x
(wall-normal, ``k``) fastest, then y (``j``), then z (``i``).  Every 3-D field has ``nx`` x
entries (Fortran ``1:nx``); only ``vx`` uses the last one.  Periodic halos of the reference
(``update_halo``) are restated with ``np.roll``.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
from scipy.linalg import lapack

__all__ = [
    "Params", "Grid", "State", "create_grid", "rk3_coefficients", "initial_state",
    "explicit_terms_vx", "explicit_terms_vy", "explicit_terms_vz", "explicit_terms_temp",
    "implicit_and_update_vx", "implicit_and_update_vy", "implicit_and_update_vz",
    "implicit_and_update_temp", "calc_local_divergence", "solve_pressure_correction",
    "remove_divergence", "correct_pressure", "calc_max_cfl", "check_divergence",
    "time_marcher", "run", "parse_bou_in", "nusselt_volume", "kinetic_energy",
]


# ----------------------------------------------------------------------------------------------
# Parameters (bou.in) and derived constants
# ----------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Params:
    """The bou.in quantities used by the flow + temperature path (``ReadInputFile.F90:20-75``)."""

    nxm: int
    nym: int
    nzm: int
    nsst: int = 3
    ntst: int = 0
    alx3: float = 1.0
    ylen: float = 1.0
    zlen: float = 1.0
    istr3: int = 4
    str3: float = 2.0
    rayt: float = 1e8
    prat: float = 1.0
    rays: float = 1e8
    pras: float = 1.0
    ffscales: int = 0
    salinity: bool = False
    idtv: int = 0
    dt: float = 5e-4
    resid: float = 1e-3
    limit_cfl: float = 1.2
    dtmin: float = 1e-8
    dtmax: float = 5e-4
    inslws: int = 1
    inslwn: int = 1
    tfixs: int = 1
    tfixn: int = 1
    active_t: int = 1
    gaxis: int = 1
    xplusu: float = 0.0
    xminusu: float = 0.0
    dpdy: float = 0.0
    dpdz: float = 0.0
    tout: float = 1e30
    tmax: float = 1e30
    # multi-resolution salinity (MULTIRES NXMR NYMR NZMR, ISTR3R, SfixS SfixN, active_S)
    multires: int = 0
    nxmr: int = 0
    nymr: int = 0
    nzmr: int = 0
    istr3r: int = 4
    sfixs: int = 1
    sfixn: int = 1
    active_s: int = 0

    @property
    def nx(self) -> int:
        return self.nxm + 1

    def derived(self):
        """ren, pect, byct, pi exactly as ``ReadInputFile.F90:109-123``."""
        rrho = abs(self.rayt) * self.pras / (abs(self.rays) * self.prat) if self.rays != 0 else math.inf
        if self.salinity and self.ffscales == 1:
            ren = math.sqrt(abs(self.rays) / self.pras)
            byct = rrho
        else:
            ren = math.sqrt(abs(self.rayt) / self.prat)
            byct = 1.0
        pect = ren * self.prat
        pi = 2.0 * math.asin(1.0)
        return ren, pect, byct, pi

    def derived_salinity(self):
        """pecs and bycs of ``ReadInputFile.F90:109-122``."""
        ren, _, _, _ = self.derived()
        rrho = abs(self.rayt) * self.pras / (abs(self.rays) * self.prat)
        bycs = 1.0 if (self.salinity and self.ffscales == 1) else 1.0 / rrho
        return ren * self.pras, bycs


def parse_bou_in(text: str) -> Params:
    """Parse the fixed-layout bou.in: 3 header lines before every value line except the first
    block, exactly the read sequence of ``ReadInputFile.F90:21-75``."""
    lines = text.splitlines()
    pos = 0

    def skip(n):
        nonlocal pos
        pos += n

    def vals():
        nonlocal pos
        v = lines[pos].split()
        pos += 1
        return v

    skip(2)
    nxm, nym, nzm, nsst = (int(float(x)) for x in vals()[:4])
    skip(3)
    multires, nxmr, nymr, nzmr = (int(float(x)) for x in vals()[:4])
    skip(3)
    flagsal, _flagpf = (int(float(x)) for x in vals()[:2])
    skip(3)
    vals()  # NREAD IRESET
    skip(3)
    v = vals()
    ntst = int(float(v[0]))
    tmax = float(v[2])
    skip(3)
    v = vals()
    tout = float(v[0])
    skip(3)
    alx3, ylen, zlen = (float(x) for x in vals()[:3])
    skip(3)
    v = vals()
    istr3, str3 = int(float(v[0])), float(v[1])
    istr3r = int(float(v[2])) if len(v) > 2 else istr3
    skip(3)
    v = vals()
    rayt, prat, rays, pras = (float(x) for x in v[:4])
    ffscales = int(float(v[4]))
    skip(3)
    v = vals()
    idtv = int(float(v[0]))
    dt, resid, limit_cfl, dtmin, dtmax = (float(x) for x in v[1:6])
    skip(3)
    v = vals()
    inslws, inslwn, tfixs, tfixn = (int(float(x)) for x in v[:4])
    sfixs, sfixn = (int(float(x)) for x in v[4:6]) if len(v) >= 6 else (1, 1)
    skip(3)
    v = vals()
    active_t, active_s, gaxis = (int(float(x)) for x in v[:3])
    skip(3)
    v = vals()
    xplusu, xminusu, dpdy, dpdz = (float(x) for x in v[:4])
    return Params(nxm=nxm, nym=nym, nzm=nzm, nsst=nsst, ntst=ntst, alx3=alx3, ylen=ylen,
                  zlen=zlen, istr3=istr3, str3=str3, rayt=rayt, prat=prat, rays=rays, pras=pras,
                  ffscales=ffscales, salinity=bool(flagsal), idtv=idtv, dt=dt, resid=resid,
                  limit_cfl=limit_cfl, dtmin=dtmin, dtmax=dtmax, inslws=inslws, inslwn=inslwn,
                  tfixs=tfixs, tfixn=tfixn, active_t=active_t, gaxis=gaxis, xplusu=xplusu,
                  xminusu=xminusu, dpdy=dpdy, dpdz=dpdz, tout=tout, tmax=tmax,
                  multires=multires, nxmr=nxmr, nymr=nymr, nzmr=nzmr, istr3r=istr3r,
                  sfixs=sfixs, sfixn=sfixn, active_s=active_s)


def rk3_coefficients(nsst: int = 3):
    """gam, rom, alm of ``InitTimeMarchScheme.F90:16-49`` (Rai-Moin RK3, or AB2 if nsst=1)."""
    if nsst > 1:
        gam = [8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0]
        rom = [0.0, -17.0 / 60.0, -5.0 / 12.0]
    else:
        gam = [1.5, 0.0, 0.0]
        rom = [-0.5, 0.0, 0.0]
    alm = [gam[n] + rom[n] for n in range(3)]
    return gam, rom, alm


# ----------------------------------------------------------------------------------------------
# Grid (CreateGrid.F90 + grid.F90)
# ----------------------------------------------------------------------------------------------
def _uniform_grid(nm, length):
    """``grid.F90:12-27``."""
    c = np.array([length * float(i) / float(nm) for i in range(nm + 1)])
    m = 0.5 * (c[:-1] + c[1:])
    return c, m


def _tanh_grid(nm, length, s):
    """``grid.F90:29-53`` (ISTR3=4)."""
    tstr = math.tanh(s)
    c = np.zeros(nm + 1)
    for i in range(2, nm + 2):
        z2 = float(2 * (i - 1) - nm) / float(nm)
        c[i - 1] = 0.5 * (1 + math.tanh(s * z2) / tstr) * length
        if c[i - 1] < 0.0 or c[i - 1] > length:
            raise ValueError("Refined grid is too streched")
    m = 0.5 * (c[:-1] + c[1:])
    return c, m


def _cheb_grid(nm, length, s, pi):
    """``grid.F90:55-92`` (ISTR3=6)."""
    nclip = int(s)
    n_ext = nm + 1 + 2 * nclip
    etazm = np.array([math.cos(pi * (float(i) - 0.5) / float(n_ext)) for i in range(1, n_ext + 1)])
    etaz = etazm[nclip:nclip + nm + 1].copy()
    delet = etaz[0] - etaz[nm]
    etaz = 2.0 * etaz / delet
    c = np.zeros(nm + 1)
    for i in range(2, nm + 1):
        c[i - 1] = 0.5 * length * (1.0 - etaz[i - 1])
    c[nm] = length
    return c, 0.5 * (c[:-1] + c[1:])


def _asym_cheb_grid(nm, length, s, pi):
    """``grid.F90:94-131`` (ISTR3=7)."""
    nclip = int(s)
    n_ext = nm + 1 + nclip
    etazm = np.array([math.cos(pi * float(i) / float(n_ext) / 2.0) for i in range(1, n_ext + 1)])
    etaz = etazm[nclip:nclip + nm + 1].copy()
    etaz = etaz / etaz[0]
    c = np.zeros(nm + 1)
    for i in range(2, nm + 1):
        c[i - 1] = length * (1.0 - etaz[i - 1])
    c[nm] = length
    return c, 0.5 * (c[:-1] + c[1:])


def _centre_focus_grid(nm, length, s):
    """``grid.F90:133-151`` (ISTR3=1)."""
    c = np.zeros(nm + 1)
    for i in range(2, nm + 1):
        t = 2.0 * (i - 1) / nm - 1
        c[i - 1] = length / 2.0 * (s * t ** 7 + 2.0 * (i - 1) / nm - 1) / (s + 1) + length / 2.0
    c[nm] = length
    return c, 0.5 * (c[:-1] + c[1:])


def _natural_bl_grid(nm, length, schmidt=None):
    """``grid.F90:153-179`` (ISTR3=2) and ``:181-213`` (ISTR3=3, symmetric)."""
    jb, c_eta, alpha, dyw = 16.0, 0.8, 1.5, 0.1

    def f(jm, sc):
        return 1 / (1.0 + (jm / jb) ** 2) * (dyw * jm + (0.75 * alpha * c_eta * jm / sc) ** (4.0 / 3.0)
                                             * (jm / jb) ** 2)
    c = np.zeros(nm + 1)
    if schmidt is None:
        for j in range(1, nm + 2):
            c[j - 1] = 1 / (1.0 + ((j - 1) / jb) ** 2) * (
                dyw * (j - 1) + (0.75 * alpha * c_eta * (j - 1)) ** (4.0 / 3.0) * ((j - 1) / jb) ** 2)
    else:
        nh = nm // 2
        for j in range(1, nh + 2):
            c[j - 1] = f(j - 1, schmidt ** 0.5)
        lh = 2.0 * c[nh]
        for j in range(1, nh + 1):
            c[nm + 1 - j] = lh - c[j - 1]
    c = c / c[nm] * length
    return c, 0.5 * (c[:-1] + c[1:])


def _second_derivative_coeff(x, xlen, fix_up, fix_low):
    """``grid.F90:264-307``: ap3, ac3, am3 with Dirichlet ghost (fix=1) or Neumann (fix=0)."""
    n = x.size
    ap3 = np.zeros(n)
    ac3 = np.zeros(n)
    am3 = np.zeros(n)
    k = 0
    a33 = 2.0 / (x[k] + x[k + 1])
    ap3[k] = a33 / (x[k + 1] - x[k])
    am3[k] = 0.0
    ac3[k] = -ap3[k] - fix_low * a33 / x[k] if x[k] != 0.0 else 0.0
    if x[k] == 0.0:
        ap3[k] = 0.0
        ac3[k] = 1.0
    for k in range(1, n - 1):
        a33 = 2.0 / (x[k + 1] - x[k - 1])
        ap3[k] = a33 / (x[k + 1] - x[k])
        am3[k] = a33 / (x[k] - x[k - 1])
        ac3[k] = -ap3[k] - am3[k]
    k = n - 1
    a33 = 2.0 / (2.0 * xlen - x[k] - x[k - 1])
    ap3[k] = 0.0
    am3[k] = a33 / (x[k] - x[k - 1])
    ac3[k] = -am3[k] - fix_up * a33 / (xlen - x[k]) if x[k] != xlen else 0.0
    if x[k] == xlen:
        am3[k] = 0.0
        ac3[k] = 1.0
    return ap3, ac3, am3


@dataclasses.dataclass
class Grid:
    """Metric tables of ``CreateGrid.F90`` and ``InitPressureSolver`` (``pressure.F90:61-114``).
    Index arrays ``kmv``/``kpv`` are 0-based here."""

    p: Params
    nx: int
    xc: np.ndarray
    xm: np.ndarray
    yc: np.ndarray
    ym: np.ndarray
    zc: np.ndarray
    zm: np.ndarray
    dx: float
    dy: float
    dz: float
    dxq: float
    dyq: float
    dzq: float
    g3rc: np.ndarray
    g3rm: np.ndarray
    d3xc: np.ndarray
    d3xm: np.ndarray
    udx3c: np.ndarray
    udx3m: np.ndarray
    kmv: np.ndarray
    kpv: np.ndarray
    kmc: np.ndarray
    kpc: np.ndarray
    ap3ck: np.ndarray
    ac3ck: np.ndarray
    am3ck: np.ndarray
    ap3sk: np.ndarray
    ac3sk: np.ndarray
    am3sk: np.ndarray
    ap3ssk: np.ndarray
    ac3ssk: np.ndarray
    am3ssk: np.ndarray
    ak1: np.ndarray
    ak2: np.ndarray
    amphk: np.ndarray
    acphk: np.ndarray
    apphk: np.ndarray
    ren: float
    pect: float
    byct: float
    pi: float
    # Test option, off for the reference behaviour: solve the singular (0,0) Poisson mode
    # exactly (last equation replaced by phi = 0) instead of through the 1+1e-15 diagonal.
    pin_zero_mode: bool = False


def create_grid(p: Params) -> Grid:
    """``CreateGrid.F90:19-177`` then the Poisson tables of ``pressure.F90:68-114``."""
    ren, pect, byct, pi = p.derived()
    nxm, nym, nzm = p.nxm, p.nym, p.nzm
    nx = nxm + 1
    kmv = np.array([max(kc - 1, 0) for kc in range(nxm)], dtype=np.int64)
    kpv = np.array([min(kc + 1, nxm - 1) for kc in range(nxm)], dtype=np.int64)
    kpc = kpv - np.arange(nxm)
    kmc = np.arange(nxm) - kmv

    zc, zm = _uniform_grid(nzm, p.zlen)
    yc, ym = _uniform_grid(nym, p.ylen)
    if p.istr3 == 0:
        xc, xm_ = _uniform_grid(nxm, p.alx3)
    elif p.istr3 == 1:
        xc, xm_ = _centre_focus_grid(nxm, p.alx3, p.str3)
    elif p.istr3 == 2:
        xc, xm_ = _natural_bl_grid(nxm, p.alx3)
    elif p.istr3 == 3:
        xc, xm_ = _natural_bl_grid(nxm, p.alx3, 1.0)
    elif p.istr3 == 4:
        xc, xm_ = _tanh_grid(nxm, p.alx3, p.str3)
    elif p.istr3 == 6:
        xc, xm_ = _cheb_grid(nxm, p.alx3, p.str3, pi)
    elif p.istr3 == 7:
        xc, xm_ = _asym_cheb_grid(nxm, p.alx3, p.str3, pi)
    else:
        raise ValueError(f"ISTR3={p.istr3} not supported by the oracle")

    dx = float(nxm) / p.alx3
    dy = float(nym) / p.ylen
    dz = float(nzm) / p.zlen
    dxq, dyq, dzq = dx * dx, dy * dy, dz * dz

    xm = np.zeros(nx)
    for kc in range(nxm):
        xm[kc] = (xc[kc] + xc[kc + 1]) * 0.5
    xm[nx - 1] = 2 * xc[nx - 1] - xm[nxm - 1]
    g3rc = np.zeros(nx)
    g3rm = np.zeros(nx)
    for kc in range(1, nxm):
        g3rc[kc] = (xc[kc + 1] - xc[kc - 1]) * dx * 0.5
        g3rm[kc] = (xm[kc + 1] - xm[kc - 1]) * dx * 0.5
    g3rm[0] = (xm[1] - (2 * xc[0] - xm[0])) * dx * 0.5
    g3rc[0] = (xc[1] - xc[0]) * dx
    g3rc[nx - 1] = (xc[nx - 1] - xc[nxm - 1]) * dx
    d3xc = np.zeros(nx)
    d3xm = np.zeros(nx)
    for kc in range(nxm):
        d3xc[kc] = (xc[kc + 1] - xc[kc]) * dx
        d3xm[kc] = (xm[kc + 1] - xm[kc]) * dx
    udx3m = np.zeros(nx)
    udx3c = np.zeros(nx)
    for kc in range(nxm):
        udx3m[kc] = dx / d3xc[kc]
        udx3c[kc] = dx / g3rc[kc]
    udx3c[nx - 1] = dx / g3rc[nx - 1]

    ap3ck, ac3ck, am3ck = _second_derivative_coeff(xc[:nx], p.alx3, 1, 1)
    ap3sk, ac3sk, am3sk = _second_derivative_coeff(xm[:nxm], p.alx3, p.inslwn, p.inslws)
    ap3ssk, ac3ssk, am3ssk = _second_derivative_coeff(xm[:nxm], p.alx3, p.tfixn, p.tfixs)

    # Modified wavenumbers (pressure.F90:78-97)
    nzmh = nzm // 2 + 1
    ao = np.array([(i - 1) * 2.0 * pi if i <= nzmh else -(nzm - i + 1) * 2.0 * pi
                   for i in range(1, nzm + 1)])
    ak1 = 2.0 * (1.0 - np.cos(ao / nzm)) * (float(nzm) / p.zlen) ** 2
    nymh = nym // 2 + 1
    ap = np.array([(j - 1) * 2.0 * pi if j <= nymh else -(nym - j + 1) * 2.0 * pi
                   for j in range(1, nym + 1)])
    ak2 = 2.0 * (1.0 - np.cos(ap / nym)) * (float(nym) / p.ylen) ** 2

    # Poisson x-coefficients (pressure.F90:103-114)
    amphk = np.zeros(nx)
    apphk = np.zeros(nx)
    acphk = np.zeros(nx)
    for kc in range(nxm):
        km = kmv[kc]
        a33icc = kmc[kc] * dxq / d3xm[km]
        a33icp = kpc[kc] * dxq / d3xm[kc]
        ugmmm = 1.0 / d3xc[kc]
        amphk[kc] = a33icc * ugmmm
        apphk[kc] = a33icp * ugmmm
        acphk[kc] = -(amphk[kc] + apphk[kc])

    return Grid(p=p, nx=nx, xc=xc, xm=xm, yc=yc, ym=ym, zc=zc, zm=zm, dx=dx, dy=dy, dz=dz,
                dxq=dxq, dyq=dyq, dzq=dzq, g3rc=g3rc, g3rm=g3rm, d3xc=d3xc, d3xm=d3xm,
                udx3c=udx3c, udx3m=udx3m, kmv=kmv, kpv=kpv, kmc=kmc, kpc=kpc,
                ap3ck=ap3ck, ac3ck=ac3ck, am3ck=am3ck, ap3sk=ap3sk, ac3sk=ac3sk, am3sk=am3sk,
                ap3ssk=ap3ssk, ac3ssk=ac3ssk, am3ssk=am3ssk, ak1=ak1, ak2=ak2,
                amphk=amphk, acphk=acphk, apphk=apphk, ren=ren, pect=pect, byct=byct, pi=pi)


# ----------------------------------------------------------------------------------------------
# State and initial condition
# ----------------------------------------------------------------------------------------------
@dataclasses.dataclass
class State:
    """Fields of ``local_arrays`` (``param.F90:100-108``), shape (nzm, nym, nx) each."""

    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    temp: np.ndarray
    pr: np.ndarray
    rux: np.ndarray
    ruy: np.ndarray
    ruz: np.ndarray
    rutemp: np.ndarray
    tempbp: np.ndarray  # (nzm, nym)
    temptp: np.ndarray  # (nzm, nym)

    def copy(self) -> "State":
        return State(**{f.name: getattr(self, f.name).copy() for f in dataclasses.fields(self)})


def temp_plates(p: Params):
    """``SetTempBCs.F90:18-41`` (no phase-field / moisture on this path)."""
    if p.rayt >= 0:
        if p.inslwn == 0:
            top, bot = 0.0, 1.0
        else:
            top, bot = -0.5, 0.5
    else:
        top, bot = 0.5, -0.5
    return (np.full((p.nzm, p.nym), bot), np.full((p.nzm, p.nym), top))


def initial_state(g: Grid, seed: int, eps: float = 1e-3) -> State:
    """Seeded synthetic initial condition: fluid at rest, conductive temperature profile
    (``CreateInitialConditions.F90:178-185``) plus a uniform perturbation of amplitude ``eps``
    clamped at the walls as ``CreateInitialConditions.F90:188-201`` does.  The reference's
    unseeded ``random_number`` is replaced by Philox4x32-10 keyed by the seed and the global
    linear cell index ``k + nx*(j + nym*i)`` (0-based), so every implementation sees the same
    numbers."""
    from oracle.philox import uniform_cells
    p = g.p
    nx = g.nx
    shape = (p.nzm, p.nym, nx)
    tempbp, temptp = temp_plates(p)
    temp = np.zeros(shape)
    xm = g.xm[:p.nxm]
    temp[:, :, :p.nxm] = tempbp[:, :, None] + (temptp - tempbp)[:, :, None] * xm[None, None, :] / p.alx3
    u = uniform_cells(seed, p.nzm, p.nym, nx)[:, :, :p.nxm]
    amp = np.where(np.abs(xm - 0.5) + eps > 0.5, 0.5 - np.abs(xm - 0.5), eps)
    temp[:, :, :p.nxm] = temp[:, :, :p.nxm] + amp[None, None, :] * (2.0 * u - 1.0)
    z = lambda: np.zeros(shape)  # noqa: E731
    return State(vx=z(), vy=z(), vz=z(), temp=temp, pr=z(), rux=z(), ruy=z(), ruz=z(),
                 rutemp=z(), tempbp=tempbp, temptp=temptp)


# ----------------------------------------------------------------------------------------------
# Periodic neighbours (update_halo restated)
# ----------------------------------------------------------------------------------------------
def _jp(a):
    return np.roll(a, -1, axis=1)


def _jm(a):
    return np.roll(a, 1, axis=1)


def _ip(a):
    return np.roll(a, -1, axis=0)


def _im(a):
    return np.roll(a, 1, axis=0)


# ----------------------------------------------------------------------------------------------
# Explicit terms
# ----------------------------------------------------------------------------------------------
def explicit_terms_vx(g: Grid, s: State, qcap: np.ndarray) -> None:
    """``ExplicitTermsVX.F90:24-127``: qcap(k=2..nxm) = -(hxx+hxy+hxz) + dyy vx + dzz vx
    (+ byct*T buoyancy for gAxis=1)."""
    p = g.p
    nxm = p.nxm
    udy = g.dy * 0.25
    udz = g.dz * 0.25
    udyq = g.dyq / g.ren
    udzq = g.dzq / g.ren
    idx = 1.0 / g.udx3m[:nxm]
    K = slice(1, nxm)
    KM = slice(0, nxm - 1)
    KP = slice(2, nxm + 1)
    vx, vy, vz = s.vx, s.vy, s.vz
    vxc = vx[..., K]
    vx_ip, vx_im, vx_jp, vx_jm = _ip(vx)[..., K], _im(vx)[..., K], _jp(vx)[..., K], _jm(vx)[..., K]
    vz_ip = _ip(vz)
    vy_jp = _jp(vy)
    udx3c = g.udx3c[K]
    hxz = udx3c * udz * (
        (idx[KM] * vz_ip[..., KM] + idx[K] * vz_ip[..., K]) * (vx_ip + vxc)
        - (idx[KM] * vz[..., KM] + idx[K] * vz[..., K]) * (vxc + vx_im))
    hxy = udx3c * udy * (
        (idx[KM] * vy_jp[..., KM] + idx[K] * vy_jp[..., K]) * (vx_jp + vxc)
        - (idx[KM] * vy[..., KM] + idx[K] * vy[..., K]) * (vxc + vx_jm))
    hxx = ((vx[..., KP] + vxc) * (vx[..., KP] + vxc)
           - (vxc + vx[..., KM]) * (vxc + vx[..., KM])) * udx3c * 0.25
    dzzvx = (vx_im - 2.0 * vxc + vx_ip) * udzq
    dyyvx = (vx_jm - 2.0 * vxc + vx_jp) * udyq
    qcap[..., K] = -(hxx + hxy + hxz) + dyyvx + dzzvx
    if p.gaxis == 1:
        tempit = p.active_t * 0.5 * (s.temp[..., K] + s.temp[..., KM])
        qcap[..., K] = qcap[..., K] + g.byct * tempit


def explicit_terms_vy(g: Grid, s: State, dph: np.ndarray) -> None:
    """``ExplicitTermsVY.F90:23-122``: dph(k=1..nxm) for vy (+ Gy, + buoyancy for gAxis=2)."""
    p = g.p
    nxm = p.nxm
    udyq = g.dyq / g.ren
    udzq = g.dzq / g.ren
    udy = g.dy * 0.25
    udz = g.dz * 0.25
    if p.inslwn == 0 or p.inslws == 0:
        gy = p.dpdy ** 2 / g.ren ** 2
    else:
        gy = 8.0 * p.dpdy ** 2 / g.ren ** 2
    KC = np.arange(nxm)
    KMM, KPP, KP = g.kmv, g.kpv, KC + 1
    vx, vy, vz = s.vx, s.vy, s.vz
    vx_jm = _jm(vx)
    c = vy[..., KC]
    vy_jp, vy_jm, vy_ip, vy_im = _jp(vy)[..., KC], _jm(vy)[..., KC], _ip(vy)[..., KC], _im(vy)[..., KC]
    vz_ip = _ip(vz)
    hyx = ((vx[..., KP] + vx_jm[..., KP]) * (vy[..., KPP] + c)
           - (vx[..., KC] + vx_jm[..., KC]) * (c + vy[..., KMM])) * g.udx3m[:nxm] * 0.25
    hyy = ((vy_jp + c) * (vy_jp + c) - (vy_jm + c) * (vy_jm + c)) * udy
    hyz = ((vy_ip + c) * (vz_ip[..., KC] + _jm(vz_ip)[..., KC])
           - (c + vy_im) * (vz[..., KC] + _jm(vz)[..., KC])) * udz
    dyyvy = (vy_jp - 2.0 * c + vy_jm) * udyq
    dzzvy = (vy_ip - 2.0 * c + vy_im) * udzq
    dph[..., :nxm] = -(hyx + hyy + hyz) + dyyvy + dzzvy + gy
    if p.gaxis == 2:
        tempit = p.active_t * 0.5 * (s.temp[..., KC] + _jm(s.temp)[..., KC])
        dph[..., :nxm] = dph[..., :nxm] + g.byct * tempit


def explicit_terms_vz(g: Grid, s: State, dq: np.ndarray) -> None:
    """``ExplicitTermsVZ.F90:23-118``: dq(k=1..nxm) for vz (+ buoyancy for gAxis=3)."""
    p = g.p
    nxm = p.nxm
    udyq = g.dyq / g.ren
    udzq = g.dzq / g.ren
    udy = g.dy * 0.25
    udz = g.dz * 0.25
    KC = np.arange(nxm)
    KMM, KPP, KP = g.kmv, g.kpv, KC + 1
    vx, vy, vz = s.vx, s.vy, s.vz
    vx_im = _im(vx)
    c = vz[..., KC]
    vz_jp, vz_jm, vz_ip, vz_im = _jp(vz)[..., KC], _jm(vz)[..., KC], _ip(vz)[..., KC], _im(vz)[..., KC]
    vy_jp = _jp(vy)
    hzz = ((vz_ip + c) * (vz_ip + c) - (vz_im + c) * (vz_im + c)) * udz
    hzy = ((vy_jp[..., KC] + _im(vy_jp)[..., KC]) * (vz_jp + c)
           - (vy[..., KC] + _im(vy)[..., KC]) * (c + vz_jm)) * udy
    hzx = ((vx[..., KP] + vx_im[..., KP]) * (vz[..., KPP] + c)
           - (vx[..., KC] + vx_im[..., KC]) * (c + vz[..., KMM])) * g.udx3m[:nxm] * 0.25
    dzzvz = (vz_ip - 2.0 * c + vz_im) * udzq
    dyyvz = (vz_jp - 2.0 * c + vz_jm) * udyq
    dq[..., :nxm] = -(hzx + hzy + hzz) + dyyvz + dzzvz
    if p.gaxis == 3:
        tempit = p.active_t * 0.5 * (s.temp[..., KC] + _im(s.temp)[..., KC])
        dq[..., :nxm] = dq[..., :nxm] + g.byct * tempit


def explicit_terms_temp(g: Grid, s: State, hro: np.ndarray) -> None:
    """``ExplicitTermsTemp.F90:22-77``: hro(k=1..nxm) with plate values at k=1 and k=nxm."""
    p = g.p
    nxm = p.nxm
    udz = g.dz * 0.5
    udy = g.dy * 0.5
    udzq = g.dzq / g.pect
    udyq = g.dyq / g.pect
    vx, vy, vz, t = s.vx, s.vy, s.vz, s.temp
    KC = np.arange(nxm)
    tc = t[..., KC]
    htx = np.empty_like(tc)
    u = g.udx3m
    if nxm > 2:
        k = np.arange(1, nxm - 1)
        htx[..., 1:nxm - 1] = (vx[..., k + 1] * (t[..., k + 1] + t[..., k])
                               - vx[..., k] * (t[..., k] + t[..., k - 1])) * 0.5 * u[k]
    if nxm > 1:
        k = nxm - 1
        htx[..., k] = (vx[..., k + 1] * 2.0 * s.temptp
                       - vx[..., k] * (t[..., k] + t[..., k - 1])) * 0.5 * u[k]
    htx[..., 0] = (vx[..., 1] * (t[..., 1] + t[..., 0]) - vx[..., 0] * 2.0 * s.tempbp) * 0.5 * u[0]
    t_ip, t_im, t_jp, t_jm = _ip(t)[..., KC], _im(t)[..., KC], _jp(t)[..., KC], _jm(t)[..., KC]
    htz = (_ip(vz)[..., KC] * (t_ip + tc) - vz[..., KC] * (tc + t_im)) * udz
    hty = (_jp(vy)[..., KC] * (t_jp + tc) - vy[..., KC] * (tc + t_jm)) * udy
    dzzt = (t_ip - 2.0 * tc + t_im) * udzq
    dyyt = (t_jp - 2.0 * tc + t_jm) * udyq
    hro[..., :nxm] = -(htx + hty + htz) + dyyt + dzzt


# ----------------------------------------------------------------------------------------------
# Implicit Crank-Nicolson updates
# ----------------------------------------------------------------------------------------------
def _columns(a, n):
    """(nzm, nym, *) array → Fortran-ordered (n, nym*nzm) right-hand-side block."""
    return np.asfortranarray(a[..., :n].reshape(-1, n).T)


def _uncolumns(b, shape):
    nzm, nym = shape[0], shape[1]
    return b.T.reshape(nzm, nym, -1)


def _dgttrs_columns(dl, d, du, rhs_cols):
    dl2, d2, du2_, du2, ipiv, info = lapack.dgttrf(dl, d, du)
    if info != 0:
        raise FloatingPointError(f"dgttrf info={info}")
    x, info = lapack.dgttrs(dl2, d2, du2_, du2, ipiv, rhs_cols)
    if info != 0:
        raise FloatingPointError(f"dgttrs info={info}")
    return x


def implicit_and_update_vx(g: Grid, s: State, qcap, al, ga, ro, dt, beta) -> None:
    """``ImplicitAndUpdateVX.F90:26-87`` + ``SolveImpEqnUpdate_X.F90:25-67``."""
    p = g.p
    nxm, nx = p.nxm, g.nx
    alre = al / g.ren
    K = slice(1, nxm)
    KM = slice(0, nxm - 1)
    KP = slice(2, nxm + 1)
    vx, pr = s.vx, s.pr
    udx3 = al * g.udx3c[K]
    dxxvx = vx[..., KP] * g.ap3ck[K] + vx[..., K] * g.ac3ck[K] + vx[..., KM] * g.am3ck[K]
    dxp = (pr[..., K] - pr[..., KM]) * udx3
    rhs = np.zeros(vx.shape)
    rhs[..., K] = (ga * qcap[..., K] + ro * s.rux[..., K] + alre * dxxvx - dxp) * dt
    s.rux[..., K] = qcap[..., K]

    betadx = beta * al
    amkl = np.zeros(nx)
    apkl = np.zeros(nx)
    ackl = np.ones(nx)
    for kc in range(1, nxm):
        ackl_b = 1.0 / (1.0 - g.ac3ck[kc] * betadx)
        amkl[kc] = -g.am3ck[kc] * betadx * ackl_b
        apkl[kc] = -g.ap3ck[kc] * betadx * ackl_b
    ackl_b = 1.0 / (1.0 - g.ac3ck[K] * betadx)
    rhs[..., K] = rhs[..., K] * ackl_b
    rhs[..., 0] = 0.0
    rhs[..., nx - 1] = 0.0
    x = _dgttrs_columns(amkl[1:nx], ackl.copy(), apkl[0:nx - 1], _columns(rhs, nx))
    x = _uncolumns(x, vx.shape)
    vx[..., K] = vx[..., K] + x[..., K]
    vx[..., 0] = 0.0
    vx[..., nx - 1] = 0.0


def _solve_yz_like(g: Grid, q, rhs, ap, ac, am, betadx):
    """``SolveImpEqnUpdate_YZ.F90:25-58`` / ``SolveImpEqnUpdate_Temp.F90:25-61``."""
    nxm = g.p.nxm
    amkl = np.zeros(nxm)
    apkl = np.zeros(nxm)
    ackl = np.ones(nxm)
    for kc in range(nxm):
        ackl_b = 1.0 / (1.0 - ac[kc] * betadx)
        amkl[kc] = -am[kc] * betadx * ackl_b
        apkl[kc] = -ap[kc] * betadx * ackl_b
    ackl_b = 1.0 / (1.0 - ac[:nxm] * betadx)
    rhs[..., :nxm] = rhs[..., :nxm] * ackl_b
    if nxm == 1:
        x = rhs[..., :1] / ackl[0]
    else:
        x = _uncolumns(_dgttrs_columns(amkl[1:nxm], ackl.copy(), apkl[0:nxm - 1],
                                       _columns(rhs, nxm)), q.shape)
    q[..., :nxm] = q[..., :nxm] + x[..., :nxm]


def implicit_and_update_vy(g: Grid, s: State, dph, al, ga, ro, dt, beta) -> None:
    """``ImplicitAndUpdateVY.F90:28-93``."""
    p = g.p
    nxm = p.nxm
    alre = al / g.ren
    udy = g.dy * al
    vy = s.vy
    KC = np.arange(nxm)
    amm, acc, app = g.am3sk[:nxm], g.ac3sk[:nxm], g.ap3sk[:nxm]
    c = vy[..., KC]
    dxxvy = vy[..., g.kpv] * app + c * acc + vy[..., g.kmv] * amm
    dxxvy[..., 0] = (vy[..., g.kpv[0]] * app[0] + c[..., 0] * acc[0]
                     - (acc[0] + app[0]) * p.xminusu * p.inslws)
    if nxm > 1:
        k = nxm - 1
        dxxvy[..., k] = (-(acc[k] + amm[k]) * p.xplusu * p.inslwn + c[..., k] * acc[k]
                         + vy[..., g.kmv[k]] * amm[k])
    dyp = (s.pr[..., KC] - _jm(s.pr)[..., KC]) * udy
    rhs = np.zeros(vy.shape)
    rhs[..., :nxm] = (ga * dph[..., KC] + ro * s.ruy[..., KC] + alre * dxxvy - dyp) * dt
    s.ruy[..., :nxm] = dph[..., :nxm]
    _solve_yz_like(g, vy, rhs, g.ap3sk, g.ac3sk, g.am3sk, beta * al)


def implicit_and_update_vz(g: Grid, s: State, dq, al, ga, ro, dt, beta) -> None:
    """``ImplicitAndUpdateVZ.F90:26-77``."""
    p = g.p
    nxm = p.nxm
    alre = al / g.ren
    vz = s.vz
    KC = np.arange(nxm)
    amm, acc, app = g.am3sk[:nxm], g.ac3sk[:nxm], g.ap3sk[:nxm]
    dxxvz = vz[..., g.kpv] * app + vz[..., KC] * acc + vz[..., g.kmv] * amm
    dzp = (s.pr[..., KC] - _im(s.pr)[..., KC]) * g.dz * al
    rhs = np.zeros(vz.shape)
    rhs[..., :nxm] = (ga * dq[..., KC] + ro * s.ruz[..., KC] + alre * dxxvz - dzp) * dt
    s.ruz[..., :nxm] = dq[..., :nxm]
    _solve_yz_like(g, vz, rhs, g.ap3sk, g.ac3sk, g.am3sk, beta * al)


def implicit_and_update_temp(g: Grid, s: State, hro, al, ga, ro, dt) -> None:
    """``ImplicitAndUpdateTemp.F90:22-74`` + ``SolveImpEqnUpdate_Temp.F90:25-61``."""
    p = g.p
    nxm = p.nxm
    alpec = al / g.pect
    t = s.temp
    am, ac, ap = g.am3ssk, g.ac3ssk, g.ap3ssk
    dxxt = np.empty(t.shape[:2] + (nxm,))
    if nxm > 2:
        k = np.arange(1, nxm - 1)
        dxxt[..., 1:nxm - 1] = t[..., k + 1] * ap[k] + t[..., k] * ac[k] + t[..., k - 1] * am[k]
    if nxm > 1:
        k = nxm - 1
        dxxt[..., k] = (t[..., k] * ac[k] + t[..., k - 1] * am[k]
                        - (am[k] + ac[k]) * s.temptp * p.tfixn)
    dxxt[..., 0] = (t[..., 1] * ap[0] + t[..., 0] * ac[0]
                    - (ap[0] + ac[0]) * s.tempbp * p.tfixs)
    rhs = np.zeros(t.shape)
    rhs[..., :nxm] = (ga * hro[..., :nxm] + ro * s.rutemp[..., :nxm] + alpec * dxxt) * dt
    s.rutemp[..., :nxm] = hro[..., :nxm]
    betadx = 0.5 * al * dt / g.pect
    _solve_yz_like(g, t, rhs, ap, ac, am, betadx)


# ----------------------------------------------------------------------------------------------
# Pressure
# ----------------------------------------------------------------------------------------------
def calc_local_divergence(g: Grid, s: State, al, dt) -> np.ndarray:
    """``pressure.F90:141-162``: dph = div(u)/(al*dt), shape (nzm, nym, nxm)."""
    nxm = g.p.nxm
    usdtal = 1.0 / (dt * al)
    KC = np.arange(nxm)
    dqcap = ((_ip(s.vz)[..., KC] - s.vz[..., KC]) * g.dz
             + (_jp(s.vy)[..., KC] - s.vy[..., KC]) * g.dy
             + (s.vx[..., KC + 1] - s.vx[..., KC]) * g.udx3m[:nxm])
    return dqcap * usdtal


def solve_tridiagonal_pressure(g: Grid, dphc: np.ndarray) -> None:
    """``pressure.F90:201-236``: per (ky, kz) a normalised complex tridiagonal with the
    ``1+1e-15`` diagonal, solved by ``zgttrf``/``zgttrs``.  ``dphc`` has shape
    (nzm, nym//2+1, nxm) and is overwritten with the solution."""
    nxm = g.p.nxm
    acphk, amphk, apphk = g.acphk[:nxm], g.amphk[:nxm], g.apphk[:nxm]
    nzm, nyh = dphc.shape[0], dphc.shape[1]
    acphT = np.full(nxm, 1.0 + 1.0e-15, dtype=np.complex128)
    for i in range(nzm):
        for j in range(nyh):
            acphT_b = 1.0 / (acphk - g.ak2[j] - g.ak1[i])
            rhs = dphc[i, j, :] * acphT_b
            if nxm == 1:
                dphc[i, j, :] = rhs / acphT[0]
                continue
            apph = (apphk[:nxm - 1] * acphT_b[:nxm - 1]).astype(np.complex128)
            amph = (amphk[1:] * acphT_b[1:]).astype(np.complex128)
            diag = acphT.copy()
            if g.pin_zero_mode and i == 0 and j == 0:
                # The reference's near-singular solve moves the non-constant part of phi by
                # ~eps * cond; CorrectPressure's wall-normal operator amplifies that in pr on
                # fine stretched grids (3.9e-9 relative at nxm = 800).
                amph[-1] = 0.0
                diag[-1] = 1.0
                rhs = rhs.copy()
                rhs[-1] = 0.0
            dl, d, du, du2, ipiv, info = lapack.zgttrf(amph, diag, apph)
            if info > 0:
                raise FloatingPointError(f"Singular value found in LAPACK routine zgttrf: info={info}")
            x, info = lapack.zgttrs(dl, d, du, du2, ipiv, rhs.reshape(nxm, 1))
            dphc[i, j, :] = x[:, 0]


def solve_pressure_correction(g: Grid, dph: np.ndarray) -> np.ndarray:
    """``pressure.F90:165-197``: forward y r2c + z c2c, normalise by 1/(nym*nzm), tridiagonal
    in x, unnormalised backward z c2c + y c2r.  Returns phi, shape (nzm, nym, nxm)."""
    nym, nzm = g.p.nym, g.p.nzm
    cy = np.fft.rfft(dph, axis=1)
    cz = np.fft.fft(cy, axis=0)
    cz = cz / float(nzm * nym)
    cz = np.ascontiguousarray(cz)
    solve_tridiagonal_pressure(g, cz)
    cy = np.fft.ifft(cz, axis=0, norm="forward")
    return np.fft.irfft(cy, n=nym, axis=1, norm="forward")


def remove_divergence(g: Grid, s: State, phi, al, dt) -> None:
    """``pressure.F90:240-267`` (through ``CorrectVelocity.F90:24``)."""
    nxm = g.p.nxm
    udy = al * dt * g.dy
    udz = al * dt * g.dz
    usukm = al * dt * g.udx3c[:nxm]
    s.vx[..., :nxm] = s.vx[..., :nxm] - (phi - phi[..., g.kmv]) * usukm
    s.vy[..., :nxm] = s.vy[..., :nxm] - (phi - _jm(phi)) * udy
    s.vz[..., :nxm] = s.vz[..., :nxm] - (phi - _im(phi)) * udz


def correct_pressure(g: Grid, s: State, phi, al, beta) -> None:
    """``pressure.F90:270-301``."""
    nxm = g.p.nxm
    be = al * beta
    amm, acc, app = g.amphk[:nxm], g.acphk[:nxm], g.apphk[:nxm]
    s.pr[..., :nxm] = s.pr[..., :nxm] + phi - be * (
        (_ip(phi) - 2.0 * phi + _im(phi)) * g.dzq
        + (_jp(phi) - 2.0 * phi + _jm(phi)) * g.dyq
        + (phi[..., g.kpv] * app + phi * acc + phi[..., g.kmv] * amm))


# ----------------------------------------------------------------------------------------------
# Diagnostics
# ----------------------------------------------------------------------------------------------
def calc_max_cfl(g: Grid, s: State) -> float:
    """``CalcMaxCFL.F90:22-43`` (initial value 1e-8)."""
    nxm = g.p.nxm
    KC = np.arange(nxm)
    qcf = (np.abs((s.vz[..., KC] + _ip(s.vz)[..., KC]) * 0.5 * g.dz)
           + np.abs((s.vy[..., KC] + _jp(s.vy)[..., KC]) * 0.5 * g.dy)
           + np.abs((s.vx[..., KC] + s.vx[..., KC + 1]) * 0.5 * g.udx3m[:nxm]))
    return max(0.00000001, float(qcf.max()))


def check_divergence(g: Grid, s: State) -> float:
    """``CheckDivergence.F90:22-42``: max |div u| (no 1/(al*dt))."""
    nxm = g.p.nxm
    KC = np.arange(nxm)
    dqcap = ((_ip(s.vz)[..., KC] - s.vz[..., KC]) * g.dz
             + (_jp(s.vy)[..., KC] - s.vy[..., KC]) * g.dy
             + (s.vx[..., KC + 1] - s.vx[..., KC]) * g.udx3m[:nxm])
    return float(np.abs(dqcap).max())


def nusselt_volume(g: Grid, s: State) -> float:
    """Volume Nusselt number of ``GlobalQuantities.F90:35-79``:
    1 + sqrt(Pr*|Ra|) * vol * sum(T * (vx_k + vx_{k+1})/2 * g3rc_k)."""
    p = g.p
    nxm = p.nxm
    vol = 1.0 / (p.alx3 * g.dx * float(p.nzm) * float(p.nym))
    vxcen = (s.vx[..., :nxm] + s.vx[..., 1:nxm + 1]) * 0.5
    anusin = float(np.sum(s.temp[..., :nxm] * vxcen * g.g3rc[:nxm]))
    return 1.0 + math.sqrt(p.prat * abs(p.rayt)) * anusin * vol


def kinetic_energy(g: Grid, s: State) -> float:
    """Volume-mean 0.5*(vx^2+vy^2+vz^2), g3rc-weighted as ``GlobalQuantities.F90:53-57, 91``."""
    p = g.p
    nxm = p.nxm
    vol = 1.0 / (p.alx3 * g.dx * float(p.nzm) * float(p.nym))
    w = g.g3rc[:nxm]
    e = (s.vz[..., :nxm] ** 2 + s.vy[..., :nxm] ** 2 + s.vx[..., :nxm] ** 2) * w
    return 0.5 * float(np.sum(e)) * vol


# ----------------------------------------------------------------------------------------------
# Substep loop and step control
# ----------------------------------------------------------------------------------------------
def time_marcher(g: Grid, s: State, dt: float) -> None:
    """``TimeMarcher.F90:28-133``: nsst substeps of explicit terms, CN updates, Poisson solve
    and projection (flow + temperature only)."""
    p = g.p
    gam, rom, alm = rk3_coefficients(p.nsst)
    beta = dt / g.ren * 0.5
    shape = s.vx.shape
    for ns in range(p.nsst):
        al, ga, ro = alm[ns], gam[ns], rom[ns]
        qcap = np.zeros(shape)
        dph = np.zeros(shape)
        dq = np.zeros(shape)
        hro = np.zeros(shape)
        explicit_terms_vx(g, s, qcap)
        explicit_terms_vy(g, s, dph)
        explicit_terms_vz(g, s, dq)
        explicit_terms_temp(g, s, hro)
        implicit_and_update_vx(g, s, qcap, al, ga, ro, dt, beta)
        implicit_and_update_vy(g, s, dph, al, ga, ro, dt, beta)
        implicit_and_update_vz(g, s, dq, al, ga, ro, dt, beta)
        implicit_and_update_temp(g, s, hro, al, ga, ro, dt)
        div = calc_local_divergence(g, s, al, dt)
        phi = solve_pressure_correction(g, div)
        remove_divergence(g, s, phi, al, dt)
        correct_pressure(g, s, phi, al, beta)


def next_dt(p: Params, ntime: int, dt: float, cflm: float):
    """Step-size rule of ``main.F90:287-304``: returns (dt, errorcode, cfl_report)."""
    err = 0
    if p.idtv == 1:
        if ntime > 1:
            dt = p.dtmax if cflm < 1.0e-8 else p.limit_cfl / cflm
            if dt > p.dtmax:
                dt = p.dtmax
        if dt < p.dtmin:
            err = 166
        return dt, err, cflm
    cflr = cflm * dt
    if cflr > p.limit_cfl:
        err = 165
    return dt, err, cflr


def run(g: Grid, s: State, nsteps: int, callback=None):
    """Main-loop restatement (``main.F90:281-313``) for ``nsteps`` steps: CFL, dt rule,
    TimeMarcher, time += dt.  Returns (time, dt, errorcode)."""
    p = g.p
    dt = p.dt
    time = 0.0
    err = 0
    for ntime in range(nsteps):
        cflm = calc_max_cfl(g, s)
        dt, err, _ = next_dt(p, ntime, dt, cflm)
        time_marcher(g, s, dt)
        time += dt
        if callback is not None:
            callback(ntime, time, dt, s)
        if err:
            break
    return time, dt, err


# ----------------------------------------------------------------------------------------------
# Wall-normal profiles (CalcMeanProfiles.F90)
# ----------------------------------------------------------------------------------------------
MEAN_PROFILE_NAMES = ("Tbar", "vybar", "vzbar", "vxT", "vyT", "vzT", "Trms", "vxrms", "vyrms", "vzrms",
                      "vxvy", "vxvz", "vyvz", "chiT", "epsilon")


def mean_profiles(g: Grid, s: State) -> dict:
    """``CalcMeanProfiles.F90:37-208``: the fifteen y-z averaged profiles written to means.h5,
    each of length nxm (names as the datasets, order of ``MEAN_PROFILE_NAMES``)."""
    p = g.p
    nxm = p.nxm
    inym, inzm = 1.0 / p.nym, 1.0 / p.nzm
    vx, vy, vz, t = s.vx, s.vy, s.vz, s.temp
    K = np.arange(nxm)
    vxc, vxp = vx[..., K], vx[..., K + 1]
    vyc, vyjp = vy[..., :nxm], _jp(vy)[..., :nxm]
    vzc, vzip = vz[..., :nxm], _ip(vz)[..., :nxm]
    tc = t[..., :nxm]

    def sums(a):
        return a.sum(axis=(0, 1))

    out = {}
    # :48-72 sums, :88-102 normalisation
    out["Tbar"] = sums(tc) * inym * inzm
    out["vybar"] = sums(0.5 * (vyc + vyjp)) * inym * inzm
    out["vzbar"] = sums(0.5 * (vzc + vzip)) * inym * inzm
    out["vxT"] = sums(0.5 * (vxc + vxp) * tc) * inym * inzm
    out["vyT"] = sums(0.5 * (vyc + vyjp) * tc) * inym * inzm
    out["vzT"] = sums(0.5 * (vzc + vzip) * tc) * inym * inzm
    out["Trms"] = np.sqrt(sums(tc ** 2) * inym * inzm)
    out["vxrms"] = np.sqrt(sums(0.5 * (vxc ** 2 + vxp ** 2)) * inym * inzm)
    out["vyrms"] = np.sqrt(sums(0.5 * (vyc ** 2 + vyjp ** 2)) * inym * inzm)
    out["vzrms"] = np.sqrt(sums(0.5 * (vzc ** 2 + vzip ** 2)) * inym * inzm)
    out["vxvy"] = sums(0.25 * (vxc + vxp) * (vyc + vyjp)) * inym * inzm
    out["vxvz"] = sums(0.25 * (vxc + vxp) * (vzc + vzip)) * inym * inzm
    out["vyvz"] = sums(0.25 * (vyc + vyjp) * (vzc + vzip)) * inym * inzm

    # :104-128 thermal dissipation
    dy, dz, dx = g.dy, g.dz, g.dx
    chi = ((_ip(t) - _im(t))[..., :nxm] * 0.5 * dz) ** 2 + ((_jp(t) - _jm(t))[..., :nxm] * 0.5 * dy) ** 2
    tdx = 0.5 * dx / g.g3rm[:nxm]
    dT = np.empty_like(tc)
    dT[..., 0] = t[..., 1] - t[..., 0] + 2.0 * p.tfixs * (t[..., 0] - s.tempbp)
    dT[..., 1:nxm - 1] = t[..., 2:nxm] - t[..., 0:nxm - 2]
    dT[..., nxm - 1] = t[..., nxm - 1] - t[..., nxm - 2] + 2.0 * p.tfixn * (s.temptp - t[..., nxm - 1])
    chi = chi + (dT * tdx) ** 2
    out["chiT"] = sums(chi) * inym * inzm / g.pect  # :203-207

    # :164-199 viscous dissipation
    vzip_, vyip_, vyim_, vxip_, vxim_ = _ip(vz), _ip(vy), _im(vy), _ip(vx), _im(vx)
    eps = (((vzip_ - vz)[..., :nxm] * dz) ** 2
           + 0.125 * dz ** 2 * ((_jp(vyip_) - _jp(vyim_))[..., :nxm] ** 2 + (vyip_ - vyim_)[..., :nxm] ** 2)
           + 0.125 * dz ** 2 * ((vxip_ - vxim_)[..., K + 1] ** 2 + (vxip_ - vxim_)[..., K] ** 2)
           + 0.125 * dy ** 2 * ((_jp(vzip_) - _jm(vzip_))[..., :nxm] ** 2 + (_jp(vz) - _jm(vz))[..., :nxm] ** 2)
           + ((_jp(vy) - vy)[..., :nxm] * dy) ** 2
           + 0.125 * dy ** 2 * ((_jp(vx) - _jm(vx))[..., K + 1] ** 2 + (_jp(vx) - _jm(vx))[..., K] ** 2)
           + ((vxp - vxc) * g.udx3m[:nxm]) ** 2)
    tdx2 = 0.125 * (dx / g.g3rm[:nxm]) ** 2
    vyjp_ = _jp(vy)
    dzx = np.empty_like(tc)
    dzx_i = np.empty_like(tc)
    dyx = np.empty_like(tc)
    dyx_j = np.empty_like(tc)
    # wall rows with the no-slip / moving-wall ghost values, interior central differences
    dzx[..., 0] = vzip_[..., 1] - vzip_[..., 0] + p.inslws * 2.0 * (vzip_[..., 0] - 0.0)
    dzx_i[..., 0] = vz[..., 1] - vz[..., 0] + p.inslws * 2.0 * (vz[..., 0] - 0.0)
    dyx[..., 0] = vyjp_[..., 1] - vyjp_[..., 0] + p.inslws * 2.0 * (vyjp_[..., 0] - p.xminusu)
    dyx_j[..., 0] = vy[..., 1] - vy[..., 0] + p.inslws * 2.0 * (vy[..., 0] - p.xminusu)
    dzx[..., 1:nxm - 1] = vzip_[..., 2:nxm] - vzip_[..., 0:nxm - 2]
    dzx_i[..., 1:nxm - 1] = vz[..., 2:nxm] - vz[..., 0:nxm - 2]
    dyx[..., 1:nxm - 1] = vyjp_[..., 2:nxm] - vyjp_[..., 0:nxm - 2]
    dyx_j[..., 1:nxm - 1] = vy[..., 2:nxm] - vy[..., 0:nxm - 2]
    n1 = nxm - 1
    dzx[..., n1] = vzip_[..., n1] - vzip_[..., n1 - 1] + p.inslwn * 2.0 * (0.0 - vzip_[..., n1])
    dzx_i[..., n1] = vz[..., n1] - vz[..., n1 - 1] + p.inslwn * 2.0 * (0.0 - vz[..., n1])
    dyx[..., n1] = vyjp_[..., n1] - vyjp_[..., n1 - 1] + p.inslwn * 2.0 * (p.xplusu - vyjp_[..., n1])
    dyx_j[..., n1] = vy[..., n1] - vy[..., n1 - 1] + p.inslwn * 2.0 * (p.xplusu - vy[..., n1])
    eps = eps + tdx2 * (dzx ** 2 + dzx_i ** 2) + tdx2 * (dyx ** 2 + dyx_j ** 2)
    out["epsilon"] = sums(eps) * inym * inzm / g.ren
    return out


# ----------------------------------------------------------------------------------------------
# Spectra (spectra.F90)
# ----------------------------------------------------------------------------------------------
def fourier_coef(g: Grid, var: np.ndarray) -> np.ndarray:
    """``CalcFourierCoef`` (spectra.F90:70-96): y r2c then z c2c of var (nzm, nym, nxm), scaled by
    1/(nzm*nym).  Returns (nzm, nym//2+1, nxm)."""
    cy = np.fft.rfft(var, axis=1)
    cz = np.fft.fft(cy, axis=0)
    return cz * (1.0 / (g.p.nzm * g.p.nym))


def spectra_update(g: Grid, s: State, dt: float, acc: dict) -> None:
    """``UpdateSpectra`` / ``AddRealSpectrum`` (spectra.F90:101-114, 139-144): acc[name] += dt*|F|^2
    for vx, vy, vz, temp at k = 1..nxm (no interpolation)."""
    nxm = g.p.nxm
    for name in ("vx", "vy", "vz", "temp"):
        f = fourier_coef(g, getattr(s, name)[..., :nxm])
        acc[name] = acc.get(name, 0.0) + dt * np.abs(f) ** 2


# ----------------------------------------------------------------------------------------------
# Plane means (h5tools/mean_zplane.F90, h5tools/means.F90)
# ----------------------------------------------------------------------------------------------
def mean_plane(field: np.ndarray, axis: int) -> np.ndarray:
    """``ymean`` (axis 1, ``means.F90:10-45``) or ``zmean`` (axis 2, ``means.F90:47-82``) of a
    field stored (nz, ny, nx_rows): plane(k, i) = sum_j var(k, j, i) / nym, or plane(k, j) =
    sum_i var(k, j, i) / nzm, summed in ascending order as the reference's loops do (one rank,
    so the MPI_REDUCE adds nothing), then divided once.  Returns (nz, nx_rows) or (ny, nx_rows).
    The refined-grid versions ``ymeanr`` / ``zmeanr`` (``means.F90:84-157`` and on) are the same
    without IBM."""
    f = np.asarray(field, dtype=np.float64)
    nz, ny, _ = f.shape
    if axis == 1:
        acc = np.zeros((nz, f.shape[2]))
        for j in range(ny):
            acc = acc + f[:, j, :]
        return acc / float(ny)
    acc = np.zeros((ny, f.shape[2]))
    for i in range(nz):
        acc = acc + f[i, :, :]
    return acc / float(nz)
