"""CPU oracle for the multi-resolution salinity scalar.  TEST INFRASTRUCTURE ONLY.

This module is test infrastructure, never the product: only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference arm may import it.  It is an FP64 NumPy restatement of
the reference routines that evolve salinity on a refined grid and couple it to the flow:

* refined grid and metrics   ``src/multires/CreateMgrdGrid.F90:11-163``
* interpolation stencils     ``src/multires/CreateMgrdStencil.F90:1-80`` with
                             ``interpolation_indices`` / ``extend_grid`` / ``construct_stencil``
                             of ``src/multires/HermiteInterpolations.F90:26-164``
* coarse -> refined          ``interpolate_xyz_to_refined`` (``HermiteInterpolations.F90:168-200``)
                             inside ``InterpVelMgrd`` (``src/multires/InterpVelMgrd.F90:1-242``):
                             velocity gradients interpolated, then integrated along x, y and z
* refined -> coarse          ``InterpSalMultigrid`` (``src/salinity.F90:455-492``) through
                             ``interpolate_xyz_to_coarse_fast`` / ``interpolate_xyz_to_coarse``
                             (``HermiteInterpolations.F90:202-288``)
* salinity explicit terms    ``ExplicitSalinity`` (``salinity.F90:268-367``, no IBM)
* salinity CN update         ``ImplicitSalinity`` + ``SolveImpEqnUpdate_Sal`` (``salinity.F90:369-453``)
* buoyancy coupling          ``AddSalBuoyancy`` (``salinity.F90:494-506``), called from
                             ``TimeMarcher.F90:50-63``
* refined CFL                ``CalcMaxCFL.F90:48-68``
* statistics                 ``CalcSalStats`` / ``CalcDissipationSal`` (``salinity.F90:508-667``)
* boundary planes and ICs    ``SetSalBCs`` / ``CreateInitialSalinity`` (``salinity.F90:105-176``);
                             the reference's unseeded ``random_number`` noise is replaced by
                             Philox4x32-10 keyed by the refined cell index k + nxr*(j + nymr*i)

Index conventions.  Arrays are C-order ``a[i, j, k]`` = Fortran ``a(k, j, i)`` (0-based).  The
Fortran index arrays (``irangs`` and friends) keep their Fortran values and their Fortran
subscripts: ``idx[io]`` holds ``idx(io)`` for io = 0 .. n_old + 1.  Stencil weights ``c[:, n]``
hold Fortran ``cx(1:4, n+1)``.  An x-extended array holds Fortran rows -1 .. n+1 at positions
0 .. n+2.

Two forms of the interpolation are restated: the reference's loop nest over source intervals
(``*_loops``, pure Python, small grids only) and a per-target form (for every target point the
first of its four source points and their weights) that the vectorised oracle and the CUDA
kernels evaluate.  The tests check the two against each other.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
from scipy.linalg import lapack

from oracle import afid_oracle as o


# ----------------------------------------------------------------------------------------------
# HermiteInterpolations.F90 stencil construction
# ----------------------------------------------------------------------------------------------
def interpolation_indices(x_old: np.ndarray, x_new: np.ndarray, x_len: float) -> np.ndarray:
    """``HermiteInterpolations.F90:26-57``: idx(io), io = 0 .. n_old+1, is the first new index
    whose coordinate is >= x_old(io) (Fortran values, 1-based)."""
    n_old, n_new = x_old.size, x_new.size
    xn = np.zeros(n_new + 2)
    xn[1:n_new + 1] = x_new
    xn[0] = -xn[1]
    if xn[0] == xn[1]:
        xn[0] = -xn[2]
    xn[n_new + 1] = 2.0 * x_len - xn[n_new]
    if xn[n_new + 1] == xn[n_new]:
        xn[n_new + 1] = 2.0 * x_len - xn[n_new - 1]
    idx = np.zeros(n_old + 2, dtype=np.int64)
    idx[0] = 1
    for io in range(1, n_old + 1):
        xo = x_old[io - 1]
        for inn in range(0, n_new + 1):
            if xn[inn] < xo and xn[inn + 1] >= xo:
                idx[io] = inn + 1
    idx[n_old + 1] = n_new + 1
    return idx


def extend_grid(x_og: np.ndarray, x_len: float, n_ext: int):
    """``HermiteInterpolations.F90:59-103``.  Returns ``x`` with Fortran x_ext(i) at
    x[i + n_ext - 1], i = 1-n_ext .. n_og+n_ext.  Mirror points that would read past the
    original grid (the reference reads out of bounds there; only possible for n_og <= n_ext)
    are filled with the nearest mirror that exists; they only ever meet a zero weight."""
    n_og = x_og.size
    x = np.zeros(n_og + 2 * n_ext)
    off = n_ext - 1

    def og(i):  # Fortran x_og(i), clamped
        return x_og[min(max(i, 1), n_og) - 1]

    x[off + 1:off + n_og + 1] = x_og
    if abs(x_og[0]) < 1e-10:
        for i in range(1, n_ext + 1):
            x[off + 1 - i] = -og(1 + i)
    else:
        for i in range(1, n_ext + 1):
            x[off + 1 - i] = -og(i)
    if abs(x_og[n_og - 1] - x_len) < 1e-10:
        for i in range(1, n_ext + 1):
            x[off + n_og + i] = 2 * x_len - og(n_og - i)
    else:
        for i in range(1, n_ext + 1):
            x[off + n_og + i] = 2 * x_len - og(n_og + 1 - i)
    return x, off


def construct_stencil(x_old, x_new, x_len, idx, axis: str) -> np.ndarray:
    """``HermiteInterpolations.F90:105-164``: cubic Hermite weights (linear next to a wall in x)
    for every new point; c[:, n] = Fortran cx(1:4, n+1)."""
    n_old, n_new = x_old.size, x_new.size
    cx = np.zeros((4, n_new))
    n_ext = 1 if axis == "x" else 2
    xo_a, oo = extend_grid(x_old, x_len, n_ext)
    xn_a, on = extend_grid(x_new, x_len, n_ext)
    xo = lambda i: xo_a[i + oo]  # noqa: E731
    xn = lambda i: xn_a[i + on]  # noqa: E731
    for io in range(0, n_old + 1):
        lo, hi = max(idx[io], 1), min(idx[io + 1] - 1, n_new)
        if axis == "x" and (io == 0 or io == n_old):
            dlc = xo(io + 1) - xo(io)
            for inn in range(lo, hi + 1):
                t = (xn(inn) - xo(io)) / dlc
                cx[:, inn - 1] = (0.0, 1 - t, t, 0.0)
        else:
            dlm = xo(io) - xo(io - 1)
            dlc = xo(io + 1) - xo(io)
            dlp = xo(io + 2) - xo(io + 1)
            for inn in range(lo, hi + 1):
                t = (xn(inn) - xo(io)) / dlc
                if t < 1e-12:
                    cx[:, inn - 1] = (0.0, 1.0, 0.0, 0.0)
                else:
                    h00 = (1.0 + 2.0 * t) * (1.0 - t) ** 2
                    h10 = t * (1.0 - t) ** 2
                    h01 = (1.0 + 2.0 * (1.0 - t)) * t ** 2
                    h11 = -(1.0 - t) * t ** 2
                    cx[0, inn - 1] = -h10 * dlc ** 2 / dlm / (dlc + dlm)
                    cx[1, inn - 1] = h00 - h11 * dlp / (dlp + dlc) + h10 * (dlc - dlm) / dlm
                    cx[2, inn - 1] = h01 + h10 * dlm / (dlm + dlc) + h11 * (dlp - dlc) / dlp
                    cx[3, inn - 1] = h11 * dlc ** 2 / dlp / (dlp + dlc)
    return cx


def starts_from_intervals(idx: np.ndarray, n_new: int, io_lo: int, io_hi: int) -> np.ndarray:
    """Per-target form of the loop ``do io=io_lo,io_hi; do in=max(idx(io),1),min(idx(io+1)-1,n_new)``
    whose body reads source rows io-1 .. io+2: returns, per new point (0-based), the 0-based
    index of its first source row (Fortran io-1, minus 1).  Every new point must be covered
    exactly once."""
    start = np.full(n_new, np.iinfo(np.int64).min, dtype=np.int64)
    for io in range(io_lo, io_hi + 1):
        for inn in range(max(idx[io], 1), min(idx[io + 1] - 1, n_new) + 1):
            if start[inn - 1] != np.iinfo(np.int64).min:
                raise ValueError("target covered twice")
            start[inn - 1] = io - 2
    if (start == np.iinfo(np.int64).min).any():
        raise ValueError("target not covered")
    return start


# ----------------------------------------------------------------------------------------------
# Refined grid (CreateMgrdGrid.F90) and stencils (CreateMgrdStencil.F90)
# ----------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Stencil:
    """Per-target interpolation along one axis: target n reads source rows start[n] .. start[n]+3
    (0-based; x rows of an extended array may be -2 .. n_src+1, y/z rows wrap periodically)
    with weights w[:, n] (Fortran cx(1:4, n+1))."""
    start: np.ndarray
    w: np.ndarray


@dataclasses.dataclass
class Mgrd:
    nxmr: int
    nymr: int
    nzmr: int
    xcr: np.ndarray      # [nxr]
    xmr: np.ndarray      # [nxr + 1]: Fortran xmr(0 .. nxr) at xmr[k]... see create_mgrd
    ycr: np.ndarray
    ymr: np.ndarray
    zcr: np.ndarray
    zmr: np.ndarray
    dxr: float
    dyr: float
    dzr: float
    dyqr: float
    dzqr: float
    g3rmr: np.ndarray    # [nxmr]
    udx3mr: np.ndarray   # [nxmr]
    ap3sskr: np.ndarray
    ac3sskr: np.ndarray
    am3sskr: np.ndarray
    pecs: float
    bycs: float
    sfixs: int
    sfixn: int
    active_s: int
    salbp: float
    saltp: float
    # Fortran index arrays and stencils (CreateMgrdStencil.F90)
    irangs: np.ndarray
    jrangs: np.ndarray
    krangs: np.ndarray
    cxrs: np.ndarray
    cyrs: np.ndarray
    czrs: np.ndarray
    fast: bool           # InterpSalMultigrid takes interpolate_xyz_to_coarse_fast
    irangb: np.ndarray
    jrangb: np.ndarray
    krangb: np.ndarray
    cxsalc: np.ndarray
    cysalc: np.ndarray
    czsalc: np.ndarray
    irangr: np.ndarray
    jrangr: np.ndarray
    krangr: np.ndarray
    cxphic: np.ndarray
    cyphic: np.ndarray
    czphic: np.ndarray
    # per-target forms
    to_ref: tuple        # (x, y, z) Stencil: coarse cell centres -> refined cell centres
    to_coarse: tuple     # (x, y, z) Stencil: refined salinity -> salc points

    @property
    def nxr(self) -> int:
        return self.nxmr + 1


def _x_grid(istr3: int, nm: int, length: float, s: float, pi: float, schmidt: float = 1.0):
    if istr3 == 0:
        return o._uniform_grid(nm, length)
    if istr3 == 1:
        return o._centre_focus_grid(nm, length, s)
    if istr3 == 3:
        return o._natural_bl_grid(nm, length, schmidt)
    if istr3 == 4:
        return o._tanh_grid(nm, length, s)
    if istr3 == 6:
        return o._cheb_grid(nm, length, s, pi)
    if istr3 == 7:
        return o._asym_cheb_grid(nm, length, s, pi)
    raise ValueError(f"ISTR3R={istr3} not supported")


def create_mgrd(g: o.Grid) -> Mgrd:
    """``CreateMgrdGrid.F90:21-163`` (refined metrics, salinity second-derivative coefficients)
    and ``CreateMgrdStencil.F90:1-80`` (interpolation stencils), for a coarse grid ``g`` whose
    Params carry MULTIRES / NXMR NYMR NZMR / ISTR3R / SfixS SfixN."""
    p = g.p
    nxm, nym, nzm = p.nxm, p.nym, p.nzm
    nxmr, nymr, nzmr = p.nxmr, p.nymr, p.nzmr
    nxr = nxmr + 1
    zcr, zmr = o._uniform_grid(nzmr, p.zlen)
    ycr, ymr = o._uniform_grid(nymr, p.ylen)
    xcr, _ = _x_grid(p.istr3r, nxmr, p.alx3, p.str3, g.pi, p.pras)
    dxr = float(nxmr) / p.alx3
    dyr = float(nymr) / p.ylen
    dzr = float(nzmr) / p.zlen
    # xmr(0 .. nxr) at xmr[0 .. nxr]
    xmr = np.zeros(nxr + 1)
    for kc in range(1, nxmr + 1):
        xmr[kc] = (xcr[kc - 1] + xcr[kc]) * 0.5
    xmr[0] = 2.0 * xcr[0] - xmr[1]
    xmr[nxr] = 2.0 * xcr[nxr - 1] - xmr[nxmr]
    g3rmr = np.zeros(nxmr)
    for kc in range(2, nxmr + 1):
        g3rmr[kc - 1] = (xmr[kc + 1] - xmr[kc - 1]) * dxr * 0.5
    g3rmr[0] = (xmr[2] - (2 * xcr[0] - xmr[1])) * dxr * 0.5
    d3xcr = np.array([(xcr[kc] - xcr[kc - 1]) * dxr for kc in range(1, nxmr + 1)])
    udx3mr = dxr / d3xcr
    ap, ac, am = o._second_derivative_coeff(xmr[1:nxmr + 1], p.alx3, p.sfixn, p.sfixs)
    pecs, bycs = p.derived_salinity()
    salbp, saltp = (-0.5, 0.5) if p.rays >= 0 else (0.5, -0.5)   # SetSalBCs (salinity.F90:105-121)

    xm = g.xm[:nxm]
    xc = g.xc[:nxm + 1]
    ym, yc, zm, zc = g.ym, g.yc[:nym], g.zm, g.zc[:nzm]
    xmr_in = xmr[1:nxmr + 1]
    # coarse cell centres -> refined cell centres (vx, vy, vz gradients, first-guess planes)
    irangs = interpolation_indices(xm, xmr_in, p.alx3)
    cxrs = construct_stencil(xm, xmr_in, p.alx3, irangs, "x")
    jrangs = interpolation_indices(ym, ymr, p.ylen)
    cyrs = construct_stencil(ym, ymr, p.ylen, jrangs, "y")
    krangs = interpolation_indices(zm, zmr, p.zlen)
    czrs = construct_stencil(zm, zmr, p.zlen, krangs, "z")
    # refined cell centres -> coarse cell centres (general path)
    irangr = interpolation_indices(xmr_in, xm, p.alx3)
    cxphic = construct_stencil(xmr_in, xm, p.alx3, irangr, "x")
    jrangr = interpolation_indices(ymr, ym, p.ylen)
    cyphic = construct_stencil(ymr, ym, p.ylen, jrangr, "y")
    krangr = interpolation_indices(zmr, zm, p.zlen)
    czphic = construct_stencil(zmr, zm, p.zlen, krangr, "z")
    # salinity to the buoyancy points: cell faces along gravity (CreateMgrdStencil.F90:26-33,...)
    if p.gaxis == 1:
        irange = interpolation_indices(xmr_in, xc, p.alx3)
        cxsalc = construct_stencil(xmr_in, xc, p.alx3, irange, "x")[:, :nxm]
        irangb = interpolation_indices(xc, xmr_in, p.alx3)
    else:
        irangb = irangs
        cxsalc = cxphic.copy()
    if p.gaxis == 2:
        jrange = interpolation_indices(ymr, yc, p.ylen)
        cysalc = construct_stencil(ymr, yc, p.ylen, jrange, "y")
        jrangb = interpolation_indices(yc, ymr, p.ylen)
    else:
        jrangb = jrangs
        cysalc = cyphic.copy()
    if p.gaxis == 3:
        krange = interpolation_indices(zmr, zc, p.zlen)
        czsalc = construct_stencil(zmr, zc, p.zlen, krange, "z")
        krangb = interpolation_indices(zc, zmr, p.zlen)
    else:
        krangb = krangs
        czsalc = czphic.copy()
    fast = bool(xmr[1] < xm[0] and xmr[nxmr] > xm[nxm - 1])   # salinity.F90:485

    to_ref = (Stencil(starts_from_intervals(irangs, nxmr, 0, nxm), cxrs),
              Stencil(starts_from_intervals(jrangs, nymr, 0, nym), cyrs),
              Stencil(starts_from_intervals(krangs, nzmr, 0, nzm), czrs))
    if fast:
        to_coarse = (Stencil(irangb[1:nxm + 1] - 3, cxsalc),
                     Stencil(jrangb[1:nym + 1] - 3, cysalc),
                     Stencil(krangb[1:nzm + 1] - 3, czsalc))
    else:
        to_coarse = (Stencil(starts_from_intervals(irangr, nxm, 0, nxmr), cxphic),
                     Stencil(starts_from_intervals(jrangr, nym, 0, nymr), cyphic),
                     Stencil(starts_from_intervals(krangr, nzm, 0, nzmr), czphic))
    return Mgrd(nxmr=nxmr, nymr=nymr, nzmr=nzmr, xcr=xcr, xmr=xmr, ycr=ycr, ymr=ymr, zcr=zcr,
                zmr=zmr, dxr=dxr, dyr=dyr, dzr=dzr, dyqr=dyr * dyr, dzqr=dzr * dzr, g3rmr=g3rmr,
                udx3mr=udx3mr, ap3sskr=ap, ac3sskr=ac, am3sskr=am, pecs=pecs, bycs=bycs,
                sfixs=p.sfixs, sfixn=p.sfixn, active_s=p.active_s, salbp=salbp, saltp=saltp,
                irangs=irangs, jrangs=jrangs, krangs=krangs, cxrs=cxrs, cyrs=cyrs, czrs=czrs,
                fast=fast, irangb=irangb, jrangb=jrangb, krangb=krangb, cxsalc=cxsalc,
                cysalc=cysalc, czsalc=czsalc, irangr=irangr, jrangr=jrangr, krangr=krangr,
                cxphic=cxphic, cyphic=cyphic, czphic=czphic, to_ref=to_ref, to_coarse=to_coarse)


# ----------------------------------------------------------------------------------------------
# Interpolation: per-target evaluation and the reference's loop nests
# ----------------------------------------------------------------------------------------------
def _rows_x(st: Stencil):
    """Positions in an x-extended array (Fortran rows -1 .. n+1 at 0 .. n+2) of the 4 sources."""
    return st.start[:, None] + 2 + np.arange(4)[None, :]


def _rows_periodic(st: Stencil, n: int):
    return np.mod(st.start[:, None] + np.arange(4)[None, :], n)


def interp3(ext: np.ndarray, sx: Stencil, sy: Stencil, sz: Stencil) -> np.ndarray:
    """Tensor-product interpolation of an x-extended, y/z-periodic array ``ext`` (nz, ny, n+3):
    out[i, j, k] = sum_a wx_a sum_b wy_b sum_c wz_c ext[...], contracted z first, then y, then x
    as ``qv2``/``qv1`` of ``HermiteInterpolations.F90:183-196``."""
    nz, ny = ext.shape[0], ext.shape[1]
    rz = _rows_periodic(sz, nz)            # (Tz, 4)
    ry = _rows_periodic(sy, ny)            # (Ty, 4)
    rx = _rows_x(sx)                       # (Tx, 4)
    out = None
    # z contraction: (Tz, ny, n+3)
    q2 = ext[rz[:, 0]] * sz.w[0][:, None, None]
    for c in range(1, 4):
        q2 = q2 + ext[rz[:, c]] * sz.w[c][:, None, None]
    # y contraction: (Tz, Ty, n+3)
    q1 = q2[:, ry[:, 0]] * sy.w[0][None, :, None]
    for b in range(1, 4):
        q1 = q1 + q2[:, ry[:, b]] * sy.w[b][None, :, None]
    # x: (Tz, Ty, Tx)
    out = q1[:, :, rx[:, 0]] * sx.w[0][None, None, :]
    for a in range(1, 4):
        out = out + q1[:, :, rx[:, a]] * sx.w[a][None, None, :]
    return out


def interp2_xz(plane: np.ndarray, sx: Stencil, sz: Stencil) -> np.ndarray:
    """First-guess plane of ``InterpVelMgrd.F90:99-116``: plane (nz, n+3) x-extended;
    z contracted first (qv1), then x.  Returns (Tz, Tx)."""
    rz = _rows_periodic(sz, plane.shape[0])
    rx = _rows_x(sx)
    q1 = plane[rz[:, 0]] * sz.w[0][:, None]
    for c in range(1, 4):
        q1 = q1 + plane[rz[:, c]] * sz.w[c][:, None]
    out = q1[:, rx[:, 0]] * sx.w[0][None, :]
    for a in range(1, 4):
        out = out + q1[:, rx[:, a]] * sx.w[a][None, :]
    return out


def interp2_xy(plane: np.ndarray, sx: Stencil, sy: Stencil) -> np.ndarray:
    """First-guess plane of ``InterpVelMgrd.F90:181-198`` (vz): plane (ny, n+3); y then x."""
    return interp2_xz(plane, sx, sy)


def to_refined_loops(m: Mgrd, g: o.Grid, cvar: np.ndarray) -> np.ndarray:
    """``interpolate_xyz_to_refined`` (``HermiteInterpolations.F90:168-200``) as written: loops
    over coarse intervals (ic, jc, kc) and the refined points inside them.  ``cvar`` is
    (nzm, nym, nx+3) x-extended; y/z halos come from periodic wrap.  Pure Python: small grids."""
    p = g.p
    nxm, nym, nzm = p.nxm, p.nym, p.nzm
    out = np.zeros((m.nzmr, m.nymr, m.nxmr))
    for ic in range(0, nzm + 1):
        zi = [(ic - 2 + c) % nzm for c in range(4)]
        for jc in range(0, nym + 1):
            yj = [(jc - 2 + b) % nym for b in range(4)]
            for kc in range(0, nxm + 1):
                qv3 = np.array([[[cvar[zi[c], yj[b], kc - 1 + a + 1] for c in range(4)]
                                 for b in range(4)] for a in range(4)])
                for icr in range(max(m.krangs[ic], 1), min(m.krangs[ic + 1] - 1, m.nzmr) + 1):
                    cz = m.czrs[:, icr - 1]
                    qv2 = qv3[:, :, 0] * cz[0] + qv3[:, :, 1] * cz[1] + qv3[:, :, 2] * cz[2] + qv3[:, :, 3] * cz[3]
                    for jcr in range(max(m.jrangs[jc], 1), min(m.jrangs[jc + 1] - 1, m.nymr) + 1):
                        cy = m.cyrs[:, jcr - 1]
                        qv1 = qv2[:, 0] * cy[0] + qv2[:, 1] * cy[1] + qv2[:, 2] * cy[2] + qv2[:, 3] * cy[3]
                        for kcr in range(max(m.irangs[kc], 1), min(m.irangs[kc + 1] - 1, m.nxmr) + 1):
                            out[icr - 1, jcr - 1, kcr - 1] = float(np.sum(qv1 * m.cxrs[:, kcr - 1]))
    return out


def to_coarse_loops(m: Mgrd, g: o.Grid, rvar: np.ndarray) -> np.ndarray:
    """``interpolate_xyz_to_coarse_fast`` (``HermiteInterpolations.F90:240-288``, when ``m.fast``)
    or ``interpolate_xyz_to_coarse`` (``:202-238``) as written; ``rvar`` (nzmr, nymr, nxmr+3)
    x-extended.  Pure Python: small grids."""
    p = g.p
    nxm, nym, nzm = p.nxm, p.nym, p.nzm
    out = np.zeros((nzm, nym, nxm))
    R = lambda i, j, k: rvar[(i - 1) % m.nzmr, (j - 1) % m.nymr, k + 1]  # noqa: E731 (Fortran idx)

    def block(k0, j0, i0):  # qv3 = rvar(k0:k0+3, j0:j0+3, i0:i0+3)
        return np.array([[[R(i0 + c, j0 + b, k0 + a) for c in range(4)] for b in range(4)]
                         for a in range(4)])

    def contract(qv3, cz, cy, cx):
        qv2 = qv3[:, :, 0] * cz[0] + qv3[:, :, 1] * cz[1] + qv3[:, :, 2] * cz[2] + qv3[:, :, 3] * cz[3]
        qv1 = qv2[:, 0] * cy[0] + qv2[:, 1] * cy[1] + qv2[:, 2] * cy[2] + qv2[:, 3] * cy[3]
        return float(np.sum(qv1 * cx))

    if m.fast:
        for ic in range(1, nzm + 1):
            icr = m.krangb[ic]
            for jc in range(1, nym + 1):
                jcr = m.jrangb[jc]
                for kc in range(1, nxm + 1):
                    kcr = m.irangb[kc]
                    out[ic - 1, jc - 1, kc - 1] = contract(block(kcr - 2, jcr - 2, icr - 2), m.czsalc[:, ic - 1],
                                                           m.cysalc[:, jc - 1], m.cxsalc[:, kc - 1])
        return out
    for icr in range(0, m.nzmr + 1):
        for jcr in range(0, m.nymr + 1):
            for kcr in range(0, m.nxmr + 1):
                qv3 = block(kcr - 1, jcr - 1, icr - 1)
                for ic in range(max(m.krangr[icr], 1), min(m.krangr[icr + 1] - 1, nzm) + 1):
                    for jc in range(max(m.jrangr[jcr], 1), min(m.jrangr[jcr + 1] - 1, nym) + 1):
                        for kc in range(max(m.irangr[kcr], 1), min(m.irangr[kcr + 1] - 1, nxm) + 1):
                            out[ic - 1, jc - 1, kc - 1] = contract(qv3, m.czphic[:, ic - 1], m.cyphic[:, jc - 1],
                                                                   m.cxphic[:, kc - 1])
    return out


# ----------------------------------------------------------------------------------------------
# Salinity state, boundary planes, initial condition
# ----------------------------------------------------------------------------------------------
@dataclasses.dataclass
class SalState:
    """Refined-grid fields of ``afid_salinity`` (``salinity.F90:13-19``), C-order (nzmr, nymr, *):
    sal/rusal (nxmr), vxr (nxr = nxmr+1), vyr/vzr (nxmr); salc (nzm, nym, nxm) on the coarse grid."""
    sal: np.ndarray
    rusal: np.ndarray
    vxr: np.ndarray
    vyr: np.ndarray
    vzr: np.ndarray
    salc: np.ndarray

    def copy(self) -> "SalState":
        return SalState(**{f.name: getattr(self, f.name).copy() for f in dataclasses.fields(self)})


def initial_salinity(m: Mgrd, g: o.Grid, seed: int, amp: float = 5e-3) -> np.ndarray:
    """``CreateInitialSalinity`` (``salinity.F90:140-170``) for the non-IBM cases: the bounded
    double-diffusive profile 0.5*(2(xmr-0.5))^7 when active_S = active_T = 1 and gAxis = 1, else
    the linear profile between the plates (``SetLinearSalinity``) plus uniform noise of
    amplitude ``amp`` limited so |S| <= 0.5 (``AddSalinityNoise``), U from Philox."""
    from oracle.philox import uniform_cells
    p = g.p
    xmr = m.xmr[1:m.nxmr + 1]
    shape = (m.nzmr, m.nymr, m.nxmr)
    if p.active_s == 1 and p.active_t == 1 and p.gaxis == 1:
        return np.broadcast_to(0.5 * (2 * (xmr - 0.5)) ** 7, shape).copy()
    sal = np.broadcast_to(m.salbp - (m.salbp - m.saltp) * xmr / m.xcr[m.nxmr], shape).copy()
    u = uniform_cells(seed, m.nzmr, m.nymr, m.nxr)[:, :, :m.nxmr]
    a2 = 0.5 - np.abs(sal)
    return np.where(np.abs(sal) + amp > 0.5, sal + a2 * (2.0 * u - 1.0), sal + amp * (2.0 * u - 1.0))


def new_sal_state(m: Mgrd, g: o.Grid, sal: np.ndarray) -> SalState:
    p = g.p
    z = lambda n: np.zeros((m.nzmr, m.nymr, n))  # noqa: E731
    return SalState(sal=sal.copy(), rusal=z(m.nxmr), vxr=z(m.nxr), vyr=z(m.nxmr), vzr=z(m.nxmr),
                    salc=np.zeros((p.nzm, p.nym, p.nxm)))


# ----------------------------------------------------------------------------------------------
# InterpVelMgrd and InterpSalMultigrid
# ----------------------------------------------------------------------------------------------
def _x_extend_coarse(g: o.Grid, interior: np.ndarray) -> np.ndarray:
    """Coarse x rows 1..nxm -> Fortran rows -1..nx+1 with the wall rule of
    ``InterpVelMgrd.F90:40-41``: row 0 = (1-2 inslwS) row 1, row nx = (1-2 inslwN) row nxm,
    rows -1 and nx+1 zero."""
    p = g.p
    nxm = p.nxm
    e = np.zeros(interior.shape[:-1] + (nxm + 4,))
    e[..., 2:nxm + 2] = interior[..., :nxm]
    e[..., 1] = (1 - 2 * p.inslws) * e[..., 2]
    e[..., nxm + 2] = (1 - 2 * p.inslwn) * e[..., nxm + 1]
    return e


def coarse_gradients(g: o.Grid, s: o.State):
    """dvx/dx, dvy/dy, dvz/dz at cell centres (``InterpVelMgrd.F90:33-39, 68-74, 152-158``)."""
    nxm = g.p.nxm
    gx = (s.vx[..., 1:nxm + 1] - s.vx[..., :nxm]) * g.udx3m[:nxm]
    gy = (o._jp(s.vy) - s.vy)[..., :nxm] * g.dy
    gz = (o._ip(s.vz) - s.vz)[..., :nxm] * g.dz
    return gx, gy, gz


def interp_vel_mgrd(m: Mgrd, g: o.Grid, s: o.State, ss: SalState, loops: bool = False) -> None:
    """``InterpVelMgrd.F90:27-239`` on one rank (the MPI_SCAN corrections vanish): the three
    velocity gradients are interpolated to the refined cell centres, then integrated from
    vxr(1) = 0 along x, from a first-guess plane at y = 0 (vy interpolated in x-z) along y, and
    from a first-guess plane at z = 0 (vz in x-y, only when nzm > 1: ``ic0 < xend(3)``) along z."""
    p = g.p
    sx, sy, sz = m.to_ref
    gx, gy, gz = coarse_gradients(g, s)
    interp = (lambda e: to_refined_loops(m, g, e)) if loops else (lambda e: interp3(e, sx, sy, sz))
    tx = interp(_x_extend_coarse(g, gx))
    ss.vxr[...] = 0.0
    lxa = m.xcr[1:] - m.xcr[:-1]
    for kcr in range(m.nxmr):
        ss.vxr[..., kcr + 1] = ss.vxr[..., kcr] + tx[..., kcr] * lxa[kcr]
    ty = interp(_x_extend_coarse(g, gy))
    ss.vyr[...] = 0.0
    ss.vyr[:, 0, :m.nxmr] = interp2_xz(_x_extend_coarse(g, s.vy[:, 0, :]), sx, sz)
    lya = 1.0 / m.dyr
    for jcr in range(m.nymr - 1):
        ss.vyr[:, jcr + 1, :] = ss.vyr[:, jcr, :] + ty[:, jcr, :] * lya
    tz = interp(_x_extend_coarse(g, gz))
    ss.vzr[...] = 0.0
    if p.nzm > 1:
        ss.vzr[0, :, :m.nxmr] = interp2_xy(_x_extend_coarse(g, s.vz[0, :, :]), sx, sy)
    lza = 1.0 / m.dzr
    for icr in range(m.nzmr - 1):
        ss.vzr[icr + 1] = ss.vzr[icr] + tz[icr] * lza


def sal_extended(m: Mgrd, sal: np.ndarray) -> np.ndarray:
    """``salinity.F90:462-481``: refined rows -1..nxr+1 with the plate ghosts
    row 0 = 2 salbp - sal(1) (SfixS) or sal(1); row nxr = 2 saltp - sal(nxmr) (SfixN) or sal(nxmr)."""
    n = m.nxmr
    e = np.zeros(sal.shape[:-1] + (n + 4,))
    e[..., 2:n + 2] = sal
    e[..., 1] = 2.0 * m.salbp - sal[..., 0] if m.sfixs == 1 else sal[..., 0]
    e[..., n + 2] = 2.0 * m.saltp - sal[..., n - 1] if m.sfixn == 1 else sal[..., n - 1]
    return e


def interp_sal_multigrid(m: Mgrd, g: o.Grid, ss: SalState, loops: bool = False) -> None:
    """``InterpSalMultigrid`` (``salinity.F90:455-492``): salc from the refined salinity."""
    e = sal_extended(m, ss.sal)
    if loops:
        ss.salc[...] = to_coarse_loops(m, g, e)
    else:
        ss.salc[...] = interp3(e, *m.to_coarse)


# ----------------------------------------------------------------------------------------------
# Salinity transport on the refined grid
# ----------------------------------------------------------------------------------------------
def _jp(a):
    return np.roll(a, -1, axis=1)


def _jm(a):
    return np.roll(a, 1, axis=1)


def _ip(a):
    return np.roll(a, -1, axis=0)


def _im(a):
    return np.roll(a, 1, axis=0)


def explicit_salinity(m: Mgrd, ss: SalState) -> np.ndarray:
    """``ExplicitSalinity`` (``salinity.F90:268-367``, no IBM): hsal = -(d(vx S)/dx + d(vy S)/dy
    + d(vz S)/dz) + (dyy + dzz) S / Pe_s."""
    n = m.nxmr
    sal, vxr, vyr, vzr = ss.sal, ss.vxr, ss.vyr, ss.vzr
    udyr, udzr = 0.5 * m.dyr, 0.5 * m.dzr
    udyrq, udzrq = m.dyqr / m.pecs, m.dzqr / m.pecs
    u = m.udx3mr
    hsx = np.empty(sal.shape)
    if n > 2:
        k = np.arange(1, n - 1)
        hsx[..., 1:n - 1] = (vxr[..., k + 1] * (sal[..., k + 1] + sal[..., k])
                             - vxr[..., k] * (sal[..., k] + sal[..., k - 1])) * u[k] * 0.5
    hsx[..., 0] = (vxr[..., 1] * (sal[..., 1] + sal[..., 0]) - vxr[..., 0] * 2.0 * m.salbp) * u[0] * 0.5
    k = n - 1
    hsx[..., k] = (vxr[..., k + 1] * 2.0 * m.saltp - vxr[..., k] * (sal[..., k] + sal[..., k - 1])) * u[k] * 0.5
    hsy = (_jp(vyr) * (_jp(sal) + sal) - vyr * (sal + _jm(sal))) * udyr
    hsz = (_ip(vzr) * (_ip(sal) + sal) - vzr * (sal + _im(sal))) * udzr
    dyys = (_jp(sal) - 2.0 * sal + _jm(sal)) * udyrq
    dzzs = (_ip(sal) - 2.0 * sal + _im(sal)) * udzrq
    return -(hsx + hsy + hsz) + dyys + dzzs


def implicit_salinity(m: Mgrd, ss: SalState, hsal, al, ga, ro, dt) -> None:
    """``ImplicitSalinity`` + ``SolveImpEqnUpdate_Sal`` (``salinity.F90:369-453``): RHS with the
    plate terms, RK3 history, CN solve in x with rows scaled by 1/(1 - ac betadx)."""
    n = m.nxmr
    sal = ss.sal
    ap, ac, am = m.ap3sskr, m.ac3sskr, m.am3sskr
    alpec = al / m.pecs
    dxxs = np.empty(sal.shape)
    if n > 2:
        k = np.arange(1, n - 1)
        dxxs[..., 1:n - 1] = sal[..., k + 1] * ap[k] + sal[..., k] * ac[k] + sal[..., k - 1] * am[k]
    dxxs[..., 0] = sal[..., 1] * ap[0] + sal[..., 0] * ac[0] - (ap[0] + ac[0]) * m.salbp * m.sfixs
    k = n - 1
    dxxs[..., k] = sal[..., k] * ac[k] + sal[..., k - 1] * am[k] - (am[k] + ac[k]) * m.saltp * m.sfixn
    rhs = (ga * hsal + ro * ss.rusal + alpec * dxxs) * dt
    ss.rusal[...] = hsal
    betadx = 0.5 * al * dt / m.pecs
    ackl_b = 1.0 / (1.0 - ac * betadx)
    amkT = -am[1:] * betadx * ackl_b[1:]
    apkT = -ap[:-1] * betadx * ackl_b[:-1]
    ackT = np.ones(n)
    cols = o._columns(rhs * ackl_b, n)
    x = o._dgttrs_columns(amkT, ackT, apkT, cols)
    ss.sal[...] = sal + o._uncolumns(x, sal.shape)


def add_sal_buoyancy(m: Mgrd, g: o.Grid, ss: SalState, qcap, dph, dq) -> None:
    """``AddSalBuoyancy`` (``salinity.F90:494-506``) into the forcing of the gravity axis
    (``TimeMarcher.F90:53-62``), rows 1..nxm."""
    if m.active_s != 1:
        return
    nxm = g.p.nxm
    tgt = {1: qcap, 2: dph, 3: dq}[g.p.gaxis]
    tgt[..., :nxm] = tgt[..., :nxm] - m.bycs * ss.salc


def calc_max_cfl_refined(m: Mgrd, ss: SalState) -> float:
    """``CalcMaxCFL.F90:48-65``: the refined-grid CFL number (initial value 1e-8)."""
    n = m.nxmr
    qcf = (np.abs((ss.vzr + _ip(ss.vzr)) * 0.5 * m.dzr)
           + np.abs((ss.vyr + _jp(ss.vyr)) * 0.5 * m.dyr)
           + np.abs((ss.vxr[..., :n] + ss.vxr[..., 1:n + 1]) * 0.5 * m.udx3mr))
    return max(1.0e-8, float(qcf.max()))


SAL_PROFILE_NAMES = ("Sbar", "Srms", "vxS", "vyS", "vzS", "chiS")


def sal_profiles(m: Mgrd, ss: SalState) -> dict:
    """``CalcSalStats`` + ``CalcDissipationSal`` (``salinity.F90:508-667``, no IBM): the six
    y-z averaged salinity profiles of means.h5, each of length nxmr."""
    n = m.nxmr
    sal, vxr, vyr, vzr = ss.sal, ss.vxr, ss.vyr, ss.vzr
    inyzmr = 1.0 / m.nymr / m.nzmr
    s2 = lambda a: a.sum(axis=(0, 1))  # noqa: E731
    sbar = s2(sal)
    srms = s2(sal ** 2)
    vxs = s2(0.5 * (vxr[..., :n] + vxr[..., 1:n + 1]) * sal)
    vys = s2(0.5 * (vyr + _jp(vyr)) * sal)
    vzs = s2(0.5 * (vzr + _ip(vzr)) * sal)
    tdxr = 0.5 * m.dxr / m.g3rmr
    chi = ((_ip(sal) - _im(sal)) * 0.5 * m.dzr) ** 2 + ((_jp(sal) - _jm(sal)) * 0.5 * m.dyr) ** 2
    cx = np.empty(sal.shape)
    cx[..., 0] = ((sal[..., 1] - sal[..., 0] + 2.0 * m.sfixs * (sal[..., 0] - m.salbp)) * tdxr[0]) ** 2
    if n > 2:
        cx[..., 1:n - 1] = ((sal[..., 2:] - sal[..., :n - 2]) * tdxr[1:n - 1]) ** 2
    cx[..., n - 1] = ((sal[..., n - 1] - sal[..., n - 2] + 2.0 * m.sfixn * (m.saltp - sal[..., n - 1]))
                      * tdxr[n - 1]) ** 2
    chis = s2(chi + cx)
    return dict(Sbar=sbar * inyzmr, Srms=np.sqrt(srms * inyzmr), vxS=vxs * inyzmr, vyS=vys * inyzmr,
                vzS=vzs * inyzmr, chiS=chis / m.pecs * inyzmr)


# ----------------------------------------------------------------------------------------------
# Substep loop with salinity
# ----------------------------------------------------------------------------------------------
def time_marcher(g: o.Grid, s: o.State, m: Mgrd, ss: SalState, dt: float) -> None:
    """``TimeMarcher.F90:28-150`` with ``salinity`` on (no phase-field, moisture or IBM):
    explicit terms, ExplicitSalinity, AddSalBuoyancy, implicit updates, ImplicitSalinity, the
    Poisson projection, then InterpVelMgrd and InterpSalMultigrid."""
    p = g.p
    gam, rom, alm = o.rk3_coefficients(p.nsst)
    beta = dt / g.ren * 0.5
    shape = s.vx.shape
    for ns in range(p.nsst):
        al, ga, ro = alm[ns], gam[ns], rom[ns]
        qcap, dph, dq, hro = (np.zeros(shape) for _ in range(4))
        o.explicit_terms_vx(g, s, qcap)
        o.explicit_terms_vy(g, s, dph)
        o.explicit_terms_vz(g, s, dq)
        o.explicit_terms_temp(g, s, hro)
        hsal = explicit_salinity(m, ss)
        add_sal_buoyancy(m, g, ss, qcap, dph, dq)
        o.implicit_and_update_vx(g, s, qcap, al, ga, ro, dt, beta)
        o.implicit_and_update_vy(g, s, dph, al, ga, ro, dt, beta)
        o.implicit_and_update_vz(g, s, dq, al, ga, ro, dt, beta)
        o.implicit_and_update_temp(g, s, hro, al, ga, ro, dt)
        implicit_salinity(m, ss, hsal, al, ga, ro, dt)
        div = o.calc_local_divergence(g, s, al, dt)
        phi = o.solve_pressure_correction(g, div)
        o.remove_divergence(g, s, phi, al, dt)
        o.correct_pressure(g, s, phi, al, beta)
        interp_vel_mgrd(m, g, s, ss)
        interp_sal_multigrid(m, g, ss)


def run(g: o.Grid, s: o.State, m: Mgrd, ss: SalState, nsteps: int):
    """``main.F90:281-313`` with salinity: the dt rule uses the refined CFL (``CFLmr``)."""
    p = g.p
    dt = p.dt
    time = 0.0
    err = 0
    for ntime in range(nsteps):
        cflmr = calc_max_cfl_refined(m, ss)
        dt, err, _ = o.next_dt(p, ntime, dt, cflmr)
        time_marcher(g, s, m, ss, dt)
        time += dt
        if err:
            break
    return time, dt, err
