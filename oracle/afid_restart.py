"""Oracle for the interpolating restart: a NumPy restatement of the branch of ReadFlowInterp that
runs when the continua files were written on another grid (ReadFlowInterp.F90:85-136).

This module is test infrastructure, never the product: the tests compare the library's native
restart (afid_read_flow_interp) with it.

Steps restated:
  CreateOldGrid           multires/IC_interpolation/CreateOldGrid.F90:11-115 (old coarse and old
                          refined coordinates from the master record: uniform y/z, wall-normal grid
                          of type istr3 / istr3r with the old STR3)
  CreateInputStencil      CreateNewInputStencil.F90:1-41 (cell centre -> cell centre Hermite
                          stencils; the cell-edge stencils it also builds are never applied)
  InterpInputVel          InterpInputVel.F90:1-350: dvx/dx, dvy/dy, dvz/dz at the old cell
                          centres with the wall rows (1 - 2 inslw) * row 1 / row nxm, interpolated
                          to the new centres (interpolate_xyz_old_to_new,
                          HermiteInterpolations.F90:314-346) and integrated: vx from vx(1) = 0
                          along x, vy from the y = 0 plane (x-z interpolation of the old vy(.,1,.))
                          along y, vz from the z = 0 plane (x-y interpolation of the old vz(.,.,1))
                          along z; temperature interpolated directly with plate ghosts
                          2 T_plate - T(1) (TfixS/N = 1) or T(1)
  CreateSalStencil,       CreateNewSalStencil.F90, InterpInputSal.F90: the refined salinity from
  InterpInputSal          the old refined grid with plate ghosts 2 S_plate - S(1) (SfixS/N = 1)
The pressure is not read in this branch and stays zero.  Single rank: the MPI_SCAN offsets of the
y and z integrations vanish.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

from oracle import afid_h5 as h5
from oracle import afid_oracle as o
from oracle import afid_salinity as sa


@dataclasses.dataclass
class Master:
    nx: int
    ny: int
    nz: int
    ylen: float
    zlen: float
    time: float
    istr3: int
    str3: float
    nxr: int = 0
    nyr: int = 0
    nzr: int = 0
    istr3r: int = 0


def read_master(directory: str, multires: bool) -> Master:
    p = os.path.join(directory, "continua_master.h5")
    v = {k: h5.read(p, k)[0] for k in ("nx", "ny", "nz", "ylen", "zlen", "time", "istr3", "str3")}
    m = Master(int(v["nx"]), int(v["ny"]), int(v["nz"]), float(v["ylen"]), float(v["zlen"]), float(v["time"]),
               int(v["istr3"]), float(v["str3"]))
    if multires:
        m.nxr, m.nyr, m.nzr, m.istr3r = (int(h5.read(p, k)[0]) for k in ("nxr", "nyr", "nzr", "istr3r"))
    return m


def _centres(xc: np.ndarray) -> np.ndarray:
    return 0.5 * (xc[:-1] + xc[1:])


def old_grids(m: Master, p: o.Params):
    """CreateOldGrid: (xmo, ymo, zmo) cell centres of the old coarse grid, and of the old refined
    grid when the master carries one (else None)."""
    pi = 2.0 * np.arcsin(1.0)
    nxmo, nymo, nzmo = m.nx - 1, m.ny - 1, m.nz - 1
    _, zmo = o._uniform_grid(nzmo, p.zlen)
    _, ymo = o._uniform_grid(nymo, p.ylen)
    xco, _ = sa._x_grid(m.istr3, nxmo, p.alx3, m.str3, pi, 1.0)
    coarse = (_centres(xco), ymo, zmo)
    refined = None
    if m.nxr:
        _, zmro = o._uniform_grid(m.nzr - 1, p.zlen)
        _, ymro = o._uniform_grid(m.nyr - 1, p.ylen)
        xcro, _ = sa._x_grid(m.istr3r, m.nxr - 1, p.alx3, m.str3, pi, 1.0)
        refined = (_centres(xcro), ymro, zmro)
    return coarse, refined


def stencils(old, new, lens):
    """Per-target centre-to-centre stencils along x, y, z (interval loops 0 .. n_old)."""
    out = []
    for axis, xo, xn, L in zip("xyz", old, new, lens):
        idx = sa.interpolation_indices(xo, xn, L)
        w = sa.construct_stencil(xo, xn, L, idx, axis)
        out.append(sa.Stencil(sa.starts_from_intervals(idx, xn.size, 0, xo.size), w))
    return tuple(out)


def _x_extend(interior: np.ndarray, low: np.ndarray, up: np.ndarray) -> np.ndarray:
    """Rows 1..n -> Fortran rows -1..n+1: row 0 = low, row n+1 = up, rows -1 and n+2 zero."""
    n = interior.shape[-1]
    e = np.zeros(interior.shape[:-1] + (n + 4,))
    e[..., 2:n + 2] = interior
    e[..., 1] = low
    e[..., n + 2] = up
    return e


def _wall_rows(a: np.ndarray, inslws: int, inslwn: int) -> np.ndarray:
    return _x_extend(a, (1 - 2 * inslws) * a[..., 0], (1 - 2 * inslwn) * a[..., -1])


def plate_values(rayt: float, inslwn: int):
    """InterpInputVel.F90: (Tlo, Tup)."""
    if rayt > 0:
        return (1.0, 0.0) if inslwn == 0 else (0.5, -0.5)
    return (-0.5, 0.5)


def interp_input_vel(old_fields: dict, m: Master, g: o.Grid):
    """vx (nzm, nym, nx), vy, vz, temp on the new grid g from the old fields (nzmo, nymo, nxo)."""
    p = g.p
    (xmo, ymo, zmo), _ = old_grids(m, p)
    nxmo = m.nx - 1
    xco_full, _ = sa._x_grid(m.istr3, nxmo, p.alx3, m.str3, 2.0 * np.arcsin(1.0), 1.0)
    st = stencils((xmo, ymo, zmo), (g.xm[:p.nxm], g.ym, g.zm), (p.alx3, p.ylen, p.zlen))
    sx, sy, sz = st
    nxm, nym, nzm = p.nxm, p.nym, p.nzm
    nx = nxm + 1
    yco, _ = o._uniform_grid(m.ny - 1, p.ylen)
    zco, _ = o._uniform_grid(m.nz - 1, p.zlen)
    dyo, dzo = 1.0 / (yco[1] - yco[0]), 1.0 / (zco[1] - zco[0])    # InterpInputVel.F90:28-29
    vxo, vyo, vzo, tempo = (old_fields[k] for k in ("vx", "vy", "vz", "temp"))
    vx = np.zeros((nzm, nym, nx))
    vy = np.zeros((nzm, nym, nx))
    vz = np.zeros((nzm, nym, nx))
    temp = np.zeros((nzm, nym, nx))
    # vx: gradient along x, integrated from vx(1) = 0
    gx = (vxo[..., 1:nxmo + 1] - vxo[..., :nxmo]) / (xco_full[1:] - xco_full[:-1])
    tx = sa.interp3(_wall_rows(gx, p.inslws, p.inslwn), sx, sy, sz)
    lxa = g.xc[1:nx] - g.xc[:nx - 1]
    for k in range(nxm):
        vx[..., k + 1] = vx[..., k] + tx[..., k] * lxa[k]
    # vy: gradient along y; first-guess plane y = 0; integrated along y
    gy = (np.roll(vyo, -1, axis=1) - vyo)[..., :nxmo] * dyo
    ty = sa.interp3(_wall_rows(gy, p.inslws, p.inslwn), sx, sy, sz)
    vy[:, 0, :nxm] = sa.interp2_xz(_wall_rows(vyo[:, 0, :nxmo], p.inslws, p.inslwn), sx, sz)
    lya = 1.0 / g.dy
    for j in range(nym - 1):
        vy[:, j + 1, :nxm] = vy[:, j, :nxm] + ty[:, j, :] * lya
    # vz: gradient along z; first-guess plane z = 0; integrated along z
    gz = (np.roll(vzo, -1, axis=0) - vzo)[..., :nxmo] * dzo
    tz = sa.interp3(_wall_rows(gz, p.inslws, p.inslwn), sx, sy, sz)
    vz[0, :, :nxm] = sa.interp2_xy(_wall_rows(vzo[0, :, :nxmo], p.inslws, p.inslwn), sx, sy)
    lza = 1.0 / g.dz
    for i in range(nzm - 1):
        vz[i + 1, :, :nxm] = vz[i, :, :nxm] + tz[i] * lza
    # temperature with the plate ghosts
    tlo, tup = plate_values(p.rayt, p.inslwn)
    t1, tn = tempo[..., 0], tempo[..., nxmo - 1]
    low = 2.0 * tlo - t1 if p.tfixs == 1 else t1
    up = 2.0 * tup - tn if p.tfixn == 1 else tn
    temp[..., :nxm] = sa.interp3(_x_extend(tempo[..., :nxmo], low, up), sx, sy, sz)
    return dict(vx=vx, vy=vy, vz=vz, temp=temp)


def interp_input_sal(salo: np.ndarray, m: Master, g: o.Grid, mg: sa.Mgrd) -> np.ndarray:
    """The refined salinity (nzmr, nymr, nxmr) from the old refined salinity (nzmro, nymro, nxmro)."""
    p = g.p
    _, (xmro, ymro, zmro) = old_grids(m, p)
    st = stencils((xmro, ymro, zmro), (mg.xmr[1:mg.nxmr + 1], mg.ymr, mg.zmr), (p.alx3, p.ylen, p.zlen))
    slo, sup = (-0.5, 0.5) if p.rays > 0 else (0.5, -0.5)
    s1, sn = salo[..., 0], salo[..., -1]
    low = 2.0 * slo - s1 if p.sfixs == 1 else s1
    up = 2.0 * sup - sn if p.sfixn == 1 else sn
    return sa.interp3(_x_extend(salo, low, up), *st)
