"""Shared helpers: build the same case for the oracle (CPU oracle) and the CUDA library."""
from __future__ import annotations

import numpy as np

from oracle import afid_oracle as o
import afid_gpu as ag

BOU_TEMPLATE = """Base grid resolution / number of substeps
NXM     NYM     NZM     NSST(>1=RK,else AB)
{nxm}     {nym}     {nzm}     {nsst}

Refined grid: on/off and grid size
MULTIRES    NXMR    NYMR    NZMR
{multires}           {nxmr}     {nymr}     {nzmr}

Salinity and Phase-field (on/off)
FLAGSAL     FLAGPF
{flagsal}           0

Read flow / Reset logs
NREAD       IRESET
{nread}           {ireset}

Time steps / time limit (wall/flow)
NTST        WALLTIMEMAX     TMAX
{ntst}        7000            {tmax}

Time interval for saving stats/movie frames
TOUT    TFRAME  SAVE_3D
{tout}     {tframe}     {save_3d}

Domain size (keep ALX3 = 1.0)
ALX3   YLEN   ZLEN
{alx3}    {ylen}    {zlen}

Grid stretching parameters
ISTR3   STR3    ISTR3R
{istr3}       {str3}     {istr3r}

Physical flow parameters / Free-fall timescale
RAYT    PRAT    RAYS    PRAS    FFscaleS
{rayt}     {prat}     {rays}     {pras}     {ffscales}

Time stepping parameters
IDTV    DT      RESID   CFLMAX  DTMIN   DTMAX
{idtv}       {dt}    {resid}   {cflmax}     1e-8    {dtmax}

Dirichlet/Neumann BC flag on upper(N) and lower(S) walls
inslwS  inslwN  TfixS   TfixN   SfixS   SfixN
{inslws}       {inslwn}       {tfixs}       {tfixn}       {sfixs}       {sfixn}

Active/passive scalar flags / Gravitational axis (x=1,y=2,z=3)
active_T    active_S    gAxis
{active_t}           {active_s}           {gaxis}

Wall velocity / Pressure gradient / Melt boundary condition
xplusU  xminusU     dPdy    dPdz    MELT
{xplusu}     {xminusu}         {dpdy}     0.0     0

Phase-field parameters
pf_D(*Pe)   pf_A    pf_S    pf_Tm   IBM     pf_IC
0.1         10.0    10.0    0.0     0       1
"""

DEFAULTS = dict(nsst=3, ntst=9, tmax=1e30, tout=1e30, alx3=1.0, ylen=1.0, zlen=1.0, istr3=4,
                str3=2.0, rayt=1e6, prat=1.0, idtv=0, dt=1e-3, resid=1e-3, cflmax=10.0,
                dtmax=1e-2, inslws=1, inslwn=1, tfixs=1, tfixn=1, active_t=1, gaxis=1,
                xplusu=0.0, xminusu=0.0, dpdy=0.0, multires=0, flagsal=0, istr3r=0, rays=1e8,
                pras=1.0, ffscales=0, sfixs=1, sfixn=1, active_s=0, nread=1, ireset=0, tframe=1.0,
                save_3d=50.0)


def bou_text(nxm, nym, nzm, **kw) -> str:
    v = dict(DEFAULTS)
    v.update(nxmr=nxm, nymr=nym, nzmr=nzm)
    v.update(kw)
    return BOU_TEMPLATE.format(nxm=nxm, nym=nym, nzm=nzm, **v)


class Case:
    """One configuration seen by both the oracle and the CUDA library."""

    def __init__(self, nxm, nym, nzm, precision=ag.PREC_FP64, **kw):
        self.text = bou_text(nxm, nym, nzm, **kw)
        self.p = o.parse_bou_in(self.text)
        self.g = o.create_grid(self.p)
        self.inp = ag.parse_bou_in(self.text)
        self.tables = ag.Tables(self.inp, precision)

    def oracle_state(self, seed=1234, random_velocity=0.0, rng_seed=7):
        s = o.initial_state(self.g, seed)
        if random_velocity:
            rng = np.random.default_rng(rng_seed)
            for f in ("vx", "vy", "vz", "pr"):
                getattr(s, f)[...] = random_velocity * rng.standard_normal(s.vx.shape)
            s.vx[..., 0] = 0.0
            s.vx[..., -1] = 0.0
            for f in ("vy", "vz", "temp", "pr"):
                getattr(s, f)[..., -1] = 0.0
        return s

    def solver(self) -> ag.Solver:
        return ag.Solver(self.tables.grid, self.tables.params)


def rel_l2(a, b) -> float:
    na = float(np.linalg.norm(b))
    d = float(np.linalg.norm(a - b))
    return d / na if na > 0 else d


def rel_l2_mod_mean(a, b) -> float:
    return rel_l2(a - a.mean(), b - b.mean())
