"""Multi-resolution salinity on the GPU (include/afid_salinity.h) against the oracle's restatement
of salinity.F90 and multires/*.F90 (oracle/afid_salinity.py).

Tolerances: interpolated fields (InterpVelMgrd, InterpSalMultigrid), the refined CFL number and
the salinity profiles 1e-12 relative to each field's largest magnitude (sums and scans run in a
different order); fields after whole RK3 steps 1e-10 relative L2 (pr after removing its mean), the
bar of the flow path.
"""
import glob
import os

import numpy as np
import pytest

import afid_gpu as ag
from helpers import bou_text, rel_l2, rel_l2_mod_mean
from oracle import afid_oracle as o
from oracle import afid_salinity as sa

pytestmark = pytest.mark.gpu

FIELDS = ("vx", "vy", "vz", "temp", "pr")


def _text(coarse, refined, **kw):
    v = dict(multires=1, nxmr=refined[0], nymr=refined[1], nzmr=refined[2], flagsal=1, rays=1e6, pras=10.0,
             active_s=1, istr3r=4, rayt=1e6, dt=1e-3)
    v.update(kw)
    return bou_text(*coarse, **v)


class SalCase:
    def __init__(self, coarse, refined, precision=ag.PREC_FP64, vel=0.05, noise=1e-2, **kw):
        self.text = _text(coarse, refined, **kw)
        self.p = o.parse_bou_in(self.text)
        self.g = o.create_grid(self.p)
        self.m = sa.create_mgrd(self.g)
        rng = np.random.default_rng(11)
        self.s = o.initial_state(self.g, 5)
        if vel:
            for f in ("vx", "vy", "vz"):
                getattr(self.s, f)[...] = vel * rng.standard_normal(self.s.vx.shape)
            self.s.vx[..., 0] = 0.0
            self.s.vx[..., -1] = 0.0
            for f in ("vy", "vz", "temp", "pr"):
                getattr(self.s, f)[..., -1] = 0.0
        sal = sa.initial_salinity(self.m, self.g, 3)
        sal = np.clip(sal + noise * rng.standard_normal(sal.shape), -0.5, 0.5)
        self.ss = sa.new_sal_state(self.m, self.g, sal)
        sa.interp_vel_mgrd(self.m, self.g, self.s, self.ss)
        sa.interp_sal_multigrid(self.m, self.g, self.ss)
        self.tables = ag.Tables(ag.parse_bou_in(self.text), precision)
        self.mgrd = ag.Mgrd(self.tables)
        assert self.mgrd.fast == self.m.fast

    def solver(self) -> ag.Solver:
        sv = ag.Solver(self.tables.grid, self.tables.params)
        sv.sal_create(self.mgrd)
        sv.upload(*(getattr(self.s, f) for f in FIELDS))
        sv.sal_upload(self.ss.sal)
        return sv


def _close(a, b, tol):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err < tol, err


GEOMS = [
    ((16, 16, 8), (32, 32, 16), dict()),                              # fast path, 3-D
    ((16, 16, 8), (24, 48, 24), dict(istr3r=0)),                      # general path
    ((24, 32, 1), (48, 64, 1), dict()),                               # 2-D
    ((16, 12, 12), (32, 24, 36), dict(istr3r=1, str3=2.0, gaxis=3)),  # gravity along z
    ((20, 16, 8), (40, 32, 16), dict(sfixs=0, sfixn=0, inslws=0)),    # zero-flux plates, free-slip bottom
    ((16, 12, 12), (32, 36, 36), dict(gaxis=2, inslwn=0)),              # gravity along y (faces in y)
    ((100, 32, 1), (300, 64, 1), dict()),                             # 12 refined rows per lane, padded
    ((200, 16, 1), (700, 32, 1), dict(istr3r=0)),                     # 24 rows per lane, general path
]


@pytest.mark.parametrize("coarse,refined,kw", GEOMS)
def test_interpolation_matches_oracle(coarse, refined, kw):
    c = SalCase(coarse, refined, **kw)
    with c.solver() as sv:
        aux = sv.sal_aux()
    _close(aux["vxr"], c.ss.vxr, 1e-12)
    _close(aux["vyr"], c.ss.vyr, 1e-12)
    if coarse[2] > 1:
        _close(aux["vzr"], c.ss.vzr, 1e-12)
    else:
        assert np.abs(aux["vzr"]).max() == 0.0
    _close(aux["salc"], c.ss.salc, 1e-12)


@pytest.mark.parametrize("coarse,refined,kw", GEOMS)
def test_steps_match_oracle(coarse, refined, kw):
    c = SalCase(coarse, refined, **kw)
    dt = 1e-3
    with c.solver() as sv:
        for n in range(3):
            sv.time_marcher(dt, n)
            sa.time_marcher(c.g, c.s, c.m, c.ss, dt)
        got = sv.download()
        sal = sv.sal_download()
        aux = sv.sal_aux()
    for f in ("vx", "vy", "vz", "temp"):
        assert rel_l2(got[f], getattr(c.s, f)) < 1e-10, f
    assert rel_l2_mod_mean(got["pr"][..., :c.p.nxm], c.s.pr[..., :c.p.nxm]) < 1e-10
    assert rel_l2(sal, c.ss.sal) < 1e-10
    assert rel_l2(aux["salc"], c.ss.salc) < 1e-10
    # the salinity buoyancy moved the flow: without it the velocities differ
    if c.m.active_s:
        assert rel_l2(sal, sa.initial_salinity(c.m, c.g, 3)) > 1e-8


def test_k1_shapes_bitwise_identical_with_salinity():
    """The salinity-coupled K1 (buoyancy from the coarse salinity) gives the same fields and
    salinity bit for bit on every launch shape of its wall-normal class, the two-column and
    persistent forms among them."""
    c = SalCase((150, 16, 8), (300, 32, 16))
    with c.solver() as sv:
        ncand = sv.autotune()["ncand"]
    assert ncand >= 2
    outs = []
    for v in range(ncand):
        with c.solver() as sv:
            sv.set_k1_shape(v)
            for n in range(2):
                sv.time_marcher(1e-3, n)
            outs.append((sv.download(), sv.sal_download()))
    for got, sal in outs[1:]:
        for f in FIELDS:
            assert np.array_equal(got[f], outs[0][0][f]), f
        assert np.array_equal(sal, outs[0][1])


def test_cfl_and_profiles_match_oracle():
    c = SalCase((16, 16, 8), (32, 32, 16))
    with c.solver() as sv:
        for n in range(2):
            sv.time_marcher(1e-3, n)
            sa.time_marcher(c.g, c.s, c.m, c.ss, 1e-3)
        cfl = sv.sal_cfl()
        prof = sv.sal_profiles()
    assert abs(cfl - sa.calc_max_cfl_refined(c.m, c.ss)) < 1e-12 * cfl
    ref = sa.sal_profiles(c.m, c.ss)
    for n in ag.SAL_PROFILE_NAMES:
        _close(prof[n], ref[n], 1e-12)


def test_salinity_diffusion_equals_temperature_diffusion_on_device():
    """Same grid, PraS = Pr, same plates, no buoyancy: the refined-grid kernel advances salinity
    as K1 advances temperature."""
    c = SalCase((24, 8, 4), (24, 8, 4), vel=0.0, noise=0.0, rays=-1e6, pras=1.0, active_s=0, active_t=0)
    with c.solver() as sv:
        sv.sal_upload(np.ascontiguousarray(c.s.temp[..., :c.p.nxm]))
        for n in range(3):
            sv.time_marcher(2e-3, n)
        t = sv.download()["temp"][..., :c.p.nxm]
        s = sv.sal_download()
    assert np.abs(s - t).max() < 1e-14


def test_mixed_precision_with_salinity_tracks_fp64():
    a = SalCase((32, 32, 16), (64, 64, 32), vel=0.02)
    b = SalCase((32, 32, 16), (64, 64, 32), precision=ag.PREC_MIXED, vel=0.02)
    with a.solver() as s64, b.solver() as smx:
        for n in range(10):
            s64.time_marcher(1e-3, n)
            smx.time_marcher(1e-3, n)
        ra, rb = s64.sal_download(), smx.sal_download()
        va, vb = s64.download()["vx"], smx.download()["vx"]
    assert rel_l2(rb, ra) < 1e-5
    assert rel_l2(vb, va) < 1e-3


def test_invalid_salinity_setups():
    c = SalCase((16, 16, 8), (32, 32, 16))
    with ag.Solver(c.tables.grid, c.tables.params) as sv:
        sv.sal_create(c.mgrd)
        with pytest.raises(ag.AfidError) as e:
            sv.sal_create(c.mgrd)  # twice
        assert e.value.status == ag.AFID_E_INVALID
    c2 = SalCase((16, 16, 8), (32, 32, 16))
    other = ag.Tables(ag.parse_bou_in(_text((20, 16, 8), (32, 32, 16))))
    with ag.Solver(other.grid, other.params) as sv:
        with pytest.raises(ag.AfidError) as e:
            sv.sal_create(c2.mgrd)  # stencils built for another coarse grid
        assert e.value.status == ag.AFID_E_INVALID


def test_host_driver_run_with_salinity_matches_oracle():
    """afid_run with MULTIRES = FLAGSAL = 1: CreateInitialSalinity (Philox key seed + 1), the dt
    rule on the refined CFL number, salinity coupled every substep; Nu and KE after 5 steps
    against the oracle main loop."""
    import ctypes
    text = _text((32, 16, 8), (64, 32, 16), idtv=1, dt=1e-3, cflmax=1.0, dtmax=4e-3, ntst=4, active_t=1)
    p = o.parse_bou_in(text)
    g = o.create_grid(p)
    m = sa.create_mgrd(g)
    s = o.initial_state(g, 99)
    ss = sa.new_sal_state(m, g, sa.initial_salinity(m, g, 100))
    sa.interp_vel_mgrd(m, g, s, ss)
    sa.interp_sal_multigrid(m, g, ss)
    sa.run(g, s, m, ss, 5)
    st = ag.RunStatsT()
    inp = ag.parse_bou_in(text)
    rc = ag.lib().afid_run(ctypes.byref(inp), ag.PREC_FP64, 99, 5, 0, None, None, ctypes.byref(st))
    assert rc == 0 and st.steps_done == 5
    assert st.nu_vol == pytest.approx(o.nusselt_volume(g, s), rel=1e-9)
    assert st.ke == pytest.approx(o.kinetic_energy(g, s), rel=1e-6)
    assert st.dt == pytest.approx(min(p.dtmax, p.limit_cfl / sa.calc_max_cfl_refined(m, ss)), rel=1e-6) or \
        st.dt == pytest.approx(p.dtmax)


def test_batches_and_jobs_refuse_salinity():
    inp = ag.parse_bou_in(_text((16, 32, 1), (32, 64, 1)))
    with pytest.raises(ag.AfidError) as e:
        ag.Batch(inp, 2, ag.PREC_FP64)
    assert e.value.status == ag.AFID_E_INVALID


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "salinity",
                                                               "*.npz"))))
def test_gpu_matches_salinity_golden_fixture(path):
    """Committed fixtures (tests/golden/salinity, from tests/golden/make_golden.py): the device
    path after 1 and 3 steps, through the C ABI, at 1e-10 relative L2."""
    d = np.load(path)
    text = str(d["bou_in"])
    tables = ag.Tables(ag.parse_bou_in(text))
    mgrd = ag.Mgrd(tables)
    with ag.Solver(tables.grid, tables.params) as sv:
        sv.sal_create(mgrd)
        sv.upload(*(d["init_" + f] for f in FIELDS))
        sv.sal_upload(d["init_sal"])
        for n in range(3):
            sv.time_marcher(float(d["dt"]), n)
            if n in (0, 2):
                got = sv.download()
                for f in ("vx", "vy", "vz", "temp"):
                    assert rel_l2(got[f], d[f"step{n + 1}_{f}"]) < 1e-10, (n, f)
                assert rel_l2(sv.sal_download(), d[f"step{n + 1}_sal"]) < 1e-10
        assert abs(sv.sal_cfl() - float(d["step3_cflmr"])) < 1e-12 * float(d["step3_cflmr"])
