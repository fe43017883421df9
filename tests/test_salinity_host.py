"""Multi-resolution salinity on the host (no GPU): the oracle's two forms of the Hermite
interpolation agree, the C++ set-up (afid_mgrd_create) reproduces the oracle's refined grid,
coefficients and per-target stencils, the stencils follow the Hermite formula of the reference's
docs/interpolation.md (and reproduce quadratics), interpolating a divergence-free coarse velocity
gives a divergence-free refined one, and the salinity CN step reduces to the temperature CN step
when both see the same grid, diffusivity and plates.

Tolerances: stencil starts and the fast/general choice are exact; grid metrics and weights 1e-14
relative (the same expressions evaluated by C++ and NumPy); weights of every stencil sum to 1
within 1e-13 (cubic Hermite reproduces constants).
"""
import glob
import os

import numpy as np
import pytest

import afid_gpu as ag
from helpers import bou_text
from oracle import afid_oracle as o
from oracle import afid_salinity as sa

CASES = [
    # coarse (nxm, nym, nzm), refined (nxmr, nymr, nzmr), extra bou.in values
    ((16, 16, 8), (32, 32, 16), dict(istr3r=4)),                 # tanh refined: fast path
    ((16, 16, 8), (24, 48, 24), dict(istr3r=0)),                 # uniform refined: general path
    ((16, 16, 8), (24, 48, 24), dict(istr3r=6, str3=2.0)),       # clipped Chebyshev
    ((12, 16, 1), (36, 48, 1), dict(istr3r=4)),                  # 2-D
    ((16, 12, 12), (32, 36, 36), dict(istr3r=4, gaxis=2, inslwn=0)),  # gravity along y: faces in y
    ((16, 12, 12), (32, 24, 36), dict(istr3r=1, str3=2.0, gaxis=3)),   # centre-focused, gravity along z
]


def _case(coarse, refined, extra, **kw):
    v = dict(multires=1, nxmr=refined[0], nymr=refined[1], nzmr=refined[2], flagsal=1, rays=1e6, pras=10.0,
             active_s=1)
    v.update(extra)
    v.update(kw)
    return bou_text(*coarse, **v)


@pytest.mark.parametrize("coarse,refined,extra", CASES)
def test_loop_and_per_target_interpolation_agree(coarse, refined, extra):
    txt = _case(coarse, refined, extra)
    g = o.create_grid(o.parse_bou_in(txt))
    m = sa.create_mgrd(g)
    rng = np.random.default_rng(3)
    p = g.p
    cvar = rng.standard_normal((p.nzm, p.nym, p.nxm + 4))
    cvar[..., 0] = 0.0
    cvar[..., -1] = 0.0
    a = sa.interp3(cvar, *m.to_ref)
    b = sa.to_refined_loops(m, g, cvar)
    assert np.array_equal(a, b)
    rvar = rng.standard_normal((m.nzmr, m.nymr, m.nxmr + 4))
    rvar[..., 0] = 0.0
    rvar[..., -1] = 0.0
    assert np.array_equal(sa.interp3(rvar, *m.to_coarse), sa.to_coarse_loops(m, g, rvar))


@pytest.mark.parametrize("coarse,refined,extra", CASES)
def test_host_tables_match_oracle(coarse, refined, extra):
    txt = _case(coarse, refined, extra)
    g = o.create_grid(o.parse_bou_in(txt))
    m = sa.create_mgrd(g)
    tables = ag.Tables(ag.parse_bou_in(txt))
    hm = ag.Mgrd(tables)
    assert hm.fast == m.fast
    v = hm.view
    assert (v.nxmr, v.nymr, v.nzmr) == (m.nxmr, m.nymr, m.nzmr)
    assert v.pecs == m.pecs and v.bycs == m.bycs
    assert (v.dxr, v.dyr, v.dzr) == (m.dxr, m.dyr, m.dzr)

    def close(a, b, tol=1e-14):
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max())

    close(hm.array("xcr"), m.xcr)
    close(hm.array("xmr"), m.xmr[1:m.nxmr + 1])
    close(hm.array("g3rmr"), m.g3rmr)
    close(hm.array("udx3mr"), m.udx3mr)
    for n in ("ap3sskr", "ac3sskr", "am3sskr"):
        close(hm.array(n), getattr(m, n))
    for d, ax in enumerate("xyz"):
        assert np.array_equal(hm.array(f"start_to_ref_{ax}").astype(np.int64), m.to_ref[d].start)
        close(hm.array(f"w_to_ref_{ax}").reshape(-1, 4).T, m.to_ref[d].w)
        assert np.array_equal(hm.array(f"start_to_coarse_{ax}").astype(np.int64), m.to_coarse[d].start)
        close(hm.array(f"w_to_coarse_{ax}").reshape(-1, 4).T, m.to_coarse[d].w)
        for st in (m.to_ref[d], m.to_coarse[d]):
            assert np.abs(st.w.sum(axis=0) - 1.0).max() < 1e-13
    hm.close()
    tables.close()


@pytest.mark.parametrize("kw", [dict(), dict(active_t=0), dict(rays=-1e6, active_s=0)])
def test_initial_salinity_matches_oracle(kw):
    txt = _case((16, 16, 8), (32, 32, 16), dict(istr3r=4), **kw)
    g = o.create_grid(o.parse_bou_in(txt))
    m = sa.create_mgrd(g)
    tables = ag.Tables(ag.parse_bou_in(txt))
    hm = ag.Mgrd(tables)
    a = hm.initial_salinity(17)
    b = sa.initial_salinity(m, g, 17)
    assert np.abs(a - b).max() < 1e-15
    assert np.abs(a).max() <= 0.5


def test_unsupported_configurations_are_rejected():
    for kw in (dict(multires=0), dict(flagsal=0), dict(istr3r=2), dict(nzmr=4)):
        txt = _case((16, 16, 1), (32, 32, 1), dict(istr3r=4), **kw)
        tables = ag.Tables(ag.parse_bou_in(txt))
        with pytest.raises(ag.AfidError) as e:
            ag.Mgrd(tables)
        assert e.value.status == ag.AFID_E_INVALID


def test_salinity_diffusion_equals_temperature_diffusion():
    """At rest with matching grids, Pr = PraS, the same plates and no buoyancy, ImplicitSalinity
    + SolveImpEqnUpdate_Sal advance salinity exactly as ImplicitAndUpdateTemp +
    SolveImpEqnUpdate_Temp advance temperature (the path pinned by the convergence test)."""
    txt = _case((24, 8, 4), (24, 8, 4), dict(istr3r=4), rays=-1e6, pras=1.0, active_s=0, active_t=0)
    p = o.parse_bou_in(txt)
    g = o.create_grid(p)
    m = sa.create_mgrd(g)
    assert m.pecs == g.pect and (m.salbp, m.saltp) == (0.5, -0.5)
    s = o.initial_state(g, 5)
    ss = sa.new_sal_state(m, g, s.temp[..., :p.nxm])
    for _ in range(3):
        sa.time_marcher(g, s, m, ss, 2e-3)
    assert np.array_equal(ss.sal, s.temp[..., :p.nxm])


def _docs_hermite_weights(xo, i, xn):
    """Weights on (f_{i-1}, f_i, f_{i+1}, f_{i+2}) of the cubic Hermite interpolant at xn with the
    second-order finite-difference derivatives stated in the reference's docs/interpolation.md
    (h00 = (1+2t)(1-t)^2, h10 = t(1-t)^2, h01 = t^2(3-2t), h11 = t^2(t-1);
    f'_k = [d-^2 (f_{k+1} - f_k) + d+^2 (f_k - f_{k-1})] / (d+ d- (d+ + d-)))."""
    d = xo[i + 1] - xo[i]
    t = (xn - xo[i]) / d

    def fprime(k):  # coefficients of f'_k on (f_{k-1}, f_k, f_{k+1})
        dp, dm = xo[k + 1] - xo[k], xo[k] - xo[k - 1]
        den = dp * dm * (dp + dm)
        return np.array([-dp * dp, dp * dp - dm * dm, dm * dm]) / den

    h00, h10, h01, h11 = (1 + 2 * t) * (1 - t) ** 2, t * (1 - t) ** 2, t * t * (3 - 2 * t), t * t * (t - 1)
    w = np.zeros(4)
    w[1] += h00
    w[2] += h01
    w[0:3] += d * h10 * fprime(i)
    w[1:4] += d * h11 * fprime(i + 1)
    return w


@pytest.mark.parametrize("coarse,refined,extra", CASES[:3])
def test_stencils_follow_the_documented_hermite_formula(coarse, refined, extra):
    """Interior weights of construct_stencil equal the formula of docs/interpolation.md, and the
    interpolation reproduces quadratics exactly (the finite-difference derivatives are exact
    for them) on the stretched wall-normal grids."""
    txt = _case(coarse, refined, extra)
    g = o.create_grid(o.parse_bou_in(txt))
    m = sa.create_mgrd(g)
    nxm = g.p.nxm
    xm = g.xm[:nxm]
    xmr = m.xmr[1:m.nxmr + 1]
    st = m.to_ref[0]
    checked = 0
    for kr in range(m.nxmr):
        i = st.start[kr] + 1  # coarse interval io - 1 (0-based), sources i-1 .. i+2
        if i - 1 < 0 or i + 2 > nxm - 1:
            continue          # wall intervals: linear, or ghost rows
        w = _docs_hermite_weights(xm, i, xmr[kr])
        assert np.abs(w - st.w[:, kr]).max() < 1e-13
        f = 0.3 + 1.7 * xm - 2.2 * xm ** 2
        val = float(np.dot(st.w[:, kr], f[i - 1:i + 3]))
        assert abs(val - (0.3 + 1.7 * xmr[kr] - 2.2 * xmr[kr] ** 2)) < 1e-13
        checked += 1
    assert checked > m.nxmr // 2


def _divergence_free_state(g, seed=4):
    """A coarse velocity field projected to zero discrete divergence by one oracle substep."""
    p = g.p
    s = o.initial_state(g, 5)
    rng = np.random.default_rng(seed)
    for f in ("vx", "vy", "vz"):
        getattr(s, f)[...] = 0.05 * rng.standard_normal(s.vx.shape)
    s.vx[..., 0] = 0.0
    s.vx[..., -1] = 0.0
    div = o.calc_local_divergence(g, s, 1.0, 1.0)
    phi = o.solve_pressure_correction(g, div)
    o.remove_divergence(g, s, phi, 1.0, 1.0)
    assert o.check_divergence(g, s) < 1e-12
    return s


def refined_divergence(m, ss):
    """Discrete divergence of (vxr, vyr, vzr) at the refined cell centres, without the periodic
    seam rows j = nymr-1 and i = nzmr-1 (where the reference's halo copy closes the
    integrated field)."""
    n = m.nxmr
    dx = (ss.vxr[..., 1:n + 1] - ss.vxr[..., :n]) * m.udx3mr
    dy = (np.roll(ss.vyr, -1, axis=1) - ss.vyr) * m.dyr
    dz = (np.roll(ss.vzr, -1, axis=0) - ss.vzr) * m.dzr
    d = dx + dy + dz
    return d[:-1, :-1] if m.nzmr > 1 else d[:, :-1]


@pytest.mark.parametrize("coarse,refined,extra", [CASES[0], CASES[1], CASES[3]])
def test_velocity_interpolation_keeps_divergence_free(coarse, refined, extra):
    """docs/interpolation.md: the velocity gradients are interpolated and integrated, so a
    divergence-free coarse field gives a divergence-free refined one (up to rounding) away from
    the periodic seam."""
    txt = _case(coarse, refined, extra)
    g = o.create_grid(o.parse_bou_in(txt))
    m = sa.create_mgrd(g)
    s = _divergence_free_state(g)
    ss = sa.new_sal_state(m, g, sa.initial_salinity(m, g, 1))
    sa.interp_vel_mgrd(m, g, s, ss)
    scale = max(np.abs(ss.vxr).max() * m.udx3mr.max(), 1e-30)
    assert np.abs(refined_divergence(m, ss)).max() < 1e-11 * scale


@pytest.mark.parametrize("coarse,refined,extra", [CASES[0], CASES[1], CASES[3], CASES[5]])
def test_c_restatement_matches_numpy_oracle(coarse, refined, extra):
    """The C + OpenMP restatement of the salinity path (the timed CPU baseline of the ddc3d
    workload) against the NumPy oracle: refined CFL and all fields after 3 RK3 steps, 1e-13."""
    from oracle import cpu_port
    txt = _case(coarse, refined, extra, rayt=1e6, dt=1e-3)
    g = o.create_grid(o.parse_bou_in(txt))
    m = sa.create_mgrd(g)
    s = o.initial_state(g, 5)
    rng = np.random.default_rng(1)
    for f in ("vx", "vy", "vz"):
        getattr(s, f)[...] = 0.05 * rng.standard_normal(s.vx.shape)
    s.vx[..., 0] = 0.0
    s.vx[..., -1] = 0.0
    for f in ("vy", "vz", "temp", "pr"):
        getattr(s, f)[..., -1] = 0.0
    sal = np.clip(sa.initial_salinity(m, g, 3) + 0.01 * rng.standard_normal((m.nzmr, m.nymr, m.nxmr)), -0.5, 0.5)
    cpu = cpu_port.CpuSalSolver(g, s.copy(), m, sal)
    ss = sa.new_sal_state(m, g, sal)
    sa.interp_vel_mgrd(m, g, s, ss)
    sa.interp_sal_multigrid(m, g, ss)
    assert abs(cpu.cfl() - sa.calc_max_cfl_refined(m, ss)) < 1e-13 * sa.calc_max_cfl_refined(m, ss)
    for _ in range(3):
        cpu.time_marcher(1e-3)
        sa.time_marcher(g, s, m, ss, 1e-3)
    out = cpu.get()
    for f in ("vx", "vy", "vz", "temp"):
        ref = getattr(s, f)
        assert np.linalg.norm(out[f] - ref) <= 1e-13 * np.linalg.norm(ref), f
    assert np.linalg.norm(cpu.sal() - ss.sal) <= 1e-13 * np.linalg.norm(ss.sal)
    cpu.close()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "salinity",
                                                               "*.npz"))))
def test_oracle_reproduces_salinity_golden_fixture(path):
    """The committed salinity fixtures (tests/golden/make_golden.py) pin the oracle against later
    changes: coarse fields and refined salinity after 1 and 3 steps to 1e-13."""
    d = np.load(path)
    p = o.parse_bou_in(str(d["bou_in"]))
    g = o.create_grid(p)
    m = sa.create_mgrd(g)
    s = o.initial_state(g, 0)
    for f in ("vx", "vy", "vz", "temp", "pr"):
        getattr(s, f)[...] = d["init_" + f]
    ss = sa.new_sal_state(m, g, d["init_sal"])
    sa.interp_vel_mgrd(m, g, s, ss)
    sa.interp_sal_multigrid(m, g, ss)
    for n in range(3):
        sa.time_marcher(g, s, m, ss, float(d["dt"]))
        if n in (0, 2):
            for f in ("vx", "vy", "vz", "temp"):
                np.testing.assert_allclose(getattr(s, f), d[f"step{n + 1}_{f}"], rtol=0, atol=1e-13)
            np.testing.assert_allclose(ss.sal, d[f"step{n + 1}_sal"], rtol=0, atol=1e-13)
    assert sa.calc_max_cfl_refined(m, ss) == pytest.approx(float(d["step3_cflmr"]), rel=1e-13)
