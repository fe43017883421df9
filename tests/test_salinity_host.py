"""Multi-resolution salinity on the host (no GPU): the oracle's two forms of the Hermite
interpolation agree, the C++ set-up (afid_mgrd_create) reproduces the oracle's refined grid,
coefficients and per-target stencils, and the salinity CN step reduces to the temperature CN step
when both see the same grid, diffusivity and plates.

Tolerances: stencil starts and the fast/general choice are exact; grid metrics and weights 1e-14
relative (the same expressions evaluated by C++ and NumPy); weights of every stencil sum to 1
within 1e-13 (cubic Hermite reproduces constants).
"""
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
