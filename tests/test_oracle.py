"""Pins of the CPU oracle (oracle/afid_oracle.py) and of its C restatement (oracle/afid_cpu.c).

The reference has no test suite and cannot be compiled here.  What pins the oracle to it:
* the published 1-D pure-diffusion errors of the temperature Crank-Nicolson path
  (docs/convergence.md:3-31, docs/figures/spatial_convergence.svg; values digitised to ~3%);
* the discrete divergence-free invariant after the projection (pressure.F90:78-97 make the
  FFT solve exact for the discrete operator, checked against resid in main.F90:357);
* the Poisson solve against the discrete operator it inverts (CorrectPressure's stencil,
  pressure.F90:291-297), and the LAPACK/FFT building blocks against dense algebra;
* Philox4x32-10 against the published known-answer vectors.
"""
import glob
import math
import os

import numpy as np
import pytest

from helpers import rel_l2, rel_l2_mod_mean
from oracle import afid_oracle as o
from oracle.philox import philox4x32

HERE = os.path.dirname(os.path.abspath(__file__))

# docs/figures/spatial_convergence.svg, digitised: N -> (L2, Linf)
PUBLISHED_1D = {8: (9.4e-2, 1.6e-1), 16: (2.1e-2, 4.2e-2), 32: (5.2e-3, 1.05e-2), 64: (1.28e-3, 2.7e-3)}


def diffusion_1d_errors(N, dt=1e-3, tf=1.0):
    """The convergence case of examples/convergence_test/bou.in (64x1x1, gAxis=3, active_T=0,
    kappa = 1/sqrt(Ra Pr) = 0.01, uniform grid) with the IC of CreateInitialConditions.F90:204-212,
    errors as defined in docs/convergence.md:22-27."""
    p = o.Params(nxm=N, nym=1, nzm=1, ylen=0.01, zlen=0.01, istr3=0, rayt=1e4, prat=1.0, dt=dt, idtv=0,
                 gaxis=3, active_t=0, limit_cfl=1.0)
    g = o.create_grid(p)
    s = o.initial_state(g, 0, eps=0.0)
    xm = g.xm[:N]
    s.temp[..., :N] = 0.5 + (-0.5 - 0.5) * xm / p.alx3 + np.sin(2.0 * g.pi * xm / p.alx3) - np.sin(6.0 * g.pi * xm / p.alx3)
    kap = 1.0 / g.pect
    l2 = linf = t = 0.0
    for _ in range(int(round(tf / dt))):
        o.time_marcher(g, s, dt)
        t += dt
        ta = (0.5 - xm + np.sin(2 * math.pi * xm) * math.exp(-kap * (2 * math.pi) ** 2 * t)
              - np.sin(6 * math.pi * xm) * math.exp(-kap * (6 * math.pi) ** 2 * t))
        e = s.temp[0, 0, :N] - ta
        l2 += np.sum(e ** 2) / N * dt
        linf = max(linf, float(np.abs(e).max()))
    return math.sqrt(l2 / tf), linf


@pytest.mark.parametrize("N", [8, 16, 32])
def test_1d_diffusion_matches_published_errors(N):
    l2, linf = diffusion_1d_errors(N)
    ref_l2, ref_linf = PUBLISHED_1D[N]
    assert abs(l2 / ref_l2 - 1) < 0.12, (l2, ref_l2)
    assert abs(linf / ref_linf - 1) < 0.12, (linf, ref_linf)


def test_1d_diffusion_second_order():
    e16 = diffusion_1d_errors(16)[0]
    e32 = diffusion_1d_errors(32)[0]
    assert 3.5 < e16 / e32 < 4.5


def _random_state(shape, seed=3, amp=0.2, **kw):
    p = o.Params(nxm=shape[0], nym=shape[1], nzm=shape[2], rayt=1e6, dt=2e-3, **kw)
    g = o.create_grid(p)
    s = o.initial_state(g, seed)
    rng = np.random.default_rng(seed)
    for f in ("vx", "vy", "vz", "pr"):
        getattr(s, f)[...] = amp * rng.standard_normal(s.vx.shape)
    s.vx[..., 0] = 0.0
    s.vx[..., -1] = 0.0
    return p, g, s


@pytest.mark.parametrize("shape", [(16, 12, 8), (24, 16, 1), (20, 10, 6)])
def test_projection_is_divergence_free(shape):
    p, g, s = _random_state(shape)
    assert o.check_divergence(g, s) > 1.0  # the random state is far from solenoidal
    o.time_marcher(g, s, p.dt)
    assert o.check_divergence(g, s) < 1e-11


def test_poisson_solve_inverts_discrete_operator():
    """phi from solve_pressure_correction satisfies L phi = rhs (modulo the mean mode), where
    L is the operator CorrectPressure applies (pressure.F90:291-297)."""
    p, g, s = _random_state((24, 16, 12), istr3=4, str3=2.0)
    nxm = p.nxm
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal((p.nzm, p.nym, nxm))
    w = g.d3xc[:nxm]  # compatibility: the x-operator is symmetric with weights d3xc
    rhs -= (rhs * w).sum() / (w.sum() * p.nym * p.nzm)
    phi = o.solve_pressure_correction(g, rhs)
    ip, im = np.roll(phi, -1, 0), np.roll(phi, 1, 0)
    jp, jm = np.roll(phi, -1, 1), np.roll(phi, 1, 1)
    lap = ((ip - 2 * phi + im) * g.dzq + (jp - 2 * phi + jm) * g.dyq
           + phi[..., g.kpv] * g.apphk[:nxm] + phi * g.acphk[:nxm] + phi[..., g.kmv] * g.amphk[:nxm])
    assert rel_l2(lap, rhs) < 1e-10


def test_fft_conventions_match_fftw():
    """numpy's pocketfft with norm='forward' on the backward transform == FFTW's unnormalised
    FFTW_BACKWARD used by the reference (pressure.F90:189,193)."""
    rng = np.random.default_rng(0)
    x = rng.standard_normal(384)
    X = np.fft.rfft(x)
    n = np.arange(384)
    direct = np.array([np.sum(x * np.exp(-2j * np.pi * k * n / 384)) for k in range(193)])
    assert np.abs(X - direct).max() < 1e-11
    back = np.fft.irfft(X, n=384, norm="forward")
    assert np.abs(back - 384 * x).max() < 1e-9


def test_lapack_tridiagonal_matches_dense():
    from scipy.linalg import lapack
    rng = np.random.default_rng(1)
    n = 37
    dl, d, du = -rng.uniform(0, .5, n - 1), np.ones(n), -rng.uniform(0, .5, n - 1)
    A = np.diag(d) + np.diag(dl, -1) + np.diag(du, 1)
    b = rng.standard_normal((n, 3))
    f = lapack.dgttrf(dl, d, du)
    x, info = lapack.dgttrs(*f[:5], b)
    assert info == 0 and np.abs(A @ x - b).max() < 1e-13


def test_philox_known_answers():
    kats = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
            ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
            ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
             (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in kats:
        c = np.array(ctr, dtype=np.uint64).reshape(4, 1)
        got = tuple(int(v[0]) for v in philox4x32(c, *key))
        assert got == want


@pytest.mark.parametrize("shape", [(16, 12, 8), (40, 10, 6), (48, 64, 1)])
def test_c_restatement_matches_numpy_oracle(shape):
    from oracle.cpu_port import CpuSolver
    p, g, s = _random_state(shape)
    cpu = CpuSolver(g, s)
    for _ in range(3):
        o.time_marcher(g, s, p.dt)
        cpu.time_marcher(p.dt)
    out = cpu.get()
    nxm = p.nxm
    assert rel_l2(out["vx"], s.vx) < 1e-13
    assert rel_l2(out["vy"][..., :nxm], s.vy[..., :nxm]) < 1e-13
    assert rel_l2(out["temp"][..., :nxm], s.temp[..., :nxm]) < 1e-13
    assert rel_l2_mod_mean(out["pr"][..., :nxm], s.pr[..., :nxm]) < 1e-11
    assert cpu.cfl() == pytest.approx(o.calc_max_cfl(g, s), rel=1e-13)
    st = cpu.stats()
    assert st["nu_vol"] == pytest.approx(o.nusselt_volume(g, s), rel=1e-13)
    assert st["ke"] == pytest.approx(o.kinetic_energy(g, s), rel=1e-13)
    tbar = o.mean_profiles(g, s)["Tbar"]
    assert st["nu_plate_lower"] == pytest.approx(-(tbar[0] - 0.5) / g.xm[0], rel=1e-13)
    assert st["nu_plate_upper"] == pytest.approx(-(-0.5 - tbar[nxm - 1]) / (1.0 - g.xm[nxm - 1]), rel=1e-13)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(HERE, "golden", "*.npz"))))
def test_oracle_reproduces_golden_fixture(path):
    d = np.load(path)
    p = o.parse_bou_in(str(d["bou_in"]))
    g = o.create_grid(p)
    s = o.initial_state(g, 0)
    for f in ("vx", "vy", "vz", "temp", "pr"):
        getattr(s, f)[...] = d["init_" + f]
    for n in range(3):
        o.time_marcher(g, s, float(d["dt"]))
        if n in (0, 2):
            for f in ("vx", "vy", "vz", "temp"):
                np.testing.assert_allclose(getattr(s, f), d[f"step{n + 1}_{f}"], rtol=0, atol=1e-13)
    assert o.nusselt_volume(g, s) == pytest.approx(float(d["step3_nu"]), rel=1e-13)


@pytest.mark.parametrize("istr3,nxm", [(4, 32), (0, 24), (6, 40)])
def test_mean_profiles_conduction_pin(istr3, nxm):
    """CalcMeanProfiles.F90 on the conductive state: Tbar is the linear profile, every velocity
    moment and epsilon vanish, and the thermal-dissipation Nusselt number Pe * int chiT dx is 1
    (discrete identity of the one-sided wall gradients with the plate values)."""
    from helpers import Case
    c = Case(nxm, 16, 8, rayt=1e6, istr3=istr3)
    s = o.initial_state(c.g, 1, eps=0.0)
    m = o.mean_profiles(c.g, s)
    assert set(m) == set(o.MEAN_PROFILE_NAMES)
    xm = c.g.xm[:nxm]
    assert np.allclose(m["Tbar"], 0.5 - xm / c.p.alx3, atol=1e-14)
    for k in ("vybar", "vzbar", "vxT", "vyT", "vzT", "vxrms", "vyrms", "vzrms", "vxvy", "vxvz", "vyvz", "epsilon"):
        assert np.abs(m[k]).max() == 0.0, k
    dxk = c.g.xc[1:nxm + 1] - c.g.xc[:nxm]
    assert abs(c.g.pect * np.sum(m["chiT"] * dxk) - 1.0) < 1e-12
