"""FP64 GPU path vs the CPU oracle, through the C ABI (``libafidgpu.so``).

Tolerance: the FP64 bar is 1e-10 relative L2 on every field after 10 steps, ``pr`` compared
after removing its volume mean (the (0,0) Poisson mode is singular, pressure.F90:219).
"""
import math

import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case, rel_l2, rel_l2_mod_mean
from oracle import afid_oracle as o

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10


def _compare(case, s, out, tol):
    nxm = case.p.nxm
    errs = {
        "vx": rel_l2(out["vx"], s.vx),
        "vy": rel_l2(out["vy"][..., :nxm], s.vy[..., :nxm]),
        "vz": rel_l2(out["vz"][..., :nxm], s.vz[..., :nxm]) if np.any(s.vz) else
        float(np.abs(out["vz"][..., :nxm]).max()),
        "temp": rel_l2(out["temp"][..., :nxm], s.temp[..., :nxm]),
        "pr": rel_l2_mod_mean(out["pr"][..., :nxm], s.pr[..., :nxm]),
    }
    bad = {k: v for k, v in errs.items() if not (v <= tol)}
    assert not bad, f"parity failed: {errs}"
    return errs


def _run_both(case, nsteps, seed=1234, random_velocity=0.0, dt=None):
    s = case.oracle_state(seed=seed, random_velocity=random_velocity)
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        dt = case.p.dt if dt is None else dt
        for n in range(nsteps):
            o.time_marcher(case.g, s, dt)
            gpu.time_marcher(dt, n)
        out = gpu.download()
    return s, out


@pytest.mark.parametrize("shape,steps,rv", [
    ((16, 12, 8), 1, 0.3),      # M=1, y radix 4*3
    ((40, 10, 6), 3, 0.2),      # M=2, y radix 2*5, z radix 2*3
    ((100, 20, 4), 2, 0.2),     # M=4 with padded rows
    ((256, 16, 8), 2, 0.1),     # M=8: the production chunk size
    ((64, 32, 16), 10, 0.0),    # RBC from rest, 10 steps
    ((48, 64, 1), 10, 0.0),     # 2-D (nzm = 1)
    ((48, 64, 1), 3, 0.2),      # 2-D with random velocity
    ((8, 384, 64), 2, 0.2),     # warp FFT: y N = 32*12, z N = 32*2
    ((8, 64, 384), 2, 0.2),     # warp FFT: z N = 32*12
    ((20, 96, 96), 2, 0.2),     # warp FFT N = 32*3 both ways
    ((21, 128, 32), 2, 0.2),    # odd nxm: the last x pair of the y transform has one point
    ((512, 32, 1), 2, 0.1),     # M=16, two rows per thread
    ((700, 8, 1), 2, 0.1),      # M=24, four rows per thread
    ((8, 512, 1), 2, 0.2),      # warp FFT y N = 32*16
    ((6, 768, 1), 2, 0.2),      # warp FFT y N = 32*24
    ((8, 1024, 1), 2, 0.2),     # warp FFT y N = 32*32
    ((4, 32, 512), 2, 0.2),     # warp FFT z N = 32*16
    ((4, 16, 1024), 1, 0.2),    # warp FFT z N = 32*32
])
def test_timemarcher_parity(shape, steps, rv):
    case = Case(*shape, rayt=1e6, dt=2e-3)
    s, out = _run_both(case, steps, random_velocity=rv)
    _compare(case, s, out, TOL_FP64)


@pytest.mark.parametrize("kw", [
    dict(gaxis=2, inslwn=0),                     # y gravity, free-slip top
    dict(gaxis=3, tfixn=0),                      # z gravity, zero-flux top plate
    dict(xplusu=0.5, xminusu=-0.25, dpdy=0.3),   # moving walls + Gy forcing
    dict(istr3=0),                               # uniform grid
    dict(istr3=6, str3=4.0),                     # clipped Chebyshev grid
    dict(nsst=1),                                # AB2 (InitTimeMarchScheme.F90:30-36)
])
def test_branch_parity(kw):
    kw = dict(kw)
    if kw.get("gaxis") == 2:
        kw.setdefault("inslwn", 0)
    case = Case(24, 16, 8, rayt=1e5, dt=1e-3, **kw)
    s, out = _run_both(case, 3, random_velocity=0.2)
    _compare(case, s, out, TOL_FP64)


def test_substep_api_matches_timemarcher():
    case = Case(32, 16, 8, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.2)
    gam, rom, alm = o.rk3_coefficients(3)
    dt = 1e-3
    beta = dt / case.g.ren * 0.5
    with case.solver() as a, case.solver() as b:
        for gpu in (a, b):
            gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        a.time_marcher(dt, 0)
        for ns in range(3):
            b.substep(ns, alm[ns], gam[ns], rom[ns], dt, beta)
        oa, ob = a.download(), b.download()
    for f in ag.Solver.FIELDS:
        np.testing.assert_array_equal(oa[f], ob[f])


def test_cfl_divergence_globals():
    case = Case(40, 24, 8, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.3)
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        assert gpu.calc_max_cfl() == pytest.approx(o.calc_max_cfl(case.g, s), rel=1e-14)
        assert gpu.check_divergence() == pytest.approx(o.check_divergence(case.g, s), rel=1e-13)
        nu, ke, _ = gpu.global_quantities(case.p.prat * abs(case.p.rayt))
        assert nu == pytest.approx(o.nusselt_volume(case.g, s), rel=1e-12)
        assert ke == pytest.approx(o.kinetic_energy(case.g, s), rel=1e-12)
        o.time_marcher(case.g, s, 1e-3)
        gpu.time_marcher(1e-3, 0)
        # after the projection both are divergence free to round-off
        assert gpu.check_divergence() < 1e-10
        assert o.check_divergence(case.g, s) < 1e-10


def test_cfl_after_timemarcher_passes_nan_on():
    """A NaN that a TimeMarcher spread through the state reaches the CFL maximum
    (CalcMaxCFL.F90:22; the main loop then turns it into 166/165)."""
    case = Case(40, 24, 8, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.1)
    s.vy[2, 3, 5] = np.nan
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        gpu.time_marcher(1e-3, 0)
        assert np.isnan(gpu.calc_max_cfl())


def test_variable_dt_main_loop():
    """Main-loop dt rule (main.F90:285-304) with the CFL from the device reduction."""
    import ctypes
    case = Case(32, 16, 8, rayt=1e7, idtv=1, dt=1e-3, cflmax=0.8, dtmax=5e-3)
    s = case.oracle_state(random_velocity=0.2)
    dt_o = dt_g = case.p.dt
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        for ntime in range(6):
            c_o = o.calc_max_cfl(case.g, s)
            c_g = gpu.calc_max_cfl()
            assert c_g == pytest.approx(c_o, rel=1e-10)
            dt_o, err_o, _ = o.next_dt(case.p, ntime, dt_o, c_o)
            dtc = ctypes.c_double(dt_g)
            err_g = ag.lib().afid_next_dt(ctypes.byref(case.inp), ntime, ctypes.byref(dtc), c_g, None)
            dt_g = dtc.value
            assert err_g == err_o
            assert dt_g == pytest.approx(dt_o, rel=1e-10)
            o.time_marcher(case.g, s, dt_o)
            gpu.time_marcher(dt_g, ntime)
        out = gpu.download()
    _compare(case, s, out, TOL_FP64)


def test_host_driver_run_matches_oracle_nu():
    """afid_run (C++ main loop) vs the oracle main loop: same Nu and KE after 5 steps."""
    import ctypes
    case = Case(32, 16, 8, rayt=1e6, idtv=1, dt=1e-3, cflmax=1.0, dtmax=4e-3, ntst=4)
    s = o.initial_state(case.g, 99)
    o.run(case.g, s, 5)
    st = ag.RunStatsT()
    rc = ag.lib().afid_run(ctypes.byref(case.inp), ag.PREC_FP64, 99, 5, 0, None, None, ctypes.byref(st))
    assert rc == 0
    assert st.steps_done == 5
    assert st.nu_vol == pytest.approx(o.nusselt_volume(case.g, s), rel=1e-9)
    assert st.ke == pytest.approx(o.kinetic_energy(case.g, s), rel=1e-6)


def test_fft_size_error():
    with pytest.raises(ag.AfidError) as e:
        Case(16, 14, 4).solver()  # 14 = 2*7
    assert e.value.status == ag.AFID_E_FFTSIZE


def test_unsupported_dpdz():
    case = Case(16, 8, 4)
    prm = case.tables.params
    prm.dpdz = 1.0
    with pytest.raises(ag.AfidError) as e:
        ag.Solver(case.tables.grid, prm)
    assert e.value.status == ag.AFID_E_INVALID


def test_halo_layout_upload():
    """Host arrays with the reference's 2-cell y/z halos (InitVariables.F90:68-73)."""
    import ctypes
    case = Case(24, 12, 6, rayt=1e5)
    s = case.oracle_state(random_velocity=0.2)
    nx, nym, nzm = case.p.nx, case.p.nym, case.p.nzm

    def with_halo(a):
        h = np.zeros((nzm + 4, nym + 4, nx))
        h[2:-2, 2:-2, :] = a
        return h
    hal = {f: with_halo(getattr(s, f)) for f in ("vx", "vy", "vz", "temp", "pr")}
    with case.solver() as gpu:
        ptr = lambda a: a[2:, 2:, :].ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        rc = ag.lib().afid_gpu_upload(gpu._h, *(ptr(hal[f]) for f in ("vx", "vy", "vz", "temp", "pr")),
                                      nx, nym + 4)
        assert rc == 0
        out = gpu.download()
    for f in ("vx", "vy", "vz", "temp", "pr"):
        np.testing.assert_array_equal(out[f], getattr(s, f))


def test_launch_count_positive():
    case = Case(16, 8, 4)
    with case.solver() as gpu:
        gpu.autotune()                     # its timing launches are counted too
        n0 = gpu.launch_count()
        gpu.time_marcher(1e-3)
        assert gpu.launch_count() - n0 == 1 + 3 * 7


@pytest.mark.parametrize("shape,precision", [((256, 24, 16), ag.PREC_FP64), ((100, 16, 8), ag.PREC_FP64),
                                             ((60, 16, 1), ag.PREC_FP64), ((500, 16, 4), ag.PREC_FP64),
                                             ((64, 32, 96), ag.PREC_FP64), ((100, 16, 8), ag.PREC_MIXED),
                                             ((64, 32, 96), ag.PREC_MIXED), ((60, 64, 64), ag.PREC_FP64),
                                             ((60, 64, 64), ag.PREC_MIXED), ((60, 16, 256), ag.PREC_MIXED),
                                             ((36, 8, 384), ag.PREC_MIXED), ((60, 16, 256), ag.PREC_FP64),
                                             ((36, 8, 384), ag.PREC_FP64), ((64, 8, 512), ag.PREC_FP64),
                                             ((36, 256, 8), ag.PREC_FP64), ((20, 384, 4), ag.PREC_FP64),
                                             ((44, 96, 4), ag.PREC_FP64), ((40, 64, 1), ag.PREC_FP64)])
def test_k4_and_fftz_forms_bitwise_identical(shape, precision):
    """Both forms of the Poisson tridiagonal (a mode per warp; persistent warps with the next
    mode prefetched), every form of the z transforms (a tile per block; persistent blocks with
    the next tile prefetched by per-thread copies, or by tensor copies) and both forms
    of the inverse y transform (per-thread copies; tensor copies for FP64 single domains with
    nym = 32 x {1, 2, 3, 4, 6, 8, 12}) and of the divergence + forward y transform (per-thread
    loads; tensor copies of the velocity rows) give the same fields bit for bit, so the autotuner's
    choices change the schedule only.  nxm = 60, 36, 20 and 44 leave partial tiles of x points."""
    case = Case(*shape, precision=precision, rayt=1e6, dt=2e-3)
    s = case.oracle_state(random_velocity=0.1)
    fp64 = precision == ag.PREC_FP64
    forms = (0, 1, 2)
    nym = shape[1]
    ify_ok = fp64 and nym % 32 == 0 and nym // 32 in (1, 2, 3, 4, 6, 8, 12)
    outs = []
    for form in forms:
        with case.solver() as g:
            g.autotune()
            g.set_k4_form(min(form, 1))
            g.set_fftz_form(form)
            if ify_ok:
                g.set_ify_form(min(form, 1))
            else:
                with pytest.raises(ag.AfidError) as e:
                    g.set_ify_form(1)
                assert e.value.status == ag.AFID_E_INVALID
                g.set_ify_form(0)
            if fp64 and nym % 32 == 0:
                g.set_div_form(min(form, 1))
            else:
                with pytest.raises(ag.AfidError) as e:
                    g.set_div_form(1)
                assert e.value.status == ag.AFID_E_INVALID
            g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
            for n in range(2):
                g.time_marcher(2e-3, n)
            outs.append(g.download())
    for o_ in outs[1:]:
        for k in ag.Solver.FIELDS:
            assert np.array_equal(outs[0][k], o_[k]), k


@pytest.mark.parametrize("name", ["rbc3d_16x12x8_rv", "rbc3d_40x10x6_rv", "rbc2d_32x48x1"])
def test_golden_fixture(name):
    """The GPU path from a committed fixture's initial state against its stored oracle steps."""
    import os
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz"))
    text = str(d["bou_in"])
    inp = ag.parse_bou_in(text)
    tab = ag.Tables(inp)
    nxm = inp.nxm
    with ag.Solver(tab.grid, tab.params) as gpu:
        gpu.upload(*(d["init_" + f] for f in ("vx", "vy", "vz", "temp", "pr")))
        for n in range(3):
            gpu.time_marcher(float(d["dt"]), n)
            if n in (0, 2):
                out = gpu.download()
                for f in ("vx", "vy", "vz", "temp"):
                    ref = d[f"step{n + 1}_{f}"][..., :nxm + (f == "vx")]
                    got = out[f][..., :nxm + (f == "vx")]
                    err = rel_l2(got, ref) if np.any(ref) else float(np.abs(got).max())
                    assert err <= TOL_FP64, (name, n, f, err)
                assert rel_l2_mod_mean(out["pr"][..., :nxm], d[f"step{n + 1}_pr"][..., :nxm]) <= TOL_FP64
        assert gpu.calc_max_cfl() == pytest.approx(float(d["step3_cfl"]), rel=1e-10)
        assert gpu.global_quantities(inp.prat * abs(inp.rayt))[0] == pytest.approx(float(d["step3_nu"]), rel=1e-10)


@pytest.mark.parametrize("shape", [(800, 8, 1), (1000, 8, 4)])
def test_timemarcher_parity_m32_exact_zero_mode(shape):
    """nxm = 800 and 1000 (M = 32, 2-D and 3-D).  The reference solves the singular (0,0)
    Poisson mode through a 1+1e-15 diagonal; at these wall-normal sizes that moves pr by ~4e-9
    relative to the exact discrete solution (CorrectPressure applies the stiff wall-normal
    operator to phi), so pr is compared with the oracle's exact (pinned) zero-mode solve; the
    velocities and temperature are compared with the reference behaviour as well."""
    case = Case(*shape, rayt=1e6, dt=2e-3)
    s_ref, out = _run_both(case, 1, random_velocity=0.1)
    nxm = case.p.nxm
    for k in ("vx", "vy", "temp"):
        assert rel_l2(out[k][..., :nxm + (k == "vx")], getattr(s_ref, k)[..., :nxm + (k == "vx")]) <= TOL_FP64, k
    assert rel_l2_mod_mean(out["pr"][..., :nxm], s_ref.pr[..., :nxm]) <= 3e-8
    case.g.pin_zero_mode = True
    s_pin = case.oracle_state(seed=1234, random_velocity=0.1)
    o.time_marcher(case.g, s_pin, 2e-3)
    _compare(case, s_pin, out, TOL_FP64)


def test_wall_normal_size_beyond_solver_is_rejected():
    """More wall-normal cells than the 32-chunk solvers cover (32 x 32) are refused at creation
    (AFID_E_INVALID), not at the first launch."""
    with pytest.raises(ag.AfidError) as e:
        Case(1100, 8, 4).solver()
    assert e.value.status == 603


@pytest.mark.parametrize("shape,precision", [((100, 16, 8), ag.PREC_FP64), ((384, 8, 4), ag.PREC_MIXED),
                                             ((500, 16, 1), ag.PREC_FP64), ((700, 8, 1), ag.PREC_FP64),
                                             ((256, 16, 8), ag.PREC_FP64), ((60, 16, 8), ag.PREC_FP64),
                                             ((256, 24, 1), ag.PREC_FP64), ((200, 16, 8), ag.PREC_MIXED)])
def test_k1_shapes_bitwise_identical(shape, precision):
    """Every launch shape the autotuner may pick (threads, rows per thread, register cap, cache
    policy, one or two columns per block, the persistent form with shared-memory tables) gives
    the same fields bit for bit, and the autotuner reports a timing for each."""
    case = Case(*shape, precision=precision, rayt=1e6, dt=2e-3)
    s = case.oracle_state(random_velocity=0.1)
    outs = []
    with case.solver() as g:
        info = g.autotune()
    assert info["ncand"] >= 2 and all(us > 0 for *_, us in info["shapes"])
    for v in range(info["ncand"]):
        with case.solver() as g:
            g.set_k1_shape(v)
            g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
            for n in range(2):
                g.time_marcher(2e-3, n)
            outs.append(g.download())
    for o in outs[1:]:
        for k in ag.Solver.FIELDS:
            assert np.array_equal(o[k], outs[0][k]), k
