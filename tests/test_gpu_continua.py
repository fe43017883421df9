"""Restart files through a device context and the host main loop (include/afid_continua.h).

A restart from the continua files continues the run: the RK3 history is zeroed on upload and the
first substep weights it by rom(1) = 0, so the restarted fields follow the uninterrupted run to
round-off (1e-12 relative L2 here; the K1 shape chosen by the autotuner may differ between the
two contexts).
"""
import ctypes
import math
import os

import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case, bou_text, rel_l2
from oracle import afid_h5 as h5

pytestmark = pytest.mark.gpu

FIELDS = ("vx", "vy", "vz", "temp", "pr")


def test_restart_through_files_continues_the_run(tmp_path):
    c = Case(16, 24, 12)
    s = c.oracle_state(random_velocity=0.05)
    m = ag.continua_master(c.inp, 0.0)
    d = str(tmp_path / "out")
    with c.solver() as a:
        a.upload(*(getattr(s, f) for f in FIELDS))
        for n in range(3):
            a.time_marcher(1e-3, n)
        m.time = 3e-3
        a.write_flow_field(d, m, final=True)
        with c.solver() as b:
            assert b.read_flow_field(d, m) == 3e-3
            got_b0 = b.download()
            got_a0 = a.download()
            for f in FIELDS:
                np.testing.assert_array_equal(got_b0[f], got_a0[f])
            for n in range(3, 6):
                a.time_marcher(1e-3, n)
                b.time_marcher(1e-3, n)
            ga, gb = a.download(), b.download()
    for f in FIELDS:
        assert rel_l2(gb[f], ga[f]) < 1e-12, f
    # the files hold what the device held at the write
    np.testing.assert_array_equal(h5.read(os.path.join(d, "continua_vx.h5"), "var"), got_a0["vx"])


def _replay_frames(t0, dt, nsteps, save_3d, tframe):
    """Frame numbers main.F90:241 and :376-381 produce for a fixed dt (same double arithmetic)."""
    nint = lambda v: int(math.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)  # noqa: E731  Fortran nint
    frames = [nint(t0 / save_3d)]
    t = t0
    for _ in range(nsteps):
        t += dt
        if math.fmod(t, save_3d) < dt and math.floor(t / tframe) != 0:
            frames.append(nint(t / save_3d))
    return t, sorted(set(frames))


@pytest.mark.parametrize("sal", [False, True])
def test_run_io_restart_matches_an_uninterrupted_run(tmp_path, sal):
    """afid_run_io: 4 steps from the seeded state (NREAD = 0), then NREAD = 1 for 3 more steps,
    against afid_run for 7 steps; the frames and the final continua files are where the main
    loop puts them."""
    kw = dict(idtv=0, dt=1e-3, save_3d=2.5e-3, tframe=1e-3, ntst=1000)
    if sal:
        kw.update(multires=1, nxmr=32, nymr=32, nzmr=16, flagsal=1, rays=1e6, pras=10.0, active_s=1, istr3r=4)
    d = str(tmp_path / "run")
    first = ag.parse_bou_in(bou_text(16, 16, 8, nread=0, **kw))
    st = ag.RunStatsT()
    assert ag.lib().afid_run_io(ctypes.byref(first), ag.PREC_FP64, 5, 4, 0, None, None, d.encode(),
                                ctypes.byref(st)) == 0
    assert st.steps_done == 4
    t1, frames1 = _replay_frames(0.0, 1e-3, 4, 2.5e-3, 1e-3)
    mm = ag.read_continua_master(d, multires=sal)
    assert mm.time == st.time == t1
    second = ag.parse_bou_in(bou_text(16, 16, 8, nread=1, **kw))
    st2 = ag.RunStatsT()
    assert ag.lib().afid_run_io(ctypes.byref(second), ag.PREC_FP64, 5, 3, 0, None, None, d.encode(),
                                ctypes.byref(st2)) == 0
    t2, frames2 = _replay_frames(t1, 1e-3, 3, 2.5e-3, 1e-3)
    assert st2.time == t2
    names = {"temp", "vx", "vy", "vz"} | ({"sal"} if sal else set())
    want = sorted(f"{fr:05d}_{k}.h5" for fr in set(frames1) | set(frames2) for k in names)
    assert sorted(os.listdir(os.path.join(d, "fields"))) == want
    assert ag.read_continua_master(d, multires=sal).time == t2
    # the plane means sit beside the cuts, frame for frame (main.F90:233-235, 337-343)
    for mean, cut in (("movie_ymean.h5", "movie_ycut.h5"), ("movie_zmean.h5", "movie_zcut.h5")):
        fm, fc = h5.H5File(os.path.join(d, "flowmov", mean)), h5.H5File(os.path.join(d, "flowmov", cut))
        assert sorted(fm.links(fm.resolve("temp"))) == sorted(fc.links(fc.resolve("temp")))
        assert sorted(fm.root()) == sorted(fc.root())
    ref = ag.RunStatsT()
    assert ag.lib().afid_run(ctypes.byref(first), ag.PREC_FP64, 5, 7, 0, None, None, ctypes.byref(ref)) == 0
    assert st2.nu_vol == pytest.approx(ref.nu_vol, rel=1e-11)
    assert st2.ke == pytest.approx(ref.ke, rel=1e-11)


def test_salinity_restart_through_files(tmp_path):
    from test_gpu_salinity import SalCase
    c = SalCase((16, 16, 8), (32, 32, 16))
    m = ag.continua_master(ag.parse_bou_in(c.text), 2e-3)
    d = str(tmp_path / "sal")
    with c.solver() as a:
        for n in range(2):
            a.time_marcher(1e-3, n)
        a.write_flow_field(d, m, final=True)
        with ag.Solver(c.tables.grid, c.tables.params) as b:
            b.sal_create(c.mgrd)
            assert b.read_flow_field(d, m) == 2e-3
            np.testing.assert_array_equal(b.sal_download(), a.sal_download())
            for n in range(2, 4):
                a.time_marcher(1e-3, n)
                b.time_marcher(1e-3, n)
            sa_, sb_ = a.sal_download(), b.sal_download()
            fa, fb = a.download(), b.download()
    assert rel_l2(sb_, sa_) < 1e-12
    for f in ("vx", "vy", "vz", "temp"):
        assert rel_l2(fb[f], fa[f]) < 1e-12, f
    s = h5.read(os.path.join(d, "continua_sal.h5"), "var")
    assert s.shape == (16, 32, 33) and np.all(s[..., 32] == 0.0)


def test_restart_on_another_grid(tmp_path):
    """NREAD = 1 with continua files from a coarser grid: the interpolating restart uploads what
    the host interpolation produces, and afid_run_io carries on from it."""
    kw = dict(idtv=0, dt=1e-3, save_3d=1e30, tframe=1e30, ntst=1000)
    d = str(tmp_path / "run")
    first = ag.parse_bou_in(bou_text(16, 16, 8, nread=0, **kw))
    st = ag.RunStatsT()
    assert ag.lib().afid_run_io(ctypes.byref(first), ag.PREC_FP64, 9, 3, 0, None, None, d.encode(),
                                ctypes.byref(st)) == 0
    text = bou_text(24, 20, 12, nread=1, **kw)
    second = ag.parse_bou_in(text)
    host = ag.read_flow_interp(d, second)
    assert host["interpolated"]
    tables = ag.Tables(second)
    with ag.Solver(tables.grid, tables.params) as sv:
        t, interp = sv.read_flow_interp(d, second)
        assert interp and t == st.time
        got = sv.download()
    for f in ("vx", "vy", "vz", "temp"):
        np.testing.assert_array_equal(got[f][..., :24], host[f][..., :24])
    assert np.all(got["pr"] == 0.0)
    st2 = ag.RunStatsT()
    assert ag.lib().afid_run_io(ctypes.byref(second), ag.PREC_FP64, 9, 2, 0, None, None, d.encode(),
                                ctypes.byref(st2)) == 0
    assert st2.steps_done == 2 and np.isfinite(st2.nu_vol) and np.isfinite(st2.ke) and st2.divmax < 1e-10
    assert ag.read_continua_master(d).nx == 25
