"""Spectra (spectra.F90), movie planes (MakeMovie{X,Y,Z}Cut.F90) and plane means
(h5tools/mean_zplane.F90, means.F90) from the device state, against the oracle's restatement and
the downloaded fields.  Plane means are bitwise equal to the oracle's (same summation order).

Tolerance for spectra: 1e-12 relative to the largest value of each spectrum in FP64 (the FFTs
differ from pocketfft in rounding only), 2e-5 with the FP32 transforms of the mixed path."""
import os

import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case
from oracle import afid_h5 as h5
from oracle import afid_oracle as o

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(24, 32, 16), (16, 96, 64), (20, 10, 6), (32, 64, 1)])
@pytest.mark.parametrize("precision", [ag.PREC_FP64, ag.PREC_MIXED])
def test_spectra_match_oracle(shape, precision):
    case = Case(*shape, precision=precision, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.2)
    acc = {}
    with case.solver() as g:
        g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        g.spectra_reset()
        g.spectra_update(0.3)
        o.spectra_update(case.g, s, 0.3, acc)
        g.time_marcher(1e-3, 0)
        o.time_marcher(case.g, s, 1e-3)
        g.spectra_update(0.2)
        o.spectra_update(case.g, s, 0.2, acc)
        got = g.spectra()
    assert abs(got["tav"] - 0.5) < 1e-15
    tol = 1e-12 if precision == ag.PREC_FP64 else 2e-5
    for name in ("vx", "vy", "vz", "temp"):
        ref = acc[name] / 0.5
        err = np.abs(got[name] - ref).max() / max(np.abs(ref).max(), 1e-300)
        assert err < tol, (name, err)


@pytest.mark.parametrize("shape", [(16, 96, 64), (24, 64, 32)])
def test_spectra_with_tensor_copy_forms(shape):
    """The spectra's field transforms take the per-thread y transform and the chosen z form
    while the step runs the tensor-copy forms of K2, K3/K5 and K6 (FP64)."""
    case = Case(*shape, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.2)
    acc = {}
    with case.solver() as g:
        g.autotune()
        g.set_div_form(1)
        g.set_fftz_form(2)
        g.set_ify_form(1)
        g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        g.spectra_reset()
        g.spectra_update(0.3)
        o.spectra_update(case.g, s, 0.3, acc)
        g.time_marcher(1e-3, 0)
        o.time_marcher(case.g, s, 1e-3)
        g.spectra_update(0.2)
        o.spectra_update(case.g, s, 0.2, acc)
        got = g.spectra()
    for name in ("vx", "vy", "vz", "temp"):
        ref = acc[name] / 0.5
        err = np.abs(got[name] - ref).max() / max(np.abs(ref).max(), 1e-300)
        assert err < 1e-12, (name, err)


def test_slices_are_planes_of_the_state():
    case = Case(20, 24, 12, rayt=1e6)
    s = case.oracle_state(random_velocity=0.2)
    with case.solver() as g:
        g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        f = g.download()
        for w, name in enumerate(ag.Solver.FIELDS):
            assert np.array_equal(g.slice(w, 0, 3), f[name][:, :, 3])
            assert np.array_equal(g.slice(w, 1, 5), f[name][:, 5, :])
            assert np.array_equal(g.slice(w, 2, 7), f[name][7, :, :])
        with pytest.raises(ag.AfidError):
            g.slice(0, 0, 21)


@pytest.mark.parametrize("shape", [(20, 24, 12), (33, 16, 40)])
def test_mean_planes_match_oracle(shape):
    case = Case(*shape, rayt=1e6)
    s = case.oracle_state(random_velocity=0.2)
    with case.solver() as g:
        g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        g.time_marcher(1e-3, 0)
        f = g.download()
        for w, name in enumerate(("vx", "vy", "vz", "temp")):
            for axis in (1, 2):
                np.testing.assert_array_equal(g.mean_plane(w, axis), o.mean_plane(f[name], axis),
                                              err_msg=f"{name} axis {axis}")
        with pytest.raises(ag.AfidError):
            g.mean_plane(4, 1)          # pr has no plane-mean file
        with pytest.raises(ag.AfidError):
            g.mean_plane(0, 0)


def test_salinity_mean_planes_match_oracle():
    from test_gpu_salinity import SalCase
    c = SalCase((16, 16, 8), (32, 32, 16))
    with c.solver() as g:
        g.time_marcher(1e-3, 0)
        sal = g.sal_download()
        for axis in (1, 2):
            np.testing.assert_array_equal(g.sal_mean_plane(axis), o.mean_plane(sal, axis))


def test_spectrum_files_hold_the_averaged_spectra(tmp_path):
    case = Case(16, 24, 8, rayt=1e6)
    s = case.oracle_state(random_velocity=0.2)
    d = str(tmp_path / "outputdir")
    with case.solver() as g:
        g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        g.spectra_reset()
        g.spectra_update(0.25)
        g.time_marcher(1e-3, 0)
        g.spectra_update(0.25)
        got = g.spectra()
        g.write_spectra(d)
    for name, fname in (("vx", "vx"), ("vy", "vy"), ("vz", "vz"), ("temp", "te")):
        a = h5.read(os.path.join(d, f"{fname}_spectrum.h5"), "var")
        assert a.shape == (8, 24, 16)
        np.testing.assert_array_equal(a[:, :13, :], got[name])
        assert np.all(a[:, 13:, :] == 0.0)
