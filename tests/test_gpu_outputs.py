"""Spectra (spectra.F90) and movie planes (MakeMovie{X,Y,Z}Cut.F90) from the device state,
against the oracle's restatement and the downloaded fields.

Tolerance for spectra: 1e-12 relative to the largest value of each spectrum in FP64 (the FFTs
differ from pocketfft in rounding only), 2e-5 with the FP32 transforms of the mixed path."""
import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case
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
