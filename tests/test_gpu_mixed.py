"""Mixed-precision path (FP32 explicit terms, y/z transforms and Poisson spectrum; FP64
tridiagonal solves, divergence, reductions and state) against the FP64 path.

Gates: per-field relative L2 after a few steps at the FP32 rounding level, and the Nusselt
number of a convecting run within 0.5% of the FP64 run (time average over the last third).
"""
import ctypes

import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case, rel_l2, rel_l2_mod_mean
from oracle import afid_oracle as o

pytestmark = pytest.mark.gpu


def _pair(shape, **kw):
    return (Case(*shape, precision=ag.PREC_FP64, **kw), Case(*shape, precision=ag.PREC_MIXED, **kw))


@pytest.mark.parametrize("shape", [(32, 32, 16), (64, 384, 1), (40, 96, 64), (24, 12, 8),
                                   (512, 32, 1), (8, 1024, 1), (16, 512, 1), (4, 16, 1024)])
def test_mixed_fields_close_to_fp64(shape):
    # dt inside the explicit horizontal-diffusion bound 0.63 dy^2 Re (Re = 1000 here)
    dt = min(1e-3, 0.3 * 1000.0 / max(shape[1], shape[2]) ** 2)
    a, b = _pair(shape, rayt=1e6, dt=dt)
    s = a.oracle_state(random_velocity=0.2)
    with a.solver() as g64, b.solver() as g32:
        for g in (g64, g32):
            g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        for n in range(5):
            g64.time_marcher(dt, n)
            g32.time_marcher(dt, n)
        o64, o32 = g64.download(), g32.download()
    nxm = shape[0]
    tv = 2e-5
    assert rel_l2(o32["vx"], o64["vx"]) < tv
    assert rel_l2(o32["vy"][..., :nxm], o64["vy"][..., :nxm]) < tv
    if shape[2] > 1:
        assert rel_l2(o32["vz"][..., :nxm], o64["vz"][..., :nxm]) < tv
    assert rel_l2(o32["temp"][..., :nxm], o64["temp"][..., :nxm]) < 1e-6
    assert rel_l2_mod_mean(o32["pr"][..., :nxm], o64["pr"][..., :nxm]) < 1e-4


def test_mixed_nusselt_within_half_percent():
    """2-D Rayleigh-Benard, Ra = 1e6, from the seeded perturbation through the onset of
    convection; Nu_vol averaged over the last third of the run."""
    a, b = _pair((64, 128, 1), rayt=1e6, ylen=2.0, zlen=0.01, idtv=1, dt=1e-3, cflmax=1.0, dtmax=5e-3)
    s = o.initial_state(a.g, 2026)
    ra_pr = a.p.prat * abs(a.p.rayt)
    nus = {}
    for name, case in (("fp64", a), ("mixed", b)):
        with case.solver() as g:
            g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
            dt = ctypes.c_double(case.p.dt)
            series = []
            for n in range(6000):
                cfl = g.calc_max_cfl()
                ag.lib().afid_next_dt(ctypes.byref(case.inp), n, ctypes.byref(dt), cfl, None)
                g.time_marcher(dt.value, n)
                if n % 10 == 0:
                    series.append(g.global_quantities(ra_pr)[0])
            nus[name] = np.array(series)
    tail = 2 * len(nus["fp64"]) // 3
    n64, n32 = nus["fp64"][tail:].mean(), nus["mixed"][tail:].mean()
    assert n64 > 2.0, f"no convection developed (Nu={n64})"
    assert abs(n32 - n64) / n64 < 5e-3, (n32, n64)
