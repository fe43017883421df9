"""Wall-normal profiles of CalcMeanProfiles.F90 computed on the device (afid_gpu_mean_profiles,
afid_batch_mean_profiles) against the oracle's restatement, on states with every velocity
component and temperature perturbation non-zero.

Tolerance: 1e-12 relative to each profile's largest magnitude (the sums run in a different
order than the reference's loops).
"""
import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case, bou_text
from oracle import afid_oracle as o

pytestmark = pytest.mark.gpu


def _random_state(case, seed=3):
    s = case.oracle_state(seed=1234, random_velocity=0.2, rng_seed=seed)
    rng = np.random.default_rng(seed + 1)
    s.temp[..., :case.p.nxm] += 0.1 * rng.standard_normal(s.temp[..., :case.p.nxm].shape)
    return s


def _compare(got, ref, tol=1e-12):
    for name in o.MEAN_PROFILE_NAMES:
        scale = max(np.abs(ref[name]).max(), 1e-300)
        err = np.abs(got[name] - ref[name]).max() / scale
        assert err < tol, (name, err)


@pytest.mark.parametrize("shape,kw", [
    ((32, 24, 16), {}),
    ((40, 16, 8), dict(inslws=0, tfixn=0, xplusu=0.3, xminusu=-0.2)),
    ((48, 64, 1), {}),
    ((256, 16, 8), dict(tfixs=0)),
])
@pytest.mark.parametrize("precision", [ag.PREC_FP64, ag.PREC_MIXED])
def test_profiles_match_oracle(shape, kw, precision):
    case = Case(*shape, precision=precision, rayt=1e7, prat=0.7, **kw)
    s = _random_state(case)
    with case.solver() as g:
        g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        got = g.mean_profiles()
    _compare(got, o.mean_profiles(case.g, s))


def test_batch_slot_profiles_match_oracle():
    nxm, nym = 32, 64
    cfgs = [dict(rayt=1e6, prat=1.0, ylen=2.0), dict(rayt=3e7, prat=4.4, ylen=1.0), dict(rayt=2e5, prat=0.7, ylen=4.0)]
    inps = [ag.parse_bou_in(bou_text(nxm, nym, 1, **c)) for c in cfgs]
    states = []
    with ag.Batch(inps[0], len(cfgs), ag.PREC_FP64) as b:
        for k, (inp, c) in enumerate(zip(inps, cfgs)):
            case = Case(nxm, nym, 1, **c)
            st = _random_state(case, seed=10 + k)
            b.configure(k, inp)
            b.upload(k, st.vx[0], st.vy[0], st.vz[0], st.temp[0], st.pr[0])
            states.append((case, st))
        for k, (case, st) in enumerate(states):
            _compare(b.mean_profiles(k), o.mean_profiles(case.g, st))


def test_profiles_after_steps_give_conduction_nusselt_at_rest():
    """From the conductive state (no perturbation) the device profiles keep Pe * int chiT dx = 1."""
    case = Case(64, 32, 16, rayt=1e5, dt=1e-3)
    s = o.initial_state(case.g, 1, eps=0.0)
    with case.solver() as g:
        g.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        for n in range(3):
            g.time_marcher(1e-3, n)
        m = g.mean_profiles()
    dxk = case.g.xc[1:65] - case.g.xc[:64]
    assert abs(case.g.pect * np.sum(m["chiT"] * dxk) - 1.0) < 1e-9
    assert np.abs(m["epsilon"]).max() < 1e-20
