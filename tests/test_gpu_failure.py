"""Failure detection without a GPU fault.

* Bounded device waits: the fused explicit/implicit kernel's staging wait is made to run out
  (afid_gpu_set_wait_test: after its copies land it also waits for an mbarrier phase that
  nothing completes, at most a few thousand polls).  Every block gives up, drains, sets the
  error flag and exits; the next synchronising call returns AFID_E_TIMEOUT, the flag stays set
  on that context, and the device stays usable: a new context on the same GPU steps and matches
  the oracle.
* Blown-up fields: a NaN in the velocity propagates through the CFL and divergence maxima
  (CalcMaxCFL.F90:22-43, CheckDivergence.F90:22-42), and the main-loop rules of
  main.F90:287-302, 357 turn it into 166 (variable dt), 165 (fixed dt) and 169 (divergence);
  in a batch only the instance with the NaN stops.
"""
import ctypes

import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case, bou_text, rel_l2
from oracle import afid_oracle as o

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_with_timeout_status():
    case = Case(32, 16, 8, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.1)
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        gpu.set_wait_test(4096)
        with pytest.raises(ag.AfidError) as e:
            gpu.time_marcher(1e-3, 0)               # stream-ordered: returns before the kernels end
            gpu.synchronize()                       # the next synchronising call reports it
        assert e.value.status == ag.AFID_E_TIMEOUT
        gpu.set_wait_test(0)
        with pytest.raises(ag.AfidError) as e:      # the flag stays set on this context
            gpu.calc_max_cfl()
        assert e.value.status == ag.AFID_E_TIMEOUT
    # the GPU itself is fine: a new context steps and matches the oracle
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        gpu.time_marcher(1e-3, 0)
        out = gpu.download()
    o.time_marcher(case.g, s, 1e-3)
    assert rel_l2(out["vx"], s.vx) < 1e-10
    assert rel_l2(out["temp"][..., :case.p.nxm], s.temp[..., :case.p.nxm]) < 1e-10


def test_bounded_wait_runs_out_in_every_k1_form():
    """The same bounded wait in every K1 form of the 129..256 wall-normal class (one column per
    block, two columns per block, the persistent form): each reports AFID_E_TIMEOUT at the next
    synchronising call and leaves no copy in flight (the device steps on in a new context)."""
    case = Case(200, 16, 8, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.1)
    with case.solver() as gpu:
        ncand = gpu.autotune()["ncand"]
    for v in range(ncand):
        with case.solver() as gpu:
            gpu.set_k1_shape(v)
            gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
            gpu.set_wait_test(4096)
            with pytest.raises(ag.AfidError) as e:
                gpu.time_marcher(1e-3, 0)
                gpu.synchronize()
            assert e.value.status == ag.AFID_E_TIMEOUT, v
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        gpu.time_marcher(1e-3, 0)
        out = gpu.download()
    o.time_marcher(case.g, s, 1e-3)
    assert rel_l2(out["vx"], s.vx) < 1e-10


def test_bounded_wait_runs_out_in_tensor_copy_transforms():
    """The tensor-copy forms of the z transforms and of both y transforms wait on an mbarrier
    for their tiles too: with the hook set their blocks give up, the next synchronising
    call reports AFID_E_TIMEOUT, and no copy is left in flight (a new context on the same device
    steps and matches the oracle)."""
    case = Case(60, 64, 256, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.1)
    with case.solver() as gpu:
        gpu.autotune()
        gpu.set_fftz_form(2)
        gpu.set_ify_form(1)
        gpu.set_div_form(1)
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        gpu.set_wait_test(4096)
        with pytest.raises(ag.AfidError) as e:
            gpu.time_marcher(1e-3, 0)
            gpu.synchronize()
        assert e.value.status == ag.AFID_E_TIMEOUT
    with case.solver() as gpu:
        gpu.autotune()
        gpu.set_fftz_form(2)
        gpu.set_ify_form(1)
        gpu.set_div_form(1)
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        gpu.time_marcher(1e-3, 0)
        out = gpu.download()
    o.time_marcher(case.g, s, 1e-3)
    assert rel_l2(out["vx"], s.vx) < 1e-10
    nxm = case.p.nxm
    assert rel_l2(out["temp"][..., :nxm], s.temp[..., :nxm]) < 1e-10


def test_bounded_wait_runs_out_in_tensor_copy_z_transform_mixed():
    """The same for the FP32 spectrum of the mixed path (two columns a warp): AFID_E_TIMEOUT at
    the next synchronising call, and a new context on the device steps to the same fields as a
    context that never ran out."""
    case = Case(60, 16, 256, precision=ag.PREC_MIXED, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.1)
    with case.solver() as gpu:
        gpu.autotune()
        gpu.set_fftz_form(2)
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        gpu.set_wait_test(4096)
        with pytest.raises(ag.AfidError) as e:
            gpu.time_marcher(1e-3, 0)
            gpu.synchronize()
        assert e.value.status == ag.AFID_E_TIMEOUT
    outs = []
    for form in (2, 1):
        with case.solver() as gpu:
            gpu.autotune()
            gpu.set_fftz_form(form)
            gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
            gpu.time_marcher(1e-3, 0)
            outs.append(gpu.download())
    for k in ag.Solver.FIELDS:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_wait_test_hook_rejects_out_of_range():
    case = Case(16, 8, 4)
    with case.solver() as gpu:
        for bad in (-1, 1 << 25):
            with pytest.raises(ag.AfidError) as e:
                gpu.set_wait_test(bad)
            assert e.value.status == ag.AFID_E_INVALID


def _next_dt(inp, ntime, dt, cflm):
    dtc = ctypes.c_double(dt)
    err = ag.lib().afid_next_dt(ctypes.byref(inp), ntime, ctypes.byref(dtc), cflm, None)
    return err, dtc.value


@pytest.mark.parametrize("field", ["vx", "vy", "vz"])
def test_nan_velocity_gives_main_loop_error_codes(field):
    case = Case(24, 16, 8, rayt=1e6, dt=1e-3, idtv=1, cflmax=1.2, dtmax=1e-2)
    s = case.oracle_state(random_velocity=0.1)
    getattr(s, field)[3, 5, 7] = np.nan
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        cflm = gpu.calc_max_cfl()
        dmax = gpu.check_divergence()
    assert np.isnan(cflm) and np.isnan(dmax)
    # variable dt: dt = CFLMAX / NaN is no valid step -> 166 (main.F90:287-298)
    err, _ = _next_dt(case.inp, 5, 1e-3, cflm)
    assert err == ag.AFID_E_DTMIN
    # fixed dt: CFL * dt > CFLMAX cannot be ruled out -> 165 (main.F90:300-302)
    fixed = ag.parse_bou_in(bou_text(24, 16, 8, rayt=1e6, dt=1e-3, idtv=0, cflmax=1.2))
    err, _ = _next_dt(fixed, 5, 1e-3, cflm)
    assert err == ag.AFID_E_CFL
    # finite values keep the reference's rules exactly
    assert _next_dt(case.inp, 5, 1e-3, 0.5)[0] == 0
    assert _next_dt(fixed, 5, 1e-3, 2000.0)[0] == ag.AFID_E_CFL


def test_nan_in_one_batch_instance_stops_only_that_instance():
    step = dict(zlen=1.0, idtv=1, dt=1e-3, cflmax=1.2, dtmax=2e-3)
    inp = ag.parse_bou_in(bou_text(32, 64, 1, rayt=1e6, **step))
    with ag.Batch(inp, 3, ag.PREC_FP64) as b:
        for slot in range(3):
            b.seed(slot, 40 + slot)
        f = b.download(1)
        f["vy"][9, 4] = np.nan                      # a 2-D slot comes back as (nym, nx)
        b.upload(1, f["vx"], f["vy"], f["vz"], f["temp"], f["pr"])
        dm = b.divmax()
        assert np.isnan(dm[1]) and np.isfinite(dm[0]) and np.isfinite(dm[2])
        b.set_active(np.ones(3, np.uint8))
        b.step(6)
        st = b.stats()
    # the first two steps use the bou.in dt (main.F90:288-296); the third computes dt from the
    # NaN CFL, raises 166, completes, and the instance stops
    assert st["errorcode"][1] == ag.AFID_E_DTMIN and st["ntime"][1] == 3
    assert st["errorcode"][0] == 0 and st["errorcode"][2] == 0
    assert st["ntime"][0] == 6 and st["ntime"][2] == 6
    assert np.isfinite(st["nu_vol"][0]) and np.isfinite(st["nu_vol"][2])
