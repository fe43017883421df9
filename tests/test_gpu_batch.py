"""Batched 2-D instances (include/afid_batch.h).

Gates:
- alone == in-mix: a slot's fields after N steps are bitwise identical whether it ran alone or
  next to other active slots with different Ra, Pr, aspect ratio and seeds (both precisions);
- an idle slot keeps its state bit for bit while the others step;
- a slot agrees with the same case run as its own context through the single-domain API with
  the main-loop dt rule driven from the host (main.F90:285-313);
- an instance that raises an error code (fixed dt, CFL > CFLMAX) stops; the others go on.
"""
import ctypes

import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case, bou_text, rel_l2

pytestmark = pytest.mark.gpu

NXM, NYM = 32, 64
SLOTS = [dict(rayt=1e6, prat=1.0, ylen=2.0), dict(rayt=3e7, prat=0.7, ylen=1.0),
         dict(rayt=2e5, prat=4.4, ylen=4.0), dict(rayt=1e8, prat=1.0, ylen=2.0),
         dict(rayt=5e6, prat=0.7, ylen=1.0)]
STEP = dict(zlen=1.0, idtv=1, dt=1e-3, cflmax=1.2, dtmax=2e-3)


def _inp(**kw):
    v = dict(STEP)
    v.update(kw)
    return ag.parse_bou_in(bou_text(NXM, NYM, 1, **v))


def _batch(precision, nslots=len(SLOTS)):
    b = ag.Batch(_inp(**SLOTS[0]), nslots, precision)
    for s in range(nslots):
        b.configure(s, _inp(**SLOTS[s % len(SLOTS)]))
        b.seed(s, 100 + s)
    return b


def _perturb(b, slot, amp=0.05):
    """Non-zero velocity so the flow terms and the CFL rule are exercised from step 1."""
    rng = np.random.default_rng(slot)
    f = b.download(slot)
    for k in ("vx", "vy"):
        f[k][...] = amp * rng.standard_normal(f[k].shape)
    f["vx"][:, 0] = 0.0
    f["vx"][:, NXM] = 0.0
    f["vy"][:, NXM] = 0.0
    b.upload(slot, f["vx"], f["vy"], f["vz"], f["temp"], f["pr"])


@pytest.mark.parametrize("precision", [ag.PREC_FP64, ag.PREC_MIXED])
def test_alone_equals_in_mix(precision):
    target, nsteps = 2, 40
    out = {}
    for mix in ("alone", "all", "odd_out"):
        with _batch(precision) as b:
            for s in range(b.nslots):
                _perturb(b, s)
            act = np.zeros(b.nslots, np.uint8)
            if mix == "alone":
                act[target] = 1
            elif mix == "all":
                act[:] = 1
            else:
                act[[0, 2, 3]] = 1
            b.set_active(act)
            b.step(nsteps // 2)
            if mix == "odd_out":  # change the mix halfway: slot 4 joins, slot 0 leaves
                act[0], act[4] = 0, 1
                b.set_active(act)
            b.step(nsteps - nsteps // 2)
            st = b.stats()
            out[mix] = (b.download(target), st)
    ref, st_ref = out["alone"]
    assert st_ref["ntime"][target] == nsteps and st_ref["errorcode"][target] == 0
    for mix in ("all", "odd_out"):
        f, st = out[mix]
        for k in ag.Batch.FIELDS:
            assert np.array_equal(f[k][:, :NXM], ref[k][:, :NXM]), (mix, k)
        assert st["dt"][target] == st_ref["dt"][target]
        assert st["time"][target] == st_ref["time"][target]
        assert st["nu_vol"][target] == st_ref["nu_vol"][target]


def test_idle_slot_keeps_state():
    with _batch(ag.PREC_FP64) as b:
        for s in range(b.nslots):
            _perturb(b, s)
        before = b.download(1)
        act = np.ones(b.nslots, np.uint8)
        act[1] = 0
        b.set_active(act)
        b.step(7)  # odd step count: the temperature buffers end swapped
        after = b.download(1)
        st = b.stats()
    for k in ag.Batch.FIELDS:
        assert np.array_equal(after[k][:, :NXM], before[k][:, :NXM]), k
    assert st["ntime"][1] == 0 and st["ntime"][0] == 7


@pytest.mark.parametrize("precision", [ag.PREC_FP64, ag.PREC_MIXED])
def test_slot_matches_single_domain(precision):
    slot, nsteps = 3, 30
    with _batch(precision) as b:
        for s in range(b.nslots):
            _perturb(b, s)
        init = b.download(slot)
        b.set_active(np.ones(b.nslots, np.uint8))
        b.step(nsteps)
        got = b.download(slot)
        st = b.stats()
    case = Case(NXM, NYM, 1, precision=precision, **dict(STEP, **SLOTS[slot]))
    dt = ctypes.c_double(case.p.dt)
    with case.solver() as g:
        g.upload(*(init[k][None] for k in ag.Solver.FIELDS))
        t = 0.0
        for n in range(nsteps):
            cfl = g.calc_max_cfl()
            assert ag.lib().afid_next_dt(ctypes.byref(case.inp), n, ctypes.byref(dt), cfl, None) == 0
            g.time_marcher(dt.value, n)
            t += dt.value
        ref = g.download()
        nu, ke, _ = g.global_quantities(case.p.prat * abs(case.p.rayt))
    tol = 1e-11 if precision == ag.PREC_FP64 else 1e-5
    for k in ("vx", "vy", "temp"):
        assert rel_l2(got[k][:, :NXM], ref[k][0][:, :NXM]) < tol, k
    assert abs(st["time"][slot] - t) < 1e-12 * t
    assert abs(st["nu_vol"][slot] - nu) < 1e-9 * abs(nu)
    assert abs(st["ke"][slot] - ke) < 1e-9 * abs(ke) + 1e-300


def test_error_stops_only_that_instance():
    with ag.Batch(_inp(**SLOTS[0]), 3, ag.PREC_FP64) as b:
        for s in range(3):
            b.configure(s, _inp(**SLOTS[s]) if s != 1 else _inp(**dict(SLOTS[1], idtv=0, dt=0.1)))
            b.seed(s, 7 + s)
            _perturb(b, s, amp=1.0)
        b.set_active(np.ones(3, np.uint8))
        b.step(5)
        st = b.stats()
    assert st["errorcode"][1] == 165
    assert st["ntime"][1] == 1  # the step that raised the code completes, then the instance stops
    assert st["ntime"][0] == 5 and st["ntime"][2] == 5
    assert st["errorcode"][0] == 0 and st["errorcode"][2] == 0


def test_configure_rejects_other_size_class():
    with ag.Batch(_inp(**SLOTS[0]), 2, ag.PREC_FP64) as b:
        other = ag.parse_bou_in(bou_text(NXM, 2 * NYM, 1, **STEP))
        with pytest.raises(ag.AfidError):
            b.configure(0, other)
        assert b.device_bytes() > 0


def test_batched_mixed_nusselt_within_half_percent():
    """Eight 2-D instances (Ra 1e6 .. 1e7, three Pr, three aspect ratios) from the seeded
    conductive state through the onset of convection, CFL-limited dt; Nu_vol averaged over the
    last third of 3000 steps, mixed against FP64, per instance."""
    cases = [dict(rayt=ra, prat=pr, ylen=asp) for ra, pr, asp in
             [(1e6, 1.0, 2.0), (2e6, 0.7, 1.0), (3e6, 4.4, 2.0), (5e6, 1.0, 4.0),
              (1e6, 0.7, 4.0), (7e6, 1.0, 1.0), (1e7, 4.4, 2.0), (4e6, 0.7, 2.0)]]
    step = dict(zlen=1.0, idtv=1, dt=1e-4, cflmax=1.2, dtmax=1e-2)
    nus = {}
    for prec in (ag.PREC_FP64, ag.PREC_MIXED):
        inp = [ag.parse_bou_in(bou_text(64, 128, 1, **dict(step, **c))) for c in cases]
        with ag.Batch(inp[0], len(cases), prec) as b:
            for s, x in enumerate(inp):
                b.configure(s, x)
                b.seed(s, 2026 + s)
            b.set_active(np.ones(len(cases), np.uint8))
            series = []
            for _ in range(300):
                b.step(10)
                series.append(b.stats()["nu_vol"])
            st = b.stats()
        assert (st["errorcode"] == 0).all() and (st["ntime"] == 3000).all()
        nus[prec] = np.array(series)
    tail = 200
    n64 = nus[ag.PREC_FP64][tail:].mean(axis=0)
    n32 = nus[ag.PREC_MIXED][tail:].mean(axis=0)
    assert (n64 > 2.0).sum() >= 4, n64
    assert np.all(np.abs(n32 - n64) / n64 < 5e-3), (n32, n64)


@pytest.mark.parametrize("precision", [ag.PREC_FP64, ag.PREC_MIXED])
def test_three_d_batch_of_one_matches_single_domain(precision):
    """A 3-D domain as a batch of one (device-side dt rule, captured step), reconfigured to a
    second Ra/Pr/aspect, against the single-domain API with the dt rule on the host."""
    shape, nsteps = (24, 32, 16), 12
    first = dict(rayt=1e5, prat=1.0, ylen=1.0, zlen=1.0)
    second = dict(rayt=4e6, prat=0.7, ylen=2.0, zlen=1.0)
    step = dict(idtv=1, dt=1e-3, cflmax=1.2, dtmax=2e-3)
    inp1 = ag.parse_bou_in(bou_text(*shape, **dict(step, **first)))
    inp2 = ag.parse_bou_in(bou_text(*shape, **dict(step, **second)))
    with ag.Batch(inp1, 1, precision) as b:
        b.seed(0, 5)  # run the first configuration, then switch: the step graph is re-captured
        b.set_active([1])
        b.step(3)
        b.configure(0, inp2)
        b.seed(0, 77)
        rng = np.random.default_rng(3)
        f = b.download(0)
        f["vy"][..., :shape[0]] = 0.05 * rng.standard_normal(f["vy"][..., :shape[0]].shape)
        b.upload(0, f["vx"], f["vy"], f["vz"], f["temp"], f["pr"])
        init = b.download(0)
        b.set_active([1])
        b.step(nsteps)
        got = b.download(0)
        st = b.stats()
    case = Case(*shape, precision=precision, **dict(step, **second))
    dt = ctypes.c_double(case.p.dt)
    with case.solver() as g:
        g.upload(*(init[k] for k in ag.Solver.FIELDS))
        for n in range(nsteps):
            cfl = g.calc_max_cfl()
            ag.lib().afid_next_dt(ctypes.byref(case.inp), n, ctypes.byref(dt), cfl, None)
            g.time_marcher(dt.value, n)
        ref = g.download()
        nu, ke, _ = g.global_quantities(case.p.prat * abs(case.p.rayt))
    nxm = shape[0]
    for k in ("vx", "vy", "vz", "temp"):
        assert np.array_equal(got[k][..., :nxm], ref[k][..., :nxm]), k
    assert st["ntime"][0] == nsteps
    assert st["nu_vol"][0] == nu and st["ke"][0] == ke


def test_step_limit_stops_slot_exactly():
    with _batch(ag.PREC_FP64) as b:
        for s in range(b.nslots):
            _perturb(b, s)
        b.set_limit(1, 7)
        b.set_active(np.ones(b.nslots, np.uint8))
        b.step(20)
        got = b.download(1)
        st = b.stats()
    with _batch(ag.PREC_FP64) as b:
        for s in range(b.nslots):
            _perturb(b, s)
        act = np.zeros(b.nslots, np.uint8)
        act[1] = 1
        b.set_active(act)
        b.step(7)
        ref = b.download(1)
        st_ref = b.stats()
    assert st["ntime"][1] == 7 and st["ntime"][0] == 20
    for k in ag.Batch.FIELDS:
        assert np.array_equal(got[k][:, :NXM], ref[k][:, :NXM]), k
    assert st["time"][1] == st_ref["time"][1]


def test_divergence_check_per_slot():
    """CheckDivergence per slot: after steps the projected fields are divergence-free to
    round-off; a slot given a divergent field reports it, the others do not."""
    with _batch(ag.PREC_FP64) as b:
        for s in range(b.nslots):
            _perturb(b, s)
        b.set_active(np.ones(b.nslots, np.uint8))
        b.step(3)
        d = b.divmax()
        assert np.all(d < 1e-9), d
        f = b.download(2)
        f["vy"][5, 3] += 1.0  # one cell, no longer divergence-free
        b.upload(2, f["vx"], f["vy"], f["vz"], f["temp"], f["pr"])
        d2 = b.divmax()
    assert d2[2] > 1.0 and np.all(np.delete(d2, 2) < 1e-9)


@pytest.mark.parametrize("precision", [ag.PREC_FP64, ag.PREC_MIXED])
def test_k1_shapes_bitwise_identical_in_batch(precision):
    """Every K1 shape a batch of the 129..256 wall-normal class can take (one or two columns per
    block, cache hints, adjacent rows) steps a batch with an idle slot to the same fields bit for
    bit, and the idle slot keeps its state; the persistent form, which holds one substep's CN
    factors per block, is refused for a batch with AFID_E_INVALID."""
    nxm, nym, nslots, idle = 200, 32, 4, 1

    def inp(**kw):
        v = dict(STEP)
        v.update(kw)
        return ag.parse_bou_in(bou_text(nxm, nym, 1, **v))

    def make():
        b = ag.Batch(inp(**SLOTS[0]), nslots, precision)
        for s in range(nslots):
            b.configure(s, inp(**SLOTS[s]))
            b.seed(s, 100 + s)
            rng = np.random.default_rng(s)
            f = b.download(s)
            for k in ("vx", "vy"):
                f[k][...] = 0.05 * rng.standard_normal(f[k].shape)
            f["vx"][:, 0] = 0.0
            f["vx"][:, nxm] = 0.0
            f["vy"][:, nxm] = 0.0
            b.upload(s, f["vx"], f["vy"], f["vz"], f["temp"], f["pr"])
        return b

    with make() as b:
        info = b.autotune()
        before = b.download(idle)
        # the forms that hold one substep's CN factors per block cannot take a batch
        usable = [v for v, (*_, us) in enumerate(info["shapes"]) if us > 0]
        for v in set(range(info["ncand"])) - set(usable):
            with pytest.raises(ag.AfidError) as e:
                b.set_k1_shape(v)
            assert e.value.status == ag.AFID_E_INVALID
    assert len(usable) >= 2
    outs = []
    for v in usable:
        with make() as b:
            b.set_k1_shape(v)
            act = np.ones(nslots, np.uint8)
            act[idle] = 0
            b.set_active(act)
            b.step(5)
            st = b.stats()
            outs.append([b.download(s) for s in range(nslots)])
        assert all(st["ntime"][s] == (0 if s == idle else 5) for s in range(nslots)), v
        assert all(st["errorcode"][s] == 0 for s in range(nslots)), v
    for v, o in zip(usable, outs):
        for k in ag.Batch.FIELDS:
            assert np.array_equal(o[idle][k], before[k]), (v, k)
            for s in range(nslots):
                assert np.array_equal(o[s][k], outs[0][s][k]), (v, s, k)
