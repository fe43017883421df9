"""Served jobs (include/afid_serve.h).

Gates:
- alone == in-mix: a job's Nu, KE, simulated time and final temperature are bitwise identical
  whether it ran alone on the server or joined pools mid-run among jobs of its own and other
  size classes (2-D and 3-D);
- every job stops at exactly its requested step count;
- admission by device-memory footprint: with room for one pool, jobs of a second class wait
  for the first class's pool to drain and be released; a job larger than the budget is refused
  at submit with AFID_E_CAPACITY; shortest-first ordering under a cells-in-flight cap;
- cancellation: a queued job leaves the queue, a running job leaves its pool at the end of the
  chunk, both come back with AFID_E_CANCELLED, and the other jobs' results do not change.
"""
import numpy as np
import pytest

import afid_gpu as ag
from helpers import bou_text

pytestmark = pytest.mark.gpu

STEP = dict(idtv=1, dt=1e-3, cflmax=1.2, dtmax=2e-3)


def _inp(nxm, nym, nzm=1, **kw):
    v = dict(STEP, rayt=1e6, prat=1.0, ylen=2.0, zlen=1.0)
    v.update(kw)
    return ag.parse_bou_in(bou_text(nxm, nym, nzm, **v))


def _run_to_completion(srv, expect, max_pumps=10000):
    got = {}
    for _ in range(max_pumps):
        srv.pump()
        for r in srv.poll():
            got[r["tag"]] = r
        if len(got) >= expect:
            return got
    raise AssertionError(f"only {len(got)} of {expect} jobs completed")


@pytest.mark.parametrize("precision", [ag.PREC_FP64, ag.PREC_MIXED])
def test_alone_equals_in_mix(precision):
    target = dict(inp=_inp(32, 64, rayt=3e6, prat=0.7), seed=11, nsteps=37)
    t_alone = np.zeros((1, 64, 33))
    with ag.Server(precision, slots_per_pool=4, chunk_steps=8) as srv:
        srv.submit(target["inp"], target["seed"], target["nsteps"], 1, t_alone)
        alone = _run_to_completion(srv, 1)[1]
    t_mix = np.zeros((1, 64, 33))
    others = [(_inp(32, 64, rayt=1e7), 21, 50), (_inp(32, 64, prat=4.4, ylen=1.0), 22, 13),
              (_inp(16, 32, rayt=2e5), 23, 40), (_inp(16, 32, 8, rayt=1e5, ylen=1.0), 24, 20),
              (_inp(32, 64, rayt=5e5), 25, 60), (_inp(32, 64), 26, 9)]
    with ag.Server(precision, slots_per_pool=4, chunk_steps=8) as srv:
        for k, (inp, seed, n) in enumerate(others[:3]):
            srv.submit(inp, seed, n, 100 + k)
        srv.pump()
        srv.pump()  # the target joins pools that are already 16 steps in
        srv.submit(target["inp"], target["seed"], target["nsteps"], 1, t_mix)
        for k, (inp, seed, n) in enumerate(others[3:]):
            srv.submit(inp, seed, n, 103 + k)
        res = _run_to_completion(srv, 1 + len(others))
    mixed = res[1]
    for k in ("nu_vol", "ke", "time", "dt", "cfl", "steps_done", "errorcode"):
        assert mixed[k] == alone[k], k
    assert np.array_equal(t_mix, t_alone)
    assert alone["steps_done"] == target["nsteps"]
    for k, (_, _, n) in enumerate(others):
        assert res[100 + k]["steps_done"] == n and res[100 + k]["errorcode"] == 0


def test_job_matches_batch_run():
    inp = _inp(32, 64, rayt=2e6)
    with ag.Server(ag.PREC_FP64, slots_per_pool=2, chunk_steps=7) as srv:
        srv.submit(inp, 5, 30, 7)
        r = _run_to_completion(srv, 1)[7]
    with ag.Batch(inp, 1, ag.PREC_FP64) as b:
        b.seed(0, 5)
        b.set_active([1])
        b.step(30)
        st = b.stats()
    assert r["steps_done"] == 30
    assert r["nu_vol"] == st["nu_vol"][0] and r["time"] == st["time"][0]


def test_admission_by_footprint():
    a, b = _inp(32, 64), _inp(16, 32)
    with ag.Batch(a, 2, ag.PREC_MIXED) as pa, ag.Batch(b, 2, ag.PREC_MIXED) as pb:
        bytes_a, bytes_b = pa.device_bytes(), pb.device_bytes()
    # room for a pool of either class, not for both
    budget = bytes_a + bytes_b // 2
    with ag.Server(ag.PREC_MIXED, hbm_budget_bytes=budget, slots_per_pool=2, chunk_steps=5) as srv:
        for k in range(3):
            srv.submit(a, k, 10 + 5 * k, k)
        srv.submit(b, 9, 10, 9)
        srv.pump()
        st = srv.status()
        assert st["pools"] == 1 and st["running"] == 2 and st["queued"] == 2
        res = _run_to_completion(srv, 4)
        assert all(res[k]["errorcode"] == 0 for k in (0, 1, 2, 9))
        # FIFO: the small-class job could only start after the large-class pool drained
        assert res[9]["t_admit"] >= max(res[k]["t_done"] for k in (0, 1, 2)) - 1e-9
        assert srv.status()["device_bytes"] <= budget
    with ag.Server(ag.PREC_MIXED, hbm_budget_bytes=4096, slots_per_pool=2) as srv:
        with pytest.raises(ag.AfidError) as e:      # larger than the whole budget: refused at submit
            srv.submit(a, 1, 10, 1)
        assert e.value.status == ag.AFID_E_CAPACITY
        assert srv.status()["queued"] == 0


def test_shortest_first_under_cell_cap():
    inp = _inp(16, 32)
    cells = 16 * 32
    with ag.Server(ag.PREC_FP64, slots_per_pool=4, chunk_steps=5, max_cells_in_flight=cells,
                   policy=ag.SERVE_SHORTEST_FIRST) as srv:
        for tag, n in ((1, 40), (2, 10), (3, 25)):
            srv.submit(inp, tag, n, tag)
        res = _run_to_completion(srv, 3)
    order = sorted(res, key=lambda t: res[t]["t_done"])
    assert order == [2, 3, 1]


def test_cancel_queued_and_running_jobs():
    inp = _inp(32, 64, rayt=2e6)
    with ag.Server(ag.PREC_FP64, slots_per_pool=2, chunk_steps=6) as srv:
        srv.submit(inp, 2, 30, 2)
        alone = _run_to_completion(srv, 1)[2]
    # room for two jobs at a time (cells in flight), so jobs 3 and 4 wait in the queue
    with ag.Server(ag.PREC_FP64, slots_per_pool=2, chunk_steps=6, policy=ag.SERVE_FIFO,
                   max_cells_in_flight=2 * 32 * 64) as srv:
        for tag in (1, 2, 3, 4):
            srv.submit(inp, tag, 30, tag)
        srv.pump()                       # jobs 1 and 2 run, 3 and 4 wait
        st = srv.status()
        assert st["running"] == 2 and st["queued"] == 2
        srv.cancel(3)                    # queued: leaves at once
        srv.cancel(1)                    # running: leaves at the end of its chunk
        with pytest.raises(ag.AfidError) as e:
            srv.cancel(99)
        assert e.value.status == ag.AFID_E_INVALID
        res = _run_to_completion(srv, 4)
    assert res[3]["errorcode"] == ag.AFID_E_CANCELLED and res[3]["steps_done"] == 0
    assert res[1]["errorcode"] == ag.AFID_E_CANCELLED and 0 < res[1]["steps_done"] < 30
    for tag in (2, 4):
        assert res[tag]["errorcode"] == 0 and res[tag]["steps_done"] == 30
    for k in ("nu_vol", "ke", "time", "dt"):
        assert res[2][k] == alone[k], k


def test_failing_pool_is_taken_out_alone():
    """A pool whose chunk launch fails (injected on the host: no CUDA call is made, no GPU
    fault) is taken out by itself: its job comes back with AFID_E_CUDA and steps_done 0, the
    job of the other pool completes with the same result as on a server without the failure,
    and a later job of the failed pool's class gets a new pool and completes."""
    a = (_inp(32, 64, rayt=3e6), 31, 24)
    b = (_inp(16, 32, rayt=2e5), 32, 40)
    with ag.Server(ag.PREC_FP64, slots_per_pool=4, chunk_steps=8) as srv:
        srv.submit(b[0], b[1], b[2], 2)
        ref = _run_to_completion(srv, 1)[2]
    with ag.Server(ag.PREC_FP64, slots_per_pool=4, chunk_steps=8) as srv:
        srv.submit(a[0], a[1], a[2], 1)   # admitted first: its pool launches first and fails
        srv.submit(b[0], b[1], b[2], 2)
        srv.set_fail_test(1)
        got = _run_to_completion(srv, 2)
        st = srv.status()
        assert st["pool_failures"] == 1 and st["last_cuda_error"] == 0   # no CUDA error behind it
        srv.submit(a[0], a[1], a[2], 3)
        got.update(_run_to_completion(srv, 1))
    assert got[1]["errorcode"] == ag.AFID_E_CUDA and got[1]["steps_done"] == 0
    for k in ("errorcode", "steps_done", "nu_vol", "ke", "time", "dt"):
        assert got[2][k] == ref[k], k
    assert got[3]["errorcode"] == 0 and got[3]["steps_done"] == a[2]
