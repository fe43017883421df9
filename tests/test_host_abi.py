"""CPU-only checks of the C ABI library: it loads, exports every symbol that include/*.h
declares, and its host-side set-up (bou.in reader, CreateGrid port, Philox IC, dt rule) agrees
with the oracle.  No CUDA call is made here."""
import ctypes
import os
import re

import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case, bou_text
from oracle import afid_oracle as o
from oracle.philox import uniform_from_counter

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in ("afid_gpu.h", "afid_host.h", "afid_batch.h", "afid_serve.h", "afid_salinity.h", "afid_continua.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(afid_\w+)\s*\(", text))
    return {n for n in names if not n.endswith("_t")}


def test_library_exports_every_declared_symbol():
    lib = ag.lib()
    declared = _declared_functions()
    assert declared, "no declarations parsed"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert declared <= set(ag.EXPORTS)


def test_tuning_setters_refuse_null_handles():
    """The autotuner overrides check their handle before any CUDA call (no GPU needed)."""
    lib = ag.lib()
    for fn in ("afid_gpu_set_k1_shape", "afid_gpu_set_k4_form", "afid_gpu_set_fftz_form", "afid_gpu_set_ify_form",
               "afid_gpu_set_div_form", "afid_batch_set_k1_shape"):
        assert getattr(lib, fn)(None, 0) == ag.AFID_E_INVALID, fn
    assert lib.afid_gpu_autotune(None, 0, None) == ag.AFID_E_INVALID
    assert lib.afid_batch_autotune(None, 0, None) == ag.AFID_E_INVALID


def test_status_strings():
    for s in (0, 8, 165, 166, 169, 444, 601, 602, 603, 604, 605, 606, 607):
        assert ag.lib().afid_gpu_status_string(s).decode() != "unknown status"


@pytest.mark.parametrize("kw", [dict(istr3=4, str3=2.0), dict(istr3=0), dict(istr3=6, str3=4.0),
                                dict(istr3=7, str3=3.0), dict(istr3=1, str3=1.5),
                                dict(istr3=2), dict(istr3=3)])
def test_tables_match_oracle_grid(kw):
    case = Case(48, 24, 12, ylen=2.0, zlen=0.5, **kw)
    g = case.g
    for name in ("xc", "xm", "g3rc", "udx3c", "udx3m", "ap3ck", "ac3ck", "am3ck", "ap3sk", "ac3sk",
                 "am3sk", "ap3ssk", "ac3ssk", "am3ssk", "amphk", "acphk", "apphk", "ak1", "ak2"):
        a = case.tables.array(name)
        ref = getattr(g, name)
        n = min(a.size, ref.size)
        np.testing.assert_allclose(a[:n], ref[:n], rtol=1e-13, atol=1e-13 * np.abs(ref).max(),
                                   err_msg=name)
    prm = case.tables.params
    assert prm.ren == pytest.approx(g.ren, rel=1e-15)
    assert prm.pect == pytest.approx(g.pect, rel=1e-15)


def test_bou_in_parse_matches_oracle():
    text = bou_text(64, 32, 16, rayt=1e9, prat=0.7, idtv=1, dt=1e-4, cflmax=1.2, dtmax=1e-2,
                    xplusu=0.25, gaxis=1)
    inp = ag.parse_bou_in(text)
    p = o.parse_bou_in(text)
    assert (inp.nxm, inp.nym, inp.nzm, inp.nsst) == (p.nxm, p.nym, p.nzm, p.nsst)
    assert inp.rayt == p.rayt and inp.prat == p.prat and inp.dt == p.dt
    assert inp.limit_cfl == p.limit_cfl and inp.dtmax == p.dtmax and inp.xplusu == p.xplusu


def test_reference_example_bou_in_parses():
    """A bou.in in the reference's own layout (examples/*/bou.in shape)."""
    text = bou_text(128, 256, 1, ylen=2.0, zlen=0.01, dt=5e-4, dtmax=5e-4, cflmax=1.2, rayt=1e8,
                    ntst=999)
    inp = ag.parse_bou_in(text)
    assert inp.ntst == 999 and inp.zlen == 0.01 and inp.nzm == 1


def test_bad_bou_in_rejected():
    with pytest.raises(ag.AfidError) as e:
        ag.parse_bou_in("garbage\n")
    assert e.value.status == ag.AFID_E_INVALID


def test_philox_c_matches_numpy():
    ns = np.array([0, 1, 2, 12345, 2**32 + 7, 2**40 + 3], dtype=np.uint64)
    for seed in (0, 1234, 20261203, 2**33 + 5):
        ref = uniform_from_counter(ns, seed)
        got = np.array([ag.lib().afid_philox_uniform(seed, int(n)) for n in ns])
        np.testing.assert_array_equal(got, ref)


def test_initial_temperature_matches_oracle():
    case = Case(32, 16, 8)
    t = case.tables.initial_temperature(777)
    s = o.initial_state(case.g, 777)
    np.testing.assert_allclose(t[..., :32], s.temp[..., :32], rtol=0, atol=1e-15)


@pytest.mark.parametrize("idtv,ntime,cflm", [(1, 0, 3.0), (1, 2, 3.0), (1, 2, 1e-9), (1, 3, 1e3),
                                             (0, 0, 100.0), (0, 5, 2e4)])
def test_next_dt_matches_oracle(idtv, ntime, cflm):
    text = bou_text(16, 8, 4, idtv=idtv, dt=1e-3, cflmax=1.2, dtmax=5e-3)
    inp = ag.parse_bou_in(text)
    inp.dtmin = 1e-3 if cflm > 100 and idtv == 1 else inp.dtmin
    p = o.parse_bou_in(text)
    p.dtmin = inp.dtmin
    dt = ctypes.c_double(1e-3)
    rep = ctypes.c_double()
    err = ag.lib().afid_next_dt(ctypes.byref(inp), ntime, ctypes.byref(dt), cflm, ctypes.byref(rep))
    dto, erro, repo = o.next_dt(p, ntime, 1e-3, cflm)
    assert err == erro
    assert dt.value == dto
    assert rep.value == repo


def test_tables_refuse_absurd_sizes():
    """Sizes far beyond what one GPU can hold are input errors answered with AFID_E_INVALID, not
    host allocations that exhaust memory."""
    import ctypes
    for dims in ((2_000_000_000, 8, 8), (64, 2_000_000_000, 8), (64, 64, 2_000_000_000), (64, 30000, 30000),
                 (-5, 8, 8), (64, 0, 8)):
        inp = ag.parse_bou_in(bou_text(16, 12, 8))
        inp.nxm, inp.nym, inp.nzm = dims
        t = ctypes.c_void_p()
        assert ag.lib().afid_tables_create(ctypes.byref(inp), 0, ctypes.byref(t)) == ag.AFID_E_INVALID, dims
        assert not t.value


def test_next_dt_refuses_nan_cfl():
    """A NaN CFL maximum (a blown-up field) is never a valid step: 166 with variable dt, 165 with
    fixed dt.  Finite values follow main.F90:287-302 (test_next_dt_matches_oracle)."""
    for idtv, want in ((1, ag.AFID_E_DTMIN), (0, ag.AFID_E_CFL)):
        inp = ag.parse_bou_in(bou_text(16, 8, 4, idtv=idtv, dt=1e-3, cflmax=1.2))
        dtc = ctypes.c_double(1e-3)
        assert ag.lib().afid_next_dt(ctypes.byref(inp), 5, ctypes.byref(dtc), float("nan"), None) == want


def test_serve_refuses_oversized_job_at_submit_and_cancels_queued_job():
    """Host side of the request loop (no pump, so no device work): a job whose pool cannot fit
    the budget is refused by afid_serve_submit itself; a queued job cancelled by its tag comes
    back from afid_serve_poll with AFID_E_CANCELLED and no steps; an unknown tag is an error."""
    small = ag.parse_bou_in(bou_text(16, 32, 1))
    big = ag.parse_bou_in(bou_text(256, 512, 1))
    # 32 slots of 257x512 FP64 cells need ~400 MB of state arrays; a 64 MB budget cannot hold them
    with ag.Server(ag.PREC_FP64, hbm_budget_bytes=64 << 20, slots_per_pool=32) as srv:
        with pytest.raises(ag.AfidError) as e:
            srv.submit(big, 1, 10, 1)
        assert e.value.status == ag.AFID_E_CAPACITY
        srv.submit(small, 2, 10, 2)
        srv.submit(small, 3, 10, 3)
        assert srv.status()["queued"] == 2
        srv.cancel(2)
        with pytest.raises(ag.AfidError) as e:
            srv.cancel(2)
        assert e.value.status == ag.AFID_E_INVALID
        st = srv.status()
        assert st["queued"] == 1 and st["running"] == 0
        res = srv.poll()
    assert len(res) == 1 and res[0]["tag"] == 2
    assert res[0]["errorcode"] == ag.AFID_E_CANCELLED and res[0]["steps_done"] == 0
