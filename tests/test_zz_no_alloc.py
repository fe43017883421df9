"""The allocation-free statistics entry point (afid_gpu_globals_noalloc) against the regular
afid_gpu_globals, through the C ABI.

Some callers cannot let a library allocate device memory (host codes with their own device
pool or a capped allocator, monitors attached to another program's run); this entry point
serves them from a static device array instead.  The check: on two calls in a row, on the
state of a running solver, it returns the same Nusselt number, kinetic energy and mean
temperature as the regular entry point, and the same Nusselt number and kinetic energy as the
CPU oracle's GlobalQuantities restatement stepped alongside, within the 1e-12 relative
tolerance the other statistics tests use.  This file is collected last so that a run that
stops at its first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import afid_gpu as ag
from helpers import Case
from oracle import afid_oracle as o

pytestmark = pytest.mark.gpu


def test_globals_noalloc_matches_regular_entry_point():
    import torch

    case = Case(40, 24, 8, rayt=1e6, dt=1e-3)
    s = case.oracle_state(random_velocity=0.3)
    ra_pr = case.p.prat * abs(case.p.rayt)
    g3rc = torch.tensor(case.tables.array("g3rc")[:case.p.nxm], dtype=torch.float64, device="cuda")
    out3 = torch.zeros(3, dtype=torch.float64, device="cuda")
    lib = ag.lib()
    with case.solver() as gpu:
        gpu.upload(s.vx, s.vy, s.vz, s.temp, s.pr)
        for call in range(2):
            # the temperature state alternates between two buffers each substep: fetch the
            # current device pointers before every call
            ptrs = [gpu.device_ptr(w) for w in range(4)]
            ldx = ptrs[0][1]
            gpu.synchronize()
            rc = lib.afid_gpu_globals_noalloc(case.p.nxm, case.p.nym, case.p.nzm, ldx, case.p.alx3, ra_pr,
                                              *(ctypes.c_void_p(p) for p, _ in ptrs),
                                              ctypes.c_void_p(g3rc.data_ptr()),
                                              ctypes.c_void_p(out3.data_ptr()), None)
            assert rc == ag.AFID_OK
            torch.cuda.synchronize()
            got = out3.cpu().numpy().copy()
            ref = np.array(gpu.global_quantities(ra_pr))
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0.0, err_msg=f"call {call}")
            assert got[0] == pytest.approx(o.nusselt_volume(case.g, s), rel=1e-12), call
            assert got[1] == pytest.approx(o.kinetic_energy(case.g, s), rel=1e-12), call
            gpu.time_marcher(1e-3, call)  # a different state for the second call
            o.time_marcher(case.g, s, 1e-3)


def test_globals_noalloc_rejects_bad_arguments():
    lib = ag.lib()
    ptrs = (ctypes.c_void_p(8),) * 7
    # a NaN Rayleigh-Prandtl product is refused like a negative one
    assert lib.afid_gpu_globals_noalloc(8, 4, 4, 16, 1.0, float("nan"), *ptrs, None) == ag.AFID_E_INVALID
    assert lib.afid_gpu_globals_noalloc(8, 4, 4, 16, 1.0, -1.0, *ptrs, None) == ag.AFID_E_INVALID
    assert lib.afid_gpu_globals_noalloc(8, 4, 4, 8, 1.0, 1.0, *ptrs, None) == ag.AFID_E_INVALID  # ldx < nxm+1


def test_globals_noalloc_rejects_oversized_grid():
    lib = ag.lib()
    # 512 x 512 = 262144 columns need 6 MiB of partial sums, more than the 4 MiB array
    rc = lib.afid_gpu_globals_noalloc(64, 512, 512, 72, 1.0, 1.0, *(ctypes.c_void_p(8),) * 7, None)
    assert rc == ag.AFID_E_CAPACITY
