"""Python mirror of the reference's TimeMarcher call sequence over the C ABI of ``libafidgpu.so``.

The reference drives the substep from ``main.F90:281-313``: ``CalcMaxCFL`` → dt rule →
``TimeMarcher`` → ``time += dt`` (with ``CheckDivergence`` on step 1 and every TOUT).  This
module exposes the same calls — :meth:`Solver.calc_max_cfl`, :meth:`Solver.time_marcher`,
:meth:`Solver.check_divergence` — on a GPU-resident state, plus the host set-up the reference
does in ``ReadInputFile`` / ``CreateGrid`` / ``InitPressureSolver`` / ``SetTempBCs`` through the
library's C++ host code (``include/afid_host.h``).

The CUDA library is required: importing this module without ``libafidgpu.so`` raises, and
every compute call goes to the sm_100a kernels (there is no CPU path).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libafidgpu.so")

AFID_OK = 0
AFID_E_ALLOC = 8
AFID_E_CFL = 165
AFID_E_DTMIN = 166
AFID_E_DIVERGENCE = 169
AFID_E_FFTSIZE = 444
AFID_E_SINGULAR = 601
AFID_E_TIMEOUT = 602
AFID_E_INVALID = 603
AFID_E_CUDA = 604
AFID_E_CAPACITY = 605
AFID_E_IO = 606
AFID_E_CANCELLED = 607
PREC_FP64 = 0
PREC_MIXED = 1

_dp = C.POINTER(C.c_double)


class GridT(C.Structure):
    _fields_ = [("nxm", C.c_int), ("nym", C.c_int), ("nzm", C.c_int),
                ("alx3", C.c_double), ("ylen", C.c_double), ("zlen", C.c_double)] + [
        (n, _dp) for n in ("xc", "xm", "g3rc", "udx3c", "udx3m", "ap3ck", "ac3ck", "am3ck",
                           "ap3sk", "ac3sk", "am3sk", "ap3ssk", "ac3ssk", "am3ssk",
                           "amphk", "acphk", "apphk", "ak1", "ak2")]


class ParamsT(C.Structure):
    _fields_ = [("ren", C.c_double), ("pect", C.c_double), ("byct", C.c_double),
                ("active_t", C.c_int), ("gaxis", C.c_int), ("inslws", C.c_int),
                ("inslwn", C.c_int), ("tfixs", C.c_int), ("tfixn", C.c_int),
                ("xplusu", C.c_double), ("xminusu", C.c_double), ("dpdy", C.c_double),
                ("dpdz", C.c_double), ("nsst", C.c_int), ("precision", C.c_int),
                ("tempbp", _dp), ("temptp", _dp)]


class InputT(C.Structure):
    _fields_ = [
        ("nxm", C.c_int), ("nym", C.c_int), ("nzm", C.c_int), ("nsst", C.c_int),
        ("multires", C.c_int), ("nxmr", C.c_int), ("nymr", C.c_int), ("nzmr", C.c_int),
        ("flagsal", C.c_int), ("flagpf", C.c_int), ("nread", C.c_int), ("ireset", C.c_int),
        ("ntst", C.c_int), ("walltimemax", C.c_double), ("tmax", C.c_double),
        ("tout", C.c_double), ("tframe", C.c_double), ("save_3d", C.c_double),
        ("alx3", C.c_double), ("ylen", C.c_double), ("zlen", C.c_double),
        ("istr3", C.c_int), ("str3", C.c_double), ("istr3r", C.c_int),
        ("rayt", C.c_double), ("prat", C.c_double), ("rays", C.c_double), ("pras", C.c_double),
        ("ffscales", C.c_int), ("idtv", C.c_int),
        ("dt", C.c_double), ("resid", C.c_double), ("limit_cfl", C.c_double),
        ("dtmin", C.c_double), ("dtmax", C.c_double),
        ("inslws", C.c_int), ("inslwn", C.c_int), ("tfixs", C.c_int), ("tfixn", C.c_int),
        ("sfixs", C.c_int), ("sfixn", C.c_int),
        ("active_t", C.c_int), ("active_s", C.c_int), ("gaxis", C.c_int),
        ("xplusu", C.c_double), ("xminusu", C.c_double), ("dpdy", C.c_double),
        ("dpdz", C.c_double), ("melt", C.c_int)]


class RunStatsT(C.Structure):
    _fields_ = [("steps_done", C.c_int), ("errorcode", C.c_int), ("time", C.c_double),
                ("dt", C.c_double), ("cfl", C.c_double), ("divmax", C.c_double),
                ("nu_vol", C.c_double), ("ke", C.c_double), ("seconds", C.c_double)]


class BatchStatT(C.Structure):
    _fields_ = [("ntime", C.c_int), ("errorcode", C.c_int), ("time", C.c_double),
                ("dt", C.c_double), ("cfl", C.c_double)]


TUNE_MAX = 8


class TuneInfoT(C.Structure):
    _fields_ = [("ncand", C.c_int), ("chosen", C.c_int), ("sample_columns", C.c_int),
                ("threads", C.c_int * TUNE_MAX), ("rows", C.c_int * TUNE_MAX), ("regcap", C.c_int * TUNE_MAX),
                ("policy", C.c_int * TUNE_MAX), ("us", C.c_double * TUNE_MAX), ("k4_chosen", C.c_int),
                ("k4_us", C.c_double * 2), ("fftz_chosen", C.c_int), ("fftz_us", C.c_double * 3),
                ("ify_chosen", C.c_int), ("ify_us", C.c_double * 2),
                ("div_chosen", C.c_int), ("div_us", C.c_double * 2)]

    def as_dict(self) -> dict:
        """shapes: [threads per column, rows per thread, register cap, memory policy,
        microseconds per sample]"""
        return {"ncand": self.ncand, "chosen": self.chosen, "sample_columns": self.sample_columns,
                "shapes": [[self.threads[v], self.rows[v], self.regcap[v], self.policy[v], round(self.us[v], 2)]
                           for v in range(self.ncand)],
                "k4": {"chosen": self.k4_chosen, "us": [round(x, 2) for x in self.k4_us]},
                "fft_z": {"chosen": self.fftz_chosen, "us": [round(x, 2) for x in self.fftz_us]},
                "ifft_y": {"chosen": self.ify_chosen, "us": [round(x, 2) for x in self.ify_us]},
                "div_fft_y": {"chosen": self.div_chosen, "us": [round(x, 2) for x in self.div_us]}}


class ServeConfigT(C.Structure):
    _fields_ = [("precision", C.c_int), ("hbm_budget_bytes", C.c_longlong), ("slots_per_pool", C.c_int),
                ("chunk_steps", C.c_int), ("max_cells_in_flight", C.c_longlong), ("policy", C.c_int)]


class ServeJobT(C.Structure):
    _fields_ = [("inp", InputT), ("seed", C.c_uint64), ("nsteps", C.c_int), ("tag", C.c_uint64),
                ("temp_out", C.POINTER(C.c_double))]


class ServeResultT(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("errorcode", C.c_int), ("steps_done", C.c_int),
                ("time", C.c_double), ("dt", C.c_double), ("cfl", C.c_double), ("nu_vol", C.c_double),
                ("ke", C.c_double), ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


class ServeStatusT(C.Structure):
    _fields_ = [("queued", C.c_int), ("running", C.c_int), ("pools", C.c_int),
                ("device_bytes", C.c_longlong), ("cells_in_flight", C.c_longlong),
                ("cell_steps_done", C.c_longlong), ("jobs_done", C.c_longlong),
                ("pool_failures", C.c_int), ("last_cuda_error", C.c_int)]


SERVE_FIFO, SERVE_SHORTEST_FIRST = 0, 1


class StencilT(C.Structure):
    _fields_ = [("n", C.c_int), ("start", C.POINTER(C.c_int)), ("w", C.POINTER(C.c_double))]


class SalGridT(C.Structure):
    _fields_ = [("nxmr", C.c_int), ("nymr", C.c_int), ("nzmr", C.c_int),
                ("dxr", C.c_double), ("dyr", C.c_double), ("dzr", C.c_double),
                ("pecs", C.c_double), ("bycs", C.c_double),
                ("active_s", C.c_int), ("sfixs", C.c_int), ("sfixn", C.c_int),
                ("xcr", C.POINTER(C.c_double)), ("udx3mr", C.POINTER(C.c_double)), ("g3rmr", C.POINTER(C.c_double)),
                ("ap3sskr", C.POINTER(C.c_double)), ("ac3sskr", C.POINTER(C.c_double)),
                ("am3sskr", C.POINTER(C.c_double)),
                ("salbp", C.POINTER(C.c_double)), ("saltp", C.POINTER(C.c_double)),
                ("to_ref", StencilT * 3), ("to_coarse", StencilT * 3)]


# afid_gpu_sal_profiles order (the means.h5 dataset names of CalcSalStats)
SAL_PROFILE_NAMES = ("Sbar", "Srms", "vxS", "vyS", "vzS", "chiS")

# afid_gpu_mean_profiles order (the means.h5 dataset names of CalcMeanProfiles.F90)
PROFILE_NAMES = ("Tbar", "vybar", "vzbar", "vxT", "vyT", "vzT", "Trms", "vxrms", "vyrms", "vzrms",
                 "vxvy", "vxvz", "vyvz", "chiT", "epsilon")

# Every symbol declared in include/afid_gpu.h, afid_host.h, afid_batch.h, afid_serve.h and
# afid_salinity.h
EXPORTS = [
    "afid_gpu_create", "afid_gpu_destroy", "afid_gpu_set_stream", "afid_gpu_get_stream",
    "afid_gpu_synchronize", "afid_gpu_upload", "afid_gpu_download", "afid_gpu_timemarcher",
    "afid_gpu_substep", "afid_gpu_cfl", "afid_gpu_divmax", "afid_gpu_globals",
    "afid_gpu_status_string", "afid_gpu_cuda_error", "afid_gpu_field_device_ptr",
    "afid_gpu_launch_count", "afid_gpu_profile_enable", "afid_gpu_profile_report",
    "afid_gpu_globals_noalloc",
    "afid_parse_bou_in", "afid_read_bou_in", "afid_tables_create", "afid_tables_destroy",
    "afid_tables_grid", "afid_tables_params", "afid_tables_array", "afid_philox_uniform",
    "afid_initial_temperature", "afid_next_dt", "afid_run",
    "afid_batch_create", "afid_batch_destroy", "afid_batch_set_stream", "afid_batch_configure",
    "afid_batch_seed", "afid_batch_upload", "afid_batch_download", "afid_batch_set_active",
    "afid_batch_step", "afid_batch_synchronize", "afid_batch_stats", "afid_batch_num_slots",
    "afid_batch_set_limit",
    "afid_batch_device_bytes", "afid_batch_launch_count",
    "afid_serve_create", "afid_serve_destroy", "afid_serve_submit", "afid_serve_pump", "afid_serve_poll",
    "afid_serve_cancel",
    "afid_serve_status", "afid_serve_now", "afid_serve_set_fail_test", "afid_gpu_autotune", "afid_batch_autotune", "afid_batch_set_k1_shape",
    "afid_gpu_set_k1_shape", "afid_gpu_set_k4_form", "afid_gpu_set_fftz_form", "afid_gpu_set_ify_form", "afid_gpu_set_div_form", "afid_gpu_set_wait_test", "afid_gpu_mean_profiles", "afid_batch_mean_profiles",
    "afid_batch_divmax", "afid_gpu_spectra_reset", "afid_gpu_spectra_update", "afid_gpu_spectra_read", "afid_gpu_slice",
    "afid_mgrd_create", "afid_mgrd_destroy", "afid_mgrd_view", "afid_mgrd_fast", "afid_mgrd_array",
    "afid_initial_salinity", "afid_gpu_sal_create", "afid_gpu_sal_upload", "afid_gpu_sal_download",
    "afid_gpu_sal_interpolate", "afid_gpu_sal_cfl", "afid_gpu_sal_profiles", "afid_gpu_sal_download_aux",
    "afid_gpu_dims", "afid_h5_write", "afid_h5_info", "afid_h5_read_f64", "afid_continua_master_from_input",
    "afid_write_flow_field", "afid_read_continua_master", "afid_read_flow_field", "afid_gpu_write_flow_field",
    "afid_gpu_read_flow_field", "afid_run_io", "afid_read_flow_interp", "afid_gpu_read_flow_interp",
    "afid_write_means", "afid_write_movie", "afid_write_grid_info", "afid_write_movie_mean",
    "afid_write_spectrum", "afid_gpu_write_spectra", "afid_gpu_mean_plane", "afid_gpu_sal_mean_plane",
]


H5_F64 = 1
H5_I32 = 2
H5_GROUP = 3
H5_MAX_RANK = 4


class H5DatasetT(C.Structure):
    _fields_ = [("name", C.c_char_p), ("dtype", C.c_int), ("rank", C.c_int), ("dims", C.c_int64 * H5_MAX_RANK),
                ("data", C.c_void_p)]


class ContinuaMasterT(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("ylen", C.c_double), ("zlen", C.c_double),
                ("time", C.c_double), ("istr3", C.c_int), ("str3", C.c_double), ("multires", C.c_int),
                ("nxr", C.c_int), ("nyr", C.c_int), ("nzr", C.c_int), ("istr3r", C.c_int)]


def load_library(path: str = _LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"libafidgpu.so not built ({path}); run afid-murphfi_b200/build.py")
    lib = C.CDLL(path)
    vp = C.c_void_p
    i = C.c_int
    d = C.c_double
    sig = {
        "afid_gpu_create": (i, [C.POINTER(GridT), C.POINTER(ParamsT), C.POINTER(vp)]),
        "afid_gpu_destroy": (i, [vp]),
        "afid_gpu_set_stream": (i, [vp, vp]),
        "afid_gpu_get_stream": (vp, [vp]),
        "afid_gpu_synchronize": (i, [vp]),
        "afid_gpu_upload": (i, [vp, _dp, _dp, _dp, _dp, _dp, i, i]),
        "afid_gpu_download": (i, [vp, _dp, _dp, _dp, _dp, _dp, i, i]),
        "afid_gpu_timemarcher": (i, [vp, d, i]),
        "afid_gpu_substep": (i, [vp, i, d, d, d, d, d]),
        "afid_gpu_cfl": (i, [vp, _dp]),
        "afid_gpu_divmax": (i, [vp, _dp]),
        "afid_gpu_globals": (i, [vp, d, _dp, _dp, _dp]),
        "afid_gpu_status_string": (C.c_char_p, [i]),
        "afid_gpu_cuda_error": (i, [vp]),
        "afid_gpu_field_device_ptr": (i, [vp, i, C.POINTER(vp), C.POINTER(i)]),
        "afid_gpu_launch_count": (C.c_longlong, [vp]),
        "afid_gpu_profile_enable": (i, [vp, i]),
        "afid_gpu_profile_report": (i, [vp, _dp, C.POINTER(C.c_longlong), i]),
        "afid_gpu_globals_noalloc": (i, [i, i, i, i, d, d, vp, vp, vp, vp, vp, vp, vp]),
        "afid_parse_bou_in": (i, [C.c_char_p, C.POINTER(InputT)]),
        "afid_read_bou_in": (i, [C.c_char_p, C.POINTER(InputT)]),
        "afid_tables_create": (i, [C.POINTER(InputT), i, C.POINTER(vp)]),
        "afid_tables_destroy": (None, [vp]),
        "afid_tables_grid": (C.POINTER(GridT), [vp]),
        "afid_tables_params": (C.POINTER(ParamsT), [vp]),
        "afid_tables_array": (_dp, [vp, C.c_char_p, C.POINTER(i)]),
        "afid_philox_uniform": (d, [C.c_uint64, C.c_uint64]),
        "afid_initial_temperature": (i, [vp, C.c_uint64, d, _dp, i, i]),
        "afid_next_dt": (i, [C.POINTER(InputT), i, _dp, d, _dp]),
        "afid_run": (i, [C.POINTER(InputT), i, C.c_uint64, i, i, vp, vp, C.POINTER(RunStatsT)]),
        "afid_batch_create": (i, [C.POINTER(InputT), i, i, C.POINTER(vp)]),
        "afid_batch_destroy": (i, [vp]),
        "afid_batch_set_stream": (i, [vp, vp]),
        "afid_batch_configure": (i, [vp, i, C.POINTER(InputT)]),
        "afid_batch_seed": (i, [vp, i, C.c_uint64]),
        "afid_batch_upload": (i, [vp, i, _dp, _dp, _dp, _dp, _dp, i, i]),
        "afid_batch_download": (i, [vp, i, _dp, _dp, _dp, _dp, _dp, i, i]),
        "afid_batch_set_active": (i, [vp, C.POINTER(C.c_ubyte)]),
        "afid_batch_set_limit": (i, [vp, i, i]),
        "afid_serve_create": (i, [C.POINTER(ServeConfigT), C.POINTER(vp)]),
        "afid_serve_destroy": (i, [vp]),
        "afid_serve_submit": (i, [vp, C.POINTER(ServeJobT)]),
        "afid_serve_pump": (i, [vp]),
        "afid_serve_cancel": (i, [vp, C.c_uint64]),
        "afid_serve_poll": (i, [vp, C.POINTER(ServeResultT), i, C.POINTER(i)]),
        "afid_serve_status": (i, [vp, C.POINTER(ServeStatusT)]),
        "afid_serve_set_fail_test": (i, [vp, i]),
        "afid_serve_now": (d, [vp]),
        "afid_gpu_autotune": (i, [vp, i, C.POINTER(TuneInfoT)]),
        "afid_gpu_set_k1_shape": (i, [vp, i]),
        "afid_gpu_set_k4_form": (i, [vp, i]),
        "afid_gpu_set_fftz_form": (i, [vp, i]),
        "afid_gpu_set_ify_form": (i, [vp, i]),
        "afid_gpu_set_div_form": (i, [vp, i]),
        "afid_gpu_set_wait_test": (i, [vp, C.c_longlong]),
        "afid_gpu_mean_profiles": (i, [vp, _dp]),
        "afid_gpu_spectra_reset": (i, [vp]),
        "afid_gpu_spectra_update": (i, [vp, d]),
        "afid_gpu_spectra_read": (i, [vp, i, _dp, _dp]),
        "afid_gpu_slice": (i, [vp, i, i, i, _dp]),
        "afid_batch_mean_profiles": (i, [vp, i, _dp]),
        "afid_batch_divmax": (i, [vp, _dp]),
        "afid_batch_autotune": (i, [vp, i, C.POINTER(TuneInfoT)]),
        "afid_batch_set_k1_shape": (i, [vp, i]),
        "afid_batch_step": (i, [vp, i]),
        "afid_batch_synchronize": (i, [vp]),
        "afid_batch_stats": (i, [vp, C.POINTER(BatchStatT), _dp, _dp]),
        "afid_batch_num_slots": (i, [vp]),
        "afid_batch_device_bytes": (C.c_longlong, [vp]),
        "afid_batch_launch_count": (C.c_longlong, [vp]),
        "afid_mgrd_create": (i, [vp, C.POINTER(vp)]),
        "afid_mgrd_destroy": (None, [vp]),
        "afid_mgrd_view": (C.POINTER(SalGridT), [vp]),
        "afid_mgrd_fast": (i, [vp]),
        "afid_mgrd_array": (_dp, [vp, C.c_char_p, C.POINTER(i)]),
        "afid_initial_salinity": (i, [vp, C.c_uint64, d, _dp, i, i]),
        "afid_gpu_sal_create": (i, [vp, C.POINTER(SalGridT)]),
        "afid_gpu_sal_upload": (i, [vp, _dp, i, i]),
        "afid_gpu_sal_download": (i, [vp, _dp, i, i]),
        "afid_gpu_sal_interpolate": (i, [vp]),
        "afid_gpu_sal_cfl": (i, [vp, _dp]),
        "afid_gpu_sal_profiles": (i, [vp, _dp]),
        "afid_gpu_sal_download_aux": (i, [vp, _dp, _dp, _dp, i, i, _dp, i, i]),
        "afid_gpu_dims": (i, [vp, C.POINTER(i)]),
        "afid_h5_write": (i, [C.c_char_p, i, C.POINTER(H5DatasetT)]),
        "afid_h5_info": (i, [C.c_char_p, C.c_char_p, C.POINTER(i), C.POINTER(i), C.POINTER(C.c_int64)]),
        "afid_h5_read_f64": (i, [C.c_char_p, C.c_char_p, _dp, C.c_int64]),
        "afid_continua_master_from_input": (i, [C.POINTER(InputT), d, C.POINTER(ContinuaMasterT)]),
        "afid_write_flow_field": (i, [C.c_char_p, i, d, C.POINTER(ContinuaMasterT), _dp, _dp, _dp, _dp, _dp, _dp]),
        "afid_read_continua_master": (i, [C.c_char_p, i, C.POINTER(ContinuaMasterT)]),
        "afid_read_flow_field": (i, [C.c_char_p, C.POINTER(ContinuaMasterT), _dp, _dp, _dp, _dp, _dp, _dp,
                                     C.POINTER(i), _dp]),
        "afid_gpu_write_flow_field": (i, [vp, C.c_char_p, i, d, C.POINTER(ContinuaMasterT)]),
        "afid_gpu_read_flow_field": (i, [vp, C.c_char_p, C.POINTER(ContinuaMasterT), _dp]),
        "afid_run_io": (i, [C.POINTER(InputT), i, C.c_uint64, i, i, vp, vp, C.c_char_p, C.POINTER(RunStatsT)]),
        "afid_read_flow_interp": (i, [C.c_char_p, C.POINTER(InputT), _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(i),
                                      C.POINTER(i), _dp]),
        "afid_gpu_read_flow_interp": (i, [vp, C.c_char_p, C.POINTER(InputT), _dp, C.POINTER(i)]),
        "afid_write_means": (i, [C.c_char_p, d, i, _dp, i, _dp, i, _dp]),
        "afid_write_movie": (i, [C.c_char_p, i, d, i, _dp, i, i, i, _dp, i, i, i, _dp]),
        "afid_write_movie_mean": (i, [C.c_char_p, i, d, i, _dp, i, i, i, _dp, i, i, i, _dp]),
        "afid_write_spectrum": (i, [C.c_char_p, i, i, i, _dp]),
        "afid_gpu_write_spectra": (i, [vp, C.c_char_p]),
        "afid_gpu_mean_plane": (i, [vp, i, i, _dp]),
        "afid_gpu_sal_mean_plane": (i, [vp, i, _dp]),
        "afid_write_grid_info": (i, [C.c_char_p, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = load_library()
    return _lib


class AfidError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        msg = lib().afid_gpu_status_string(status).decode()
        super().__init__(f"{what}: status {status} ({msg})")
        self.status = status


def _check(status: int, what: str) -> None:
    if status != AFID_OK:
        raise AfidError(status, what)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def parse_bou_in(text: str) -> InputT:
    inp = InputT()
    _check(lib().afid_parse_bou_in(text.encode(), C.byref(inp)), "afid_parse_bou_in")
    return inp


class Tables:
    """Host-side set-up (CreateGrid + InitPressureSolver + SetTempBCs) built by the C++ code."""

    def __init__(self, inp: InputT, precision: int = PREC_FP64):
        self.inp = inp
        self._h = C.c_void_p()
        _check(lib().afid_tables_create(C.byref(inp), precision, C.byref(self._h)), "afid_tables_create")

    def array(self, name: str) -> np.ndarray:
        n = C.c_int()
        p = lib().afid_tables_array(self._h, name.encode(), C.byref(n))
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    @property
    def grid(self) -> GridT:
        return lib().afid_tables_grid(self._h).contents

    @property
    def params(self) -> ParamsT:
        return lib().afid_tables_params(self._h).contents

    def initial_temperature(self, seed: int, eps: float = 1e-3) -> np.ndarray:
        i = self.inp
        t = np.zeros((i.nzm, i.nym, i.nxm + 1))
        _check(lib().afid_initial_temperature(self._h, seed, eps, _ptr(t), i.nxm + 1, i.nym),
               "afid_initial_temperature")
        return t

    def close(self):
        if self._h:
            lib().afid_tables_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mgrd:
    """Refined salinity grid and stencils (CreateMgrdGrid + CreateMgrdStencil) built by the C++
    host code from the coarse ``Tables`` of a bou.in with MULTIRES = FLAGSAL = 1."""

    def __init__(self, tables: Tables):
        self.tables = tables
        self._h = C.c_void_p()
        _check(lib().afid_mgrd_create(tables._h, C.byref(self._h)), "afid_mgrd_create")

    @property
    def view(self) -> SalGridT:
        return lib().afid_mgrd_view(self._h).contents

    @property
    def fast(self) -> bool:
        return bool(lib().afid_mgrd_fast(self._h))

    @property
    def shape(self):
        v = self.view
        return (v.nzmr, v.nymr, v.nxmr)

    def array(self, name: str) -> np.ndarray:
        n = C.c_int()
        p = lib().afid_mgrd_array(self._h, name.encode(), C.byref(n))
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def initial_salinity(self, seed: int, amp: float = 5e-3) -> np.ndarray:
        nz, ny, nx = self.shape
        out = np.zeros((nz, ny, nx))
        _check(lib().afid_initial_salinity(self._h, seed, amp, _ptr(out), nx, ny), "afid_initial_salinity")
        return out

    def close(self):
        if self._h:
            lib().afid_mgrd_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """GPU-resident AFiD flow + temperature state.

    Arrays cross the boundary in the reference's Fortran layout: numpy shape (nzm, nym, nx)
    C-order == Fortran (nx, nym, nzm), x fastest.  ``grid`` / ``params`` are ``GridT`` /
    ``ParamsT`` (e.g. from :class:`Tables`); the arrays they point to must outlive creation.
    """

    FIELDS = ("vx", "vy", "vz", "temp", "pr")

    def __init__(self, grid: GridT, params: ParamsT):
        self.nxm, self.nym, self.nzm = grid.nxm, grid.nym, grid.nzm
        self.nx = self.nxm + 1
        self._h = C.c_void_p()
        _check(lib().afid_gpu_create(C.byref(grid), C.byref(params), C.byref(self._h)), "afid_gpu_create")

    @property
    def shape(self):
        return (self.nzm, self.nym, self.nx)

    def _arr(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"expected shape {self.shape}, got {a.shape}")
        return a

    def upload(self, vx=None, vy=None, vz=None, temp=None, pr=None):
        arrs = [self._arr(a) for a in (vx, vy, vz, temp, pr)]
        ptrs = [(_ptr(a) if a is not None else None) for a in arrs]
        _check(lib().afid_gpu_upload(self._h, *ptrs, self.nx, self.nym), "afid_gpu_upload")

    def download(self) -> dict:
        out = {f: np.zeros(self.shape) for f in self.FIELDS}
        _check(lib().afid_gpu_download(self._h, *(_ptr(out[f]) for f in self.FIELDS), self.nx, self.nym),
               "afid_gpu_download")
        return out

    def time_marcher(self, dt: float, ntime: int = 0) -> None:
        _check(lib().afid_gpu_timemarcher(self._h, dt, ntime), "afid_gpu_timemarcher")

    def substep(self, ns: int, al: float, ga: float, ro: float, dt: float, beta: float) -> None:
        _check(lib().afid_gpu_substep(self._h, ns, al, ga, ro, dt, beta), "afid_gpu_substep")

    def calc_max_cfl(self) -> float:
        v = C.c_double()
        _check(lib().afid_gpu_cfl(self._h, C.byref(v)), "afid_gpu_cfl")
        return v.value

    def check_divergence(self) -> float:
        v = C.c_double()
        _check(lib().afid_gpu_divmax(self._h, C.byref(v)), "afid_gpu_divmax")
        return v.value

    def global_quantities(self, ra_pr: float):
        nu, ke, tm = C.c_double(), C.c_double(), C.c_double()
        _check(lib().afid_gpu_globals(self._h, ra_pr, C.byref(nu), C.byref(ke), C.byref(tm)),
               "afid_gpu_globals")
        return nu.value, ke.value, tm.value

    def synchronize(self) -> None:
        _check(lib().afid_gpu_synchronize(self._h), "afid_gpu_synchronize")

    def set_stream(self, stream_handle: int | None) -> None:
        _check(lib().afid_gpu_set_stream(self._h, C.c_void_p(stream_handle or 0)), "afid_gpu_set_stream")

    def stream(self) -> int:
        return lib().afid_gpu_get_stream(self._h) or 0

    def launch_count(self) -> int:
        return int(lib().afid_gpu_launch_count(self._h))

    PROFILE_CLASSES = ("cn_tables", "explicit_implicit", "div_fft_y", "fft_z_fwd", "tridiag_pressure",
                       "fft_z_inv", "ifft_y", "correct", "reductions", "sal_step", "sal_interp")

    def autotune(self, force: bool = False) -> dict:
        info = TuneInfoT()
        _check(lib().afid_gpu_autotune(self._h, int(force), C.byref(info)), "afid_gpu_autotune")
        return info.as_dict()

    def mean_profiles(self) -> dict:
        """CalcMeanProfiles.F90 profiles (means.h5 dataset names) from the device state."""
        out = np.zeros((len(PROFILE_NAMES), self.nxm))
        _check(lib().afid_gpu_mean_profiles(self._h, _ptr(out)), "afid_gpu_mean_profiles")
        return dict(zip(PROFILE_NAMES, out))

    def spectra_reset(self) -> None:
        _check(lib().afid_gpu_spectra_reset(self._h), "afid_gpu_spectra_reset")

    def spectra_update(self, dt: float) -> None:
        _check(lib().afid_gpu_spectra_update(self._h, dt), "afid_gpu_spectra_update")

    def spectra(self) -> dict:
        """Time-averaged spectra {vx, vy, vz, temp}: arrays (nzm, nym//2+1, nxm) (Fortran
        (nxm, nyh, nzm)), and the averaging interval under 'tav'."""
        out, tav = {}, C.c_double()
        for w, name in enumerate(("vx", "vy", "vz", "temp")):
            a = np.zeros((self.nzm, self.nym // 2 + 1, self.nxm))
            _check(lib().afid_gpu_spectra_read(self._h, w, _ptr(a), C.byref(tav)), "afid_gpu_spectra_read")
            out[name] = a
        out["tav"] = tav.value
        return out

    def mean_plane(self, which: int, axis: int) -> np.ndarray:
        """afid_gpu_mean_plane: the y-mean (axis 1, (nzm, nx)) or z-mean (axis 2, (nym, nx)) of
        vx, vy, vz or temp (which 0..3)."""
        a = np.zeros((self.nzm, self.nx) if axis == 1 else (self.nym, self.nx))
        _check(lib().afid_gpu_mean_plane(self._h, which, axis, _ptr(a)), "afid_gpu_mean_plane")
        return a

    def sal_mean_plane(self, axis: int) -> np.ndarray:
        nzmr, nymr, nxmr = self._sal_shape
        a = np.zeros((nzmr, nxmr) if axis == 1 else (nymr, nxmr))
        _check(lib().afid_gpu_sal_mean_plane(self._h, axis, _ptr(a)), "afid_gpu_sal_mean_plane")
        return a

    def write_spectra(self, directory: str) -> None:
        _check(lib().afid_gpu_write_spectra(self._h, directory.encode()), "afid_gpu_write_spectra")

    def slice(self, which: int, axis: int, index: int) -> np.ndarray:
        shape = {0: (self.nzm, self.nym), 1: (self.nzm, self.nx), 2: (self.nym, self.nx)}[axis]
        a = np.zeros(shape)
        _check(lib().afid_gpu_slice(self._h, which, axis, index, _ptr(a)), "afid_gpu_slice")
        return a

    # ---- multi-resolution salinity (include/afid_salinity.h) ----
    def sal_create(self, mgrd: "Mgrd") -> None:
        _check(lib().afid_gpu_sal_create(self._h, C.byref(mgrd.view)), "afid_gpu_sal_create")
        self._sal_shape = mgrd.shape

    def sal_upload(self, sal: np.ndarray) -> None:
        nz, ny, nx = self._sal_shape
        a = np.ascontiguousarray(sal, dtype=np.float64)
        if a.shape != (nz, ny, nx):
            raise ValueError(f"salinity shape {a.shape} != {(nz, ny, nx)}")
        _check(lib().afid_gpu_sal_upload(self._h, _ptr(a), nx, ny), "afid_gpu_sal_upload")

    def sal_download(self) -> np.ndarray:
        nz, ny, nx = self._sal_shape
        out = np.zeros((nz, ny, nx))
        _check(lib().afid_gpu_sal_download(self._h, _ptr(out), nx, ny), "afid_gpu_sal_download")
        return out

    def sal_interpolate(self) -> None:
        _check(lib().afid_gpu_sal_interpolate(self._h), "afid_gpu_sal_interpolate")

    def sal_cfl(self) -> float:
        v = C.c_double()
        _check(lib().afid_gpu_sal_cfl(self._h, C.byref(v)), "afid_gpu_sal_cfl")
        return v.value

    def sal_profiles(self) -> dict:
        nxmr = self._sal_shape[2]
        out = np.zeros(6 * nxmr)
        _check(lib().afid_gpu_sal_profiles(self._h, _ptr(out)), "afid_gpu_sal_profiles")
        return {n: out[q * nxmr:(q + 1) * nxmr].copy() for q, n in enumerate(SAL_PROFILE_NAMES)}

    def sal_aux(self) -> dict:
        """vxr (nzmr, nymr, nxmr+1), vyr / vzr (.., nxmr+1, last row unused) and salc (nzm, nym, nxm)."""
        nz, ny, nx = self._sal_shape
        nzm, nym, nxc = self.shape
        vxr, vyr, vzr = (np.zeros((nz, ny, nx + 1)) for _ in range(3))
        salc = np.zeros((nzm, nym, nxc - 1))
        _check(lib().afid_gpu_sal_download_aux(self._h, _ptr(vxr), _ptr(vyr), _ptr(vzr), nx + 1, ny, _ptr(salc),
                                               nxc - 1, nym), "afid_gpu_sal_download_aux")
        return dict(vxr=vxr, vyr=vyr[..., :nx], vzr=vzr[..., :nx], salc=salc)

    def dims(self) -> tuple:
        d = (C.c_int * 6)()
        _check(lib().afid_gpu_dims(self._h, d), "afid_gpu_dims")
        return tuple(d)

    def write_flow_field(self, directory: str, master: "ContinuaMasterT", final: bool = True,
                         save_3d: float = 1.0) -> None:
        """WriteFlowField: the resident fields (and salinity) to directory's continua files."""
        _check(lib().afid_gpu_write_flow_field(self._h, directory.encode(), int(final), save_3d, C.byref(master)),
               "afid_gpu_write_flow_field")

    def read_flow_field(self, directory: str, master: "ContinuaMasterT") -> float:
        """Same-grid restart from directory's continua files; returns the master's time."""
        t = C.c_double()
        _check(lib().afid_gpu_read_flow_field(self._h, directory.encode(), C.byref(master), C.byref(t)),
               "afid_gpu_read_flow_field")
        return t.value

    def read_flow_interp(self, directory: str, inp: "InputT") -> tuple:
        """ReadFlowInterp (either branch) onto this context; returns (time, interpolated)."""
        t, interp = C.c_double(), C.c_int()
        _check(lib().afid_gpu_read_flow_interp(self._h, directory.encode(), C.byref(inp), C.byref(t),
                                               C.byref(interp)), "afid_gpu_read_flow_interp")
        return t.value, bool(interp.value)

    def set_k1_shape(self, index: int) -> None:
        _check(lib().afid_gpu_set_k1_shape(self._h, index), "afid_gpu_set_k1_shape")

    def set_k4_form(self, form: int) -> None:
        _check(lib().afid_gpu_set_k4_form(self._h, form), "afid_gpu_set_k4_form")

    def set_fftz_form(self, form: int) -> None:
        _check(lib().afid_gpu_set_fftz_form(self._h, form), "afid_gpu_set_fftz_form")

    def set_ify_form(self, form: int) -> None:
        _check(lib().afid_gpu_set_ify_form(self._h, form), "afid_gpu_set_ify_form")

    def set_div_form(self, form: int) -> None:
        _check(lib().afid_gpu_set_div_form(self._h, form), "afid_gpu_set_div_form")

    def set_wait_test(self, polls: int) -> None:
        """Test hook: make the bounded staging wait run out after `polls` polls (0 = off)."""
        _check(lib().afid_gpu_set_wait_test(self._h, polls), "afid_gpu_set_wait_test")

    def profile(self, enable: bool = True) -> None:
        _check(lib().afid_gpu_profile_enable(self._h, int(enable)), "afid_gpu_profile_enable")

    def profile_report(self) -> dict:
        n = len(self.PROFILE_CLASSES)
        ms = (C.c_double * n)()
        cnt = (C.c_longlong * n)()
        _check(lib().afid_gpu_profile_report(self._h, ms, cnt, n), "afid_gpu_profile_report")
        return {k: (ms[i], int(cnt[i])) for i, k in enumerate(self.PROFILE_CLASSES)}

    def device_ptr(self, which: int):
        p, ld = C.c_void_p(), C.c_int()
        _check(lib().afid_gpu_field_device_ptr(self._h, which, C.byref(p), C.byref(ld)), "field_device_ptr")
        return p.value, ld.value

    def close(self):
        if self._h:
            lib().afid_gpu_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent 2-D instances of one size class advanced together (include/afid_batch.h).

    Slot state crosses the boundary as numpy (nym, nx) arrays, x fastest.  Each slot carries
    its own bou.in (Ra, Pr, YLEN, dt rule); ``step`` runs the reference's main-loop step
    (CFL, dt rule, TimeMarcher) for every active slot.
    """

    FIELDS = ("vx", "vy", "vz", "temp", "pr")

    def __init__(self, proto: InputT, nslots: int, precision: int = PREC_FP64):
        self.nxm, self.nym, self.nzm, self.nslots = proto.nxm, proto.nym, proto.nzm, nslots
        self.nx = self.nxm + 1
        self._h = C.c_void_p()
        _check(lib().afid_batch_create(C.byref(proto), nslots, precision, C.byref(self._h)),
               "afid_batch_create")

    @property
    def shape(self):
        return (self.nym, self.nx) if self.nzm == 1 else (self.nzm, self.nym, self.nx)

    def set_limit(self, slot: int, nsteps: int) -> None:
        _check(lib().afid_batch_set_limit(self._h, slot, nsteps), "afid_batch_set_limit")

    def configure(self, slot: int, inp: InputT) -> None:
        _check(lib().afid_batch_configure(self._h, slot, C.byref(inp)), "afid_batch_configure")

    def seed(self, slot: int, seed: int) -> None:
        _check(lib().afid_batch_seed(self._h, slot, seed), "afid_batch_seed")

    def upload(self, slot: int, vx=None, vy=None, vz=None, temp=None, pr=None) -> None:
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(self.shape)
                for a in (vx, vy, vz, temp, pr)]
        ptrs = [(_ptr(a) if a is not None else None) for a in arrs]
        _check(lib().afid_batch_upload(self._h, slot, *ptrs, self.nx, self.nym), "afid_batch_upload")

    def download(self, slot: int) -> dict:
        out = {f: np.zeros(self.shape) for f in self.FIELDS}
        _check(lib().afid_batch_download(self._h, slot, *(_ptr(out[f]) for f in self.FIELDS),
                                         self.nx, self.nym), "afid_batch_download")
        return out

    def set_active(self, active) -> None:
        a = np.ascontiguousarray(np.asarray(active, dtype=np.uint8).reshape(self.nslots))
        _check(lib().afid_batch_set_active(self._h, a.ctypes.data_as(C.POINTER(C.c_ubyte))),
               "afid_batch_set_active")

    def step(self, nsteps: int = 1) -> None:
        _check(lib().afid_batch_step(self._h, nsteps), "afid_batch_step")

    def synchronize(self) -> None:
        _check(lib().afid_batch_synchronize(self._h), "afid_batch_synchronize")

    def set_stream(self, stream_handle: int | None) -> None:
        _check(lib().afid_batch_set_stream(self._h, stream_handle), "afid_batch_set_stream")

    def stats(self, globals_: bool = True) -> dict:
        st = (BatchStatT * self.nslots)()
        nu = np.zeros(self.nslots)
        ke = np.zeros(self.nslots)
        _check(lib().afid_batch_stats(self._h, st, _ptr(nu) if globals_ else None,
                                      _ptr(ke) if globals_ else None), "afid_batch_stats")
        out = {k: np.array([getattr(x, k) for x in st]) for k in ("ntime", "errorcode", "time", "dt", "cfl")}
        if globals_:
            out["nu_vol"], out["ke"] = nu, ke
        return out

    def device_bytes(self) -> int:
        return int(lib().afid_batch_device_bytes(self._h))

    def divmax(self) -> np.ndarray:
        out = np.zeros(self.nslots)
        _check(lib().afid_batch_divmax(self._h, _ptr(out)), "afid_batch_divmax")
        return out

    def mean_profiles(self, slot: int) -> dict:
        out = np.zeros((len(PROFILE_NAMES), self.nxm))
        _check(lib().afid_batch_mean_profiles(self._h, slot, _ptr(out)), "afid_batch_mean_profiles")
        return dict(zip(PROFILE_NAMES, out))

    def autotune(self, force: bool = False) -> dict:
        info = TuneInfoT()
        _check(lib().afid_batch_autotune(self._h, int(force), C.byref(info)), "afid_batch_autotune")
        return info.as_dict()

    def set_k1_shape(self, index: int) -> None:
        """Use K1 shape `index` (as Solver.set_k1_shape) for this batch from now on."""
        _check(lib().afid_batch_set_k1_shape(self._h, index), "afid_batch_set_k1_shape")

    def launch_count(self) -> int:
        return int(lib().afid_batch_launch_count(self._h))

    def close(self):
        if self._h:
            lib().afid_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop for simulation jobs (include/afid_serve.h)."""

    def __init__(self, precision: int = PREC_MIXED, hbm_budget_bytes: int = 64 << 30, slots_per_pool: int = 32,
                 chunk_steps: int = 50, max_cells_in_flight: int = 0, policy: int = SERVE_FIFO):
        cfg = ServeConfigT(precision, hbm_budget_bytes, slots_per_pool, chunk_steps, max_cells_in_flight, policy)
        self._h = C.c_void_p()
        self._keep = {}
        _check(lib().afid_serve_create(C.byref(cfg), C.byref(self._h)), "afid_serve_create")

    def submit(self, inp: InputT, seed: int, nsteps: int, tag: int, temp_out: np.ndarray | None = None) -> None:
        job = ServeJobT(inp, seed, nsteps, tag, None)
        if temp_out is not None:
            assert temp_out.dtype == np.float64 and temp_out.flags.c_contiguous
            job.temp_out = _ptr(temp_out)
            self._keep[tag] = temp_out
        _check(lib().afid_serve_submit(self._h, C.byref(job)), "afid_serve_submit")

    def pump(self) -> None:
        _check(lib().afid_serve_pump(self._h), "afid_serve_pump")

    def cancel(self, tag: int) -> None:
        """afid_serve_cancel: the job comes back as a result with errorcode AFID_E_CANCELLED."""
        _check(lib().afid_serve_cancel(self._h, C.c_uint64(tag)), "afid_serve_cancel")

    def poll(self, max_results: int = 1024) -> list:
        buf = (ServeResultT * max_results)()
        n = C.c_int()
        _check(lib().afid_serve_poll(self._h, buf, max_results, C.byref(n)), "afid_serve_poll")
        out = []
        for r in buf[:n.value]:
            out.append({k: getattr(r, k) for k, _ in ServeResultT._fields_})
            self._keep.pop(r.tag, None)
        return out

    def status(self) -> dict:
        st = ServeStatusT()
        _check(lib().afid_serve_status(self._h, C.byref(st)), "afid_serve_status")
        return {k: getattr(st, k) for k, _ in ServeStatusT._fields_}

    def now(self) -> float:
        return float(lib().afid_serve_now(self._h))

    def set_fail_test(self, nth: int) -> None:
        """Test hook: the nth next chunk launch counts as failed (no CUDA call); 0 = off."""
        _check(lib().afid_serve_set_fail_test(self._h, nth), "afid_serve_set_fail_test")

    def close(self):
        if self._h:
            lib().afid_serve_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def h5_write(path: str, datasets: dict) -> None:
    """afid_h5_write: path -> array (float64 or int32, rank 1-4, C order), or None for a group;
    '/' in a path nests groups."""
    keep, sets = [], (H5DatasetT * len(datasets))()
    for i, (name, a) in enumerate(datasets.items()):
        if a is None:
            sets[i].name = name.encode()
            sets[i].dtype = H5_GROUP
            continue
        a = np.ascontiguousarray(a)
        if a.dtype not in (np.float64, np.int32):
            raise TypeError(f"{name}: dtype {a.dtype}")
        keep.append(a)
        sets[i].name = name.encode()
        sets[i].dtype = H5_F64 if a.dtype == np.float64 else H5_I32
        sets[i].rank = a.ndim
        for r in range(a.ndim):
            sets[i].dims[r] = a.shape[r]
        sets[i].data = a.ctypes.data
    _check(lib().afid_h5_write(path.encode(), len(datasets), sets), "afid_h5_write")


def h5_info(path: str, name: str) -> tuple:
    """(dtype class, shape) of one dataset."""
    dt, rk, dims = C.c_int(), C.c_int(), (C.c_int64 * H5_MAX_RANK)()
    _check(lib().afid_h5_info(path.encode(), name.encode(), C.byref(dt), C.byref(rk), dims), "afid_h5_info")
    return dt.value, tuple(dims[i] for i in range(rk.value))


def h5_read(path: str, name: str) -> np.ndarray:
    """afid_h5_read_f64: the dataset converted to float64, in its own shape."""
    _, shape = h5_info(path, name)
    out = np.empty(shape, dtype=np.float64)
    _check(lib().afid_h5_read_f64(path.encode(), name.encode(), _ptr(out), out.size), "afid_h5_read_f64")
    return out


def write_grid_info(directory: str, tables: "Tables", mgrd: "Mgrd" = None) -> None:
    """afid_write_grid_info: cordin_info.h5 of the grid (and the refined grid)."""
    _check(lib().afid_write_grid_info(directory.encode(), tables._h, mgrd._h if mgrd is not None else None),
           "afid_write_grid_info")


def write_means(directory: str, tout: float, times, profiles: np.ndarray, sal_profiles: np.ndarray = None) -> None:
    """afid_write_means: profiles (nsamples, 15, nxm) as Solver.mean_profiles stacks them,
    sal_profiles (nsamples, 6, nxmr) or None."""
    times = np.ascontiguousarray(times, dtype=np.float64)
    prof = np.ascontiguousarray(profiles, dtype=np.float64)
    ns, nq, nxm = prof.shape
    if nq != len(PROFILE_NAMES) or times.shape != (ns,):
        raise ValueError("profiles must be (nsamples, 15, nxm) with one time per sample")
    sal = None if sal_profiles is None else np.ascontiguousarray(sal_profiles, dtype=np.float64)
    nxmr = 0 if sal is None else sal.shape[2]
    _check(lib().afid_write_means(directory.encode(), tout, ns, _ptr(times), nxm, _ptr(prof), nxmr,
                                  _ptr(sal) if sal is not None else None), "afid_write_means")


def write_movie(directory: str, axis: int, tframe: float, times, planes: np.ndarray, nxm: int, nym: int,
                nzm: int, sal_planes: np.ndarray = None, refined: tuple = (0, 0, 0)) -> None:
    """afid_write_movie: planes (nframes, 4, rows, cols) in Solver.slice's layout for the axis,
    sal_planes (nframes, rows_r, cols_r) or None with refined = (nxmr, nymr, nzmr)."""
    times = np.ascontiguousarray(times, dtype=np.float64)
    pl = np.ascontiguousarray(planes, dtype=np.float64)
    sal = None if sal_planes is None else np.ascontiguousarray(sal_planes, dtype=np.float64)
    _check(lib().afid_write_movie(directory.encode(), axis, tframe, times.size, _ptr(times), nxm, nym, nzm,
                                  _ptr(pl), *refined, _ptr(sal) if sal is not None else None), "afid_write_movie")


def write_movie_mean(directory: str, axis: int, tframe: float, times, planes: np.ndarray, nxm: int, nym: int,
                     nzm: int, sal_planes: np.ndarray = None, refined: tuple = (0, 0, 0)) -> None:
    """afid_write_movie_mean: flowmov/movie_ymean.h5 (axis 1) or movie_zmean.h5 (axis 2) from
    planes (nframes, 4, rows, nx) in Solver.mean_plane's layout, sal_planes (nframes, rows_r,
    nxmr) or None."""
    times = np.ascontiguousarray(times, dtype=np.float64)
    pl = np.ascontiguousarray(planes, dtype=np.float64)
    sal = None if sal_planes is None else np.ascontiguousarray(sal_planes, dtype=np.float64)
    _check(lib().afid_write_movie_mean(directory.encode(), axis, tframe, times.size, _ptr(times), nxm, nym, nzm,
                                       _ptr(pl), *refined, _ptr(sal) if sal is not None else None),
           "afid_write_movie_mean")


def write_spectrum_file(path: str, half: np.ndarray, nym: int) -> None:
    """afid_write_spectrum: the half spectrum (nzm, nym//2 + 1, nxm) as the 'var' dataset
    (nzm, nym, nxm) of write_3D_spectrum, the rows past nym//2 at 0."""
    a = np.ascontiguousarray(half, dtype=np.float64)
    nzm, nyh, nxm = a.shape
    if nyh != nym // 2 + 1:
        raise ValueError(f"half spectrum has {nyh} rows, nym = {nym} needs {nym // 2 + 1}")
    _check(lib().afid_write_spectrum(path.encode(), nxm, nym, nzm, _ptr(a)), "afid_write_spectrum")


class Recorder:
    """The outputs the reference's main loop writes besides the restart files, for a run driven
    from Python: cordin_info.h5 at construction (WriteGridInfo), a mean-profile sample per
    ``profiles(time)`` call (CalcMeanProfiles / CalcSalStats at TOUT), the three movie cuts per
    ``frame(time)`` call (Mkmov_xcut / Mkmov_ycut / Mkmov_zcut at TFRAME, and mean_yplane /
    mean_zplane when nym > 1 and nzm > 1, main.F90:42, 340-343), and ``flush()`` writing means.h5,
    flowmov/movie_{x,y,z}cut.h5 and flowmov/movie_{y,z}mean.h5 from everything sampled so far.

    The cuts sit where the reference puts them (0-based here): x at index 0 (vx at 1; index
    nxm/2 - 1, vx max(nxm/2, 2) - 1, when RAYS and RAYT are both negative), y at nym/2, z at nzm/2;
    the refined salinity likewise on its own grid, cut on the host from a download of the field."""

    def __init__(self, solver, inp: InputT, directory: str, tables: "Tables", mgrd: "Mgrd" = None):
        self.solver, self.inp, self.dir, self.sal = solver, inp, directory, mgrd is not None
        write_grid_info(directory, tables, mgrd)
        self.ptimes, self.prof, self.salprof = [], [], []
        self.ftimes, self.planes, self.salplanes = [], {0: [], 1: [], 2: []}, {0: [], 1: [], 2: []}
        self.mean_planes = inp.nym > 1 and inp.nzm > 1          # write_mean_planes (main.F90:42)
        self.mplanes, self.salmplanes = {1: [], 2: []}, {1: [], 2: []}
        both_neg = inp.rays < 0 and inp.rayt < 0
        ic = inp.nxm // 2 if both_neg else 1                      # 1-based, MakeMovieXCut.F90
        self.xcut = (max(ic, 2) - 1, ic - 1)                       # (vx, the others)
        self.ycut, self.zcut = inp.nym // 2, inp.nzm // 2         # nym/2 + 1, nzm/2 + 1 (1-based)
        if self.sal:
            icr = inp.nxmr // 2 if both_neg else 1
            self.salcut = (icr - 1, inp.nymr // 2, inp.nzmr // 2)

    def profiles(self, time: float) -> None:
        p = self.solver.mean_profiles()
        self.ptimes.append(time)
        self.prof.append(np.stack([p[n] for n in PROFILE_NAMES]))
        if self.sal:
            q = self.solver.sal_profiles()
            self.salprof.append(np.stack([q[n] for n in SAL_PROFILE_NAMES]))

    def frame(self, time: float) -> None:
        self.ftimes.append(time)
        for axis in (0, 1, 2):
            planes = []
            for which in range(4):
                idx = (self.xcut[0] if which == 0 else self.xcut[1]) if axis == 0 else \
                    (self.ycut if axis == 1 else self.zcut)
                planes.append(self.solver.slice(which, axis, idx))
            self.planes[axis].append(np.stack(planes))
        if self.mean_planes:
            for axis in (1, 2):
                self.mplanes[axis].append(np.stack([self.solver.mean_plane(w, axis) for w in range(4)]))
                if self.sal:
                    self.salmplanes[axis].append(self.solver.sal_mean_plane(axis))
        if self.sal:
            sal = self.solver.sal_download()                       # (nzmr, nymr, nxmr)
            ix, iy, iz = self.salcut
            self.salplanes[0].append(np.ascontiguousarray(sal[:, :, ix]))
            self.salplanes[1].append(np.ascontiguousarray(sal[:, iy, :]))
            self.salplanes[2].append(np.ascontiguousarray(sal[iz, :, :]))

    def flush(self) -> None:
        inp = self.inp
        nxm = inp.nxm
        prof = np.stack(self.prof) if self.prof else np.zeros((0, len(PROFILE_NAMES), nxm))
        salprof = (np.stack(self.salprof) if self.salprof else np.zeros((0, 6, inp.nxmr))) if self.sal else None
        write_means(self.dir, inp.tout, np.array(self.ptimes, dtype=np.float64), prof, salprof)
        if not self.ftimes:
            return
        refined = (inp.nxmr, inp.nymr, inp.nzmr) if self.sal else (0, 0, 0)
        for axis in (0, 1, 2):
            sp = np.stack(self.salplanes[axis]) if self.sal else None
            write_movie(self.dir, axis, inp.tframe, np.array(self.ftimes, dtype=np.float64),
                        np.stack(self.planes[axis]), nxm, inp.nym, inp.nzm, sp, refined)
        if self.mean_planes:
            for axis in (1, 2):
                sp = np.stack(self.salmplanes[axis]) if self.sal else None
                write_movie_mean(self.dir, axis, inp.tframe, np.array(self.ftimes, dtype=np.float64),
                                 np.stack(self.mplanes[axis]), nxm, inp.nym, inp.nzm, sp, refined)


def continua_master(inp: InputT, time: float = 0.0) -> ContinuaMasterT:
    m = ContinuaMasterT()
    _check(lib().afid_continua_master_from_input(C.byref(inp), time, C.byref(m)), "afid_continua_master_from_input")
    return m


def read_continua_master(directory: str, multires: bool = False) -> ContinuaMasterT:
    m = ContinuaMasterT()
    _check(lib().afid_read_continua_master(directory.encode(), int(multires), C.byref(m)), "afid_read_continua_master")
    return m


def write_flow_field(directory: str, master: ContinuaMasterT, fields: dict, final: bool = True,
                     save_3d: float = 1.0) -> None:
    """afid_write_flow_field from packed host arrays: vx, vy, vz, temp, pr of shape (nzm, nym, nx)
    and optionally sal of shape (nzmr, nymr, nxmr)."""
    arrs = {k: (np.ascontiguousarray(v, dtype=np.float64) if v is not None else None) for k, v in fields.items()}

    def p(k):
        a = arrs.get(k)
        return _ptr(a) if a is not None else None
    _check(lib().afid_write_flow_field(directory.encode(), int(final), save_3d, C.byref(master), p("vx"), p("vy"),
                                       p("vz"), p("temp"), p("pr"), p("sal")), "afid_write_flow_field")


def read_flow_field(directory: str, current: ContinuaMasterT, with_sal: bool = False) -> dict:
    """afid_read_flow_field into packed arrays; pr is None when continua_pr.h5 is absent."""
    shape = (current.nz - 1, current.ny - 1, current.nx)
    f = {k: np.zeros(shape) for k in ("vx", "vy", "vz", "temp", "pr")}
    sal = np.zeros((current.nzr - 1, current.nyr - 1, current.nxr - 1)) if with_sal else None
    t, pr_read = C.c_double(), C.c_int()
    _check(lib().afid_read_flow_field(directory.encode(), C.byref(current), C.byref(t), _ptr(f["vx"]), _ptr(f["vy"]),
                                      _ptr(f["vz"]), _ptr(f["temp"]), _ptr(f["pr"]), C.byref(pr_read),
                                      _ptr(sal) if sal is not None else None), "afid_read_flow_field")
    if not pr_read.value:
        f["pr"] = None
    f["sal"] = sal
    f["time"] = t.value
    return f


def read_flow_interp(directory: str, inp: InputT) -> dict:
    """afid_read_flow_interp (either branch of ReadFlowInterp) for the run described by inp."""
    shape = (inp.nzm, inp.nym, inp.nxm + 1)
    f = {k: np.zeros(shape) for k in ("vx", "vy", "vz", "temp", "pr")}
    sal = np.zeros((inp.nzmr, inp.nymr, inp.nxmr)) if inp.multires else None
    t, pr_read, interp = C.c_double(), C.c_int(), C.c_int()
    _check(lib().afid_read_flow_interp(directory.encode(), C.byref(inp), C.byref(t), _ptr(f["vx"]), _ptr(f["vy"]),
                                       _ptr(f["vz"]), _ptr(f["temp"]), _ptr(f["pr"]), C.byref(pr_read),
                                       C.byref(interp), _ptr(sal) if sal is not None else None),
           "afid_read_flow_interp")
    f.update(sal=sal, time=t.value, pr_read=bool(pr_read.value), interpolated=bool(interp.value))
    return f


def grid_from_arrays(nxm, nym, nzm, alx3, ylen, zlen, arrays: dict, keep: list) -> GridT:
    """Build a GridT from named numpy tables (0-based copies of the reference arrays);
    ``keep`` collects the contiguous copies, which must outlive the solver creation."""
    g = GridT()
    g.nxm, g.nym, g.nzm = nxm, nym, nzm
    g.alx3, g.ylen, g.zlen = alx3, ylen, zlen
    for name, _ in GridT._fields_[6:]:
        a = np.ascontiguousarray(arrays[name], dtype=np.float64)
        keep.append(a)
        setattr(g, name, _ptr(a))
    return g


def params_from_values(ren, pect, byct, active_t, gaxis, inslws, inslwn, tfixs, tfixn,
                       xplusu, xminusu, dpdy, dpdz, nsst, precision, tempbp, temptp,
                       keep: list) -> ParamsT:
    p = ParamsT()
    p.ren, p.pect, p.byct = ren, pect, byct
    p.active_t, p.gaxis, p.inslws, p.inslwn, p.tfixs, p.tfixn = active_t, gaxis, inslws, inslwn, tfixs, tfixn
    p.xplusu, p.xminusu, p.dpdy, p.dpdz = xplusu, xminusu, dpdy, dpdz
    p.nsst, p.precision = nsst, precision
    for name, a in (("tempbp", tempbp), ("temptp", temptp)):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        setattr(p, name, _ptr(a))
    return p
