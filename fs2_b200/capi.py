"""ctypes binding of libfs2gpu.so (include/fs2gpu.h).

The C ABI is the product's boundary; this module declares every entry point
with its argument types so that Python callers (tests, bench.py, the torch
adjoint wrapper) can call it directly.  Raises FS2GError on a non-zero
status, with fs2g_last_error()'s message.
"""
from __future__ import annotations

import ctypes as C
import os
import re

from . import LIB_PATH

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(
    __file__))), "include", "fs2gpu.h")

OK = 0
ERR = {-1: "RUNTIME", -2: "ASSERTION", -3: "IO", -4: "MEMORY", -5: "VALUE",
       -6: "FFT", -7: "CUDA", -8: "INDEX", -9: "DEVICE"}
FIELD_X, FIELD_V, FIELD_DX1, FIELD_DX2, FIELD_FORCE, FIELD_ID = range(6)
DEPOSIT_ATOMIC, DEPOSIT_DETERMINISTIC = 0, 1
FFT_AUTO, FFT_CUFFT, FFT_FUSED = 0, 1, 2
ENSEMBLE_LOOP, ENSEMBLE_GRAPH = 0, 1


class FS2GError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%s): %s" % (ERR.get(code, code), code, msg))
        self.code = code


vp = C.c_void_p
i32 = C.c_int
f32 = C.c_float
f64 = C.c_double
sz = C.c_size_t
PF = C.POINTER(C.c_float)
PD = C.POINTER(C.c_double)
PVP = C.POINTER(C.c_void_p)
PI = C.POINTER(C.c_int)

_SIGS = {
    "fs2g_version": ([], i32),
    "fs2g_last_error": ([], C.c_char_p),
    "fs2g_ctx_create": ([i32, PVP], i32),
    "fs2g_ctx_destroy": ([vp], i32),
    "fs2g_ctx_set_stream": ([vp, vp], i32),
    "fs2g_ctx_get_stream": ([vp, PVP], i32),
    "fs2g_ctx_synchronize": ([vp], i32),
    "fs2g_ctx_set_timing": ([vp, i32], i32),
    "fs2g_ctx_reset_timing": ([vp], i32),
    "fs2g_ctx_get_timing": ([vp, PD, C.POINTER(C.c_long), i32], i32),
    "fs2g_stage_count": ([], i32),
    "fs2g_stage_name": ([i32], C.c_char_p),
    "fs2g_ctx_kernel_launches": ([vp, C.POINTER(C.c_long)], i32),
    "fs2g_cosmology_init": ([f64], i32),
    "fs2g_cosmology_omega_m": ([PD], i32),
    "fs2g_cosmology_D_growth": ([f64, PD], i32),
    "fs2g_cosmology_D2_growth": ([f64, f64, PD], i32),
    "fs2g_cosmology_Dv_growth": ([f64, f64, PD], i32),
    "fs2g_cosmology_D2v_growth": ([f64, f64, PD], i32),
    "fs2g_cosmology_f_growth_rate": ([f64, PD], i32),
    "fs2g_cosmology_hubble_function": ([f64, PD], i32),
    "fs2g_power_alloc": ([C.c_char_p, PVP], i32),
    "fs2g_power_from_table": ([PD, PD, i32, PVP], i32),
    "fs2g_power_free": ([vp], i32),
    "fs2g_power_n": ([vp, C.POINTER(C.c_int)], i32),
    "fs2g_power_i": ([vp, i32, PD, PD], i32),
    "fs2g_power_P": ([vp, f64, PD], i32),
    "fs2g_power_sigma": ([vp, f64, PD], i32),
    "fs2g_particles_alloc": ([vp, sz, f64, PVP], i32),
    "fs2g_particles_free": ([vp], i32),
    "fs2g_particles_len": ([vp, C.POINTER(C.c_size_t)], i32),
    "fs2g_particles_np_allocated": ([vp, C.POINTER(C.c_size_t)], i32),
    "fs2g_particles_np_total": ([vp, C.POINTER(C.c_uint64)], i32),
    "fs2g_particles_update_np_total": ([vp], i32),
    "fs2g_particles_boxsize": ([vp, PD], i32),
    "fs2g_particles_get_a": ([vp, PD, PD, PD], i32),
    "fs2g_particles_set_a": ([vp, f64, f64, f64], i32),
    "fs2g_particles_set_np": ([vp, sz], i32),
    "fs2g_particles_append": ([vp, PD, sz, C.c_ssize_t, C.c_ssize_t], i32),
    "fs2g_particles_clear": ([vp], i32),
    "fs2g_particles_periodic_wrapup": ([vp], i32),
    "fs2g_particles_copy_out": ([vp, i32, vp, sz, sz], i32),
    "fs2g_particles_copy_in": ([vp, i32, vp, sz, sz], i32),
    "fs2g_particles_device_field": ([vp, i32, PVP, C.POINTER(C.c_size_t)], i32),
    "fs2g_cola_velocity": ([vp, vp, PF], i32),
    "fs2g_pm_init": ([vp, i32, f64, f64], i32),
    "fs2g_pm_free": ([vp], i32),
    "fs2g_pm_send_positions": ([vp, vp], i32),
    "fs2g_pm_compute_density": ([vp, vp], i32),
    "fs2g_pm_check_total_density": ([vp], i32),
    "fs2g_pm_compute_force": ([vp, vp], i32),
    "fs2g_pm_get_forces": ([vp, vp], i32),
    "fs2g_pm_force": ([vp, vp], i32),
    "fs2g_pm_set_deposit_mode": ([vp, i32], i32),
    "fs2g_pm_set_bin_tile": ([vp, i32], i32),
    "fs2g_pm_get_bin_tile": ([vp, PI, PI, PI, PI], i32),
    "fs2g_pm_get_bin_pass": ([vp, PI], i32),
    "fs2g_pm_set_check": ([vp, i32], i32),
    "fs2g_pm_status": ([vp, C.POINTER(C.c_int)], i32),
    "fs2g_pm_set_fft_engine": ([vp, i32], i32),
    "fs2g_pm_set_keep_delta_k": ([vp, i32], i32),
    "fs2g_pm_fft_engine": ([vp, C.POINTER(C.c_int)], i32),
    "fs2g_pm_set_fft_tile": ([vp, i32], i32),
    "fs2g_pm_nc": ([vp, C.POINTER(C.c_int)], i32),
    "fs2g_pm_fft": ([vp, PVP], i32),
    "fs2g_pm_delta_k_copy_out": ([vp, PF], i32),
    "fs2g_pm_force_mesh_copy_out": ([vp, i32, PF], i32),
    "fs2g_cola_kick": ([vp, vp, f64], i32),
    "fs2g_cola_drift": ([vp, vp, f64], i32),
    "fs2g_cola_kick_drift": ([vp, vp, f64, f64], i32),
    "fs2g_cola_kick_coef": ([f64, f64, f64, PD, PF, PF, PF], i32),
    "fs2g_cola_drift_coef": ([f64, f64, f64, PD, PF, PF], i32),
    "fs2g_cola_step": ([vp, vp, f64, f64], i32),
    "fs2g_lpt": ([vp, i32, f64, f64, C.c_ulong, vp, C.c_char_p, PVP], i32),
    "fs2g_lpt_from_draws": ([vp, i32, f64, f64, PD, PD, vp, C.c_char_p, PVP],
                            i32),
    "fs2g_lpt_from_delta_k": ([vp, i32, f64, f64, PF, C.c_char_p, PVP], i32),
    "fs2g_lpt_draws": ([vp, i32, C.c_ulong, PD, PD], i32),
    "fs2g_lpt_set_offset": ([f64], i32),
    "fs2g_lpt_set_zeldovich_force": ([vp, vp, f64], i32),
    "fs2g_fft_alloc": ([vp, i32, PVP], i32),
    "fs2g_fft_free": ([vp], i32),
    "fs2g_fft_nc": ([vp, C.POINTER(C.c_int)], i32),
    "fs2g_fft_set_test_data": ([vp], i32),
    "fs2g_fft_fx_copy_out": ([vp, PF], i32),
    "fs2g_diff_create": ([vp, i32, i32, f64, vp, f64, i32, PD, PD, PVP], i32),
    "fs2g_diff_free": ([vp], i32),
    "fs2g_diff_forward": ([vp, vp, vp], i32),
    "fs2g_diff_backward": ([vp, vp, vp], i32),
    "fs2g_diff_particles": ([vp, PVP], i32),
    "fs2g_leapfrog_initial_velocity": ([vp, vp, f64], i32),
    "fs2g_leapfrog_kick": ([vp, vp, f64], i32),
    "fs2g_leapfrog_drift": ([vp, vp, f64], i32),
    "fs2g_leapfrog_coef": ([f64, f64, f64, f64, PF, PD], i32),
    "fs2g_ensemble_create": ([vp, i32, PI, PI, PD, vp, f64, i32, PD, PD, i32,
                              PVP], i32),
    "fs2g_ensemble_free": ([vp], i32),
    "fs2g_ensemble_size": ([vp, PI], i32),
    "fs2g_ensemble_member": ([vp, i32, PVP, PVP, PVP, PVP, PI, PI], i32),
    "fs2g_ensemble_tuning": ([vp, i32, PI, PI, PD], i32),
    "fs2g_ensemble_forward_member": ([vp, i32], i32),
    "fs2g_ensemble_run": ([vp, i32], i32),
    "fs2g_ensemble_losses": ([vp, PD], i32),
    "fs2g_ensemble_graph_kernels": ([vp, C.POINTER(C.c_long)], i32),
    "fs2g_cic_density_noalloc": ([vp, vp, vp, sz, vp, i32, f64, f64, vp],
                                 i32),
}

# exported for tests and profiler captures, not part of include/fs2gpu.h
# (declared in fs2_b200/csrc/probe.h)
_INTERNAL_SIGS = {
    "fs2g_fused_pass_probe": ([i32, i32, i32, PD], i32),
}

_lib = None


def header_functions(path: str = HEADER):
    """Names of the functions include/fs2gpu.h declares."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fs2g_\w+)\s*\(", text)))


def lib(path: str = LIB_PATH):
    """The loaded library with argument types set (loads once)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError("libfs2gpu.so is not built (%s); run "
                              "python -m fs2_b200.build" % path)
        L = C.CDLL(path)
        for name, (args, res) in list(_SIGS.items()) + list(
                _INTERNAL_SIGS.items()):
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def last_error() -> str:
    return (lib().fs2g_last_error() or b"").decode()


def check(rc: int):
    if rc != OK:
        raise FS2GError(rc, last_error())
    return rc


def call(name: str, *args):
    return check(getattr(lib(), name)(*args))


def ptr(a):
    """ctypes void pointer to a numpy array's data."""
    return C.c_void_p(a.ctypes.data)


def fptr(a):
    return a.ctypes.data_as(PF)


def dptr(a):
    return a.ctypes.data_as(PD)
