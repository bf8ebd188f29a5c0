"""ctypes binding of libespecgpu.so (the C-ABI declared in include/espec_gpu.h).

There is no CPU fallback: if the library or a CUDA device is missing every
entry point raises EspecError.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libespecgpu.so")

OK, EINVAL, ECUDA, ENOMEM = 0, -1, -2, -3
FP64, MIXED = 0, 1
ABS_NONE, ABS_VOPTIC, ABS_SMOOTHW = 0, 1, 2
Q_SPO_INPLACE = 1
Q_SOD_SMOOTHW = 2
Q_SIL_INPLACE = 4
Q_FFTNT_SP = 8
Q_DIGT_ND = 16
Q_PSOD_COPY = 32
PULSE_NONE, PULSE_GAUS, PULSE_GGAUS, PULSE_SIN2 = 0, 1, 2, 3
SPO, SOD, SIL, PSOD = 0, 1, 2, 3
MEM_HOST, MEM_DEVICE, MEM_HOST_ASYNC = 0, 1, 2
LAUNCH_CLASSES, LAUNCH_PERSISTENT = 0, 1
VARIANT_TC = 5
SHFS = 2.4188843243e-2

# every symbol the header declares (checked by the CPU test suite)
EXPORTS = [
    "espec_last_error", "espec_version", "espec_device_ok", "espec_spo_create", "espec_spo_load",
    "espec_spo_run", "espec_spo_results", "espec_spo_device_c", "espec_spo_npoints",
    "espec_spo_destroy", "espec_spo_set_variant", "espec_spo_variant_count",
    "espec_spo_run_static", "espec_spo_set_launch", "espec_spo_set_item_cost", "espec_prop_nonfinite",
    "espec_spo_tc_status",
    "espec_prop_create", "espec_prop_previous", "espec_prop_continue",
    "espec_prop_energies", "espec_format_crl_row", "pspofft_", "psodfft_", "espec_grid_create",
    "espec_grid_load", "espec_grid_run", "espec_grid_continue", "espec_grid_results",
    "espec_grid_energies", "espec_grid_npoints", "espec_grid_destroy", "espec_grid_basis",
    "espec_grid_previous", "espec_grid_energies_at", "espec_grid_set_pulse", "espec_pulse_field",
    "espec_ppsod_field", "espec_pplnz_field", "plnz_", "psod_", "ppsod_", "pplnz_",
    "espec_grid_project", "espec_run_deck", "espec_run_scan", "espec_spectrum_dev",
    "espec_spectrum_work_bytes", "hwhm_", "spectrumtd_", "espec_eig_solve_dev",
    "espec_eig_lcg_start", "espec_eig_morse2d", "espec_gemm_f64", "espec_gemm_f32",
    "espec_gemm_bf16", "espec_gemm_bf16_status", "espec_mlp_bias_gelu", "espec_mlp_gelu_back",
    "espec_to_bf16", "espec_mlp_adam_bf16", "espec_mlp_colsum", "espec_mlp_mse", "espec_sep_basis",
    "espec_convert", "espec_spond_create", "espec_spond_load", "espec_spond_run",
    "espec_spond_results", "espec_spond_destroy", "espec_spond_continue", "espec_spond_energies",
    "espec_spond_create_method", "espec_spond_previous",
    "espec_set_wait_limit", "espec_selftest_short_arrivals", "espec_selftest_mbar_wait",
    "espec_grid_set_ctas",
    "espec_pot_kind", "espec_gvpot_1d", "espec_gvpot_nd",
]


class EspecError(RuntimeError):
    pass


_lib = None


def load():
    """Load the in-tree library (building it first if sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _b
        _b.build()
    lib = C.CDLL(LIB_PATH)
    d, i, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
    lib.espec_last_error.restype = C.c_char_p
    lib.espec_version.restype = C.c_char_p
    lib.espec_device_ok.restype = C.c_int
    lib.espec_spo_create.argtypes = [C.POINTER(vp), C.c_int, i, d, d, C.c_double, C.c_int,
                                     C.c_int, C.c_int]
    lib.espec_prop_create.argtypes = [C.POINTER(vp), C.c_int, i, d, d, C.c_double, C.c_int,
                                      C.c_int, C.c_int, C.c_int]
    lib.espec_prop_previous.argtypes = [vp, vp, vp, C.c_int, vp]
    lib.espec_spo_load.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp]
    lib.espec_spo_run.argtypes = [vp, C.c_int, vp]
    lib.espec_spo_results.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp]
    lib.espec_spo_device_c.argtypes = [vp]
    lib.espec_spo_device_c.restype = vp
    lib.espec_spo_npoints.argtypes = [vp]
    lib.espec_spo_set_variant.argtypes = [vp, C.c_int, C.c_int]
    lib.espec_spo_set_launch.argtypes = [vp, C.c_int]
    lib.espec_prop_nonfinite.argtypes = [vp, C.POINTER(C.c_int), vp]
    lib.espec_spo_tc_status.argtypes = [C.POINTER(C.c_int)]
    lib.espec_set_wait_limit.argtypes = [C.c_long]
    lib.espec_grid_set_ctas.argtypes = [vp, C.c_int]
    lib.espec_pot_kind.argtypes = [C.c_char_p, C.c_size_t, C.c_int]
    lib.espec_gvpot_1d.argtypes = [C.c_int, vp, vp, vp, C.c_int, vp, C.c_int, vp, vp, vp]
    lib.espec_gvpot_nd.argtypes = [C.c_int, vp, vp, vp, vp, C.c_int, vp, C.c_int, C.c_int, vp, vp]
    lib.espec_selftest_short_arrivals.argtypes = [C.c_int]
    lib.espec_selftest_mbar_wait.argtypes = [C.c_long, C.POINTER(C.c_int)]
    lib.espec_spo_set_item_cost.argtypes = [vp, C.c_int, C.c_double]
    lib.espec_spo_variant_count.restype = C.c_int
    lib.espec_spo_run_static.argtypes = [C.c_int, i, d, d, C.c_double, C.c_int, vp, vp, C.c_int,
                                         vp, vp, vp]
    lib.espec_prop_continue.argtypes = [vp, C.c_int, vp]
    lib.espec_prop_energies.argtypes = [vp, vp, vp, vp]
    lib.espec_format_crl_row.argtypes = [C.c_double] * 6 + [C.c_char_p, C.c_int]
    # Fortran drop-ins: every argument by reference, then one size_t length
    # per CHARACTER*(*) argument
    lib.pspofft_.argtypes = [vp] * 30 + [C.c_size_t] * 3
    lib.pspofft_.restype = None
    lib.psodfft_.argtypes = [vp] * 32 + [C.c_size_t] * 3
    lib.psodfft_.restype = None
    lib.espec_grid_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, i, d, C.c_double,
                                      C.c_int, C.c_int, C.c_int, C.c_int]
    lib.espec_grid_load.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp]
    lib.espec_grid_run.argtypes = [vp, C.c_int, vp]
    lib.espec_grid_continue.argtypes = [vp, C.c_int, vp]
    lib.espec_grid_results.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp]
    lib.espec_grid_energies.argtypes = [vp, vp, vp, vp]
    lib.espec_grid_npoints.argtypes = [vp]
    lib.espec_grid_npoints.restype = C.c_long
    lib.espec_grid_basis.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, vp]
    lib.espec_grid_previous.argtypes = [vp, vp, vp, C.c_int, vp]
    lib.espec_grid_energies_at.argtypes = [vp, C.c_double, vp, vp, vp]
    lib.espec_grid_set_pulse.argtypes = [vp, vp, vp, C.c_long, C.c_int]
    lib.espec_pulse_field.argtypes = [C.c_int, vp, C.c_double]
    lib.espec_pulse_field.restype = C.c_double
    lib.espec_ppsod_field.argtypes = [C.c_int, vp, C.c_double, C.c_double, C.c_double, vp,
                                      C.c_long]
    lib.espec_ppsod_field.restype = C.c_long
    lib.espec_pplnz_field.argtypes = [C.c_int, vp, C.c_double, C.c_double, C.c_double, vp,
                                      C.c_long]
    lib.espec_pplnz_field.restype = C.c_long
    lib.plnz_.argtypes = [vp] * 33 + [C.c_size_t] * 3
    lib.plnz_.restype = None
    lib.psod_.argtypes = [vp] * 28 + [C.c_size_t] * 3
    lib.psod_.restype = None
    lib.ppsod_.argtypes = [vp] * 51 + [C.c_size_t] * 4
    lib.ppsod_.restype = None
    lib.pplnz_.argtypes = [vp] * 51 + [C.c_size_t] * 4
    lib.pplnz_.restype = None
    lib.espec_grid_project.argtypes = [vp, vp, C.c_int, vp, vp]
    lib.espec_run_deck.argtypes = [C.c_char_p]
    lib.espec_run_scan.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), C.c_char_p]
    lib.espec_spectrum_dev.argtypes = [C.c_int, C.c_int, vp, C.c_long, C.c_int, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                       C.c_int, vp, vp, vp]
    lib.espec_spectrum_work_bytes.argtypes = [C.c_int, C.c_int]
    lib.espec_spectrum_work_bytes.restype = C.c_size_t
    lib.hwhm_.argtypes = [vp] * 7
    lib.hwhm_.restype = None
    lib.spectrumtd_.argtypes = [vp] * 8 + [C.c_size_t]
    lib.spectrumtd_.restype = None
    lib.espec_eig_solve_dev.argtypes = [C.c_int, i, d, vp, vp, C.c_int, C.c_int, C.c_double,
                                        C.c_int, vp, vp, vp, vp, vp, vp, vp]
    lib.espec_eig_lcg_start.argtypes = [vp, C.c_int, C.c_int, vp]
    lib.espec_eig_morse2d.argtypes = [C.c_int, vp, i, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_double, vp, vp]
    ci, cd, cf, cl = C.c_int, C.c_double, C.c_float, C.c_long
    lib.espec_gemm_f64.argtypes = [ci, ci, ci, cd, vp, ci, ci, vp, ci, ci, cd, vp, ci, vp]
    lib.espec_gemm_f32.argtypes = [ci, ci, ci, cf, vp, ci, ci, vp, ci, ci, cf, vp, ci, vp]
    lib.espec_mlp_colsum.argtypes = [vp, ci, ci, vp, vp]
    lib.espec_mlp_mse.argtypes = [vp, vp, ci, ci, vp, vp, vp]
    lib.espec_gemm_bf16.argtypes = [ci, ci, ci, cf, vp, ci, ci, vp, ci, ci, cf, vp, ci, vp]
    lib.espec_gemm_bf16_status.argtypes = [C.POINTER(ci)]
    lib.espec_mlp_bias_gelu.argtypes = [vp, vp, ci, ci, ci, vp, vp]
    lib.espec_mlp_gelu_back.argtypes = [vp, vp, cl, vp, vp]
    lib.espec_to_bf16.argtypes = [vp, vp, cl, vp]
    lib.espec_mlp_adam_bf16.argtypes = [vp, vp, vp, vp, cl, vp, cf, cf, cf, vp, vp]
    lib.espec_spond_create.argtypes = [C.POINTER(vp), ci, i, d, d, cd, ci, ci, ci]
    lib.espec_spond_load.argtypes = [vp, vp, vp, vp, vp, ci, vp]
    lib.espec_spond_run.argtypes = [vp, ci, vp]
    lib.espec_spond_results.argtypes = [vp, vp, vp, vp, vp, ci, vp]
    lib.espec_spond_continue.argtypes = [vp, ci, vp]
    lib.espec_spond_create_method.argtypes = [C.POINTER(vp), ci, ci, i, d, d, cd, ci, ci, ci]
    lib.espec_spond_previous.argtypes = [vp, vp, vp, ci, vp]
    lib.espec_spond_energies.argtypes = [vp, vp, vp, vp]
    lib.espec_spond_destroy.argtypes = [vp]
    lib.espec_spond_destroy.restype = None
    lib.espec_sep_basis.argtypes = [ci, ci, ci, ci, ci, vp, vp, vp, vp, cf, vp]
    lib.espec_convert.argtypes = [vp, vp, cl, ci, cd, vp]
    lib.espec_grid_destroy.argtypes = [vp]
    lib.espec_grid_destroy.restype = None
    lib.espec_spo_destroy.argtypes = [vp]
    lib.espec_spo_destroy.restype = None
    _lib = lib
    return lib


def check(rc, what):
    if rc != OK:
        msg = load().espec_last_error().decode(errors="replace")
        raise EspecError(f"{what} failed ({rc}): {msg}")


def ptr(a):
    """Address of a numpy array, a torch tensor or an int (device pointer)."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)
