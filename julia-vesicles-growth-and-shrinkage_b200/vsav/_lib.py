"""ctypes binding of libvsav (include/vsav.h).  No torch types cross the
boundary: plain pointers to float64 host (or device) buffers and sizes."""
import ctypes as ct
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libvsav.so")

VSAV_OK = 0
VSAV_E_INVALID = -1
VSAV_E_CUDA = -2
VSAV_E_WC_NEGATIVE = -3
VSAV_E_NONFINITE = -4
VSAV_W_NOT_CONVERGED = 1

FIELDS = ("phi", "phi_hat", "psi", "psi_hat", "u", "u_hat", "p", "p_hat", "mu", "mu_hat", "nu", "nu_hat")
FIELD_ID = {k: i for i, k in enumerate(FIELDS)}

# every function declared in include/vsav.h
EXPORTS = ("vsav_create", "vsav_destroy", "vsav_last_error", "vsav_create_error", "vsav_default_options",
           "vsav_set_field", "vsav_get_field", "vsav_export_f32", "vsav_set_scalars", "vsav_get_scalars", "vsav_set_dt",
           "vsav_get_dt", "vsav_set_A0", "vsav_get_A0", "vsav_init_state", "vsav_init_shapes2d", "vsav_generate_initial_condition", "vsav_step1", "vsav_step2", "vsav_step3",
           "vsav_step4", "vsav_step5", "vsav_step6", "vsav_step7", "vsav_update_state", "vsav_run",
           "vsav_monitor", "vsav_get_work", "vsav_get_scalar_work", "vsav_transform", "vsav_time_run",
           "vsav_profile", "vsav_profile_read", "vsav_launch_count", "vsav_get_tuning",
           "vsav_net_create", "vsav_net_destroy", "vsav_net_last_error", "vsav_net_nparams",
           "vsav_net_set_params", "vsav_net_get_params", "vsav_net_forward", "vsav_net_grad", "vsav_net_train",
           "vsav_net_eval", "vsav_set_psi_net", "vsav_psi_harvest", "vsav_psi_harvest_read",
           "vsav_irfft2d_f32_noalloc", "vsav_noalloc_error")


class VsavConfig(ct.Structure):
    _fields_ = [("ndim", ct.c_int32), ("Nx", ct.c_int32), ("Ny", ct.c_int32), ("Nz", ct.c_int32),
                ("N", ct.c_int32),
                ("epsilon", ct.c_double), ("M_phi", ct.c_double), ("M0_psi", ct.c_double), ("eta", ct.c_double),
                ("gamma_surf", ct.c_double), ("gamma_area", ct.c_double), ("gamma_bend", ct.c_double),
                ("gamma_in", ct.c_double), ("beta_in", ct.c_double), ("gamma_out", ct.c_double),
                ("beta_out", ct.c_double), ("lamda", ct.c_double),
                ("S1", ct.c_double), ("S2", ct.c_double), ("S3", ct.c_double), ("S4", ct.c_double),
                ("C1", ct.c_double), ("C2", ct.c_double), ("C3", ct.c_double),
                ("dt", ct.c_double), ("T", ct.c_double), ("Lx", ct.c_double), ("Ly", ct.c_double),
                ("Lz", ct.c_double), ("tol", ct.c_double),
                ("psi_in_v", ct.POINTER(ct.c_double)), ("psi_out_v", ct.POINTER(ct.c_double))]


class VsavOptions(ct.Structure):
    _fields_ = [("precision", ct.c_int32), ("psi_form", ct.c_int32), ("psi_precond", ct.c_int32),
                ("psi_itmax", ct.c_int32), ("psi_rtol", ct.c_double), ("psi_atol", ct.c_double),
                ("n_runs", ct.c_int32), ("run_sizes", ct.POINTER(ct.c_int32)), ("device", ct.c_int32),
                ("graph", ct.c_int32), ("psi3d_variable", ct.c_int32), ("psi_stop", ct.c_int32),
                ("psi_check", ct.c_int32)]


class VsavShape2D(ct.Structure):
    _fields_ = [("cx", ct.c_double), ("cy", ct.c_double), ("a", ct.c_double), ("b", ct.c_double),
                ("rot", ct.c_double), ("psi_in", ct.c_double), ("psi_out", ct.c_double),
                ("nmodes", ct.c_int32), ("m", ct.c_int32 * 8), ("amp", ct.c_double * 8), ("phase", ct.c_double * 8)]


class VsavStatus(ct.Structure):
    _fields_ = [("err_flags", ct.c_int32), ("psi_systems", ct.c_int32), ("psi_max_iters", ct.c_int32),
                ("psi_not_converged", ct.c_int32)]


_lib = None


def load(path: str = LIB_PATH):
    """Loads libvsav.so.  Fails loudly when the CUDA library has not been built:
    there is no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libvsav.so not found at {path}: build it with "
                           "`python julia-vesicles-growth-and-shrinkage_b200/build.py`")
    lib = ct.CDLL(path)
    H = ct.c_void_p
    D = ct.POINTER(ct.c_double)
    i32 = ct.c_int32
    sig = {
        "vsav_create": ([ct.POINTER(VsavConfig), ct.POINTER(VsavOptions), ct.POINTER(ct.c_void_p)], ct.c_int),
        "vsav_destroy": ([H], ct.c_int),
        "vsav_last_error": ([H], ct.c_char_p),
        "vsav_create_error": ([], ct.c_char_p),
        "vsav_default_options": ([ct.POINTER(VsavOptions), ct.POINTER(VsavConfig)], None),
        "vsav_set_field": ([H, i32, i32, D], ct.c_int),
        "vsav_get_field": ([H, i32, i32, D], ct.c_int),
        "vsav_export_f32": ([H, ct.c_int32, ct.c_int32, ct.POINTER(ct.c_float)], ct.c_int),
        "vsav_set_scalars": ([H, i32, D], ct.c_int),
        "vsav_get_scalars": ([H, i32, D], ct.c_int),
        "vsav_set_dt": ([H, D], ct.c_int),
        "vsav_get_dt": ([H, D], ct.c_int),
        "vsav_init_shapes2d": ([H, ct.POINTER(VsavShape2D)], ct.c_int),
        "vsav_generate_initial_condition": ([H, ct.c_int32, ct.c_int32, D], ct.c_int),
        "vsav_set_A0": ([H, D], ct.c_int),
        "vsav_get_A0": ([H, D], ct.c_int),
        "vsav_init_state": ([H, i32], ct.c_int),
        "vsav_step1": ([H, i32, ct.POINTER(VsavStatus)], ct.c_int),
        "vsav_step2": ([H, i32], ct.c_int),
        "vsav_step3": ([H], ct.c_int),
        "vsav_step4": ([H, i32], ct.c_int),
        "vsav_step5": ([H, i32], ct.c_int),
        "vsav_step6": ([H], ct.c_int),
        "vsav_step7": ([H, i32], ct.c_int),
        "vsav_update_state": ([H], ct.c_int),
        "vsav_run": ([H, i32, i32, D, D, D, ct.POINTER(VsavStatus)], ct.c_int),
        "vsav_monitor": ([H, D, D], ct.c_int),
        "vsav_get_work": ([H, i32, i32, D], ct.c_int),
        "vsav_get_scalar_work": ([H, i32, D], ct.c_int),
        "vsav_transform": ([H, i32, i32, D, D], ct.c_int),
        "vsav_time_run": ([H, i32, i32, D, i32, D], ct.c_int),
        "vsav_profile": ([H, i32], ct.c_int),
        "vsav_profile_read": ([H, i32, D], ct.c_int),
        "vsav_launch_count": ([], ct.c_int64),
        "vsav_get_tuning": ([H, ct.c_char_p, ct.c_int64, ct.POINTER(ct.c_int64)], ct.c_int),
        "vsav_irfft2d_f32_noalloc": ([ct.c_void_p, ct.c_void_p, i32, i32, i32, ct.c_double, ct.c_double, i32,
                                      ct.c_void_p], ct.c_int),
        "vsav_noalloc_error": ([], ct.c_char_p),
        "vsav_net_create": ([ct.c_int64, i32, ct.POINTER(ct.c_void_p)], ct.c_int),
        "vsav_net_destroy": ([H], ct.c_int),
        "vsav_net_last_error": ([H], ct.c_char_p),
        "vsav_net_nparams": ([], ct.c_int),
        "vsav_net_set_params": ([H, D], ct.c_int),
        "vsav_net_get_params": ([H, D, i32], ct.c_int),
        "vsav_net_forward": ([H, ct.c_void_p, i32, i32, i32, i32, i32, ct.c_void_p], ct.c_int),
        "vsav_net_grad": ([H, ct.c_void_p, ct.c_void_p, i32, i32, i32, i32, i32, ct.c_double, D, D], ct.c_int),
        "vsav_net_train": ([H, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int64, i32, i32, i32, ct.c_double,
                            ct.c_uint64, i32, i32, ct.c_double, D], ct.c_int),
        "vsav_net_eval": ([H, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int64, i32, i32, i32, ct.c_double, D],
                          ct.c_int),
        "vsav_set_psi_net": ([H, D], ct.c_int),
        "vsav_psi_harvest": ([H, i32], ct.c_int),
        "vsav_psi_harvest_read": ([H, ct.c_void_p, ct.c_int64, ct.POINTER(i32), ct.POINTER(ct.c_int64)], ct.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def dptr(a: np.ndarray):
    assert a.dtype in (np.float64, np.complex128) and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ct.POINTER(ct.c_double))
