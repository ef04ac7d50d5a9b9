"""ctypes binding of libwildfires_b200.so (the C-ABI in include/wildfires_b200.h).

The library is built in-tree by wildfires_b200/build.py.  Loading fails
loudly when it is missing: there is no CPU implementation behind this API.
"""
import ctypes as C
import os

from ._params import Parameters

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwildfires_b200.so")

WF_OK, WF_ERR_ARG, WF_ERR_CUDA, WF_ERR_IO, WF_ERR_PARSE, WF_ERR_OOM, WF_ERR_NAN, WF_ERR_NO_DEVICE = range(8)
WF_FP64, WF_FP32_STENCIL = 0, 1
WF_NPHASES = 9

#: every symbol include/wildfires_b200.h declares
EXPORTS = [
    "wf_read_parameters", "wf_free_parameters", "wf_set_topography", "wf_state_size",
    "wf_load_fields", "wf_save_fields", "wf_create", "wf_destroy", "wf_upload_state", "wf_upload_state_async",
    "wf_download_state", "wf_step", "wf_synchronize", "wf_time", "wf_diagnostics",
    "wf_device_state", "wf_stream", "wf_phi", "wf_pressure", "wf_launches_per_step",
    "wf_status_string", "wf_last_error", "wf_profile_phases", "wf_phase_name",
    "wf_pressure_noalloc", "wf_rk", "wf_pressure_report",
    "wf_ensemble_create", "wf_ensemble_destroy", "wf_ensemble_size", "wf_ensemble_member",
    "wf_ensemble_step", "wf_ensemble_synchronize",
    "wf_closure_param_count", "wf_set_closure", "wf_closure_coefficients", "wf_mlp_loss_grad", "wf_mlp_train",
    "wf_timestep_reports", "wf_dump_async", "wf_dump_wait", "wf_save_domain", "wf_save_topography",
    "wf_initial_conditions", "wf_stage_tile", "wf_set_stage_tile",
    "wf_set_stream", "wf_phi_device", "wf_rk_device", "wf_pressure_device",
    "wf_closure_predict", "wf_set_closure_wait_limit",
    "wf_ibm_parameters_device", "wf_set_topography_hills", "wf_ensemble_stream",
    "wf_inject_allocation_failure",
]


class WfDiag(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "mass", "energy", "fuel", "fuel_consumed", "max_abs_u", "max_abs_v", "max_abs_w",
        "cfl", "T_min", "T_max", "Y_min", "Y_max")] + [("nan_count", C.c_longlong)]


class WfReport(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("cfl", "Y_min", "Y_max", "T_min", "T_max")] + \
        [(n, C.c_int) for n in ("nan_field", "nan_i", "nan_j", "nan_k")]


class WfError(RuntimeError):
    def __init__(self, status, where, msg):
        super().__init__("%s: status %d (%s): %s" % (where, status, _status_name(status), msg))
        self.status = status


_names = {WF_OK: "ok", WF_ERR_ARG: "invalid argument", WF_ERR_CUDA: "CUDA error", WF_ERR_IO: "I/O error",
          WF_ERR_PARSE: "parse error", WF_ERR_OOM: "out of memory", WF_ERR_NAN: "NaN in state",
          WF_ERR_NO_DEVICE: "no sm_100 device"}


def _status_name(s):
    return _names.get(s, "unknown")


_lib = None


def lib():
    """Load the library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libwildfires_b200.so is not built (run python wildfires_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER(Parameters)
    dp = C.POINTER(C.c_double)
    fp = C.POINTER(C.c_float)
    vp = C.c_void_p
    sig = {
        "wf_read_parameters": (C.c_int, [C.c_char_p, P]),
        "wf_free_parameters": (None, [P]),
        "wf_set_topography": (C.c_int, [P, dp]),
        "wf_state_size": (C.c_size_t, [P]),
        "wf_load_fields": (C.c_int, [P, C.c_char_p, dp, dp]),
        "wf_save_fields": (C.c_int, [P, C.c_char_p, C.c_int, dp, dp]),
        "wf_create": (C.c_int, [P, C.c_int, C.POINTER(vp)]),
        "wf_destroy": (C.c_int, [vp]),
        "wf_upload_state": (C.c_int, [vp, dp, dp]),
        "wf_upload_state_async": (C.c_int, [vp, dp, dp]),
        "wf_download_state": (C.c_int, [vp, dp, dp]),
        "wf_step": (C.c_int, [vp, C.c_int]),
        "wf_synchronize": (C.c_int, [vp]),
        "wf_time": (C.c_int, [vp, C.POINTER(C.c_int), dp]),
        "wf_diagnostics": (C.c_int, [vp, C.POINTER(WfDiag)]),
        "wf_device_state": (C.c_int, [vp, C.POINTER(vp), C.POINTER(dp)]),
        "wf_stream": (vp, [vp]),
        "wf_phi": (C.c_int, [vp, dp, dp]),
        "wf_pressure": (C.c_int, [vp, dp, dp, dp, C.POINTER(C.c_int)]),
        "wf_launches_per_step": (C.c_int, [vp]),
        "wf_status_string": (C.c_char_p, [C.c_int]),
        "wf_profile_phases": (C.c_int, [vp, C.c_int, dp, C.POINTER(C.c_int)]),
        "wf_phase_name": (C.c_char_p, [C.c_int]),
        "wf_pressure_noalloc": (C.c_int, [P, vp, vp, vp]),
        "wf_rk": (C.c_int, [vp, dp, dp]),
        "wf_ensemble_create": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(vp)]),
        "wf_ensemble_destroy": (C.c_int, [vp]),
        "wf_ensemble_size": (C.c_int, [vp]),
        "wf_ensemble_member": (vp, [vp, C.c_int]),
        "wf_ensemble_step": (C.c_int, [vp, C.c_int]),
        "wf_ensemble_synchronize": (C.c_int, [vp]),
        "wf_closure_param_count": (C.c_int, []),
        "wf_set_closure": (C.c_int, [vp, C.c_int, fp]),
        "wf_closure_coefficients": (C.c_int, [vp, dp, dp]),
        "wf_mlp_loss_grad": (C.c_int, [fp, fp, fp, C.c_size_t, dp, fp]),
        "wf_mlp_train": (C.c_int, [fp, fp, fp, C.c_size_t, C.c_int, C.c_int, C.c_float, C.c_ulonglong, dp]),
        "wf_pressure_report": (C.c_int, [vp, dp, C.POINTER(C.c_int)]),
        "wf_last_error": (C.c_char_p, []),
        "wf_timestep_reports": (C.c_int, [vp, C.POINTER(WfReport)]),
        "wf_dump_async": (C.c_int, [vp, C.c_char_p, C.c_int]),
        "wf_dump_wait": (C.c_int, [vp]),
        "wf_save_domain": (C.c_int, [P, C.c_char_p]),
        "wf_save_topography": (C.c_int, [P, C.c_char_p]),
        "wf_initial_conditions": (C.c_int, [vp]),
        "wf_stage_tile": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "wf_set_stage_tile": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
        "wf_set_stream": (C.c_int, [vp, vp]),
        "wf_phi_device": (C.c_int, [vp, vp, vp]),
        "wf_rk_device": (C.c_int, [vp, vp, vp]),
        "wf_pressure_device": (C.c_int, [vp, vp, vp, vp]),
        "wf_closure_predict": (C.c_int, [fp, fp, C.c_size_t, fp]),
        "wf_set_closure_wait_limit": (C.c_int, [vp, C.c_int]),
        "wf_ibm_parameters_device": (C.c_int, [P]),
        "wf_set_topography_hills": (C.c_int, [P, C.c_int, dp]),
        "wf_ensemble_stream": (vp, [vp]),
        "wf_inject_allocation_failure": (None, [C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status, where):
    if status != WF_OK:
        raise WfError(status, where, lib().wf_last_error().decode(errors="replace"))
