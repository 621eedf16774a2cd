"""ctypes binding of the C ABI in include/vdi.h (libvdi.so).

There is no fallback: if the library is missing or a call fails, an
exception says so.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libvdi.so")

# status codes (include/vdi.h)
VDI_OK = 0
VDI_ERR_INVALID_ARGUMENT = 1
VDI_ERR_UNSUPPORTED_SIZE = 2
VDI_ERR_CUDA = 3
VDI_ERR_OUT_OF_MEMORY = 4
VDI_ERR_MG_NOT_CONVERGED = 5
VDI_ERR_NEWTON_NOT_CONVERGED = 6
VDI_ERR_TRI_SINGULAR = 7
VDI_ERR_NONFINITE = 8
VDI_ERR_CONFIG = 9
VDI_ERR_NOT_READY = 10

VDI_MG_FP64 = 0
VDI_MG_MIXED = 1
VDI_MG_HYBRID = 2
VDI_GUESS_EXTRAPOLATE = 0
VDI_GUESS_LEARNED = 1
VDI_GUESS_QUADRATIC = 2

VDI_LIFTOFF_OFF = 0
VDI_LIFTOFF_SMOOTHED = 1
VDI_LIFTOFF_RAW = 2

VDI_MG_MAC = 0
VDI_MG_FEM = 1
VDI_MG_VISC_U = 2
VDI_MG_VISC_V = 3
VDI_MG_MAC_NEUMANN = 4


class VdiParams(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("x_sym", C.c_int), ("implicit_visc", C.c_int),
                ("ax", C.c_double), ("ay", C.c_double), ("bx", C.c_double), ("by", C.c_double),
                ("mu", C.c_double), ("rho", C.c_double), ("tmult", C.c_double), ("t_end", C.c_double),
                ("nframes", C.c_int),
                ("alpha", C.c_double), ("mug", C.c_double), ("Pamb", C.c_double), ("h0", C.c_double),
                ("R", C.c_double), ("V", C.c_double), ("sigma", C.c_double),
                ("mg_rtol", C.c_double), ("mg_max_vcycles", C.c_int), ("mg_precision", C.c_int),
                ("mg_guess", C.c_int),
                ("ntrace", C.c_int), ("nif_mode", C.c_int), ("nif_a", C.c_int), ("nif_b", C.c_int)]


_dp = C.POINTER(C.c_double)


class VdiState(C.Structure):
    _fields_ = [("time", C.c_double), ("Vframe", C.c_double),
                ("u", _dp), ("v", _dp), ("p", _dp),
                ("gp", _dp), ("tau", _dp), ("h", _dp), ("fbd", _dp), ("pg", _dp), ("ht", _dp)]


class VdiStats(C.Structure):
    _fields_ = [("steps", C.c_long), ("solves", C.c_long * 4), ("vcycles", C.c_long * 4),
                ("newton_steps", C.c_long), ("tri_pivot_fallbacks", C.c_long),
                ("height_fixed_point_iters", C.c_long), ("last_rel_res", C.c_double * 4),
                ("kernel_launches", C.c_long)]


class VdiMgResult(C.Structure):
    _fields_ = [("vcycles", C.c_int), ("rel_res", C.c_double)]


class VdiLiftoff(C.Structure):
    _fields_ = [("states", C.c_long), ("min_state", C.c_long), ("min_height", C.c_double), ("min_x", C.c_double),
                ("interval", C.c_double), ("t_rel", C.c_double), ("t_rel_ev", C.c_double), ("percent", C.c_double),
                ("searching", C.c_int), ("ev_found", C.c_int), ("last_x", C.c_double),
                ("last_height", C.c_double)]


class VdiTune(C.Structure):
    _fields_ = [("blk_x", C.c_int), ("blk_y", C.c_int), ("cta_limit", C.c_long * 4), ("tiled_levels", C.c_int * 4),
                ("stencil_ms", C.c_float), ("vcycle_ms", C.c_float * 4), ("from_cache", C.c_int)]


class VdiError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: status {status} ({_status_string(status)}): {detail}")
        self.status = status


_lib = None


def _status_string(s: int) -> str:
    try:
        return lib().vdi_status_string(s).decode()
    except Exception:  # pragma: no cover - the library itself failed to load
        return "?"


# (name, restype, argtypes)
_SIGS = [
    ("vdi_status_string", C.c_char_p, [C.c_int]),
    ("vdi_abi_version", C.c_int, []),
    ("vdi_last_error", C.c_char_p, []),
    ("vdi_params_from_cfg", C.c_int, [C.c_char_p, C.POINTER(VdiParams)]),
    ("vdi_sim_create", C.c_int, [C.POINTER(VdiParams), C.c_void_p, C.POINTER(C.c_void_p)]),
    ("vdi_sim_destroy", C.c_int, [C.c_void_p]),
    ("vdi_sim_init_fields", C.c_int, [C.c_void_p]),
    ("vdi_sim_timestep_select", C.c_int, [C.c_void_p, C.c_double, _dp, C.POINTER(C.c_int)]),
    ("vdi_sim_step_forward", C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    ("vdi_sim_use_graph", C.c_int, [C.c_void_p, C.c_int]),
    ("vdi_sim_synchronize", C.c_int, [C.c_void_p]),
    ("vdi_sim_get_state", C.c_int, [C.c_void_p, C.POINTER(VdiState)]),
    ("vdi_sim_set_state", C.c_int, [C.c_void_p, C.POINTER(VdiState)]),
    ("vdi_sim_get_tracers", C.c_int, [C.c_void_p, _dp, C.c_long]),
    ("vdi_sim_set_tracers", C.c_int, [C.c_void_p, _dp, C.c_long]),
    ("vdi_sim_stats", C.c_int, [C.c_void_p, C.POINTER(VdiStats), C.c_int]),
    ("vdi_sim_device_field", C.c_int, [C.c_void_p, C.c_int, C.POINTER(_dp), C.POINTER(C.c_size_t)]),
    ("vdi_sim_vcycle_bytes", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    ("vdi_sim_get_params", C.c_int, [C.c_void_p, C.POINTER(VdiParams)]),
    ("vdi_unet_guess", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    ("vdi_unet_tensor_path", C.c_int, []),
    ("vdi_mg_tile_path", C.c_int, [C.POINTER(C.c_longlong)]),
    ("vdi_sim_init_tracers", C.c_int, [C.c_void_p]),
    ("vdi_sim_update_tracers", C.c_int, [C.c_void_p, C.c_double]),
    ("vdi_sim_set_nif_mode", C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    ("vdi_gas_update", C.c_int, [C.c_void_p, C.c_double]),
    ("vdi_gas_init_fields", C.c_int, [C.c_void_p]),
    ("vdi_sim_autotune", C.c_int, [C.c_void_p, C.POINTER(VdiTune)]),
    ("vdi_sim_set_tuning", C.c_int, [C.c_void_p, C.POINTER(VdiTune)]),
    ("vdi_sim_profile", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_float)]),
    ("vdi_batch_create", C.c_int, [C.POINTER(VdiParams), C.c_int, C.POINTER(C.c_void_p)]),
    ("vdi_batch_destroy", C.c_int, [C.c_void_p]),
    ("vdi_batch_size", C.c_int, [C.c_void_p]),
    ("vdi_batch_sim", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    ("vdi_batch_init_fields", C.c_int, [C.c_void_p]),
    ("vdi_batch_autotune", C.c_int, [C.c_void_p, C.c_void_p]),
    ("vdi_batch_step_forward", C.c_int, [C.c_void_p, _dp, C.c_int]),
    ("vdi_sim_liftoff_setup", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_long]),
    ("vdi_sim_liftoff", C.c_int, [C.c_void_p, C.POINTER(VdiLiftoff), C.c_void_p, C.c_void_p, C.c_long]),
    ("vdi_profile_min", C.c_int, [C.c_int, C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p, _dp, _dp]),
    ("vdi_mg_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_void_p,
                                C.POINTER(C.c_void_p)]),
    ("vdi_mg_destroy", C.c_int, [C.c_void_p]),
    ("vdi_mg_setup", C.c_int, [C.c_void_p]),
    ("vdi_mg_solve", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_int,
                               C.POINTER(VdiMgResult)]),
    ("vdi_mg_v_cycle", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vdi_mg_residual", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _dp]),
    ("vdi_mg_apply", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vdi_mg_profile", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_float),
                                 _dp]),
    ("vdi_mg_coarse_cycle", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("vdi_unet_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint, C.c_void_p, C.POINTER(C.c_void_p)]),
    ("vdi_unet_destroy", C.c_int, [C.c_void_p]),
    ("vdi_unet_param_count", C.c_long, [C.c_void_p]),
    ("vdi_unet_forward", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    ("vdi_unet_train_step", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                      C.POINTER(C.c_float)]),
    ("vdi_unet_gradients", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                     C.POINTER(C.c_float)]),
    ("vdi_unet_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_int]),
    ("vdi_sim_attach_unet", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_double]),
    ("vdi_tri_solve", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_int)]),
]

# Optional entry points bound when present in the built library.
_OPTIONAL = []


def declared_symbols() -> list[str]:
    """Every entry point include/vdi.h declares (parsed from the header)."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "vdi.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(vdi_[a-z0-9_]+)\s*\(", text)))


def lib() -> C.CDLL:
    """Loads libvdi.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m vdropimpact_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIGS + _OPTIONAL:
            if not hasattr(L, name):
                if (name, res, args) in _OPTIONAL:
                    continue
                raise ImportError(f"{LIB_PATH} does not export {name}")
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str):
    if status != VDI_OK:
        detail = lib().vdi_last_error().decode(errors="replace")
        raise VdiError(status, where, detail)
