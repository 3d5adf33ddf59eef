"""ctypes binding of libsurfatt_gpu.so (the C ABI declared in include/surfatt_gpu.h).

There is no CPU fallback: if the library is missing or no CUDA device is
present, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# SURFATT_GPU_LIB selects another build of the same library (same C ABI).
LIB_PATH = os.environ.get("SURFATT_GPU_LIB") or os.path.join(_HERE, "libsurfatt_gpu.so")

(SA_OK, SA_ERR_ARG, SA_ERR_CUDA, SA_ERR_NOCONV, SA_ERR_NOROOT, SA_ERR_NONFINITE, SA_ERR_NOMEM,
 SA_ERR_TEAM) = range(8)
SA_FP64, SA_FP32 = 0, 1
STATUS_NAMES = {0: "SA_OK", 1: "SA_ERR_ARG", 2: "SA_ERR_CUDA", 3: "SA_ERR_NOCONV",
                4: "SA_ERR_NOROOT", 5: "SA_ERR_NONFINITE", 6: "SA_ERR_NOMEM", 7: "SA_ERR_TEAM"}

# Every symbol include/surfatt_gpu.h declares.
EXPORTED = (
    "sa_ctx_create", "sa_ctx_destroy", "sa_ctx_error", "sa_version",
    "sa_eik_fwd_field", "sa_eik_adj_field", "sa_mask_uniform_grid",
    "sa_plan_create", "sa_plan_destroy", "sa_plan_set_graph", "sa_plan_forward_adjoint",
    "sa_forward_for_events", "sa_plan_debug_fields", "sa_plan_kernel_timing", "sa_plan_kernel_ms",
    "sa_plan_autotune", "sa_plan_set_tune", "sa_plan_get_tune",
    "sa_surfdisp_columns", "sa_depthkernel_columns", "sa_combine_kernels_vs",
    "sa_depthkernel_columns_group",
    "sa_eik_fwd_field_noalloc", "sa_math_eval", "sa_plan_adjoint_source",
    "sa_grad_forward", "sa_grad_vjp", "sa_plan_set_deterministic",
    "sa_grad_set_data_type", "sa_plan_kden_output", "sa_grad_set_kden", "sa_grad_ker_den",
    "sa_plan_set_adjoint", "sa_grad_root_derivatives",
    "sa_kernel_precondition", "sa_multi_create", "sa_multi_destroy",
    "sa_multi_forward_adjoint", "sa_multi_kernel_ms", "sa_multi_status",
    "sa_depthkernel_columns_love", "sa_grad_set_wave_type", "sa_multigrid_create",
    "sa_multigrid_destroy", "sa_multigrid_smooth",
    "sa_grad_create", "sa_grad_destroy", "sa_grad_run", "sa_grad_sen", "sa_grad_combine",
    "sa_pde_smooth_nstep", "sa_pde_smooth",
    "sa_lbfgs_create", "sa_lbfgs_destroy", "sa_lbfgs_store", "sa_lbfgs_direction", "sa_dot",
    "sa_grad_normalization", "sa_descent_angle", "sa_wolfe_condition", "sa_model_update_vs",
    "sa_grid_topography", "sa_topo_media", "sa_correct_depth_with_topo",
    "sa_srcrec_load", "sa_srcrec_destroy", "sa_srcrec_sizes", "sa_srcrec_periods",
    "sa_srcrec_observations", "sa_srcrec_events", "sa_srcrec_event_name", "sa_srcrec_write",
)


class SAError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class NoConvergence(SAError):
    pass


_lib = None
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = C.c_void_p


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m surfattpp_b200.build`")
    L = C.CDLL(LIB_PATH)
    i, d = C.c_int, C.c_double
    L.sa_ctx_create.argtypes = [i, C.POINTER(_vp)]
    L.sa_ctx_destroy.argtypes = [_vp]
    L.sa_ctx_error.argtypes = [_vp]
    L.sa_ctx_error.restype = C.c_char_p
    L.sa_version.restype = i
    L.sa_eik_fwd_field.argtypes = [_vp, i, i, i, _dp, _dp, _dp, _dp, _dp, _dp, d, d, _dp,
                                   C.POINTER(i)]
    L.sa_eik_adj_field.argtypes = [_vp, i, i, i, _dp, _dp, _dp, _dp, _dp, _dp, i, _vp, _vp, _vp,
                                   _dp, C.POINTER(i)]
    L.sa_mask_uniform_grid.argtypes = [i, i, _dp, _dp, _dp, d, d]
    L.sa_plan_create.argtypes = [_vp, i, i, i, i, _dp, _dp, i, _vp, _vp, _vp, _vp, _vp, i, _vp,
                                 _vp, C.POINTER(_vp)]
    L.sa_plan_destroy.argtypes = [_vp]
    L.sa_plan_set_graph.argtypes = [_vp, i]
    L.sa_plan_forward_adjoint.argtypes = [_vp] + [_vp] * 6 + [i] + [_vp] * 6 + [_vp]
    L.sa_plan_debug_fields.argtypes = [_vp, _vp, _vp]
    L.sa_plan_kernel_timing.argtypes = [_vp, i]
    L.sa_plan_kernel_ms.argtypes = [_vp, C.POINTER(C.c_float)]
    L.sa_plan_autotune.argtypes = [_vp] * 7 + [i, _vp, C.POINTER(C.c_float), C.POINTER(i),
                                              C.POINTER(i), _vp]
    L.sa_plan_set_tune.argtypes = [_vp, i, i]
    L.sa_plan_get_tune.argtypes = [_vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.sa_forward_for_events.argtypes = [_vp, i, i, i, i, _dp, _dp, _dp, _vp, _vp, _vp, i, _dp,
                                        _dp, _ip, _ip, _ip, i, _dp, _dp, _dp, _dp, i, _dp, _dp,
                                        C.POINTER(d), _ip, _ip]
    L.sa_surfdisp_columns.argtypes = [_vp, i, i, i, _dp, _vp, i, _dp, i, i, _vp, _vp, _vp]
    L.sa_depthkernel_columns.argtypes = [_vp, i, i, i, _dp, _vp, i, _dp, _vp, _vp, _vp, _vp, _vp]
    L.sa_depthkernel_columns_group.argtypes = [_vp, i, i, i, _dp, _vp, i, _dp, _vp, _vp, _vp,
                                               _vp, _vp]
    L.sa_combine_kernels_vs.argtypes = [_vp, i, i, i, i] + [_vp] * 7 + [_vp]
    L.sa_eik_fwd_field_noalloc.argtypes = [i, i] + [_vp] * 6 + [d, d] + [_vp] * 4
    L.sa_math_eval.argtypes = [i, C.c_size_t, _vp, _vp, _vp]
    L.sa_plan_adjoint_source.argtypes = [_vp] * 9 + [_vp]
    L.sa_grad_forward.argtypes = [_vp] * 5 + [_vp]
    L.sa_grad_vjp.argtypes = [_vp] * 4 + [i] + [_vp] * 4 + [_vp]
    L.sa_plan_set_deterministic.argtypes = [_vp, i, C.c_size_t]
    L.sa_grad_set_data_type.argtypes = [_vp, i]
    L.sa_grad_set_wave_type.argtypes = [_vp, i]
    L.sa_multigrid_create.argtypes = [i, i, i, i, _dp, _dp, _dp, _ip, i, C.POINTER(_vp)]
    L.sa_multigrid_destroy.argtypes = [_vp]
    L.sa_multigrid_smooth.argtypes = [_vp, _vp, _vp, _vp]
    L.sa_plan_kden_output.argtypes = [_vp, _vp]
    L.sa_plan_set_adjoint.argtypes = [_vp, i]
    L.sa_grad_root_derivatives.argtypes = [_vp] * 4
    L.sa_grad_set_kden.argtypes = [_vp, i]
    L.sa_grad_ker_den.argtypes = [_vp] * 4 + [_vp]
    L.sa_kernel_precondition.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp]
    L.sa_multi_create.argtypes = [C.POINTER(_vp), i, C.POINTER(_vp)]
    L.sa_multi_destroy.argtypes = [_vp]
    L.sa_multi_forward_adjoint.argtypes = [_vp] + [C.POINTER(_vp)] * 6 + [i] + \
        [C.POINTER(_vp)] * 4 + [_vp]
    L.sa_multi_kernel_ms.argtypes = [_vp, C.POINTER(C.c_float)]
    L.sa_multi_status.argtypes = [_vp, C.POINTER(i)]
    L.sa_depthkernel_columns_love.argtypes = [_vp, i, i, i, _dp, _vp, i, _dp, i, _vp, _vp, _vp,
                                              _vp]
    L.sa_grad_create.argtypes = [_vp, i, _dp, _dp, C.POINTER(_vp)]
    L.sa_grad_destroy.argtypes = [_vp]
    L.sa_grad_run.argtypes = [_vp] + [_vp] * 9 + [_vp]
    L.sa_grad_sen.argtypes = [_vp] * 5
    L.sa_grad_combine.argtypes = [_vp] * 6
    L.sa_pde_smooth_nstep.argtypes = [i, d, d, d, _dp, d, d, C.POINTER(i), C.POINTER(d),
                                      C.POINTER(d)]
    z = C.c_size_t
    L.sa_lbfgs_create.argtypes = [_vp, z, C.POINTER(_vp)]
    L.sa_lbfgs_destroy.argtypes = [_vp]
    L.sa_lbfgs_store.argtypes = [_vp, i, _vp, _vp]
    L.sa_lbfgs_direction.argtypes = [_vp, i, _vp]
    L.sa_dot.argtypes = [_vp, z, _vp, _vp, C.POINTER(d)]
    L.sa_grad_normalization.argtypes = [_vp, z, _vp, C.POINTER(d)]
    L.sa_descent_angle.argtypes = [_vp, z, _vp, _vp, C.POINTER(d)]
    L.sa_wolfe_condition.argtypes = [d, d, d, C.POINTER(d), C.POINTER(d), d, d, i, d, d, i, d,
                                     C.POINTER(d)]
    L.sa_model_update_vs.argtypes = [_vp, z, _vp, _vp, d, _vp, _vp, _vp, _vp]
    L.sa_srcrec_load.argtypes = [C.c_char_p, C.POINTER(_vp)]
    L.sa_srcrec_destroy.argtypes = [_vp]
    L.sa_srcrec_sizes.argtypes = [_vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.sa_srcrec_periods.argtypes = [_vp, _vp, _vp, _vp]
    L.sa_srcrec_observations.argtypes = [_vp] + [_vp] * 7
    L.sa_srcrec_events.argtypes = [_vp] + [_vp] * 5
    L.sa_srcrec_event_name.argtypes = [_vp, i]
    L.sa_srcrec_event_name.restype = C.c_char_p
    L.sa_srcrec_write.argtypes = [_vp, C.c_char_p, _vp]
    L.sa_grid_topography.argtypes = [_vp, i, i, _dp, _dp, _dp, i, i, _dp, _dp, _vp]
    L.sa_topo_media.argtypes = [_vp, i, i, _dp, _dp, _vp, i, _dp, _vp, _vp, _vp, _vp, _vp]
    L.sa_correct_depth_with_topo.argtypes = [_vp, i, i, i, i, _dp, _vp, _vp, _vp, _vp, _vp]
    L.sa_pde_smooth.argtypes = [_vp, i, i, i, d, d, d, _dp, _dp, d, d, _vp, _vp, C.POINTER(i),
                                _vp]
    _lib = L
    return L


def check(ctx, rc):
    if rc == SA_OK:
        return
    msg = lib().sa_ctx_error(ctx).decode() if ctx else ""
    if rc == SA_ERR_NOCONV:
        raise NoConvergence(rc, msg)
    raise SAError(rc, msg)


class Context:
    """One CUDA device + stream (sa_ctx)."""

    def __init__(self, device: int = 0):
        h = _vp()
        rc = lib().sa_ctx_create(device, C.byref(h))
        if rc != SA_OK:
            raise SAError(rc, "sa_ctx_create failed (no CUDA device?)")
        self.h = h

    def close(self):
        if self.h:
            lib().sa_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(int(os.environ.get("SA_DEVICE", "0")))
    return _default_ctx


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (or None)."""
    if t is None:
        return None
    return t.data_ptr()
