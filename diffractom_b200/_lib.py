"""ctypes binding of the C ABI (include/diffractom_b200.h) implemented by diffractom_b200/_lib/libdfx_b200.so.

There is no fallback: if the library is missing (python -m diffractom_b200.build makes it) or cannot be loaded,
every operator call fails with an ImportError. Status codes become the exception types of the reference's Python
API: bad arguments ValueError, scratch too small MemoryError, launch / CUDA errors RuntimeError, a device-side wait
that ran out TimeoutError.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libdfx_b200.so"

DFX_OK, DFX_EINVAL, DFX_ENOMEM, DFX_ELAUNCH, DFX_ETIMEOUT, DFX_ECUDA = range(6)
ABI_VERSION = 1


class PFGeometry(ctypes.Structure):
    """dfx_pf_geometry: device pointers of the operator's PF inputs and their sizes."""
    _fields_ = [("coords", c_void_p), ("poles", c_void_p), ("axis_start", c_void_p), ("axis_count", c_void_p),
                ("inv_sigma2", c_void_p), ("norm", c_void_p), ("quad_w", c_void_p), ("intens", c_void_p),
                ("R", c_int32), ("C", c_int32), ("P", c_int32), ("A", c_int32), ("S", c_int32),
                ("S_eta", c_int32), ("K", c_int32), ("cut", c_float),
                ("axis_w", c_void_p), ("axis_sin", c_void_p), ("axis_cos", c_void_p),
                ("wp_pos", c_void_p), ("wp_cov", c_void_p), ("wp_b", c_void_p), ("wp_ax", c_void_p),
                ("wp_ch", c_void_p), ("wp_invD", c_float), ("wp_eta", c_float)]


P, I, L, F, S = c_void_p, c_int, c_int64, c_float, c_void_p   # pointer, int, int64, float, stream
SIGNATURES = {
    "dfx_abi_version": ([], c_int),
    "dfx_last_error": ([], ctypes.c_char_p),
    "dfx_launch_count": ([], ctypes.c_uint64),
    "dfx_gather_channels": ([P, P, L, I, I, I, S], c_int),
    "dfx_scatter_channels": ([P, P, L, I, I, I, S], c_int),
    "dfx_radon_forward": ([P, P, P, I, I, I, I, I, I, I, F, S], c_int),
    "dfx_radon_backward": ([P, P, P, I, I, I, I, I, I, I, I, S], c_int),
    "dfx_radon_backward_pixels": ([P, P, P, I, I, I, I, I, I, I, I, P, L, S], c_int),
    "dfx_radon_backward_spdhg": ([P, P, I, I, I, I, I, I, I, I, P, P, P, F, F, S], c_int),
    "dfx_radon_forward_bf16": ([P, P, L, P, I, I, I, I, I, I, I, F, S], c_int),
    "dfx_radon_backward_bf16": ([P, L, P, P, I, I, I, I, I, I, I, I, S], c_int),
    "dfx_radon_backward_spdhg_bf16": ([P, L, P, I, I, I, I, I, I, I, I, P, P, P, F, F, P, S], c_int),
    "dfx_radon_backward_spdhg_tc": ([P, L, P, I, I, I, I, I, I, I, I, P, P, P, F, F, P, S], c_int),
    "dfx_convert_rows": ([I, P, L, P, L, L, I, S], c_int),
    "dfx_radon_forward_tc": ([P, P, L, I, P, I, I, I, I, I, I, I, F, P, I, S], c_int),
    "dfx_radon_tc_weights_bytes": ([I, I, I], c_int64),
    "dfx_radon_tc_weights": ([P, I, I, I, I, I, I, P, P, S], c_int),
    "dfx_radon_forward_tc_table": ([P, P, L, I, P, P, P, I, I, I, I, I, F, P, I, S], c_int),
    "dfx_radon_table_count": ([P, I, I, I, I, I, P, P, S], c_int),
    "dfx_radon_table_fill": ([P, I, I, I, I, I, P, P, P, S], c_int),
    "dfx_radon_forward_table": ([P, P, P, P, P, I, I, I, I, F, S], c_int),
    "dfx_radon_gtable_count": ([P, I, I, I, I, I, P, P, S], c_int),
    "dfx_radon_gtable_fill": ([P, I, I, I, I, I, P, P, P, P, S], c_int),
    "dfx_radon_forward_gtable": ([P, P, P, P, P, P, I, I, I, I, F, S], c_int),
    "dfx_radon_forward_table_bf16": ([P, P, L, P, P, P, I, I, I, I, F, S], c_int),
    "dfx_radon_forward_table_bf16_bf16": ([P, P, L, P, P, P, I, I, I, I, F, S], c_int),
    "dfx_batch_support": ([P, P, P, L, I, I, F, I, S], c_int),
    "dfx_pf_dense": ([POINTER(PFGeometry), I, I, P, S], c_int),
    "dfx_pf_csr_count": ([POINTER(PFGeometry), P, I, I, I, I, P, S], c_int),
    "dfx_pf_csr_fill": ([POINTER(PFGeometry), P, I, I, I, I, P, P, P, S], c_int),
    "dfx_scan_scratch_bytes": ([L], c_size_t),
    "dfx_scan_exclusive_i32": ([P, P, L, P, c_size_t, S], c_int),
    "dfx_scan_exclusive_i32_static": ([P, P, L, S], c_int),
    "dfx_spmm_pf_forward": ([P, P, P, P, P, P, I, I, I, I, I, I, S], c_int),
    "dfx_spmm_pf_adjoint": ([P, P, P, P, P, P, I, I, I, I, I, F, I, S], c_int),
    "dfx_pf_dense_products": ([I, P, I, I, I, P, P, I, I, F, S], c_int),
    "dfx_pf_fblock_rows": ([I, I, I], c_int64),
    "dfx_pf_fblock_count": ([P, P, I, I, I, P, P, S], c_int),
    "dfx_pf_fblock_fill": ([P, P, P, I, I, I, P, P, P, S], c_int),
    "dfx_spmm_pf_forward_blocked": ([P, P, P, P, P, P, P, I, I, I, I, I, I, S], c_int),
    "dfx_spmm_pf_forward_zt_floats": ([I, I, I], c_int64),
    "dfx_spmm_pf_forward_blocked_zt": ([P, P, L, P, P, P, P, P, P, I, I, I, I, I, I, I, S], c_int),
    "dfx_spmm_pf_adjoint_zt_floats": ([I, I, I], c_int64),
    "dfx_spmm_pf_adjoint_zt": ([P, P, L, P, P, P, P, P, I, I, I, I, I, F, I, I, S], c_int),
    "dfx_zero_rows": ([P, P, I, L, S], c_int),
    "dfx_fill_f32": ([P, F, L, S], c_int),
    "dfx_spdhg_dual_update": ([P, P, P, P, P, L, P, L, P, L, F, P, I, L, S], c_int),
    "dfx_spdhg_primal_update": ([P, P, P, P, F, F, L, S], c_int),
    "dfx_spdhg_primal_update_t16": ([P, P, P, P, F, F, L, S], c_int),
    "dfx_f32_to_bf16_rz": ([P, P, L, S], c_int),
    "dfx_dual_steps": ([P, P, P, L, F, L, S], c_int),
    "dfx_set_mask_ones": ([P, P, L, L, S], c_int),
    "dfx_tinit": ([P, L, S], c_int),
    "dfx_tmin": ([P, P, P, L, F, L, S], c_int),
    "dfx_tfinal": ([P, L, S], c_int),
    "dfx_support_ones": ([P, P, L, L, S], c_int),
    "dfx_project_support": ([P, P, L, L, S], c_int),
    "dfx_reduce_scratch_bytes": ([L], c_size_t),
    "dfx_poisson_value_grad": ([P, P, P, L, P, L, P, L, F, I, I, F, L, P, P, c_size_t, S], c_int),
    "dfx_mean_counted": ([P, P, L, L, P, P, c_size_t, S], c_int),
    "dfx_dot_f64": ([P, P, L, P, P, c_size_t, S], c_int),
    "dfx_ls_residual": ([P, P, P, L, I, F, L, P, P, c_size_t, S], c_int),
    "dfx_fista_ls_blocks": ([], c_int),
    "dfx_fista_ls_update": ([P, P, P, P, L, I, I, F, F, F, I, P, S], c_int),
    "dfx_sum_partials": ([P, I, I, P, S], c_int),
    "dfx_score_z": ([P, P, P, L, S], c_int),
    "dfx_local_scatter": ([P, P, P, P, P, I, I, I, I, P, P, S], c_int),
    "dfx_local_gather": ([P, P, P, P, P, I, I, I, I, P, P, S], c_int),
    "dfx_poisson_term": ([P, P, P, L, P, L, P, L, F, F, I, P, P, L, S], c_int),
    "dfx_osem_update": ([P, P, P, P, L, F, L, S], c_int),
    "dfx_tv_dual_local": ([P, P, P, P, P, P, P, P, F, F, L, S], c_int),
    "dfx_tv_adjoint_update_local": ([P, P, P, P, P, P, P, F, F, L, S], c_int),
    "dfx_tv_value_local": ([P, P, P, P, L, P, P, c_size_t, S], c_int),
    "dfx_tv_adjoint_local": ([P, P, P, P, P, L, S], c_int),
    "dfx_tree_sums": ([P, P, P, P, L, S], c_int),
    "dfx_tree_scatter": ([P, P, P, L, S], c_int),
    "dfx_pdhg_dual_update": ([P, P, P, P, P, L, P, L, P, L, F, L, S], c_int),
    "dfx_pdhg_primal_update": ([P, P, P, P, F, L, S], c_int),
    "dfx_pdhg_average": ([P, P, L, S], c_int),
    "dfx_pdhg_primal_steps": ([P, P, P, L, F, L, S], c_int),
    "dfx_tv_dual": ([P, P, P, P, P, P, I, I, I, F, F, S], c_int),
    "dfx_tv_adjoint_update": ([P, P, P, P, P, I, I, I, F, F, S], c_int),
    "dfx_tv_value": ([P, P, I, I, I, P, P, c_size_t, S], c_int),
    "dfx_pf_param_nq": ([I, I], c_int),
    "dfx_pf_param_vjp": ([POINTER(PFGeometry), P, P, P, P, P, I, I, I, I, I, P, P, P, P, P, P, I, P, S], c_int),
    "dfx_pf_rows_sum": ([P, I, I, I, P, S], c_int),
    "dfx_radon_dtable_fill": ([P, I, I, I, I, I, P, P, S], c_int),
    "dfx_angle_dot": ([P, P, I, I, I, I, P, S], c_int),
    "dfx_fr_scratch_bytes": ([P, I], c_size_t),
    "dfx_fr_forward": ([P, P, P, I, I, I, P, c_size_t, S], c_int),
    "dfx_fr_backward": ([P, P, P, I, I, I, P, c_size_t, S], c_int),
    "dfx_times_curvature": ([P, P, P, P, L, P, L, P, L, F, I, L, P, P, c_size_t, S], c_int),
    "dfx_support_sum": ([P, P, L, L, P, P, c_size_t, S], c_int),
    "dfx_weighted_sums": ([P, P, P, L, L, P, P, c_size_t, S], c_int),
    "dfx_step_sums": ([P, P, P, P, L, P, P, c_size_t, S], c_int),
    "dfx_invert_metric": ([P, P, P, L, L, S], c_int),
    "dfx_metric_step": ([P, P, P, P, F, F, L, S], c_int),
    "dfx_extrapolate": ([P, P, P, F, L, S], c_int),
    "dfx_copy_f32": ([P, P, L, S], c_int),
    "dfx_scale_f32": ([P, F, L, S], c_int),
    "dfx_pf_dense_bf16": ([POINTER(PFGeometry), I, I, L, L, I, P, S], c_int),
    "dfx_pf_dense_bf16_rows": ([POINTER(PFGeometry), P, I, I, I, L, L, I, P, S], c_int),
    "dfx_pf_tc_forward": ([P, L, L, L, I, I, I, P, P, I, I, P, I, I, S], c_int),
    "dfx_pf_tc_adjoint": ([P, L, L, L, I, I, I, P, P, I, I, F, P, I, S], c_int),
    "dfx_tc_status": ([POINTER(ctypes.c_uint), I], c_int),
    "dfx_rows_to_bf16": ([P, P, P, I, I, I, I, S], c_int),
    "dfx_f32_to_bf16": ([P, P, L, S], c_int),
}

_lib = None


def lib():
    """The loaded library (ImportError if it is missing or does not export the ABI)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"the CUDA library {LIB_PATH} is missing: build it with `python -m diffractom_b200.build`")
    try:
        h = ctypes.CDLL(str(LIB_PATH))
    except OSError as e:
        raise ImportError(f"cannot load {LIB_PATH}: {e}") from e
    for name, (args, res) in SIGNATURES.items():
        f = getattr(h, name, None)
        if f is None:
            raise ImportError(f"{LIB_PATH} does not export {name}")
        f.argtypes = args
        f.restype = res
    if h.dfx_abi_version() != ABI_VERSION:
        raise ImportError(f"{LIB_PATH}: ABI version {h.dfx_abi_version()}, expected {ABI_VERSION}")
    _lib = h
    return h


_EXC = {DFX_EINVAL: ValueError, DFX_ENOMEM: MemoryError, DFX_ELAUNCH: RuntimeError, DFX_ETIMEOUT: TimeoutError,
        DFX_ECUDA: RuntimeError}


def check(status: int) -> None:
    if status != DFX_OK:
        msg = lib().dfx_last_error().decode(errors="replace")
        raise _EXC.get(status, RuntimeError)(msg or f"diffractom_b200 error {status}")


def call(name: str, *args) -> None:
    """Call an entry point that returns a status; raise on error."""
    check(getattr(lib(), name)(*args))
