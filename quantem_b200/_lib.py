"""ctypes binding of libptycho_b200.so (the C ABI declared in include/ptycho_b200.h).

The library is loaded from ``quantem_b200/lib`` inside this source tree.  There
is no fallback: if the library is missing or cannot be loaded, every call raises
``RuntimeError`` with the reason.
"""
from __future__ import annotations

import ctypes
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libptycho_b200.so")

PTYCHO_OK = 0
VARIANTS = {"auto": 0, "serial": 1, "cluster": 2}
ERR_NAMES = {1: "invalid argument", 2: "unsupported configuration", 3: "CUDA error", 4: "non-finite values"}

LOSS_TYPES = {
    "l2_amplitude": 0,
    "l1_amplitude": 1,
    "l2_intensity": 2,
    "l1_intensity": 3,
    "poisson": 4,
}

# Every symbol include/ptycho_b200.h declares.
EXPORTED = (
    "ptycho_get_last_error",
    "ptycho_abi_version",
    "ptycho_sm_count",
    "ptycho_workspace_elems",
    "ptycho_batch_plan",
    "ptycho_forward_loss",
    "ptycho_forward_adjoint",
    "ptycho_forward_adjoint_multi",
    "ptycho_fft2",
    "ptycho_reduce_partials",
    "ptycho_reduce_loss",
    "ptycho_obj_constrain",
    "ptycho_obj_constrain_vjp",
    "ptycho_obj_transmission",
    "ptycho_obj_transmission_vjp",
    "ptycho_reduce_blocks",
    "ptycho_adam_step",
    "ptycho_sgd_step",
    "ptycho_adam_step_dev",
    "ptycho_add_scalar",
    "ptycho_patch_energy_max",
    "ptycho_analytic_obj_finalize",
    "ptycho_analytic_probe_finalize",
    "ptycho_fp32_fma_probe",
    "ptycho_forward_loss_noalloc",
    "ptycho_gemm_bf16",
    "ptycho_cnn_im2col3x3",
    "ptycho_cnn_col2im3x3",
    "ptycho_cnn_convT_gather",
    "ptycho_cnn_convT_im2col",
    "ptycho_cnn_transpose",
    "ptycho_cnn_bn_forward",
    "ptycho_cnn_bn_backward",
    "ptycho_cnn_colsum",
    "ptycho_cnn_maxpool2",
    "ptycho_cnn_maxpool2_backward",
    "ptycho_cnn_cast_bf16",
    "ptycho_cnn_mse",
    "ptycho_cnn_bin_features",
    "ptycho_pattern_com",
    "ptycho_pattern_prepare",
    "ptycho_pattern_shift_ramp",
    "ptycho_pattern_center",
    "ptycho_pattern_bilinear",
    "ptycho_adam_amsgrad_step",
    "ptycho_sgd_momentum_step",
    "ptycho_cnn_dropout",
    "ptycho_probe_ortho_work_elems",
    "ptycho_probe_orthogonalize",
    "ptycho_probe_orthogonalize_vjp",
    "ptycho_probe_center_work_elems",
    "ptycho_probe_center",
    "ptycho_probe_center_vjp",
    "ptycho_probe_tv_work_elems",
    "ptycho_probe_tv",
    "ptycho_obj_constraint_work_elems",
    "ptycho_probe_overlap",
    "ptycho_obj_constrain_fov",
    "ptycho_obj_constrain_fov_vjp",
    "ptycho_obj_potential_base",
    "ptycho_obj_potential_base_vjp",
    "ptycho_phase_exp",
    "ptycho_phase_exp_vjp",
    "ptycho_obj_blur",
    "ptycho_obj_slice_mean",
    "ptycho_obj_soft_loss",
    "ptycho_obj_butterworth",
    "ptycho_obj_butterworth_vjp",
)

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_flt = ctypes.c_float


class BatchArgs(ctypes.Structure):
    """Mirror of ``ptycho_batch_args``."""

    _fields_ = [
        ("obj", _vp), ("probe_hat", _vp), ("prop", _vp), ("positions", _vp), ("batch_idx", _vp),
        ("targets", _vp), ("mask", _vp), ("grad_obj", _vp), ("probe_grad_part", _vp),
        ("scratch", _vp), ("loss_part", _vp), ("out_intensity", _vp), ("out_exit", _vp),
        ("out_waves", _vp), ("status", _vp), ("prop_r", _vp), ("prop_c", _vp),
        ("n", _int), ("S", _int), ("P", _int), ("B", _int), ("Ho", _int), ("Wo", _int),
        ("npos", _int), ("grid", _int), ("loss_type", _int),
        ("loss_scale", _flt), ("inv_mean_intensity", _flt), ("variant", _int),
        ("analytic", _int), ("an_norm", _vp), ("recompute_every", _int), ("grad_positions", _vp),
        ("descan", _vp), ("grad_descan", _vp), ("grad_prop", _vp),
    ]


_lock = threading.Lock()
_lib = None


def _declare(lib):
    sig = {
        "ptycho_get_last_error": (_int, [ctypes.c_char_p, ctypes.c_size_t]),
        "ptycho_abi_version": (_int, []),
        "ptycho_sm_count": (_int, [ctypes.POINTER(_int)]),
        "ptycho_workspace_elems": (_int, [_int, _int, _int, _int, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
        "ptycho_batch_plan": (_int, [ctypes.POINTER(BatchArgs), _int, ctypes.POINTER(_int), ctypes.POINTER(_int),
                                     ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_int)]),
        "ptycho_forward_loss": (_int, [ctypes.POINTER(BatchArgs), _vp]),
        "ptycho_forward_adjoint": (_int, [ctypes.POINTER(BatchArgs), _vp]),
        "ptycho_forward_adjoint_multi": (_int, [_vp, _int, _vp]),
        "ptycho_adam_step_dev": (_int, [_vp, _vp, _vp, _vp, _i64, _vp, _vp, _flt, _flt, _flt, _flt, _int, _vp]),
        "ptycho_add_scalar": (_int, [_vp, _flt, _vp]),
        "ptycho_fft2": (_int, [_vp, _vp, _int, _int, _int, _flt, _vp]),
        "ptycho_reduce_partials": (_int, [_vp, _vp, _int, _i64, _vp]),
        "ptycho_reduce_loss": (_int, [_vp, _int, _vp, _vp]),
        "ptycho_obj_constrain": (_int, [_vp, _vp, _i64, _vp, _int, _vp]),
        "ptycho_obj_constrain_vjp": (_int, [_vp, _vp, _vp, _i64, _vp, _int, _vp, _vp]),
        "ptycho_obj_transmission": (_int, [_vp, _vp, _i64, _int, _int, _int, _flt, _vp, _int, _vp]),
        "ptycho_obj_transmission_vjp": (_int, [_vp, _vp, _vp, _i64, _int, _int, _int, _flt, _vp, _int, _vp, _vp]),
        "ptycho_reduce_blocks": (_int, []),
        "ptycho_adam_step": (_int, [_vp, _vp, _vp, _vp, _i64, _flt, _vp, _flt, _flt, _flt, _flt, _int, _flt, _flt,
                                    _vp]),
        "ptycho_sgd_step": (_int, [_vp, _vp, _i64, _flt, _vp, _flt, _vp]),
        "ptycho_fp32_fma_probe": (_int, [_vp, _int, _int, _vp]),
        "ptycho_patch_energy_max": (_int, [_vp, _vp, _vp, _int, _int, _int, _int, _int, _int, _vp, _vp]),
        "ptycho_analytic_obj_finalize": (_int, [_vp, _vp, _vp, _int, _int, _i64, _vp, _vp]),
        "ptycho_analytic_probe_finalize": (_int, [_vp, _i64, _vp, _flt, _vp]),
        "ptycho_forward_loss_noalloc": (_int, [ctypes.POINTER(BatchArgs), _vp, _vp]),
        "ptycho_gemm_bf16": (_int, [_vp, _int, _vp, _int, _vp, _int, _int, _int, _int, _vp, _int, _int, _vp, _vp]),
        "ptycho_cnn_im2col3x3": (_int, [_vp, _int, _int, _int, _int, _int, _vp, _int, _vp]),
        "ptycho_cnn_col2im3x3": (_int, [_vp, _int, _int, _int, _int, _int, _vp, _int, _int, _vp]),
        "ptycho_cnn_convT_gather": (_int, [_vp, _int, _int, _int, _int, _int, _vp, _vp, _int, _vp]),
        "ptycho_cnn_convT_im2col": (_int, [_vp, _int, _int, _int, _int, _int, _vp, _int, _vp]),
        "ptycho_cnn_transpose": (_int, [_vp, _int, _int, _int, _int, _i64, _vp, _int, _int, _i64, _int, _vp]),
        "ptycho_cnn_bn_forward": (_int, [_vp, _int, _int, _int, _vp, _vp, _vp, _vp, _flt, _flt, _int, _vp, _vp, _vp,
                                         _i64, _vp, _int, _vp]),
        "ptycho_cnn_bn_backward": (_int, [_vp, _int, _vp, _int, _int, _int, _vp, _vp, _vp, _int, _int, _vp, _vp,
                                          _vp, _i64, _vp, _vp, _int, _vp]),
        "ptycho_cnn_colsum": (_int, [_vp, _int, _int, _int, _vp, _int, _vp, _i64, _vp]),
        "ptycho_cnn_maxpool2": (_int, [_vp, _int, _int, _int, _int, _int, _vp, _int, _vp, _vp]),
        "ptycho_cnn_maxpool2_backward": (_int, [_vp, _int, _vp, _int, _int, _int, _int, _vp, _int, _int, _vp]),
        "ptycho_cnn_cast_bf16": (_int, [_vp, _vp, _i64, _vp]),
        "ptycho_cnn_mse": (_int, [_vp, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp]),
        "ptycho_cnn_bin_features": (_int, [_vp, _int, _int, _int, _int, _flt, _vp, _flt, _vp, _int, _vp]),
        "ptycho_pattern_com": (_int, [_vp, _vp, _int, _int, _int, _vp, _vp]),
        "ptycho_pattern_prepare": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp, _vp]),
        "ptycho_pattern_shift_ramp": (_int, [_vp, _vp, _int, _int, _vp]),
        "ptycho_pattern_center": (_int, [_vp, _int, _int, _flt, _vp, _vp, _vp]),
        "ptycho_pattern_bilinear": (_int, [_vp, _vp, _int, _int, _vp, _vp, _vp]),
        "ptycho_adam_amsgrad_step": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _flt, _vp, _flt, _flt, _flt, _flt, _int,
                                             _flt, _flt, _vp]),
        "ptycho_sgd_momentum_step": (_int, [_vp, _vp, _vp, _i64, _flt, _vp, _flt, _flt, _flt, _int, _int, _vp]),
        "ptycho_cnn_dropout": (_int, [_vp, _int, _int, _int, _int, _flt, ctypes.c_uint64, _vp]),
        "ptycho_probe_ortho_work_elems": (_i64, [_int, _i64]),
        "ptycho_probe_orthogonalize": (_int, [_vp, _vp, _int, _i64, _vp, _i64, _vp]),
        "ptycho_probe_orthogonalize_vjp": (_int, [_vp, _vp, _vp, _int, _i64, _vp, _i64, _vp]),
        "ptycho_probe_center_work_elems": (_i64, [_int, _int]),
        "ptycho_probe_center": (_int, [_vp, _vp, _int, _int, _vp, _i64, _vp]),
        "ptycho_probe_center_vjp": (_int, [_vp, _vp, _vp, _int, _int, _vp, _i64, _vp]),
        "ptycho_probe_tv_work_elems": (_int, []),
        "ptycho_probe_tv": (_int, [_vp, _int, _int, _flt, _vp, _vp, _vp, _int, _vp]),
        "ptycho_obj_constraint_work_elems": (_int, []),
        "ptycho_probe_overlap": (_int, [_vp, _int, _vp, _int, _int, _int, _vp, _vp]),
        "ptycho_obj_constrain_fov": (_int, [_vp, _vp, _i64, _vp, _i64, _int, _vp, _int, _vp]),
        "ptycho_obj_constrain_fov_vjp": (_int, [_vp, _vp, _i64, _vp, _vp, _i64, _int, _vp, _int, _vp]),
        "ptycho_obj_potential_base": (_int, [_vp, _vp, _vp, _i64, _vp, _i64, _int, _int, _flt, _vp, _int, _vp]),
        "ptycho_obj_potential_base_vjp": (_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i64, _int, _int, _flt, _vp, _int,
                                                 _vp]),
        "ptycho_phase_exp": (_int, [_vp, _vp, _i64, _vp]),
        "ptycho_phase_exp_vjp": (_int, [_vp, _vp, _vp, _i64, _vp]),
        "ptycho_obj_blur": (_int, [_vp, _vp, _vp, _int, _int, _int, _int, _vp, _int, _vp]),
        "ptycho_obj_slice_mean": (_int, [_vp, _vp, _int, _i64, _int, _vp]),
        "ptycho_obj_soft_loss": (_int, [_vp, _int, _int, _int, _int, _flt, _flt, _flt, _vp, _int, _vp, _vp, _vp]),
        "ptycho_obj_butterworth": (_int, [_vp, _vp, _int, _int, _int, _int, _vp, _vp, _vp, _vp]),
        "ptycho_obj_butterworth_vjp": (_int, [_vp, _vp, _int, _int, _int, _int, _vp, _vp, _vp, _vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def lib():
    """The loaded library; raises RuntimeError (never falls back) if unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"libptycho_b200.so not found at {LIB_PATH}; build it with "
                    "`python -m quantem_b200.build` (the CUDA path has no CPU fallback)")
            try:
                handle = ctypes.CDLL(LIB_PATH)
            except OSError as exc:  # pragma: no cover - depends on the machine
                raise RuntimeError(f"cannot load {LIB_PATH}: {exc}") from exc
            _declare(handle)
            _lib = handle
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    lib().ptycho_get_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = "") -> None:
    if rc != PTYCHO_OK:
        kind = ERR_NAMES.get(rc, f"status {rc}")
        raise RuntimeError(f"ptycho_b200 {what} failed ({kind}): {last_error()}")
