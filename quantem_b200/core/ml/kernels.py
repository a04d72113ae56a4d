"""Torch-facing wrappers of the CNN kernels of libptycho_b200 (C ABI).

Tensors are CUDA tensors; 2-D views may be strided along their first dimension
(leading dimension = ``t.stride(0)``) but must be contiguous along the second,
so channel slices of a wider channels-last buffer are passed without copies.
Every call raises ``RuntimeError`` with the library's message on failure; there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes

import torch

from ... import _lib

GEMM_BF16 = 1
GEMM_RELU = 2
GEMM_ATOMIC = 4
# activation ids of the GEMM epilogue and the batch-norm backward (core/ml/activation_functions.py:
# 166-181, torch's default parameters); 0 = identity
ACT_IDS = {"identity": 0, "eye": 0, "ident": 0, "relu": 1, "leaky_relu": 2, "leakyrelu": 2, "lrelu": 2, "elu": 3,
           "tanh": 4, "sigmoid": 5, "softplus": 6}

_F32, _BF16 = 0, 1


def _s():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _ld(t: torch.Tensor, name: str) -> int:
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor (the B200 path has no CPU fallback)")
    if t.dim() != 2 or t.stride(1) != 1:
        raise ValueError(f"{name} must be a 2-D view contiguous along its last dimension")
    return int(t.stride(0))


def _dt(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _F32
    if t.dtype == torch.bfloat16:
        return _BF16
    raise TypeError(f"unsupported dtype {t.dtype}")


def _call(name: str, *args):
    _lib.check(getattr(_lib.lib(), name)(*args), name)


def gemm(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, bias: torch.Tensor | None = None, relu: bool = False,
         splits: int = 1, status: torch.Tensor | None = None, accumulate: bool = False, act: int = 0) -> torch.Tensor:
    """C (op)= A @ B.T (+ bias) (activation) on the tcgen05 tensor cores.

    A (M, K) and B (N, K) are BF16; C (M, N) is FP32 or BF16.  splits > 1
    splits K over CTAs with FP32 atomics (C is cleared first); accumulate=True
    adds into FP32 C atomically without clearing it.  ``act`` is an activation id
    (``ACT_IDS``); ``relu=True`` is act 1."""
    if A.dtype != torch.bfloat16 or B.dtype != torch.bfloat16:
        raise TypeError("gemm operands must be bfloat16")
    M, K = A.shape
    N, K2 = B.shape
    if K2 != K or tuple(C.shape) != (M, N):
        raise ValueError(f"gemm shapes: A {tuple(A.shape)}, B {tuple(B.shape)}, C {tuple(C.shape)}")
    flags = (GEMM_BF16 if C.dtype == torch.bfloat16 else 0) | (GEMM_RELU if relu else (int(act) << 8)) | \
        (GEMM_ATOMIC if accumulate else 0)
    _call("ptycho_gemm_bf16", _p(A), _ld(A, "A"), _p(B), _ld(B, "B"), _p(C), _ld(C, "C"), M, N, K, _p(bias), flags,
          int(splits), _p(status), _s())
    return C


def im2col3x3(x: torch.Tensor, B: int, H: int, W: int, col: torch.Tensor) -> torch.Tensor:
    C = x.shape[1]
    _call("ptycho_cnn_im2col3x3", _p(x), B, H, W, C, _ld(x, "x"), _p(col), _ld(col, "col"), _s())
    return col


def col2im3x3(dcol: torch.Tensor, B: int, H: int, W: int, C: int, dx: torch.Tensor, accumulate: bool = False):
    _call("ptycho_cnn_col2im3x3", _p(dcol), _ld(dcol, "dcol"), B, H, W, C, _p(dx), _ld(dx, "dx"), int(accumulate),
          _s())
    return dx


def convT_gather(colT: torch.Tensor, B: int, H: int, W: int, Co: int, bias, out: torch.Tensor):
    _call("ptycho_cnn_convT_gather", _p(colT), _ld(colT, "colT"), B, H, W, Co, _p(bias), _p(out), _ld(out, "out"),
          _s())
    return out


def convT_im2col(dout: torch.Tensor, B: int, H: int, W: int, Co: int, dcol: torch.Tensor):
    _call("ptycho_cnn_convT_im2col", _p(dout), _ld(dout, "dout"), B, H, W, Co, _p(dcol), _ld(dcol, "dcol"), _s())
    return dcol


def transpose(x: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
    """out (C, R) = x (R, C).T, also 3-D batched (Z, R, C) -> (Z, C, R) for contiguous tensors."""
    if x.dim() == 3:
        Z, R, C = x.shape
        if not (x.is_contiguous() and out.is_contiguous() and tuple(out.shape) == (Z, C, R)):
            raise ValueError("batched transpose needs contiguous (Z, R, C) -> (Z, C, R)")
        _call("ptycho_cnn_transpose", _p(x), _dt(x), R, C, C, R * C, _p(out), _dt(out), R, R * C, Z, _s())
        return out
    R, C = x.shape
    if tuple(out.shape) != (C, R):
        raise ValueError("transpose: out must be (C, R)")
    _call("ptycho_cnn_transpose", _p(x), _dt(x), R, C, _ld(x, "x"), 0, _p(out), _dt(out), _ld(out, "out"), 0, 1,
          _s())
    return out


def bn_forward(x, gamma, beta, run_mean, run_var, momentum, eps, training, mean, rstd, work, out):
    R, C = x.shape
    _call("ptycho_cnn_bn_forward", _p(x), _ld(x, "x"), R, C, _p(gamma), _p(beta), _p(run_mean), _p(run_var),
          ctypes.c_float(momentum), ctypes.c_float(eps), int(training), _p(mean), _p(rstd), _p(work), work.numel(),
          _p(out), _ld(out, "out"), _s())
    return out


def bn_backward(dy, x, gamma, mean, rstd, training, act, dgamma, dbeta, work, dz32=None, dz16=None):
    """Batch-norm backward (gamma given) times the derivative of activation ``act`` (an id of
    ``ACT_IDS``; True is ReLU) evaluated from its output x."""
    R, C = x.shape
    z = dz32 if dz32 is not None else dz16
    if dz32 is not None and dz16 is not None and dz32.stride(0) != dz16.stride(0):
        raise ValueError("dz32 and dz16 must share a leading dimension")
    _call("ptycho_cnn_bn_backward", _p(dy), _ld(dy, "dy"), _p(x), _ld(x, "x"), R, C, _p(gamma), _p(mean), _p(rstd),
          int(training), int(act), _p(dgamma), _p(dbeta), _p(work), work.numel(), _p(dz32), _p(dz16),
          _ld(z, "dz"), _s())


def dropout(x: torch.Tensor, p: float, seed: int) -> torch.Tensor:
    """x (R, C) FP32 or BF16, in place: keep / (1 - p) with the mask of ``seed``."""
    R, C = x.shape
    _call("ptycho_cnn_dropout", _p(x), _dt(x), R, C, _ld(x, "x"), ctypes.c_float(p),
          ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), _s())
    return x


def colsum(a: torch.Tensor, out: torch.Tensor, work: torch.Tensor, accumulate: bool = False):
    R, C = a.shape
    _call("ptycho_cnn_colsum", _p(a), _ld(a, "a"), R, C, _p(out), int(accumulate), _p(work), work.numel(), _s())
    return out


def maxpool2(x: torch.Tensor, B: int, H: int, W: int, out: torch.Tensor, argmax: torch.Tensor):
    C = x.shape[1]
    _call("ptycho_cnn_maxpool2", _p(x), _ld(x, "x"), B, H, W, C, _p(out), _ld(out, "out"), _p(argmax), _s())
    return out


def maxpool2_backward(dout, argmax, B, H, W, din, accumulate=False):
    C = dout.shape[1]
    _call("ptycho_cnn_maxpool2_backward", _p(dout), _ld(dout, "dout"), _p(argmax), B, H, W, C, _p(din),
          _ld(din, "din"), int(accumulate), _s())
    return din


def cast_bf16(x: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
    if not (x.is_contiguous() and out.is_contiguous()) or x.numel() != out.numel():
        raise ValueError("cast_bf16 needs contiguous tensors of equal size")
    _call("ptycho_cnn_cast_bf16", _p(x), _p(out), x.numel(), _s())
    return out


def mse(pred, target, loss, work, dpred32=None, dpred16=None):
    if not (pred.is_contiguous() and target.is_contiguous()) or pred.numel() != target.numel():
        raise ValueError("mse needs contiguous tensors of equal size")
    _call("ptycho_cnn_mse", _p(pred), _p(target), pred.numel(), _p(loss), _p(dpred32), _p(dpred16), _p(work),
          work.numel(), _s())
    return loss


def bin_features(patterns: torch.Tensor, bin: int, out: torch.Tensor, mean: torch.Tensor | None = None,
                 scale: float = 1.0, amplitudes: bool = False, norm: float = 1.0) -> torch.Tensor:
    """Rows (npos, (n/bin)^2) BF16 of sqrt-binned pattern features (see ptycho_cnn_bin_features)."""
    if patterns.dtype != torch.float32 or not patterns.is_contiguous() or patterns.dim() != 3:
        raise ValueError("patterns must be contiguous float32 (npos, n, n)")
    npos, n, _ = patterns.shape
    _call("ptycho_cnn_bin_features", _p(patterns), npos, n, int(bin), int(amplitudes), ctypes.c_float(norm),
          _p(mean), ctypes.c_float(scale), _p(out), _ld(out, "out"), _s())
    return out
