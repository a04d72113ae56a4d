"""The C ABI library loads and exports every symbol include/ptycho_b200.h declares
(no GPU needed: nothing here launches work)."""
import ctypes
import os
import re

from tests.conftest import ROOT


def _declared():
    txt = open(os.path.join(ROOT, "include", "ptycho_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|int64_t)\s+(ptycho_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from quantem_b200 import _lib

    lib = _lib.lib()
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(_lib.EXPORTED) == names


def test_host_side_validation_without_gpu():
    from quantem_b200 import _lib

    lib = _lib.lib()
    assert lib.ptycho_abi_version() >= 1
    # NULL arguments are rejected before any CUDA call, with a message
    assert lib.ptycho_forward_loss(None, None) == 1
    assert "NULL" in _lib.last_error()
    a = _lib.BatchArgs()
    a.n = 80
    assert lib.ptycho_forward_adjoint(ctypes.byref(a), None) == 2  # 80 x 80 window not built
    assert "80" in _lib.last_error()
    a.n, a.recompute_every, a.S = 256, 5, 3
    assert lib.ptycho_forward_adjoint(ctypes.byref(a), None) == 1  # checkpoint interval beyond S
    a.recompute_every = 0
    a.n, a.S, a.P, a.B, a.Ho, a.Wo, a.npos = 128, 2, 1, 4, 64, 64, 4
    assert lib.ptycho_forward_loss(ctypes.byref(a), None) == 1      # missing pointers
    assert lib.ptycho_reduce_loss(None, 1, None, None) == 1
    assert lib.ptycho_fft2(None, None, 1, 128, 0, 1.0, None) == 1
    # probe orthogonalisation: mode count and work size are checked before the launch
    dummy = ctypes.c_void_p(16)  # never dereferenced: the calls fail validation
    we = lib.ptycho_probe_ortho_work_elems(4, 128 * 128)
    assert we >= 2 * 4 * 128 * 128
    assert lib.ptycho_probe_orthogonalize(dummy, dummy, 17, 128 * 128, dummy, we, None) == 1
    assert "P <= 16" in _lib.last_error()
    assert lib.ptycho_probe_orthogonalize(dummy, ctypes.c_void_p(32), 4, 128 * 128, dummy, we - 1, None) == 1
    assert "work" in _lib.last_error()
    assert lib.ptycho_probe_orthogonalize(dummy, dummy, 4, 128 * 128, ctypes.c_void_p(64), we, None) == 1
    assert "alias" in _lib.last_error()
    assert lib.ptycho_probe_orthogonalize_vjp(None, dummy, dummy, 4, 128 * 128, dummy, we, None) == 1
    # the gradient output must not alias any input of the VJP
    a1, a2, a3 = ctypes.c_void_p(16), ctypes.c_void_p(48), ctypes.c_void_p(80)
    for gp in (a1, a2, a3):  # grad_probe == probe, == grad_sorted, == work
        assert lib.ptycho_probe_orthogonalize_vjp(a1, a2, gp, 4, 128 * 128, a3, we, None) == 1
        assert "alias" in _lib.last_error()
    buf = ctypes.create_string_buffer(8)
    assert lib.ptycho_get_last_error(buf, 8) == 0 and len(buf.value) <= 7


def test_product_has_no_cpu_fallback():
    """Compute entry points refuse CPU tensors instead of computing elsewhere."""
    import pytest
    import torch

    from quantem_b200 import ops

    x = torch.zeros((1, 64, 64), dtype=torch.complex64)
    with pytest.raises(RuntimeError, match="CUDA"):
        ops.fft2(x)
    with pytest.raises(RuntimeError, match="CUDA"):
        ops.obj_constrain(x)


def test_extension_arguments_are_validated_without_gpu():
    """Descan shifts and the descan / propagator gradients (ABI 3): rejected, before any
    CUDA call, where they are not built or are inconsistent."""
    from quantem_b200 import _lib

    lib = _lib.lib()
    assert lib.ptycho_abi_version() >= 3
    a = _lib.BatchArgs()
    d = ctypes.c_void_p(256)  # never dereferenced: every call below fails validation
    for f in ("obj", "probe_hat", "prop", "positions", "batch_idx", "targets", "mask", "loss_part", "grad_obj",
              "probe_grad_part", "scratch"):
        setattr(a, f, d)
    a.n, a.S, a.P, a.B, a.Ho, a.Wo, a.npos, a.grid = 128, 3, 2, 4, 256, 256, 4, 4
    a.grad_descan = d
    assert lib.ptycho_forward_adjoint(ctypes.byref(a), None) == 1  # grad_descan without descan
    assert "descan" in _lib.last_error()
    a.descan = d
    assert lib.ptycho_forward_loss(ctypes.byref(a), None) == 2     # gradients need the adjoint launch
    a.grad_descan = None
    a.grad_prop, a.S = d, 18
    assert lib.ptycho_forward_adjoint(ctypes.byref(a), None) == 2  # propagator gradients up to 17 slices
    assert "17" in _lib.last_error()
    a.grad_prop, a.S = None, 3
    a.analytic, a.an_norm = 1, d
    assert lib.ptycho_forward_adjoint(ctypes.byref(a), None) == 2  # descan with the analytic update
    a.analytic, a.an_norm = 0, None
    a.n = 256
    assert lib.ptycho_forward_loss(ctypes.byref(a), None) == 2     # not built for 256 x 256 windows
    assert "256" in _lib.last_error()
    sets = (_lib.BatchArgs * 1)(a)
    sets[0].n = 128
    assert lib.ptycho_forward_adjoint_multi(sets, 1, None) == 2    # not in the multi-dataset launch
    assert "multi" in _lib.last_error()


def test_lazy_conjugate_views_are_rejected_or_resolved():
    """Kernels read raw memory: a lazily conjugated tensor (autograd hands complex
    gradients in that form) is either resolved by ops.dense or refused by the argument
    checks, never read with its conjugate bit dropped."""
    import pytest
    import torch

    from quantem_b200 import ops

    z = torch.tensor([1 + 2j, 3 - 1j], dtype=torch.complex64)
    with pytest.raises(ValueError, match="conjugate"):
        ops._req(z.conj(), "x", torch.complex64)
    d = ops.dense(z.conj())
    assert not d.is_conj() and torch.equal(d, torch.tensor([1 - 2j, 3 + 1j], dtype=torch.complex64))


def test_new_entry_points_validate_arguments_without_gpu():
    """Probe constraints, bilinear centring, AMSGrad / momentum steps, dropout and the GEMM
    activation flags: bad arguments are rejected before any CUDA call."""
    from quantem_b200 import _lib

    lib = _lib.lib()
    d = ctypes.c_void_p(256)  # never dereferenced: every call below fails validation
    assert lib.ptycho_probe_center_work_elems(2, 64) == 2 * 2 * 64 * 64 + 6 * 16
    assert lib.ptycho_probe_center(d, d, 17, 64, ctypes.c_void_p(512), 10 ** 9, None) == 1   # P <= 16
    assert lib.ptycho_probe_center(d, d, 2, 100, ctypes.c_void_p(512), 10 ** 9, None) == 2   # n not built
    assert lib.ptycho_probe_center(d, d, 2, 64, ctypes.c_void_p(512), 10, None) == 1         # work too small
    assert lib.ptycho_probe_center(d, d, 2, 64, ctypes.c_void_p(512), 10 ** 9, None) == 1    # out aliases probe
    assert lib.ptycho_probe_center_vjp(d, ctypes.c_void_p(512), d, 2, 64, ctypes.c_void_p(768), 10 ** 9,
                                       None) == 1                                             # grad aliases probe
    nw = lib.ptycho_probe_tv_work_elems()
    assert lib.ptycho_probe_tv(d, 2, 64, ctypes.c_float(0.1), ctypes.c_void_p(512), None, ctypes.c_void_p(768),
                               nw - 1, None) == 1                                             # work too small
    assert lib.ptycho_probe_tv(d, 2, 64, ctypes.c_float(0.1), ctypes.c_void_p(512), d, ctypes.c_void_p(768), nw,
                               None) == 1                                                     # grad aliases probe
    assert lib.ptycho_pattern_bilinear(d, ctypes.c_void_p(512), 4, 63, ctypes.c_void_p(768), None, None) == 1  # odd n
    assert lib.ptycho_pattern_bilinear(d, ctypes.c_void_p(512), 4, 64, d, None, None) == 1   # output aliases input
    assert lib.ptycho_adam_amsgrad_step(d, d, d, d, None, 10, ctypes.c_float(1e-3), None, ctypes.c_float(0.9),
                                        ctypes.c_float(0.999), ctypes.c_float(1e-8), ctypes.c_float(0), 0,
                                        ctypes.c_float(0.1), ctypes.c_float(0.1), None) == 1  # no max buffer
    assert lib.ptycho_sgd_momentum_step(d, d, None, 10, ctypes.c_float(0.1), None, ctypes.c_float(0),
                                        ctypes.c_float(0.9), ctypes.c_float(0), 0, 1, None) == 1  # no buffer
    assert lib.ptycho_cnn_dropout(d, 0, 4, 4, 4, ctypes.c_float(1.5), ctypes.c_uint64(1), None) == 1  # p > 1
    assert lib.ptycho_cnn_dropout(d, 2, 4, 4, 4, ctypes.c_float(0.5), ctypes.c_uint64(1), None) == 1  # dtype
    flags = 1 | (9 << 8)  # BF16 output with an activation id that does not exist
    assert lib.ptycho_gemm_bf16(d, 64, d, 64, d, 64, 128, 64, 64, None, flags, 1, None, None) == 1
    assert "activation" in _lib.last_error()
    assert lib.ptycho_gemm_bf16(d, 64, d, 64, d, 64, 128, 64, 64, None, 4 | (4 << 8), 1, None, None) == 1
    assert "atomic" in _lib.last_error()
    for act in (-1, 7):  # activation ids of the batch-norm backward: 0 .. 6
        assert lib.ptycho_cnn_bn_backward(d, 8, d, 8, 16, 8, None, None, None, 1, act, None, None, None, 0, d, None, 8,
                                          None) == 1
