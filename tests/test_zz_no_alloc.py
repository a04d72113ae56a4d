"""The allocation-free forward + loss entry point, called through the C ABI.

ptycho_forward_loss_noalloc exists for callers that cannot allocate device
memory (their memory is owned by another framework's allocator, or allocation
is not allowed where they run): it keeps its per-CTA loss partials in a static
device array of the library instead of a caller buffer.  This test checks that
two calls in a row give the same intensities and loss as the allocating entry
point (ptycho_forward_loss + ptycho_reduce_loss), within the forward tolerance
of the other GPU tests, and that a grid above the array's size is rejected.
It is collected last so a stop-at-first-failure run has run everything else.
"""
import ctypes

import numpy as np
import pytest
import torch

from tests.conftest import load_golden, rel

pytestmark = pytest.mark.gpu

TOL_I = 1e-5


def test_forward_loss_noalloc_matches_allocating_entry_point(cuda_device):
    from quantem_b200 import _lib, ops

    dev = cuda_device
    z = load_golden("mixed128")
    n = int(z["H"])
    t = lambda x, dt=None: torch.as_tensor(np.ascontiguousarray(x), device=dev, dtype=dt)  # noqa: E731
    obj_c, _ = ops.obj_constrain(t(z["obj_perturbed"]))
    probe_o = t(z["probe_ortho"])
    prop = t(z["propagators"])
    positions = t(z["positions"], torch.float32)
    targets = t(z["targets"], torch.float32)
    mask = torch.ones((n, n), device=dev, dtype=torch.float32)
    bidx = t(z["batch_indices"].astype(np.int64))
    npos, mean_i = int(z["positions"].shape[0]), float(z["mean_intensity"])

    ref = ops.batch_forward(obj_c, probe_o, prop, positions, bidx, targets, mask, npos, mean_i)
    ref_i = ref["intensity"].cpu().numpy()
    ref_loss = ref["loss"].item()

    probe_hat = ops.fft2(probe_o)
    geom = ops.BatchGeometry.of(obj_c, probe_o, npos)
    B = int(bidx.numel())
    lib = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        out_i = torch.full((B, n, n), float("nan"), device=dev)
        out_loss = torch.full((1,), float("nan"), device=dev)
        a = _lib.BatchArgs()
        a.obj, a.probe_hat, a.prop = obj_c.data_ptr(), probe_hat.data_ptr(), prop.data_ptr()
        a.positions, a.batch_idx = positions.data_ptr(), bidx.data_ptr()
        a.targets, a.mask = targets.data_ptr(), mask.data_ptr()
        a.loss_part = None  # ignored: the partials live in the library's static array
        a.out_intensity = out_i.data_ptr()
        a.n, a.S, a.P, a.B = geom.n, geom.S, geom.P, B
        a.Ho, a.Wo, a.npos = geom.Ho, geom.Wo, npos
        grid = ctypes.c_int(0)
        _lib.check(lib.ptycho_batch_plan(ctypes.byref(a), 0, None, ctypes.byref(grid), None, None, None), "plan")
        a.grid = grid.value
        a.loss_type = _lib.LOSS_TYPES["l2_amplitude"]
        a.loss_scale = ops.loss_scale_of("l2_amplitude", B, npos, mean_i)
        a.inv_mean_intensity = 1.0 / mean_i
        _lib.check(lib.ptycho_forward_loss_noalloc(ctypes.byref(a), ctypes.c_void_p(out_loss.data_ptr()), stream),
                   "forward_loss_noalloc")
        torch.cuda.synchronize()
        assert rel(out_i.cpu().numpy(), ref_i) < TOL_I, f"call {call}"
        assert abs(out_loss.item() - ref_loss) / abs(ref_loss) < TOL_I, f"call {call}"

    a.grid = 1025  # above PTYCHO_NOALLOC_MAX_GRID
    rc = lib.ptycho_forward_loss_noalloc(ctypes.byref(a), ctypes.c_void_p(out_loss.data_ptr()), stream)
    assert rc == 1
    assert "PTYCHO_NOALLOC_MAX_GRID" in _lib.last_error()
