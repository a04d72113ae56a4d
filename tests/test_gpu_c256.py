"""256 x 256 probe windows: the cluster FFT and the cluster batch kernel (four
CTAs per position, distributed-shared-memory exchanges) against numpy / the FP64
oracle, with every slice's wave kept and with checkpoint + recompute in the
adjoint.  Tolerances as for 64 / 128: intensities 1e-5, gradients 1e-4."""
import numpy as np
import pytest
import torch

from oracle import ptycho_oracle as O
from tests.conftest import rel

pytestmark = pytest.mark.gpu

TOL_I = 1e-5
TOL_G = 1e-4


def _t(x, dev, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(x), device=dev, dtype=dtype)


@pytest.mark.parametrize("inverse", [False, True])
def test_fft256_matches_numpy(cuda_device, inverse):
    from quantem_b200 import ops

    rng = np.random.default_rng(3 + inverse)
    x = (rng.standard_normal((5, 256, 256)) + 1j * rng.standard_normal((5, 256, 256))).astype(np.complex64)
    got = ops.fft2(_t(x, cuda_device), inverse=inverse, scale=0.25).cpu().numpy()
    xd = x.astype(np.complex128)
    ref = (np.fft.ifft2(xd) * 256 * 256 if inverse else np.fft.fft2(xd)) * 0.25
    assert rel(got, ref) < 2e-6
    # in place
    xt = _t(x, cuda_device)
    ops.fft2(xt, inverse=inverse, scale=0.25, out=xt)
    assert rel(xt.cpu().numpy(), ref) < 2e-6


def _c5_like(rng, S=5, P=3, n=256, Ho=640, B=6):
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / 800.0)
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    positions = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    targets = np.abs(rng.standard_normal((B, n, n))) * 3
    return obj, probe, props, positions, targets


@pytest.mark.parametrize("recompute_every", [0, 1, 2, 3])
@pytest.mark.parametrize("separable", [False, True])
def test_c256_batch_matches_fp64_oracle(cuda_device, recompute_every, separable):
    """5 slices, 3 modes at 256^2 on a 640^2 object (the large multislice geometry,
    shortened): forward intensities, loss, object and probe gradients."""
    from quantem_b200 import ops

    rng = np.random.default_rng(11)
    obj, probe, props, positions, targets = _c5_like(rng)
    dev = cuda_device
    B, npos, mean_i, n = positions.shape[0], 16384, 50.0, 256
    obj_c = O.constrain_object(obj)
    loss_o, g_obj_o, g_probe_o, st = O.batch_loss_and_grads(obj_c, probe, positions, props, targets,
                                                            np.ones((n, n)), npos, mean_i)
    pos_full = np.zeros((npos, 2))
    pos_full[:B] = positions
    tg_full = np.zeros((B, n, n))
    tg_full[:B] = targets
    if separable:
        prop = ops.separable_propagators(n, (0.2, 0.2), 300e3, [20.0] * (obj.shape[0] - 1), device=dev)
    else:
        prop = _t(props.astype(np.complex64), dev)
    # targets only for the batch's own indices 0..B-1 (npos counts the full scan for the loss scale)
    args = (_t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev), prop,
            _t(pos_full[:B], dev, torch.float32), torch.arange(B, device=dev, dtype=torch.int64),
            _t(tg_full, dev, torch.float32), torch.ones((n, n), device=dev), npos, mean_i)
    out = ops.batch_forward(*args)
    assert rel(out["intensity"].cpu().numpy(), O.detector_intensities(st)) < TOL_I
    loss, g_obj, g_probe = ops.batch_forward_adjoint(*args, recompute_every=recompute_every)
    assert abs(loss.item() - loss_o) / loss_o < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G


@pytest.mark.parametrize("S,P,recompute_every", [(1, 1, 0), (1, 2, 1), (3, 1, 2), (4, 2, 3)])
def test_c256_slice_and_mode_counts(cuda_device, S, P, recompute_every):
    """Single-slice and single-mode 256^2 batches, and checkpoint intervals that do not
    divide the slice count: loss and gradients against the FP64 oracle."""
    from quantem_b200 import ops

    rng = np.random.default_rng(100 + 10 * S + P)
    n, Ho, B, npos, mean_i = 256, 384, 3, 64, 20.0
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / 800.0)
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    pos = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    targets = np.abs(rng.standard_normal((B, n, n))) * 3
    obj_c = O.constrain_object(obj)
    loss_o, g_obj_o, g_probe_o, _ = O.batch_loss_and_grads(obj_c, probe, pos, props, targets, np.ones((n, n)),
                                                           npos, mean_i)
    dev = cuda_device
    prop = _t(props.astype(np.complex64), dev) if S > 1 else torch.zeros((0, n, n), dtype=torch.complex64,
                                                                           device=dev)
    loss, g_obj, g_probe = ops.batch_forward_adjoint(
        _t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev), prop, _t(pos, dev, torch.float32),
        torch.arange(B, device=dev, dtype=torch.int64), _t(targets, dev, torch.float32), torch.ones((n, n), device=dev),
        npos, mean_i, recompute_every=recompute_every)
    assert abs(loss.item() - loss_o) / abs(loss_o) < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G
