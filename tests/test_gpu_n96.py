"""96 x 96 probe windows (mixed-radix 3 x 2^k register FFT engine, 192-thread CTAs):
FFT against numpy and the fused batch kernel against the FP64 oracle."""
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
def test_fft96_matches_numpy(cuda_device, inverse):
    from quantem_b200 import ops

    rng = np.random.default_rng(9 + inverse)
    x = (rng.standard_normal((7, 96, 96)) + 1j * rng.standard_normal((7, 96, 96))).astype(np.complex64)
    got = ops.fft2(_t(x, cuda_device), inverse=inverse, scale=0.5).cpu().numpy()
    xd = x.astype(np.complex128)
    ref = (np.fft.ifft2(xd) * 96 * 96 if inverse else np.fft.fft2(xd)) * 0.5
    assert rel(got, ref) < 2e-6


@pytest.mark.parametrize("separable", [False, True])
def test_n96_batch_matches_fp64_oracle(cuda_device, separable):
    from quantem_b200 import ops

    rng = np.random.default_rng(21)
    S, P, n, Ho, B = 4, 3, 96, 300, 7
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / 150.0)
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    positions = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    targets = np.abs(rng.standard_normal((B, n, n))) * 3
    npos, mean_i = 1024, 40.0
    obj_c = O.constrain_object(obj)
    loss_o, g_obj_o, g_probe_o, st = O.batch_loss_and_grads(obj_c, probe, positions, props, targets,
                                                            np.ones((n, n)), npos, mean_i)
    dev = cuda_device
    prop = (ops.separable_propagators(n, (0.2, 0.2), 300e3, [20.0] * (S - 1), device=dev) if separable
            else _t(props.astype(np.complex64), dev))
    args = (_t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev), prop,
            _t(positions, dev, torch.float32), torch.arange(B, device=dev, dtype=torch.int64),
            _t(targets, dev, torch.float32), torch.ones((n, n), device=dev), npos, mean_i)
    out = ops.batch_forward(*args)
    assert rel(out["intensity"].cpu().numpy(), O.detector_intensities(st)) < TOL_I
    loss, g_obj, g_probe = ops.batch_forward_adjoint(*args)
    assert abs(loss.item() - loss_o) / loss_o < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G
