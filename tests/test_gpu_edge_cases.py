"""Edge cases of the fused batch kernels against the FP64 oracle: empty batches, one
position repeated inside a batch (its object-gradient scatters collide on the same
addresses), batches that repeat a position across the window sizes, and positions
exactly on the wrap-around seam of the object (periodic patch indices,
dataset_models.py:514-535).  Tolerances: loss 1e-5 relative, gradients 1e-4 relative L2."""
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


def _problem(n, S, P, Ho, seed):
    rng = np.random.default_rng(seed)
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / (n * 2.0))
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1)) if S > 1 else np.zeros((0, n, n))
    return rng, O.constrain_object(obj), probe, props


def _run(dev, obj_c, probe, props, positions, batch, targets, npos, mean_i):
    from quantem_b200 import ops

    n = probe.shape[-1]
    return ops.batch_forward_adjoint(
        _t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev), _t(props.astype(np.complex64), dev),
        _t(positions, dev, torch.float32), _t(batch, dev, torch.int64), _t(targets, dev, torch.float32),
        torch.ones((n, n), device=dev), npos, mean_i)


@pytest.mark.parametrize("n", [64, 96, 128])
def test_empty_batch(cuda_device, n):
    """No positions: loss 0, no object gradient, zero probe gradient, and nothing launched
    that reads the (empty) index list."""
    _, obj_c, probe, props = _problem(n, 2, 2, n + 32, 3)
    pos = np.array([[10.2, 11.7]])
    loss, g_obj, g_probe = _run(cuda_device, obj_c, probe, props, pos, np.zeros(0, np.int64),
                                np.ones((1, n, n)), 1, 1.0)
    assert float(loss) == 0.0
    assert not g_obj.abs().any() and not g_probe.abs().any()


@pytest.mark.parametrize("n", [64, 96, 128])
def test_repeated_positions_in_one_batch(cuda_device, n):
    """The same scan position three times in a batch with two others: every copy adds its
    full gradient (colliding float atomics), as the reference's index scatter does."""
    rng, obj_c, probe, props = _problem(n, 3, 2, n + 40, 11 + n)
    Ho = obj_c.shape[-1]
    positions = np.stack([rng.uniform(0, Ho, 4), rng.uniform(0, Ho, 4)], 1).astype(np.float32).astype(np.float64)
    targets = np.abs(rng.standard_normal((4, n, n))) * 2
    batch = np.array([2, 0, 2, 3, 2])
    npos, mean_i = 40, 7.0
    loss_o, g_obj_o, g_probe_o, _ = O.batch_loss_and_grads(obj_c, probe, positions[batch], props, targets[batch],
                                                           np.ones((n, n)), npos, mean_i)
    loss, g_obj, g_probe = _run(cuda_device, obj_c, probe, props, positions, batch, targets, npos, mean_i)
    assert abs(loss.item() - loss_o) / abs(loss_o) < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G


@pytest.mark.parametrize("n", [64, 128])
def test_positions_on_the_wrap_seam(cuda_device, n):
    """Integer and half-integer positions at 0 and at the object's last row / column: the
    window straddles the periodic seam, and round-half-to-even picks the integer corner."""
    rng, obj_c, probe, props = _problem(n, 2, 3, n + 24, 5 + n)
    Ho = obj_c.shape[-1]
    positions = np.array([[0.0, 0.0], [Ho - 1.0, Ho - 1.0], [0.5, Ho - 0.5], [Ho - 1.5, 2.5], [1.5, 0.5]])
    targets = np.abs(rng.standard_normal((len(positions), n, n))) * 2
    batch = np.arange(len(positions))
    npos, mean_i = 20, 5.0
    loss_o, g_obj_o, g_probe_o, _ = O.batch_loss_and_grads(obj_c, probe, positions, props, targets,
                                                           np.ones((n, n)), npos, mean_i)
    loss, g_obj, g_probe = _run(cuda_device, obj_c, probe, props, positions, batch, targets, npos, mean_i)
    assert abs(loss.item() - loss_o) / abs(loss_o) < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G
