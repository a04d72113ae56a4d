"""Run-to-run determinism of the fused batch kernels on identical inputs: the loss and the
probe gradient come from fixed-order reductions of per-CTA partials and must repeat bit
for bit; the object gradient is accumulated with float atomics (order-dependent at the
rounding level) and must repeat to within a few float32 ulps of its scale; the
forward-only intensities repeat bit for bit."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,S,P", [(64, 1, 1), (96, 3, 2), (128, 8, 4)])
def test_batch_kernels_repeat(cuda_device, n, S, P):
    from quantem_b200 import ops

    dev = cuda_device
    g = torch.Generator(device="cpu").manual_seed(5 + n)
    Ho, B = 2 * n + 64, 300

    def crand(*shape):
        return torch.complex(torch.randn(*shape, generator=g), torch.randn(*shape, generator=g))

    obj = torch.polar(1 - 0.2 * torch.rand((S, Ho, Ho), generator=g), 0.3 * torch.randn((S, Ho, Ho), generator=g))
    probe = crand(P, n, n) * torch.exp(-(torch.fft.fftfreq(n) * n)[:, None] ** 2 / (2.0 * n)
                                       - (torch.fft.fftfreq(n) * n)[None] ** 2 / (2.0 * n))
    props = ops.separable_propagators(n, (0.2, 0.2), 300e3, [20.0] * (S - 1), device=dev) if S > 1 else \
        torch.zeros((0, n, n), dtype=torch.complex64, device=dev)
    pos = (torch.rand((B, 2), generator=g) * Ho).to(dev)
    tg = (torch.rand((B, n, n), generator=g) * 3).to(dev)
    idx = torch.randperm(B, generator=g).to(dev)
    args = (obj.to(torch.complex64).to(dev), probe.to(torch.complex64).to(dev), props, pos, idx, tg,
            torch.ones((n, n), device=dev), B, 20.0)
    runs = [ops.batch_forward_adjoint(*args) for _ in range(3)]
    torch.cuda.synchronize()
    l0, go0, gp0 = (t.cpu() for t in runs[0])
    for loss, go, gp in runs[1:]:
        assert torch.equal(loss.cpu(), l0)
        assert torch.equal(gp.cpu(), gp0)
        d = (go.cpu() - go0).abs().max().item()
        assert d <= 1e-6 * go0.abs().max().item(), d
    f = [ops.batch_forward(*args)["intensity"].cpu() for _ in range(2)]
    assert torch.equal(f[0], f[1])
    assert np.isfinite(l0.item())
