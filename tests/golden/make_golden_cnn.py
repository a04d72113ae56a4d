"""Golden fixtures for the learned initialiser's CNN, made by the reference itself.

Run in a container where the reference source tree is mounted:

    python tests/golden/make_golden_cnn.py <reference checkout>/src

Builds the reference's ``quantem.core.ml.cnn.CNN2d`` (UNet topology of
core/ml/cnn.py:17-212 with the blocks of core/ml/blocks.py) for a few small
configurations, with torch's default initialisation under a fixed seed, and
records in FP64: the state dict, an input, the training-mode output (batch-norm
batch statistics), the gradients of sum(output * dy) with respect to every
parameter and to the input, the running statistics after that step and the
eval-mode output.  The fixtures pin the FP64 NumPy oracle (``oracle/cnn_oracle.py``)
and the CUDA network (``quantem_b200.core.ml.cnn.CNN2d``).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from baseline.reference_import import import_reference  # noqa: E402

CASES = {
    # name: (in_ch, out_ch, start_filters, num_layers, num_per_layer, skip, batchnorm, B, H, W)
    "cnn_unet2": (4, 3, 8, 2, 2, True, True, 2, 16, 16),
    "cnn_unet2_noskip": (8, 2, 8, 2, 2, False, True, 2, 16, 24),
    "cnn_unet1_nobn": (16, 5, 16, 1, 2, True, False, 3, 8, 8),
}


# the other real activations of the reference (activation_functions.py:166-181) on a
# small U-Net: name: (config as above, hidden activation, final activation)
ACT_CASES = {
    "cnn_act_leaky_relu": ((4, 3, 8, 2, 2, True, True, 2, 16, 16), "leaky_relu", "identity"),
    "cnn_act_elu": ((4, 3, 8, 2, 2, True, True, 2, 16, 16), "elu", "sigmoid"),
    "cnn_act_tanh": ((4, 2, 8, 1, 2, True, False, 2, 16, 16), "tanh", "tanh"),
    "cnn_act_sigmoid": ((4, 3, 8, 2, 2, False, True, 2, 16, 16), "sigmoid", "softplus"),
    "cnn_act_softplus": ((4, 3, 8, 2, 2, True, True, 2, 16, 16), "softplus", "relu"),
}


def run_case(name, cfg, activation="relu", final_activation="identity"):
    import torch
    from quantem.core.ml.cnn import CNN2d

    cin, cout, sf, L, npl, skip, bn, B, H, W = cfg
    torch.manual_seed(1234 + len(name))
    net = CNN2d(cin, cout, start_filters=sf, num_layers=L, num_per_layer=npl, use_skip_connections=skip,
                use_batchnorm=bn, dtype=torch.float32, activation=activation,
                final_activation=final_activation).double()
    net.train()
    g = torch.Generator().manual_seed(99)
    x = torch.randn(B, cin, H, W, generator=g, dtype=torch.float64).requires_grad_(True)
    dy = torch.randn(B, cout, H, W, generator=g, dtype=torch.float64)
    sd0 = {k: v.detach().clone() for k, v in net.state_dict().items()}
    y = net(x)
    (y * dy).sum().backward()
    out = {"x": x.detach().numpy(), "dy": dy.numpy(), "y_train": y.detach().numpy(),
           "dx": x.grad.numpy(), "config": np.array(cfg[:5] + (int(skip), int(bn)), dtype=np.int64),
           "activation": np.asarray(activation), "final_activation": np.asarray(final_activation)}
    for k, v in sd0.items():
        out["sd/" + k] = v.numpy()
    for k, p in net.named_parameters():  # unused parameters (the upsample bn without batch norm) get zeros
        out["grad/" + k] = p.grad.numpy() if p.grad is not None else np.zeros(tuple(p.shape))
    for k, v in net.state_dict().items():
        if "running" in k:
            out["after/" + k] = v.numpy()
    net.eval()
    with torch.no_grad():
        out["y_eval"] = net(x.detach()).numpy()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "params", sum(p.numel() for p in net.parameters()))


def _to_fp64(net):
    """complex parameters / buffers to complex128, real ones to float64 (Module.double()
    leaves complex tensors alone and Module.to(complex128) would make the batch norms
    complex)."""
    import torch

    for mod in net.modules():
        for name, t in list(mod._parameters.items()) + list(mod._buffers.items()):
            if t is None:
                continue
            if t.is_complex():
                t.data = t.data.to(torch.complex128)
            elif t.is_floating_point():
                t.data = t.data.double()
    return net


def run_complex_case(name, cfg):
    """A complex CNN2d (dtype=complex64: complex convolutions, ComplexBatchNorm2D,
    Complex_ReLU, complex pooling), run in complex128: the loss is
    Re(sum(conj(dy) * y)), so every recorded gradient follows torch's complex
    convention (dL/dRe + i dL/dIm)."""
    import torch
    from quantem.core.ml.cnn import CNN2d

    cin, cout, sf, L, npl, skip, bn, B, H, W = cfg
    torch.manual_seed(4321 + len(name))
    net = _to_fp64(CNN2d(cin, cout, start_filters=sf, num_layers=L, num_per_layer=npl, use_skip_connections=skip,
                         use_batchnorm=bn, dtype=torch.complex64))
    net.train()
    g = torch.Generator().manual_seed(77)

    def crandn(*shape):
        return torch.complex(torch.randn(*shape, generator=g, dtype=torch.float64),
                             torch.randn(*shape, generator=g, dtype=torch.float64))

    x = crandn(B, cin, H, W).requires_grad_(True)
    dy = crandn(B, cout, H, W)
    sd0 = {k: v.detach().clone() for k, v in net.state_dict().items()}
    y = net(x)
    (torch.conj(dy) * y).real.sum().backward()
    out = {"x": x.detach().numpy(), "dy": dy.numpy(), "y_train": y.detach().numpy(),
           "dx": x.grad.numpy(), "config": np.array(cfg[:5] + (int(skip), int(bn)), dtype=np.int64)}
    for k, v in sd0.items():
        out["sd/" + k] = v.numpy()
    for k, p in net.named_parameters():
        out["grad/" + k] = p.grad.numpy() if p.grad is not None else np.zeros(tuple(p.shape), p.detach().numpy().dtype)
    for k, v in net.state_dict().items():
        if "running" in k:
            out["after/" + k] = v.numpy()
    net.eval()
    with torch.no_grad():
        out["y_eval"] = net(x.detach()).numpy()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "params", sum(p.numel() for p in net.parameters()))


COMPLEX_CASES = {
    "cnn_complex_unet2": (2, 2, 8, 2, 2, True, True, 2, 16, 16),
}


def main():
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.relpath(__file__)} <reference source dir (the one holding quantem/)>")
    src = sys.argv[1]
    import_reference(src)
    if os.environ.get("GOLDEN_ONLY") == "activations":
        for name, (cfg, act, fin) in ACT_CASES.items():
            run_case(name, cfg, act, fin)
        return
    if os.environ.get("GOLDEN_ONLY") != "complex":
        for name, cfg in CASES.items():
            run_case(name, cfg)
    for name, cfg in COMPLEX_CASES.items():
        run_complex_case(name, cfg)


if __name__ == "__main__":
    main()
