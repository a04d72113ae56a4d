"""The FP64 NumPy CNN2d oracle against the golden fixtures made by the reference's
own CNN2d (tests/golden/make_golden_cnn.py): training-mode output, input and
parameter gradients, running statistics and eval-mode output."""
import numpy as np
import pytest

from oracle.cnn_oracle import CNN2dOracle, bf16
from tests.conftest import load_golden

CASES = ["cnn_unet2", "cnn_unet2_noskip", "cnn_unet1_nobn"]
# the reference's other real activations (hidden / final), fixtures made with them
ACT_CASES = ["cnn_act_leaky_relu", "cnn_act_elu", "cnn_act_tanh", "cnn_act_sigmoid", "cnn_act_softplus"]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_for(z, **kw):
    cfg = [int(c) for c in z["config"]]
    sd = {k[3:]: z[k] for k in z if k.startswith("sd/")}
    if "activation" in z:
        kw = dict(activation=str(z["activation"]), final_activation=str(z["final_activation"]), **kw)
    return CNN2dOracle(sd, *cfg[:5], use_skip_connections=bool(cfg[5]), use_batchnorm=bool(cfg[6]), **kw)


@pytest.mark.parametrize("name", CASES + ACT_CASES)
def test_cnn_oracle_matches_reference(name):
    z = load_golden(name)
    net = oracle_for(z)
    assert _rel(net.forward(z["x"], training=True), z["y_train"]) < 1e-12
    dx, grads = net.backward(z["dy"])
    assert _rel(dx, z["dx"]) < 1e-12
    gscale = np.sqrt(sum(np.linalg.norm(z[k]) ** 2 for k in z if k.startswith("grad/")))
    for k in z:
        if k.startswith("grad/"):
            # biases right before a batch norm have an exactly-zero gradient: compare on the global scale
            assert np.linalg.norm(grads[k[5:]] - z[k]) <= 1e-12 * gscale, k
    for k in z:
        if k.startswith("after/"):
            assert _rel(net.sd[k[6:]], z[k]) < 1e-12, k
    assert _rel(net.forward(z["x"], training=False), z["y_eval"]) < 1e-12


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-40, 65504.0, np.inf])
    r = bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie -> even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.isinf(r[6])


def test_complex_cnn_is_the_real_network_with_block_weights():
    """The reference's complex CNN2d (tests/golden/cnn_complex_unet2.npz) equals the real
    CNN2d with doubled channels and [[A, -B], [B, A]] weights
    (quantem_b200.core.ml.complex_map): the FP64 oracle run on that real network
    reproduces the complex outputs, input and parameter gradients and running
    statistics of the reference to 1e-12."""
    import torch

    from quantem_b200.core.ml.complex_map import complex_to_real_state, real_grads_to_complex

    z = load_golden("cnn_complex_unet2")
    cfg = [int(c) for c in z["config"]]
    cin, cout, sf, L, npl, skip, bn = cfg
    sd = {k[3:]: torch.as_tensor(z[k]) for k in z if k.startswith("sd/")}
    rsd = {k: v.numpy() for k, v in complex_to_real_state(sd, bool(skip)).items()}
    net = CNN2dOracle(rsd, 2 * cin, 2 * cout, 2 * sf, L, npl, use_skip_connections=bool(skip),
                      use_batchnorm=bool(bn))
    x = z["x"]
    y = net.forward(np.concatenate([x.real, x.imag], axis=1), training=True)
    assert _rel(y[:, :cout] + 1j * y[:, cout:], z["y_train"]) < 1e-12
    dy = z["dy"]
    dx, grads = net.backward(np.concatenate([dy.real, dy.imag], axis=1))
    assert _rel(dx[:, :cin] + 1j * dx[:, cin:], z["dx"]) < 1e-12
    cg = real_grads_to_complex({k: torch.as_tensor(v) for k, v in grads.items()}, sd, bool(skip))
    gscale = np.sqrt(sum(np.linalg.norm(z[k]) ** 2 for k in z if k.startswith("grad/")))
    for k in z:
        if k.startswith("grad/"):
            assert np.linalg.norm(cg[k[5:]].numpy() - z[k]) <= 1e-12 * gscale, k
    back = {}
    for k in z:
        if k.startswith("after/"):
            name = k[6:]
            pref, half, field = name.rsplit(".", 2)
            full = net.sd[f"{pref}.{field}"]
            C = full.shape[0] // 2
            assert _rel(full[:C] if half == "real_bn" else full[C:], z[k]) < 1e-12, k
    y_eval = net.forward(np.concatenate([x.real, x.imag], axis=1), training=False)
    assert _rel(y_eval[:, :cout] + 1j * y_eval[:, cout:], z["y_eval"]) < 1e-12
