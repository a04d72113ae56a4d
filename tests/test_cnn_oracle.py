"""The FP64 NumPy CNN2d oracle against the golden fixtures made by the reference's
own CNN2d (tests/golden/make_golden_cnn.py): training-mode output, input and
parameter gradients, running statistics and eval-mode output."""
import numpy as np
import pytest

from oracle.cnn_oracle import CNN2dOracle, bf16
from tests.conftest import load_golden

CASES = ["cnn_unet2", "cnn_unet2_noskip", "cnn_unet1_nobn"]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_for(z, **kw):
    cfg = [int(c) for c in z["config"]]
    sd = {k[3:]: z[k] for k in z if k.startswith("sd/")}
    return CNN2dOracle(sd, *cfg[:5], use_skip_connections=bool(cfg[5]), use_batchnorm=bool(cfg[6]), **kw)


@pytest.mark.parametrize("name", CASES)
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
