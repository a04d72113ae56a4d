"""FP64 NumPy restatement of the reference's CNN2d (TEST INFRASTRUCTURE ONLY).

Follows src/quantem/core/ml/cnn.py:113-201 (topology and forward) with the
blocks of src/quantem/core/ml/blocks.py: Conv2dBlock (:53-140, Conv2d 3x3 with
padding_mode="circular" -> activation -> BatchNorm2d per layer), Upsample2dBlock
(:143-205, ConvTranspose2d(3, stride 2, padding 1, output_padding 1) -> 1x1
Conv2d -> BatchNorm2d), MaxPool2d(2, 2) and channel concatenation.  Forward and
a hand-written backward, NCHW, parameters under the reference's state-dict names
in torch layouts.  Pinned by tests/golden/cnn_*.npz (made by the reference).

``emulate_bf16=True`` rounds to BF16 at exactly the points where the CUDA path
stores BF16 (layer inputs / batch-norm outputs, weights, transposed-conv
outputs, and the gradients fed to the tensor-core products), so the CUDA
network can be checked far below the BF16 noise floor.

Only tests/, smoke() and the bench's CPU baseline use this module.
"""
from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32).astype(np.float64)
    return np.where(np.isfinite(f), out, f.astype(np.float64))


# ----------------------------------------------------------------------------- layers
def conv3x3_circ(x, w, b):
    """nn.Conv2d(k=3, padding=1, padding_mode='circular') (blocks.py:120-129)."""
    y = np.zeros((x.shape[0], w.shape[0]) + x.shape[2:])
    for ky in range(3):
        for kx in range(3):
            xs = np.roll(x, shift=(1 - ky, 1 - kx), axis=(2, 3))  # xs[.., i, j] = x[.., i+ky-1, j+kx-1]
            y += np.einsum("oc,bchw->bohw", w[:, :, ky, kx], xs, optimize=True)
    return y + b[None, :, None, None]


def conv3x3_circ_bwd(x, w, dy, need_dx=True):
    dw = np.zeros_like(w)
    dx = np.zeros_like(x) if need_dx else None
    for ky in range(3):
        for kx in range(3):
            xs = np.roll(x, shift=(1 - ky, 1 - kx), axis=(2, 3))
            dw[:, :, ky, kx] = np.einsum("bohw,bchw->oc", dy, xs, optimize=True)
            if need_dx:
                g = np.einsum("oc,bohw->bchw", w[:, :, ky, kx], dy, optimize=True)
                dx += np.roll(g, shift=(ky - 1, kx - 1), axis=(2, 3))
    return dx, dw, dy.sum(axis=(0, 2, 3))


def conv_transpose3x3_s2(x, w, b):
    """nn.ConvTranspose2d(k=3, stride=2, padding=1, output_padding=1) (blocks.py:178-186);
    w has torch's (in, out, kh, kw) layout.  out[oy] gathers x[iy] with oy = 2 iy - 1 + ky."""
    B, _, H, W = x.shape
    yp = np.zeros((B, w.shape[1], 2 * H + 2, 2 * W + 2))
    for ky in range(3):
        for kx in range(3):
            yp[:, :, ky:ky + 2 * H:2, kx:kx + 2 * W:2] += np.einsum("bchw,co->bohw", x, w[:, :, ky, kx],
                                                                    optimize=True)
    return yp[:, :, 1:2 * H + 1, 1:2 * W + 1] + b[None, :, None, None]


def conv_transpose3x3_s2_bwd(x, w, dy, dcol_round=None):
    B, _, H, W = x.shape
    dyp = np.zeros((B, dy.shape[1], 2 * H + 2, 2 * W + 2))
    dyp[:, :, 1:2 * H + 1, 1:2 * W + 1] = dy if dcol_round is None else dcol_round(dy)
    dw = np.zeros_like(w)
    dx = np.zeros_like(x)
    for ky in range(3):
        for kx in range(3):
            g = dyp[:, :, ky:ky + 2 * H:2, kx:kx + 2 * W:2]
            dx += np.einsum("bohw,co->bchw", g, w[:, :, ky, kx], optimize=True)
            dw[:, :, ky, kx] = np.einsum("bchw,bohw->co", x, g, optimize=True)
    return dx, dw, dy.sum(axis=(0, 2, 3))


def conv1x1(x, w, b):
    return np.einsum("oc,bchw->bohw", w[:, :, 0, 0], x, optimize=True) + b[None, :, None, None]


def conv1x1_bwd(x, w, dy):
    dx = np.einsum("oc,bohw->bchw", w[:, :, 0, 0], dy, optimize=True)
    dw = np.einsum("bohw,bchw->oc", dy, x, optimize=True)[:, :, None, None]
    return dx, dw, dy.sum(axis=(0, 2, 3))


def batchnorm_train(x, g, b, eps=1e-5):
    """nn.BatchNorm2d in training mode: batch statistics, biased variance."""
    m = x.mean(axis=(0, 2, 3))
    v = x.var(axis=(0, 2, 3))
    rstd = 1.0 / np.sqrt(v + eps)
    xh = (x - m[None, :, None, None]) * rstd[None, :, None, None]
    return xh * g[None, :, None, None] + b[None, :, None, None], (xh, rstd, m, v)


def batchnorm_eval(x, g, b, rm, rv, eps=1e-5):
    return (x - rm[None, :, None, None]) / np.sqrt(rv[None, :, None, None] + eps) * g[None, :, None, None] + \
        b[None, :, None, None]


def batchnorm_train_bwd(dy, g, cache):
    xh, rstd, _, _ = cache
    n = dy.shape[0] * dy.shape[2] * dy.shape[3]
    db = dy.sum(axis=(0, 2, 3))
    dg = (dy * xh).sum(axis=(0, 2, 3))
    dx = (g * rstd)[None, :, None, None] * (dy - db[None, :, None, None] / n - xh * dg[None, :, None, None] / n)
    return dx, dg, db


def maxpool2(x):
    B, C, H, W = x.shape
    v = x.reshape(B, C, H // 2, 2, W // 2, 2).transpose(0, 1, 2, 4, 3, 5).reshape(B, C, H // 2, W // 2, 4)
    arg = v.argmax(axis=-1)  # first maximum in row-major window order
    return np.take_along_axis(v, arg[..., None], -1)[..., 0], arg


def maxpool2_bwd(dy, arg, shape):
    B, C, H, W = shape
    d = np.zeros((B, C, H // 2, W // 2, 4))
    np.put_along_axis(d, arg[..., None], dy[..., None], -1)
    return d.reshape(B, C, H // 2, W // 2, 2, 2).transpose(0, 1, 2, 4, 3, 5).reshape(B, C, H, W)


# ----------------------------------------------------------------------------- network
ACTIVATIONS = {"relu": "relu", "leaky_relu": "leaky_relu", "leakyrelu": "leaky_relu", "lrelu": "leaky_relu",
               "elu": "elu", "tanh": "tanh", "sigmoid": "sigmoid", "softplus": "softplus",
               "identity": None, "eye": None, "ident": None}


def act_fwd(name, z):
    """The real activations of activation_functions.py:166-181 (torch defaults: leaky slope
    0.01, ELU alpha 1, softplus beta 1 with threshold 20)."""
    if name is None:
        return z
    if name == "relu":
        return np.maximum(z, 0.0)
    if name == "leaky_relu":
        return np.where(z > 0, z, 0.01 * z)
    if name == "elu":
        return np.where(z > 0, z, np.expm1(np.minimum(z, 0.0)))
    if name == "tanh":
        return np.tanh(z)
    if name == "sigmoid":
        return 1.0 / (1.0 + np.exp(-z))
    if name == "softplus":
        return np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, 20.0))))
    raise ValueError(name)


def act_grad(name, z):
    """d act / dz at the pre-activation z."""
    if name is None:
        return np.ones_like(z)
    if name == "relu":
        return (z > 0).astype(z.dtype)
    if name == "leaky_relu":
        return np.where(z > 0, 1.0, 0.01)
    if name == "elu":
        return np.where(z > 0, 1.0, np.exp(np.minimum(z, 0.0)))
    if name == "tanh":
        return 1.0 - np.tanh(z) ** 2
    if name == "sigmoid":
        s = 1.0 / (1.0 + np.exp(-z))
        return s * (1.0 - s)
    if name == "softplus":
        return np.where(z > 20, 1.0, 1.0 / (1.0 + np.exp(-np.minimum(z, 20.0))))
    raise ValueError(name)


class CNN2dOracle:
    """CNN2d (cnn.py:17-212) in FP64 from a reference-format state dict."""

    def __init__(self, sd: dict, in_channels, out_channels, start_filters, num_layers, num_per_layer,
                 use_skip_connections=True, use_batchnorm=True, final_relu=False, emulate_bf16=False,
                 momentum=0.1, eps=1e-5, activation="relu", final_activation=None):
        self.sd = {k: np.array(v, dtype=np.float64) for k, v in sd.items()}
        self.cin, self.cout, self.sf = in_channels, out_channels, start_filters
        self.L, self.npl = num_layers, num_per_layer
        self.skip, self.bn = use_skip_connections, use_batchnorm
        self.act = ACTIVATIONS[str(activation).lower()]
        fa = final_activation if final_activation is not None else ("relu" if final_relu else "identity")
        self.final_act = ACTIVATIONS[str(fa).lower()]
        self.emu = emulate_bf16
        self.momentum, self.eps = momentum, eps
        self.r = bf16 if emulate_bf16 else (lambda a: a)

    def _w(self, k):
        return self.r(self.sd[k]) if (self.emu and k.endswith("weight") and self.sd[k].ndim == 4) else self.sd[k]

    def _conv_names(self, prefix, j):
        step = 3 if self.bn else 2
        return f"{prefix}.block.{step * j}", (f"{prefix}.block.{step * j + 2}" if self.bn else None)

    def _conv_layer(self, x, prefix, j, training, tape, with_bn=True, relu=True):
        cname, bname = self._conv_names(prefix, j) if with_bn else (f"{prefix}.block.{2 * j}", None)
        z = conv3x3_circ(x, self._w(cname + ".weight"), self.sd[cname + ".bias"])
        act = self.act if relu else None
        a = act_fwd(act, z)
        if bname is None:
            tape.append(("conv", prefix, j, x, a, None, (act, z), with_bn))
            return a if not with_bn else self.r(a)
        if training:
            y, cache = batchnorm_train(a, self.sd[bname + ".weight"], self.sd[bname + ".bias"], self.eps)
            self._update_running(bname, a, cache)
        else:
            y = batchnorm_eval(a, self.sd[bname + ".weight"], self.sd[bname + ".bias"],
                               self.sd[bname + ".running_mean"], self.sd[bname + ".running_var"], self.eps)
            cache = None
        tape.append(("conv", prefix, j, x, a, cache, (act, z), with_bn))
        return self.r(y)

    def _update_running(self, bname, a, cache):
        _, _, m, v = cache
        n = a.shape[0] * a.shape[2] * a.shape[3]
        unb = v * n / max(n - 1, 1)
        self.sd[bname + ".running_mean"] = (1 - self.momentum) * self.sd[bname + ".running_mean"] + self.momentum * m
        self.sd[bname + ".running_var"] = (1 - self.momentum) * self.sd[bname + ".running_var"] + self.momentum * unb

    def _block(self, x, prefix, training, tape, layers=None):
        for j in range(self.npl if layers is None else layers):
            x = self._conv_layer(x, prefix, j, training, tape)
        return x

    def forward(self, x, training=True):
        """Returns the output; keeps the tape for ``backward``."""
        tape = []
        skips = []
        x = self.r(np.asarray(x, dtype=np.float64))
        self.x_shape = x.shape
        for l in range(self.L):
            x = self._block(x, f"down_conv_blocks.{l}", training, tape)
            skips.append(x)
            pooled, arg = maxpool2(x)
            tape.append(("pool", l, x.shape, arg))
            x = pooled
        x = self._block(x, "bottleneck", training, tape)
        for u in range(self.L):
            p = f"upsample_blocks.{u}"
            t = self.r(conv_transpose3x3_s2(x, self._w(p + ".upsample2x.weight"), self.sd[p + ".upsample2x.bias"]))
            a = conv1x1(t, self._w(p + ".conv.weight"), self.sd[p + ".conv.bias"])
            if self.bn:
                if training:
                    y, cache = batchnorm_train(a, self.sd[p + ".bn.weight"], self.sd[p + ".bn.bias"], self.eps)
                    self._update_running(p + ".bn", a, cache)
                else:
                    y = batchnorm_eval(a, self.sd[p + ".bn.weight"], self.sd[p + ".bn.bias"],
                                       self.sd[p + ".bn.running_mean"], self.sd[p + ".bn.running_var"], self.eps)
                    cache = None
            else:
                y, cache = a, None
            y = self.r(y)
            tape.append(("up", u, x, t, a, cache))
            if self.skip:
                y = np.concatenate([y, skips[self.L - 1 - u]], axis=1)
            x = self._block(y, f"up_conv_blocks.{u}", training, tape)
        z = conv3x3_circ(x, self._w("final_conv.block.0.weight"), self.sd["final_conv.block.0.bias"])
        out = act_fwd(self.final_act, z)
        tape.append(("final", x, z))
        self.tape = tape
        self.training = training
        return out

    def _dz(self, g):
        """Gradient fed to the tensor-core products (BF16 in the CUDA path)."""
        return self.r(g)

    def backward(self, dout):
        """Gradients of sum(out * dout): (dx, {param name: grad}) for the last forward."""
        grads = {}
        tape = list(self.tape)
        _, xin, zf = tape.pop()
        g = np.asarray(dout, dtype=np.float64) * act_grad(self.final_act, zf)
        dxf, dw, db = conv3x3_circ_bwd(xin, self._w("final_conv.block.0.weight"), self._dz(g))
        grads["final_conv.block.0.weight"] = dw
        grads["final_conv.block.0.bias"] = g.sum(axis=(0, 2, 3))
        g = dxf
        dskips = [None] * self.L
        for u in range(self.L - 1, -1, -1):
            g = self._block_bwd(g, f"up_conv_blocks.{u}", tape, grads)
            _, uu, x, t, a, cache = tape.pop()
            assert uu == u
            p = f"upsample_blocks.{u}"
            co = a.shape[1]
            if self.skip:
                dskips[self.L - 1 - u] = g[:, co:]
                g = g[:, :co]
            if self.bn:
                g, dg, dbb = batchnorm_train_bwd(g, self.sd[p + ".bn.weight"], cache)
                grads[p + ".bn.weight"], grads[p + ".bn.bias"] = dg, dbb
            else:
                grads[p + ".bn.weight"] = np.zeros_like(self.sd[p + ".bn.weight"])
                grads[p + ".bn.bias"] = np.zeros_like(self.sd[p + ".bn.bias"])
            grads[p + ".conv.bias"] = g.sum(axis=(0, 2, 3))
            dt, dw1, _ = conv1x1_bwd(t, self._w(p + ".conv.weight"), self._dz(g))
            grads[p + ".conv.weight"] = dw1
            grads[p + ".upsample2x.bias"] = dt.sum(axis=(0, 2, 3))
            dx, dwt, _ = conv_transpose3x3_s2_bwd(x, self._w(p + ".upsample2x.weight"), dt, dcol_round=self._dz)
            grads[p + ".upsample2x.weight"] = dwt
            g = dx
        g = self._block_bwd(g, "bottleneck", tape, grads)
        for l in range(self.L - 1, -1, -1):
            _, ll, shape, arg = tape.pop()
            assert ll == l
            g = maxpool2_bwd(g, arg, shape)
            if self.skip:
                g = g + dskips[l]
            g = self._block_bwd(g, f"down_conv_blocks.{l}", tape, grads, need_dx_first=True)
        return g, grads

    def _block_bwd(self, g, prefix, tape, grads, need_dx_first=True):
        for j in range(self.npl - 1, -1, -1):
            _, pre, jj, x, a, cache, (act, z), with_bn = tape.pop()
            assert pre == prefix and jj == j
            cname, bname = self._conv_names(prefix, j)
            if bname is not None:
                g, dg, dbb = batchnorm_train_bwd(g, self.sd[bname + ".weight"], cache)
                grads[bname + ".weight"], grads[bname + ".bias"] = dg, dbb
            if act is not None:
                g = g * act_grad(act, z)
            grads[cname + ".bias"] = g.sum(axis=(0, 2, 3))
            dx, dw, _ = conv3x3_circ_bwd(x, self._w(cname + ".weight"), self._dz(g))
            grads[cname + ".weight"] = dw
            g = dx
        return g
