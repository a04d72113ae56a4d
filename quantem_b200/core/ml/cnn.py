"""UNet-like CNN2d on the B200 kernels (reference: src/quantem/core/ml/cnn.py:17-212).

Same topology, constructor and parameter names as the reference's ``CNN2d``:
``num_layers`` encoder levels of ``Conv2dBlock`` (``num_per_layer`` x [3x3 conv with
circular padding -> ReLU -> BatchNorm2d], core/ml/blocks.py:53-140) each followed
by a 2x2 max pool, a bottleneck block, ``num_layers`` decoder levels of
``Upsample2dBlock`` (ConvTranspose2d 3x3 stride 2 -> 1x1 conv -> BatchNorm2d,
blocks.py:143-205), skip concatenation ``cat((up, skip), dim=1)`` and a
``Conv2dBlock``, then a final 3x3 conv without batch norm.

B200 design: activations are channels-last BF16 matrices (rows = pixels); every
convolution is a tcgen05 BF16 GEMM with FP32 accumulation (``kernels.gemm``),
fed by im2col / transposed-convolution gather kernels; ReLU and bias are fused
into the GEMM epilogue, batch norm runs on the FP32 GEMM output and writes the
BF16 input of the next layer (directly into the skip-concatenation buffer).
All parameters live in one flat FP32 master tensor (``self.flat``, an
``nn.Parameter``; its ``.grad`` is filled by backward) with a BF16 copy for the
GEMMs, so one fused optimiser launch updates the whole network.
``state_dict()`` / ``load_state_dict()`` use the reference's module names and
torch layouts.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from . import kernels as kk
from .kernels import ACT_IDS


def _up8(n: int) -> int:
    return (n + 7) // 8 * 8


@dataclass
class _Seg:
    name: str       # reference parameter name
    off: int        # element offset in the flat buffers
    shape: tuple    # shape inside the flat buffer
    numel: int


def _activation_name(a) -> str:
    """Canonical name of an activation given as a string or a torch module (the reference's
    get_activation_function names, activation_functions.py:150-181)."""
    if isinstance(a, torch.nn.Module):
        for cls, name in ((torch.nn.Identity, "identity"), (torch.nn.ReLU, "relu"), (torch.nn.Tanh, "tanh"),
                          (torch.nn.Sigmoid, "sigmoid")):
            if type(a) is cls:
                return name
        if type(a) is torch.nn.LeakyReLU and a.negative_slope == 0.01:
            return "leaky_relu"
        if type(a) is torch.nn.ELU and a.alpha == 1.0:
            return "elu"
        if type(a) is torch.nn.Softplus and a.beta == 1.0 and a.threshold == 20.0:
            return "softplus"
        raise NotImplementedError(f"activation {a!r} is not one of the B200 kernels' activations")
    name = str(a).lower()
    if name not in ACT_IDS:
        raise NotImplementedError(f"activation {a!r}: the B200 kernels implement {sorted(set(ACT_IDS))}")
    return {"eye": "identity", "ident": "identity", "leakyrelu": "leaky_relu", "lrelu": "leaky_relu"}.get(name, name)


class CNN2d(torch.nn.Module):
    """UNet-like CNN for 2-D images (reference core/ml/cnn.py:17-212).

    Input (B, in_channels, H, W) FP32 with H, W divisible by 2**num_layers;
    output (B, out_channels, H, W) FP32.  Computation is BF16 x BF16 -> FP32 on
    the tensor cores."""

    def __init__(self, in_channels: int, out_channels: int | None = None, start_filters: int = 16,
                 num_layers: int = 3, num_per_layer: int = 2, use_skip_connections: bool = True,
                 dtype: torch.dtype = torch.float32, dropout: float = 0, activation="relu",
                 final_activation="identity", use_batchnorm: bool = True, device="cuda", seed: int | None = 0):
        super().__init__()
        self.in_channels = int(in_channels)
        self.out_channels = int(out_channels) if out_channels is not None else int(in_channels)
        self.start_filters = int(start_filters)
        self.num_layers = int(num_layers)
        self._num_per_layer = int(num_per_layer)
        if use_skip_connections and num_per_layer < 2:
            raise ValueError("If using skip connections, num_per_layer must be at least 2 to allow for "
                             "channel concatenation.")
        if dtype.is_complex:
            raise NotImplementedError("complex CNN2d is not part of the B200 path (real phase maps only)")
        if not 0.0 <= float(dropout) <= 1.0:
            raise ValueError(f"dropout must be in [0, 1], got {dropout}")
        self.dropout = float(dropout)
        self._dropout_calls = 0
        self._dropout_seed = int(seed) if seed is not None else 0
        self._act_name = _activation_name(activation)
        fa = _activation_name(final_activation)
        self._final_act_name = fa
        self._act = ACT_IDS[self._act_name]
        self._final_act = ACT_IDS[fa]
        if self.start_filters % 8:
            raise ValueError("start_filters must be a multiple of 8 (16-byte rows of the BF16 operands)")
        self.use_skip_connections = bool(use_skip_connections)
        self._use_batchnorm = bool(use_batchnorm)
        self._final_relu = fa == "relu"
        self.dtype = dtype
        self.device = torch.device(device)
        self.cin_pad = _up8(self.in_channels)
        self.momentum = 0.1
        self.eps = 1e-5
        # when a dict, each pass records every layer's inputs / outputs / gradients
        # (used by the per-layer parity tests)
        self.trace = None
        self._build()
        self._init_params(seed)

    # ------------------------------------------------------------------ layout
    def _build(self):
        segs: list[_Seg] = []
        off = 0

        def add(name, shape):
            nonlocal off
            n = int(math.prod(shape))
            segs.append(_Seg(name, off, tuple(shape), n))
            off += _up8(n)
            return segs[-1]

        self.convs = {}  # prefix -> dict(ci, co, w, b, bn)
        npl, bn = self._num_per_layer, self._use_batchnorm
        # conv, activation, (batch norm), (dropout) per layer of a Conv2dBlock (blocks.py:117-136)
        drop = 1 if self.dropout > 0 else 0
        step = (3 if bn else 2) + drop

        def conv_block(prefix, ci, co, layers, with_bn=True):
            out = []
            for j in range(layers):
                cin = ci if j == 0 else co
                cin_store = self.cin_pad if (prefix == "down_conv_blocks.0" and j == 0) else cin
                p = f"{prefix}.block.{step * j if with_bn else (2 + drop) * j}"
                w = add(p + ".weight", (co, 9 * cin_store))
                b = add(p + ".bias", (co,))
                layer = dict(ci=cin, ci_store=cin_store, co=co, w=w, b=b, bn=None)
                if with_bn and bn:
                    pb = f"{prefix}.block.{step * j + 2}"
                    layer["bn"] = (add(pb + ".weight", (co,)), add(pb + ".bias", (co,)), pb)
                out.append(layer)
            return out

        self.down = []
        ci, co = self.in_channels, self.start_filters
        for l in range(self.num_layers):
            if l:
                co = ci * 2
            self.down.append(conv_block(f"down_conv_blocks.{l}", ci, co, npl))
            ci = co
        co = ci * 2
        self.bottleneck = conv_block("bottleneck", ci, co, npl)
        ci = co
        self.up = []
        for u in range(self.num_layers):
            co = self.start_filters if u == self.num_layers - 1 else ci // 2
            ci2 = ci if self.use_skip_connections else co
            p = f"upsample_blocks.{u}"
            wt = add(p + ".upsample2x.weight", (9 * ci, ci))
            bt = add(p + ".upsample2x.bias", (ci,))
            w1 = add(p + ".conv.weight", (co, ci))
            b1 = add(p + ".conv.bias", (co,))
            ubn = (add(p + ".bn.weight", (co,)), add(p + ".bn.bias", (co,)), p + ".bn")
            block = conv_block(f"up_conv_blocks.{u}", ci2, co, npl)
            self.up.append(dict(ci=ci, co=co, wt=wt, bt=bt, w1=w1, b1=b1, bn=ubn, block=block))
            ci = co
        self.final = conv_block("final_conv", self.start_filters, self.out_channels, 1, with_bn=False)[0]
        self.segs = segs
        self.total = off
        dev = self.device
        self.flat = torch.nn.Parameter(torch.zeros(off, device=dev))
        self.flat16 = torch.zeros(off, dtype=torch.bfloat16, device=dev)
        # batch-norm running statistics (buffers) per bn prefix
        self.running = {}
        for seg in segs:
            if seg.name.endswith(".weight") and self._is_bn(seg.name):
                c = seg.shape[0]
                pref = seg.name[: -len(".weight")]
                self.running[pref] = (torch.zeros(c, device=dev), torch.ones(c, device=dev))
        self.num_batches_tracked = 0

    def _is_bn(self, name: str) -> bool:
        for layer in self._all_conv_layers():
            if layer["bn"] is not None and layer["bn"][0].name == name:
                return True
        return any(u["bn"][0].name == name for u in self.up)

    def _all_conv_layers(self):
        for blk in self.down:
            yield from blk
        yield from self.bottleneck
        for u in self.up:
            yield from u["block"]
        yield self.final

    def view(self, seg: _Seg, t: torch.Tensor | None = None) -> torch.Tensor:
        t = self.flat.data if t is None else t
        return t[seg.off: seg.off + seg.numel].view(seg.shape)

    def _init_params(self, seed):
        """torch's default initialisation of Conv2d / ConvTranspose2d / BatchNorm2d."""
        g = torch.Generator().manual_seed(0 if seed is None else int(seed))
        flat = torch.zeros(self.total)

        def uni(seg, bound, fill_shape=None):
            v = (torch.rand(seg.shape if fill_shape is None else fill_shape, generator=g) * 2 - 1) * bound
            return v

        for layer in self._all_conv_layers():
            fan_in = 9 * layer["ci"]
            bound = 1.0 / math.sqrt(fan_in)
            w = uni(layer["w"], bound, (layer["co"], 9, layer["ci"]))
            full = torch.zeros(layer["co"], 9, layer["ci_store"])
            full[:, :, : layer["ci"]] = w
            flat[layer["w"].off: layer["w"].off + layer["w"].numel] = full.reshape(-1)
            flat[layer["b"].off: layer["b"].off + layer["b"].numel] = uni(layer["b"], bound)
            if layer["bn"] is not None:
                flat[layer["bn"][0].off: layer["bn"][0].off + layer["bn"][0].numel] = 1.0
        for u in self.up:
            bt = 1.0 / math.sqrt(9 * u["ci"])  # ConvTranspose2d fan_in = weight.size(1) * 9
            flat[u["wt"].off: u["wt"].off + u["wt"].numel] = uni(u["wt"], bt).reshape(-1)
            flat[u["bt"].off: u["bt"].off + u["bt"].numel] = uni(u["bt"], bt)
            b1 = 1.0 / math.sqrt(u["ci"])
            flat[u["w1"].off: u["w1"].off + u["w1"].numel] = uni(u["w1"], b1).reshape(-1)
            flat[u["b1"].off: u["b1"].off + u["b1"].numel] = uni(u["b1"], b1)
            flat[u["bn"][0].off: u["bn"][0].off + u["bn"][0].numel] = 1.0
        self.flat.data.copy_(flat.to(self.device))
        self.sync_weights()

    # ------------------------------------------------------------------ state
    def sync_weights(self):
        """Refresh the BF16 GEMM copy of the FP32 master weights."""
        kk.cast_bf16(self.flat.data, self.flat16)

    def train(self, mode: bool = True):
        self.training = bool(mode)
        return self

    def eval(self):
        return self.train(False)

    def config(self) -> dict:
        """Construction arguments (a checkpoint rebuilds the network from them)."""
        return dict(in_channels=self.in_channels, out_channels=self.out_channels, start_filters=self.start_filters,
                    num_layers=self.num_layers, num_per_layer=self._num_per_layer,
                    use_skip_connections=self.use_skip_connections, use_batchnorm=self._use_batchnorm,
                    activation=self._act_name, final_activation=self._final_act_name, dropout=self.dropout)

    def state_dict(self, *args, **kwargs):
        """Parameters and batch-norm buffers under the reference's module names, torch layouts."""
        return self._export(self.flat.data, buffers=True)

    def named_gradients(self) -> dict:
        """Gradients of the last backward (``self.flat.grad``) under the reference's names and layouts."""
        if self.flat.grad is None:
            return {}
        return self._export(self.flat.grad, buffers=False)

    def _export(self, src: torch.Tensor, buffers: bool) -> dict:
        sd = {}
        for layer in self._all_conv_layers():
            w = self.view(layer["w"], src).reshape(layer["co"], 3, 3, layer["ci_store"])[..., : layer["ci"]]
            sd[layer["w"].name] = w.permute(0, 3, 1, 2).contiguous().clone()
            sd[layer["b"].name] = self.view(layer["b"], src).clone()
            if layer["bn"] is not None:
                self._bn_state(sd, layer["bn"], src, buffers)
        for u in self.up:
            ci = u["ci"]
            wt = self.view(u["wt"], src).reshape(3, 3, ci, ci)
            sd[u["wt"].name] = wt.permute(3, 2, 0, 1).contiguous().clone()
            sd[u["bt"].name] = self.view(u["bt"], src).clone()
            sd[u["w1"].name] = self.view(u["w1"], src).reshape(u["co"], ci, 1, 1).clone()
            sd[u["b1"].name] = self.view(u["b1"], src).clone()
            self._bn_state(sd, u["bn"], src, buffers)
        return sd

    def _bn_state(self, sd, bn, src, buffers):
        gseg, bseg, pref = bn
        sd[gseg.name] = self.view(gseg, src).clone()
        sd[bseg.name] = self.view(bseg, src).clone()
        if not buffers:
            return
        rm, rv = self.running[pref]
        sd[pref + ".running_mean"] = rm.clone()
        sd[pref + ".running_var"] = rv.clone()
        sd[pref + ".num_batches_tracked"] = torch.tensor(self.num_batches_tracked)

    def load_state_dict(self, sd, strict: bool = True):
        """Load a reference CNN2d state dict (same module names, torch layouts)."""
        flat = self.flat.data
        used = set()

        def put(seg, val):
            flat[seg.off: seg.off + seg.numel] = val.reshape(-1).to(flat)
            used.add(seg.name)

        for layer in self._all_conv_layers():
            w = torch.as_tensor(sd[layer["w"].name]).float().permute(0, 2, 3, 1)  # (co, ky, kx, ci)
            full = torch.zeros(layer["co"], 3, 3, layer["ci_store"])
            full[..., : layer["ci"]] = w
            put(layer["w"], full)
            put(layer["b"], torch.as_tensor(sd[layer["b"].name]).float())
            if layer["bn"] is not None:
                self._load_bn(sd, layer["bn"], put, used)
        for u in self.up:
            wt = torch.as_tensor(sd[u["wt"].name]).float()  # (in, out, ky, kx)
            put(u["wt"], wt.permute(2, 3, 1, 0))
            put(u["bt"], torch.as_tensor(sd[u["bt"].name]).float())
            put(u["w1"], torch.as_tensor(sd[u["w1"].name]).float())
            put(u["b1"], torch.as_tensor(sd[u["b1"].name]).float())
            self._load_bn(sd, u["bn"], put, used)
        if strict:
            missing = [k for k in sd if k not in used and not k.endswith(("running_mean", "running_var",
                                                                            "num_batches_tracked"))]
            if missing:
                raise KeyError(f"unexpected keys in state dict: {missing[:5]}")
        self.sync_weights()

    def _load_bn(self, sd, bn, put, used):
        gseg, bseg, pref = bn
        put(gseg, torch.as_tensor(sd[gseg.name]).float())
        put(bseg, torch.as_tensor(sd[bseg.name]).float())
        rm, rv = self.running[pref]
        rm.copy_(torch.as_tensor(sd[pref + ".running_mean"]).float())
        rv.copy_(torch.as_tensor(sd[pref + ".running_var"]).float())
        if pref + ".num_batches_tracked" in sd:
            self.num_batches_tracked = int(torch.as_tensor(sd[pref + ".num_batches_tracked"]).item())

    # ------------------------------------------------------------------ compute
    def forward(self, x: torch.Tensor, rows: tuple | None = None) -> torch.Tensor:
        """x: (B, in_channels, H, W) FP32, or with ``rows=(B, H, W)`` the channels-last
        BF16 input matrix (B*H*W, in_channels rounded up to 8) itself."""
        if rows is not None:
            B, H, W = (int(v) for v in rows)
            if x.dtype != torch.bfloat16 or x.dim() != 2 or tuple(x.shape) != (B * H * W, self.cin_pad):
                raise ValueError(f"row input must be bfloat16 ({B * H * W}, {self.cin_pad})")
            f = 2 ** self.num_layers
            if H % f or W % f:
                raise ValueError(f"H and W must be divisible by 2**num_layers = {f}")
            return _CNNFn.apply(x, self.flat, self, (B, H, W))
        if x.dim() != 4 or x.shape[1] != self.in_channels:
            raise ValueError(f"expected (B, {self.in_channels}, H, W), got {tuple(x.shape)}")
        if not x.is_cuda:
            raise RuntimeError("CNN2d runs on the CUDA kernels only (no CPU fallback)")
        f = 2 ** self.num_layers
        if x.shape[2] % f or x.shape[3] % f:
            raise ValueError(f"H and W must be divisible by 2**num_layers = {f}")
        return _CNNFn.apply(x.float().contiguous(), self.flat, self, None)

    __call__ = forward


class _Run:
    """One forward pass: buffers and saved tensors for its backward."""

    def __init__(self, net: CNN2d, B: int, H: int, W: int, training: bool):
        self.net, self.B, self.H, self.W, self.training = net, B, H, W, training
        dev = net.device
        maxc = max(2 * net.start_filters * 2 ** net.num_layers, net.cin_pad, 64)
        self.work = torch.empty(2 * 592 * maxc, dtype=torch.float64, device=dev)
        self.dev = dev
        self.saved = {}

    def empty(self, *shape, dtype=torch.float32):
        return torch.empty(*shape, dtype=dtype, device=self.dev)

    # --- conv3x3 + bias + activation (+ BN) -> bf16 into `out` ------------------
    def conv_fwd(self, key, layer, x16, B, H, W, out16, act=None, final=False):
        net = self.net
        R = B * H * W
        co = layer["co"]
        col = self.empty(R, 9 * layer["ci_store"], dtype=torch.bfloat16)
        kk.im2col3x3(x16, B, H, W, col)
        w16 = net.view(layer["w"], net.flat16)
        r = self.empty(R, co if not final else co)
        kk.gemm(col, w16, r, bias=net.view(layer["b"]), act=net._act if act is None else act)
        del col
        tr = self.net.trace
        seed = self._next_dropout_seed()
        if final:
            # the activation's output r stays for the backward; the dropped copy is the output
            y = r if seed is None else kk.dropout(r.clone(), net.dropout, seed)
            self.saved[key] = (x16, r, None, None, seed)
            if tr is not None:
                tr[("fwd",) + key] = dict(x=x16.clone(), r=r.clone())
            return y
        if layer["bn"] is not None:
            gseg, bseg, pref = layer["bn"]
            mean, rstd = self.empty(co), self.empty(co)
            rm, rv = net.running[pref]
            kk.bn_forward(r, net.view(gseg), net.view(bseg), rm, rv, net.momentum, net.eps, self.training, mean,
                          rstd, self.work, out16)
        else:
            mean = rstd = None
            kk.bn_forward(r, None, None, None, None, 0.0, 0.0, False, None, None, self.work, out16)
        if seed is not None:
            kk.dropout(out16, net.dropout, seed)
        self.saved[key] = (x16, r, mean, rstd, seed)
        if tr is not None:
            tr[("fwd",) + key] = dict(x=x16.clone(), r=r.clone(), y=out16.clone())
        return out16

    def _next_dropout_seed(self):
        """A fresh mask seed per layer and pass in training mode with dropout, else None."""
        net = self.net
        if not (self.training and net.dropout > 0):
            return None
        net._dropout_calls += 1
        return (net._dropout_seed * 0x9E3779B1 + net._dropout_calls) & 0xFFFFFFFFFFFF

    def block_fwd(self, prefix, layers, x16, B, H, W, out16_last):
        y = x16
        for j, layer in enumerate(layers):
            out = out16_last if j == len(layers) - 1 else self.empty(B * H * W, layer["co"], dtype=torch.bfloat16)
            y = self.conv_fwd((prefix, j), layer, y, B, H, W, out)
        return y

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        net = self.net
        B, H, W = self.B, self.H, self.W
        L = net.num_layers
        if x.dim() == 2:  # channels-last BF16 rows given directly
            x16 = x
        else:
            x16 = self._to_rows(x)
        return self._forward_rows(x16)

    def _to_rows(self, x: torch.Tensor) -> torch.Tensor:
        net = self.net
        B, H, W = self.B, self.H, self.W
        # NCHW FP32 -> channels-last BF16 (padded channels stay zero)
        x16 = self.empty(B * H * W, net.cin_pad, dtype=torch.bfloat16)
        if net.cin_pad != net.in_channels:
            x16.zero_()
        xc = x.reshape(B, net.in_channels, H * W)
        if net.cin_pad == net.in_channels:
            kk.transpose(xc, x16.view(B, H * W, net.cin_pad))
        else:
            tmp = self.empty(B, H * W, net.in_channels, dtype=torch.bfloat16)
            kk.transpose(xc, tmp)
            x16.view(B, H * W, net.cin_pad)[..., : net.in_channels].copy_(tmp)
        return x16

    def _forward_rows(self, x16: torch.Tensor) -> torch.Tensor:
        net = self.net
        B, H, W = self.B, self.H, self.W
        L = net.num_layers
        self.cat = []
        self.pool_arg = []
        y = x16
        for l in range(L):
            h, w = H >> l, W >> l
            co = net.down[l][-1]["co"]
            R = B * h * w
            if net.use_skip_connections:
                cat = self.empty(R, 2 * co, dtype=torch.bfloat16)
                skip = cat[:, co:]
            else:
                cat = None
                skip = self.empty(R, co, dtype=torch.bfloat16)
            self.cat.append(cat)
            self.block_fwd(("down", l), net.down[l], y, B, h, w, skip)
            pooled = self.empty(R // 4, co, dtype=torch.bfloat16)
            arg = self.empty(R // 4, co, dtype=torch.uint8)
            kk.maxpool2(skip, B, h, w, pooled, arg)
            self.pool_arg.append((skip, arg))
            y = pooled
        h, w = H >> L, W >> L
        cb = net.bottleneck[-1]["co"]
        yb = self.empty(B * h * w, cb, dtype=torch.bfloat16)
        y = self.block_fwd(("bott",), net.bottleneck, y, B, h, w, yb)
        for u, up in enumerate(net.up):
            l = L - 1 - u
            hin, win = H >> (l + 1), W >> (l + 1)
            h, w = H >> l, W >> l
            ci, co = up["ci"], up["co"]
            Rin, R = B * hin * win, B * h * w
            colT = self.empty(Rin, 9 * ci)
            kk.gemm(y, net.view(up["wt"], net.flat16), colT)
            t16 = self.empty(R, ci, dtype=torch.bfloat16)
            kk.convT_gather(colT, B, hin, win, ci, net.view(up["bt"]), t16)
            del colT
            r = self.empty(R, co)
            kk.gemm(t16, net.view(up["w1"], net.flat16), r, bias=net.view(up["b1"]))
            cat = self.cat[l]
            dst = cat[:, :co] if cat is not None else self.empty(R, co, dtype=torch.bfloat16)
            if net._use_batchnorm:
                gseg, bseg, pref = up["bn"]
                mean, rstd = self.empty(co), self.empty(co)
                rm, rv = net.running[pref]
                kk.bn_forward(r, net.view(gseg), net.view(bseg), rm, rv, net.momentum, net.eps, self.training, mean,
                              rstd, self.work, dst)
            else:
                mean = rstd = None
                kk.bn_forward(r, None, None, None, None, 0.0, 0.0, False, None, None, self.work, dst)
            self.saved[("upT", u)] = (y, t16, r, mean, rstd, hin, win)
            if net.trace is not None:
                net.trace[("upfwd", u)] = dict(x=y.clone(), t=t16.clone(), r=r.clone(), y=dst.clone())
            src = cat if cat is not None else dst
            out = self.empty(R, up["block"][-1]["co"], dtype=torch.bfloat16)
            y = self.block_fwd(("upc", u), up["block"], src, B, h, w, out)
        fin = net.final
        r = self.conv_fwd(("final",), fin, y, B, H, W, None, act=net._final_act, final=True)
        out = self.empty(B, net.out_channels, H * W)
        kk.transpose(r.view(B, H * W, net.out_channels), out)
        return out.view(B, net.out_channels, H, W)

    # ------------------------------------------------------------------ backward
    def conv_bwd(self, key, layer, dy, B, H, W, grad, dx_out=None, dx_accumulate=False, act=None):
        """dy: FP32 gradient w.r.t. the layer output (after BN).  Accumulates the
        weight / bias / BN gradients into `grad` and writes dx (FP32) if asked."""
        net = self.net
        x16, r, mean, rstd, seed = self.saved.pop(key)
        if seed is not None:  # the forward's dropout mask on the incoming gradient
            dy = kk.dropout(dy.contiguous().clone(), net.dropout, seed)
        tr = net.trace
        if tr is not None:
            tr[("bwd",) + key] = dict(dy=dy.clone())
        R = B * H * W
        co, ci_store = layer["co"], layer["ci_store"]
        ldz = _up8(co)
        dz32 = self.empty(R, ldz)[:, :co]
        dz16 = self.empty(R, ldz, dtype=torch.bfloat16)[:, :co]
        act = net._act if act is None else act
        if layer["bn"] is not None:
            gseg, bseg, _ = layer["bn"]
            kk.bn_backward(dy, r, net.view(gseg), mean, rstd, self.training, act, net.view(gseg, grad),
                           net.view(bseg, grad), self.work, dz32=dz32, dz16=dz16)
        else:
            kk.bn_backward(dy, r, None, None, None, self.training, act, None, None, self.work, dz32=dz32, dz16=dz16)
        kk.colsum(dz32, net.view(layer["b"], grad), self.work)
        del dz32
        # weight gradient: dW[co][9ci] = dz^T @ col
        col = self.empty(R, 9 * ci_store, dtype=torch.bfloat16)
        kk.im2col3x3(x16, B, H, W, col)
        colT = self.empty(9 * ci_store, _up8(R), dtype=torch.bfloat16)[:, :R]
        kk.transpose(col, colT)
        del col
        dzT = self.empty(co, _up8(R), dtype=torch.bfloat16)[:, :R]
        kk.transpose(dz16, dzT)
        gw = net.view(layer["w"], grad)
        _gemm_acc(dzT, colT, gw, self)
        del colT, dzT
        if dx_out is not None:
            # dx = col2im(dz @ W): W^T operand (9ci x co)
            wT = self.empty(9 * ci_store, ldz, dtype=torch.bfloat16)[:, :co]
            kk.transpose(net.view(layer["w"], net.flat16), wT)
            dcol = self.empty(R, 9 * ci_store)
            kk.gemm(dz16, wT, dcol)
            kk.col2im3x3(dcol, B, H, W, ci_store, dx_out, accumulate=dx_accumulate)
            if tr is not None:
                tr[("bwd",) + key]["dx"] = dx_out.clone()

    def block_bwd(self, prefix, layers, dy, B, H, W, grad, dx_out, dx_accumulate=False):
        g = dy
        for j in range(len(layers) - 1, -1, -1):
            layer = layers[j]
            if j > 0:
                dx = self.empty(B * H * W, layer["ci_store"])
                self.conv_bwd((prefix, j), layer, g, B, H, W, grad, dx)
                g = dx
            else:
                self.conv_bwd((prefix, 0), layer, g, B, H, W, grad, dx_out, dx_accumulate)

    def backward(self, dout: torch.Tensor, grad: torch.Tensor, need_dx: bool):
        net = self.net
        B, H, W = self.B, self.H, self.W
        L = net.num_layers
        R0 = B * H * W
        dfin = self.empty(R0, net.out_channels)
        kk.transpose(dout.reshape(B, net.out_channels, H * W), dfin.view(B, H * W, net.out_channels))
        dy = self.empty(R0, net.final["ci_store"])
        self.conv_bwd(("final",), net.final, dfin, B, H, W, grad, dy, act=net._final_act)
        dcat = [None] * L
        # decoder, last level first
        for u in range(L - 1, -1, -1):
            up = net.up[u]
            l = L - 1 - u
            h, w = H >> l, W >> l
            ci, co = up["ci"], up["co"]
            R = B * h * w
            cin_block = up["block"][0]["ci_store"]
            dsrc = self.empty(R, cin_block)
            self.block_bwd(("upc", u), up["block"], dy, B, h, w, grad, dsrc)
            dcat[l] = dsrc
            dup = dsrc[:, :co] if net.use_skip_connections else dsrc
            yin, t16, r, mean, rstd, hin, win = self.saved.pop(("upT", u))
            Rin = B * hin * win
            ldz = _up8(co)
            dz32 = self.empty(R, ldz)[:, :co]
            dz16 = self.empty(R, ldz, dtype=torch.bfloat16)[:, :co]
            if net._use_batchnorm:
                gseg, bseg, _ = up["bn"]
                kk.bn_backward(dup, r, net.view(gseg), mean, rstd, self.training, False, net.view(gseg, grad),
                               net.view(bseg, grad), self.work, dz32=dz32, dz16=dz16)
            else:
                kk.bn_backward(dup, r, None, None, None, self.training, False, None, None, self.work, dz32=dz32,
                               dz16=dz16)
            kk.colsum(dz32, net.view(up["b1"], grad), self.work)
            # 1x1 conv: dW1 = dz^T t ; dt = dz W1
            dzT = self.empty(co, _up8(R), dtype=torch.bfloat16)[:, :R]
            kk.transpose(dz16, dzT)
            tT = self.empty(ci, _up8(R), dtype=torch.bfloat16)[:, :R]
            kk.transpose(t16, tT)
            _gemm_acc(dzT, tT, net.view(up["w1"], grad), self)
            del dzT, tT
            w1T = self.empty(ci, ldz, dtype=torch.bfloat16)[:, :co]
            kk.transpose(net.view(up["w1"], net.flat16), w1T)
            dt = self.empty(R, ci)
            kk.gemm(dz16, w1T, dt)
            # transposed convolution: bias, weight and input gradients
            kk.colsum(dt, net.view(up["bt"], grad), self.work)
            dcolT = self.empty(Rin, 9 * ci, dtype=torch.bfloat16)
            kk.convT_im2col(dt, B, hin, win, ci, dcolT)
            dcolTT = self.empty(9 * ci, _up8(Rin), dtype=torch.bfloat16)[:, :Rin]
            kk.transpose(dcolT, dcolTT)
            yT = self.empty(ci, _up8(Rin), dtype=torch.bfloat16)[:, :Rin]
            kk.transpose(yin, yT)
            _gemm_acc(dcolTT, yT, net.view(up["wt"], grad), self)
            del dcolTT, yT
            wtT = self.empty(ci, 9 * ci, dtype=torch.bfloat16)
            kk.transpose(net.view(up["wt"], net.flat16), wtT)
            dy = self.empty(Rin, ci)
            kk.gemm(dcolT, wtT, dy)
            if net.trace is not None:
                net.trace[("upbwd", u)] = dict(dup=dup.clone(), dt=dt.clone(), dx=dy.clone())
        # bottleneck
        h, w = H >> L, W >> L
        cin = net.bottleneck[0]["ci_store"]
        dpool = self.empty(B * h * w, cin)
        self.block_bwd(("bott",), net.bottleneck, dy, B, h, w, grad, dpool)
        # encoder, deepest first
        for l in range(L - 1, -1, -1):
            h, w = H >> l, W >> l
            R = B * h * w
            co = net.down[l][-1]["co"]
            skip, arg = self.pool_arg[l]
            if net.use_skip_connections:
                dskip = dcat[l][:, co:]
                kk.maxpool2_backward(dpool, arg, B, h, w, dskip, accumulate=True)
            else:
                dskip = self.empty(R, co)
                kk.maxpool2_backward(dpool, arg, B, h, w, dskip)
            cin = net.down[l][0]["ci_store"]
            if l > 0:
                dpool = self.empty(R, cin)
                self.block_bwd(("down", l), net.down[l], dskip, B, h, w, grad, dpool)
            else:
                dx = self.empty(R, cin) if need_dx else None
                self.block_bwd(("down", 0), net.down[0], dskip, B, h, w, grad, dx)
                if need_dx:
                    out = self.empty(B, net.in_channels, H * W)
                    src = dx.view(B, H * W, cin)[..., : net.in_channels]
                    kk.transpose(src.contiguous(), out)
                    return out.view(B, net.in_channels, H, W)
        return None


def _gemm_acc(A: torch.Tensor, B: torch.Tensor, out: torch.Tensor, run: _Run):
    """out (FP32 parameter-gradient view) += A @ B.T with a long K (pixels): split-K
    across CTAs, each adding its partial product atomically."""
    M, K = A.shape
    N = B.shape[0]
    bn = 32 if N <= 32 else (64 if N <= 64 else 128)
    tiles = ((M + 127) // 128) * ((N + bn - 1) // bn)
    nkb = (K + 63) // 64
    splits = max(1, min(nkb // 4, (2 * 148) // max(tiles, 1)))
    kk.gemm(A, B, out.view(M, N), splits=splits, accumulate=True)


class _CNNFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, flat, net, rows):
        B, H, W = rows if rows is not None else (x.shape[0], x.shape[2], x.shape[3])
        net.sync_weights()
        run = _Run(net, B, H, W, net.training)
        y = run.forward(x)
        if net.training:
            net.num_batches_tracked += 1
        ctx.run = run
        ctx.needs_x = ctx.needs_input_grad[0] and rows is None
        return y

    @staticmethod
    def backward(ctx, dy):
        run = ctx.run
        ctx.run = None
        grad = torch.zeros_like(run.net.flat.data)
        dx = run.backward(dy.float().resolve_neg().contiguous(), grad, ctx.needs_x)
        return dx, grad, None, None


def mse_loss(pred: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
    """Mean squared error on the CUDA kernel (torch.nn.functional.mse_loss semantics)."""
    return _MSEFn.apply(pred, target)


class _MSEFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pred, target):
        p = pred.float().resolve_neg().contiguous()
        t = target.float().resolve_neg().contiguous()
        loss = torch.empty(1, device=p.device)
        work = torch.empty(296, dtype=torch.float64, device=p.device)
        dp = torch.empty_like(p)
        kk.mse(p, t, loss, work, dpred32=dp)
        ctx.save_for_backward(dp)
        return loss.view(())

    @staticmethod
    def backward(ctx, g):
        (dp,) = ctx.saved_tensors
        return dp * g, None


class ComplexCNN2d(torch.nn.Module):
    """The reference's CNN2d with ``dtype=torch.complex64`` (complex convolutions,
    ComplexBatchNorm2D, Complex_ReLU, complex pooling) on the B200 kernels.

    It runs as a real ``CNN2d`` with doubled channels whose tensors hold the real parts
    followed by the imaginary parts and whose weights have the block structure
    [[A, -B], [B, A]] of a complex weight A + iB (``complex_map``).  The complex
    parameters live in one flat FP32 tensor (``self.flat``: every complex tensor as its
    real view, batch-norm parameters as they are); each forward writes the real
    network's weights as a signed gather of it, and the gradient of the real weights
    flows back through the same gather (so dA and dB sum the two blocks each feeds).
    ``state_dict`` / ``load_state_dict`` use the reference's names, complex dtypes and
    layouts (``real_bn`` / ``imag_bn`` batch-norm halves)."""

    def __init__(self, in_channels: int, out_channels: int | None = None, start_filters: int = 16,
                 num_layers: int = 3, num_per_layer: int = 2, use_skip_connections: bool = True,
                 dtype: torch.dtype = torch.complex64, dropout: float = 0, activation="relu",
                 final_activation="identity", use_batchnorm: bool = True, device="cuda", seed: int | None = 0):
        super().__init__()
        from .complex_map import complex_to_real_state

        if not dtype.is_complex:
            raise ValueError("ComplexCNN2d takes a complex dtype (use CNN2d for real networks)")
        if dropout:  # nn.Dropout drops a complex element whole; the doubled real network would not
            raise NotImplementedError("dropout in complex networks is not part of the B200 path")
        # Complex_ReLU acts on the real and imaginary parts separately, which the doubled real
        # network reproduces; modReLU and the phase ReLU couple them and are not built
        act = str(activation).lower() if not isinstance(activation, torch.nn.Module) else activation
        if act in ("complexrelu", "complex_relu"):
            act = "relu"
        if act != "relu":
            raise NotImplementedError(f"activation {activation!r}: complex networks take complexrelu")
        fin = final_activation
        if isinstance(fin, str) and fin.lower() in ("complexrelu", "complex_relu"):
            fin = "relu"
        if _activation_name(fin) not in ("identity", "relu"):
            raise NotImplementedError(f"final_activation {final_activation!r}: complex networks take identity or "
                                      "complexrelu")
        activation, final_activation = act, fin
        self.in_channels = int(in_channels)
        self.out_channels = int(out_channels) if out_channels is not None else int(in_channels)
        self.start_filters = int(start_filters)
        self.num_layers = int(num_layers)
        self.use_skip_connections = bool(use_skip_connections)
        self.dtype = dtype
        self.device = torch.device(device)
        self.real = CNN2d(2 * self.in_channels, 2 * self.out_channels, start_filters=2 * self.start_filters,
                          num_layers=num_layers, num_per_layer=num_per_layer,
                          use_skip_connections=use_skip_connections, dtype=torch.float32, dropout=dropout,
                          activation=activation, final_activation=final_activation, use_batchnorm=use_batchnorm,
                          device=device, seed=seed)
        # the reference's complex state-dict template, from the real network's
        self.template = self._complex_template(self.real.state_dict())
        self.keys = [k for k, v in self.template.items()
                     if not k.endswith(("running_mean", "running_var", "num_batches_tracked"))]
        self.offsets = {}
        off = 0
        for k in self.keys:
            t = self.template[k]
            n = t.numel() * (2 if t.is_complex() else 1)
            self.offsets[k] = (off, n)
            off += n
        if off >= 2 ** 24:
            raise ValueError("network too large for the float32 index map of ComplexCNN2d")
        self.flat = torch.nn.Parameter(torch.zeros(off, device=self.device))
        # signed gather map: real flat element e = sign[e] * self.flat[src[e]]
        probe_sd = {}
        for k, t in self.template.items():
            if k in self.offsets:
                o, n = self.offsets[k]
                idx = torch.arange(o + 1, o + n + 1, dtype=torch.float64)
                probe_sd[k] = torch.view_as_complex(idx.view(*t.shape, 2)) if t.is_complex() else idx.view(t.shape)
            else:
                probe_sd[k] = t.clone().double() if t.is_floating_point() else t.clone()
        self.real.load_state_dict(complex_to_real_state(probe_sd, self.use_skip_connections))
        code = self.real.flat.data.clone()
        self.src = (code.abs().round().long() - 1).clamp(min=0)
        self.sign = torch.sign(code)
        for pref, (rm, rv) in self.real.running.items():
            rm.zero_()
            rv.fill_(1.0)
        self.real.num_batches_tracked = 0
        self._init_params(seed)

    @staticmethod
    def _complex_template(rsd: dict) -> dict:
        """Complex state-dict entries (names, shapes, dtypes) of the real network's."""
        bn_prefixes = {k[: -len(".running_mean")] for k in rsd if k.endswith(".running_mean")}
        out = {}
        for k, v in rsd.items():
            pref = k.rsplit(".", 1)[0]
            field = k.rsplit(".", 1)[1]
            if pref in bn_prefixes:
                if field == "num_batches_tracked":
                    for half in ("real_bn", "imag_bn"):
                        out[f"{pref}.{half}.{field}"] = v.clone()
                else:
                    C = v.shape[0] // 2
                    for half in ("real_bn", "imag_bn"):
                        out[f"{pref}.{half}.{field}"] = torch.zeros(C, dtype=torch.float32)
            elif field == "bias":
                out[k] = torch.zeros(v.shape[0] // 2, dtype=torch.complex64)
            elif ".upsample2x." in k:
                out[k] = torch.zeros((v.shape[0] // 2, v.shape[1] // 2) + tuple(v.shape[2:]), dtype=torch.complex64)
            else:
                out[k] = torch.zeros((v.shape[0] // 2, v.shape[1] // 2) + tuple(v.shape[2:]), dtype=torch.complex64)
        return out

    def _init_params(self, seed):
        """torch's default initialisation of complex Conv2d / ConvTranspose2d (real and
        imaginary parts uniform in +-1/sqrt(fan_in)) and of the batch norms (1, 0)."""
        g = torch.Generator().manual_seed(0 if seed is None else int(seed))
        flat = torch.zeros(self.flat.numel())
        for k in self.keys:
            t = self.template[k]
            o, n = self.offsets[k]
            if not t.is_complex():  # batch norm: weight 1, bias 0
                flat[o:o + n] = 1.0 if k.endswith(".weight") else 0.0
                continue
            wkey = k[: -len(".bias")] + ".weight" if k.endswith(".bias") else k
            w = self.template[wkey]
            fan_in = (w.shape[0] if ".upsample2x." in wkey else w.shape[1]) * int(math.prod(w.shape[2:]))
            bound = 1.0 / math.sqrt(fan_in)
            flat[o:o + n] = (torch.rand(n, generator=g) * 2 - 1) * bound
        self.flat.data.copy_(flat.to(self.device))

    def _real_flat(self) -> torch.Tensor:
        return self.sign * self.flat[self.src]

    def train(self, mode: bool = True):
        self.training = bool(mode)
        self.real.train(mode)
        return self

    def eval(self):
        return self.train(False)

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x: (B, in_channels, H, W) complex; returns (B, out_channels, H, W) complex64."""
        if not x.is_complex():
            raise TypeError("ComplexCNN2d takes a complex input")
        if not x.is_cuda:
            raise RuntimeError("ComplexCNN2d runs on the CUDA kernels only (no CPU fallback)")
        xr = torch.cat([x.real, x.imag], dim=1).float().contiguous()
        w = self._real_flat()
        self.real.flat.data.copy_(w.detach())
        y = _CNNFn.apply(xr, w, self.real, None)
        C = self.out_channels
        return torch.complex(y[:, :C], y[:, C:])

    __call__ = forward

    def config(self) -> dict:
        """Construction arguments (a checkpoint rebuilds the network from them)."""
        r = self.real
        return dict(in_channels=self.in_channels, out_channels=self.out_channels, start_filters=self.start_filters,
                    num_layers=self.num_layers, num_per_layer=r._num_per_layer,
                    use_skip_connections=self.use_skip_connections, use_batchnorm=r._use_batchnorm,
                    final_activation=r._final_act_name)

    def state_dict(self, *args, **kwargs):
        from .complex_map import real_to_complex_state

        self.real.flat.data.copy_(self._real_flat().detach())
        return real_to_complex_state(self.real.state_dict(), self.template, self.use_skip_connections)

    def load_state_dict(self, sd, strict: bool = True):
        from .complex_map import complex_to_real_state

        flat = torch.zeros(self.flat.numel())
        for k in self.keys:
            if k not in sd:
                if strict:
                    raise KeyError(f"missing key {k}")
                continue
            o, n = self.offsets[k]
            v = torch.as_tensor(sd[k])
            flat[o:o + n] = (torch.view_as_real(v.to(torch.complex64)) if v.is_complex() else v.float()).reshape(-1)
        self.flat.data.copy_(flat.to(self.device))
        full = dict(self.template)
        full.update({k: torch.as_tensor(v) for k, v in sd.items()})
        self.real.load_state_dict(complex_to_real_state(full, self.use_skip_connections), strict=False)
        self.real.flat.data.copy_(self._real_flat().detach())
        self.real.sync_weights()

    def named_gradients(self) -> dict:
        """Gradients of the last backward under the reference's names (complex tensors
        in torch's convention dL/dRe + i dL/dIm)."""
        if self.flat.grad is None:
            return {}
        out = {}
        for k in self.keys:
            o, n = self.offsets[k]
            t = self.template[k]
            g = self.flat.grad[o:o + n]
            out[k] = torch.view_as_complex(g.view(*t.shape, 2).contiguous()) if t.is_complex() else g.view(t.shape)
        return out
