"""Complex CNN2d as a real CNN2d with doubled channels (reference: core/ml/cnn.py with
dtype=complex64, core/ml/blocks.py, core/ml/activation_functions.py).

The reference's complex network is built from complex convolutions and transposed
convolutions (complex multiply-accumulate), ``ComplexBatchNorm2D`` (an independent
BatchNorm2d on the real and on the imaginary channels), ``Complex_ReLU`` (ReLU of
the real and of the imaginary part) and ``complex_pool`` (the pooling of each part).
All of these act on the real and imaginary parts as one real network whose tensors
hold 2C channels -- the C real parts followed by the C imaginary parts -- and whose
weights have the block structure

    [out_re]   [A  -B] [in_re]
    [out_im] = [B   A] [in_im]     for a complex weight A + iB,

biases [Re b; Im b] and batch-norm parameters [real_bn; imag_bn].  A skip
concatenation cat((up, skip)) of complex tensors becomes, on the real tensors,
[up_re, up_im, skip_re, skip_im], so the first convolution of each decoder level
reads its complex input channel j from real channels (j, Cu + j) for j < Cu and
(2Cu + j', 2Cu + Cs + j') for the skip channels j' = j - Cu.

``complex_to_real_state`` maps a complex state dict (the reference's names and
layouts) onto the real network's state dict; ``real_to_complex_state`` maps it back.
The GPU network (``ComplexCNN2d``) uses the same map as a signed gather of its
complex parameters, so the tensor-core GEMMs of the real network do the work.
"""
from __future__ import annotations

import re

import torch


def _in_maps(C: int, concat_first: int | None = None):
    """Real channel indices (of the real and of the imaginary part) of the C complex
    input channels; ``concat_first`` = Cu for a skip concatenation input."""
    ar = torch.arange(C)
    if concat_first is None:
        return ar, C + ar
    cu, cs = concat_first, C - concat_first
    r = torch.cat([torch.arange(cu), 2 * cu + torch.arange(cs)])
    i = torch.cat([cu + torch.arange(cu), 2 * cu + cs + torch.arange(cs)])
    return r, i


_BN = re.compile(r"^(.*)\.(real_bn|imag_bn)\.(weight|bias|running_mean|running_var|num_batches_tracked)$")


def _concat_split(key: str, cin: int, skip: bool):
    """Cu of the skip concatenation feeding ``key``'s convolution, or None."""
    if skip and key.startswith("up_conv_blocks.") and ".block.0." in key:
        return cin // 2
    return None


def complex_to_real_state(sd: dict, skip: bool = True) -> dict:
    """Real-network state dict of a complex CNN2d state dict (see the module docstring).
    Complex tensors map to float tensors of the complex dtype's real precision."""
    out = {}
    bn_parts: dict = {}
    for key, v in sd.items():
        m = _BN.match(key)
        if m:
            bn_parts.setdefault((m.group(1), m.group(3)), {})[m.group(2)] = v
            continue
        v = torch.as_tensor(v)
        if not v.is_complex():
            out[key] = v.clone()
            continue
        A, B = v.real, v.imag
        if key.endswith(".bias"):
            out[key] = torch.cat([A, B])
        elif ".upsample2x.weight" in key:  # ConvTranspose2d (in, out, kh, kw)
            ci, co = v.shape[:2]
            ri, ii = _in_maps(ci)
            ro, io = _in_maps(co)
            R = torch.zeros((2 * ci, 2 * co) + tuple(v.shape[2:]), dtype=A.dtype)
            R[ri[:, None], ro[None, :]] = A
            R[ii[:, None], ro[None, :]] = -B
            R[ri[:, None], io[None, :]] = B
            R[ii[:, None], io[None, :]] = A
            out[key] = R
        elif key.endswith(".weight"):  # Conv2d (out, in, kh, kw)
            co, ci = v.shape[:2]
            ri, ii = _in_maps(ci, _concat_split(key, ci, skip))
            ro, io = _in_maps(co)
            R = torch.zeros((2 * co, 2 * ci) + tuple(v.shape[2:]), dtype=A.dtype)
            R[ro[:, None], ri[None, :]] = A
            R[ro[:, None], ii[None, :]] = -B
            R[io[:, None], ri[None, :]] = B
            R[io[:, None], ii[None, :]] = A
            out[key] = R
        else:
            raise KeyError(f"unexpected complex entry {key}")
    for (pref, field), parts in bn_parts.items():
        if field == "num_batches_tracked":
            out[f"{pref}.{field}"] = torch.as_tensor(parts["real_bn"]).clone()
        else:
            out[f"{pref}.{field}"] = torch.cat([torch.as_tensor(parts["real_bn"]), torch.as_tensor(parts["imag_bn"])])
    return out


def real_to_complex_state(rsd: dict, template: dict, skip: bool = True) -> dict:
    """Inverse of ``complex_to_real_state``: complex entries of ``template`` (names,
    shapes, dtypes) read back from the real network's state dict."""
    out = {}
    for key, t in template.items():
        t = torch.as_tensor(t)
        m = _BN.match(key)
        if m:
            v = torch.as_tensor(rsd[f"{m.group(1)}.{m.group(3)}"])
            if m.group(3) == "num_batches_tracked":
                out[key] = v.clone()
            else:
                C = t.shape[0]
                out[key] = (v[:C] if m.group(2) == "real_bn" else v[C:]).clone().to(t.dtype)
            continue
        v = torch.as_tensor(rsd[key])
        if not t.is_complex():
            out[key] = v.clone().to(t.dtype)
        elif key.endswith(".bias"):
            C = t.shape[0]
            out[key] = torch.complex(v[:C], v[C:]).to(t.dtype)
        elif ".upsample2x.weight" in key:
            ci, co = t.shape[:2]
            ri, ii = _in_maps(ci)
            ro, io = _in_maps(co)
            out[key] = torch.complex(v[ri[:, None], ro[None, :]], v[ri[:, None], io[None, :]]).to(t.dtype)
        else:
            co, ci = t.shape[:2]
            ri, ii = _in_maps(ci, _concat_split(key, ci, skip))
            ro, io = _in_maps(co)
            out[key] = torch.complex(v[ro[:, None], ri[None, :]], v[io[:, None], ri[None, :]]).to(t.dtype)
    return out


def real_grads_to_complex(rgrads: dict, template: dict, skip: bool = True) -> dict:
    """Gradients of the complex parameters (torch convention dL/dA + i dL/dB) from the
    gradients of the real network's weights: a complex weight feeds two blocks each of
    A and B, dL/dA = G_rr + G_ii and dL/dB = G_ir - G_ri."""
    out = {}
    for key, t in template.items():
        t = torch.as_tensor(t)
        if key.endswith(("running_mean", "running_var", "num_batches_tracked")):
            continue
        m = _BN.match(key)
        if m:
            v = torch.as_tensor(rgrads[f"{m.group(1)}.{m.group(3)}"])
            C = t.shape[0]
            out[key] = (v[:C] if m.group(2) == "real_bn" else v[C:]).clone()
            continue
        v = torch.as_tensor(rgrads[key])
        if key.endswith(".bias"):
            C = t.shape[0]
            out[key] = torch.complex(v[:C], v[C:])
            continue
        if ".upsample2x.weight" in key:
            ci, co = t.shape[:2]
            ri, ii = _in_maps(ci)
            ro, io = _in_maps(co)
            gA = v[ri[:, None], ro[None, :]] + v[ii[:, None], io[None, :]]
            gB = v[ri[:, None], io[None, :]] - v[ii[:, None], ro[None, :]]
        else:
            co, ci = t.shape[:2]
            ri, ii = _in_maps(ci, _concat_split(key, ci, skip))
            ro, io = _in_maps(co)
            gA = v[ro[:, None], ri[None, :]] + v[io[:, None], ii[None, :]]
            gB = v[io[:, None], ri[None, :]] - v[ro[:, None], ii[None, :]]
        out[key] = torch.complex(gA, gB)
    return out
