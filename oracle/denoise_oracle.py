"""CPU oracle of the mesh denoiser -- test infrastructure only.

The denoiser has no counterpart in the reference, so its oracle is a plain
restatement of the same network in torch float64 on the CPU (F.conv3d,
avg_pool3d, nearest upsampling, concatenation, autograd).  Tests compare the
device forward pass, the data and weight gradients of every layer and the
parameter gradients of the whole network against it, within tolerances set by
the BF16 operands.

Parameter layout (shared with the device code): per 3x3x3 layer W[cout][27][cin]
with tap = 9 (dz+1) + 3 (dy+1) + (dx+1), then b[cout]; head w[16], b.
"""
from __future__ import annotations

import numpy as np

SPECS = [(1, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16),
         (16, 16)]


def param_count() -> int:
    return sum(co * 27 * ci + co for ci, co in SPECS) + 17


def unpack(params):
    """Flat parameters -> [(W (cout, cin, 3, 3, 3), b)] * 10 + [(w_head (16,), b_head)] as
    float64 torch tensors."""
    import torch
    p = torch.as_tensor(np.asarray(params, np.float64))
    out, o = [], 0
    for ci, co in SPECS:
        n = co * 27 * ci
        w = p[o:o + n].reshape(co, 3, 3, 3, ci).permute(0, 4, 1, 2, 3).contiguous()
        o += n
        out.append((w, p[o:o + co].clone()))
        o += co
    out.append((p[o:o + 16].clone(), p[o + 16:o + 17].clone()))
    return out


def pack(layers) -> np.ndarray:
    """Inverse of unpack (for gradients)."""
    parts = []
    for (w, b), (ci, co) in zip(layers[:10], SPECS):
        parts.append(w.permute(0, 2, 3, 4, 1).reshape(-1).detach().numpy())
        parts.append(b.reshape(-1).detach().numpy())
    parts.append(layers[10][0].reshape(-1).detach().numpy())
    parts.append(layers[10][1].reshape(-1).detach().numpy())
    return np.concatenate(parts)


def conv3(x, w, b=None, relu=False):
    import torch.nn.functional as F
    y = F.conv3d(x, w, b, padding=1)
    return F.relu(y) if relu else y


def up2(x):
    return x.repeat_interleave(2, dim=2).repeat_interleave(2, dim=3).repeat_interleave(2, dim=4)


def forward(layers, x):
    """x: float64 (nb, D, H, W) -> network output (nb, D, H, W)."""
    import torch
    import torch.nn.functional as F
    L = layers
    x5 = x[:, None]
    e1a = conv3(x5, *L[0], relu=True)
    s1 = conv3(e1a, *L[1], relu=True)
    e2a = conv3(F.avg_pool3d(s1, 2), *L[2], relu=True)
    s2 = conv3(e2a, *L[3], relu=True)
    b1 = conv3(F.avg_pool3d(s2, 2), *L[4], relu=True)
    b2 = conv3(b1, *L[5], relu=True)
    d2a = conv3(torch.cat([up2(b2), s2], 1), *L[6], relu=True)
    d2b = conv3(d2a, *L[7], relu=True)
    d1a = conv3(torch.cat([up2(d2b), s1], 1), *L[8], relu=True)
    d1b = conv3(d1a, *L[9], relu=True)
    wh, bh = L[10]
    return x + (d1b * wh[None, :, None, None, None]).sum(1) + bh


def loss_and_grads(params, x, target, weight=None):
    """Mean (weighted) squared error of the network output against target,
    its parameter gradients (flat, same layout) and the output."""
    import torch
    layers = unpack(params)
    for w, b in layers:
        w.requires_grad_(True)
        b.requires_grad_(True)
    xt = torch.as_tensor(np.asarray(x, np.float64))
    tt = torch.as_tensor(np.asarray(target, np.float64))
    out = forward(layers, xt)
    d2 = (out - tt) ** 2
    if weight is not None:
        d2 = d2 * torch.as_tensor(np.asarray(weight, np.float64))
    loss = d2.mean()
    loss.backward()
    grads = pack([(w.grad, b.grad) for w, b in layers])
    return float(loss.detach()), grads, out.detach().numpy()


def conv_layer(src0, src1, w, b, relu, up0):
    """One layer on NDHWC float arrays: src0 (nb, d, h, w, c0) or None, src1
    (nb, D, H, W, c1), w (cout, 27, cin) -> (nb, D, H, W, cout) float64."""
    import torch
    parts = []
    if src0 is not None:
        s0 = torch.as_tensor(np.asarray(src0, np.float64)).permute(0, 4, 1, 2, 3)
        parts.append(up2(s0) if up0 else s0)
    parts.append(torch.as_tensor(np.asarray(src1, np.float64)).permute(0, 4, 1, 2, 3))
    x = torch.cat(parts, 1)
    co, _, ci = w.shape
    wt = torch.as_tensor(np.asarray(w, np.float64)).reshape(co, 3, 3, 3, ci).permute(0, 4, 1, 2, 3)
    bt = None if b is None else torch.as_tensor(np.asarray(b, np.float64))
    return conv3(x, wt, bt, relu).permute(0, 2, 3, 4, 1).numpy()


def wgrad_layer(src0, src1, g, up0):
    """dW[co][tap][ci] = sum_v g[v][co] X[v + off(tap)][ci] and db[co] = sum_v g[v][co]
    (float64), X = concat(upsampled src0, src1)."""
    import torch
    parts = []
    if src0 is not None:
        s0 = torch.as_tensor(np.asarray(src0, np.float64)).permute(0, 4, 1, 2, 3)
        parts.append(up2(s0) if up0 else s0)
    parts.append(torch.as_tensor(np.asarray(src1, np.float64)).permute(0, 4, 1, 2, 3))
    x = torch.cat(parts, 1)
    gt = torch.as_tensor(np.asarray(g, np.float64)).permute(0, 4, 1, 2, 3)
    co, ci = gt.shape[1], x.shape[1]
    w = torch.zeros(co, ci, 3, 3, 3, dtype=torch.float64, requires_grad=True)
    y = conv3(x, w)
    (y * gt).sum().backward()
    dw = w.grad.permute(0, 2, 3, 4, 1).reshape(co, 27, ci).numpy()
    return dw, gt.sum(dim=(0, 2, 3, 4)).numpy()
