"""FP64 restatement of the learned proposal network (test infrastructure only).

The reference has no learned proposal; this module is the oracle of the
network kernels in cistem_downstream_bah_b200/csrc/tm_proposal.cu: the same
layers, tie rules and loss written as plain numpy in float64, with the
backward pass derived by hand.  ``bf16=True`` rounds the weights to BF16
(round to nearest even) before use, as the kernels do; the weight gradient is
then the gradient with respect to those rounded values.  The backward pass is
itself pinned by central differences in float64 (tests/test_proposal_cpu.py).
Only the tests import this module; the product never does.

Network (tile x tile input, cin channels):
  conv3x3(cin->32)+ReLU, maxpool2; conv3x3(32->64)+ReLU, maxpool2;
  conv3x3(64->128)+ReLU, maxpool2; conv3x3(128->128)+ReLU, global max;
  fully connected 128 -> 4 (objectness logit, direction x, y, z).
"""
from __future__ import annotations

import numpy as np

CHANNELS = (32, 64, 128, 128)
N_OUT = 4


def layout(cin):
    """[(name, shape)] in the flat parameter order of the kernels."""
    chans = (cin,) + CHANNELS
    out = []
    for i in range(4):
        out.append((f"w{i + 1}", (chans[i + 1], chans[i], 3, 3)))
        out.append((f"b{i + 1}", (chans[i + 1],)))
    out.append(("w5", (N_OUT, CHANNELS[-1])))
    out.append(("b5", (N_OUT,)))
    return out


def param_count(cin):
    return int(sum(np.prod(s) for _, s in layout(cin)))


def unflatten(flat, cin):
    d, o = {}, 0
    for name, shape in layout(cin):
        n = int(np.prod(shape))
        d[name] = np.asarray(flat[o:o + n], np.float64).reshape(shape)
        o += n
    return d


def flatten(d, cin):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in layout(cin)])


def bf16_round(x):
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    b = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def _conv(x, w, b):
    n, ci, h, wd = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    out = np.zeros((n, w.shape[0], h, wd))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("nihw,oi->nohw", xp[:, :, ky:ky + h, kx:kx + wd], w[:, :, ky, kx], optimize=True)
    if b is not None:
        out += b[None, :, None, None]
    return out


def _conv_wgrad(x, g):
    n, ci, h, wd = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    dw = np.zeros((g.shape[1], ci, 3, 3))
    for ky in range(3):
        for kx in range(3):
            dw[:, :, ky, kx] = np.einsum("nohw,nihw->oi", g, xp[:, :, ky:ky + h, kx:kx + wd], optimize=True)
    return dw, g.sum(axis=(0, 2, 3))


def _conv_dgrad(g, w):
    n, co, h, wd = g.shape
    dxp = np.zeros((n, w.shape[1], h + 2, wd + 2))
    for ky in range(3):
        for kx in range(3):
            dxp[:, :, ky:ky + h, kx:kx + wd] += np.einsum("nohw,oi->nihw", g, w[:, :, ky, kx], optimize=True)
    return dxp[:, :, 1:-1, 1:-1]


def _pool(a):
    n, c, h, w = a.shape
    cand = a.reshape(n, c, h // 2, 2, w // 2, 2).transpose(0, 1, 2, 4, 3, 5).reshape(n, c, h // 2, w // 2, 4)
    arg = np.argmax(cand, axis=-1)          # first maximum in (0,0), (0,1), (1,0), (1,1) order
    return np.take_along_axis(cand, arg[..., None], -1)[..., 0], arg


def _pool_bwd(g, arg, act):
    n, c, h2, w2 = g.shape
    sel = np.zeros((n, c, h2, w2, 4))
    np.put_along_axis(sel, arg[..., None], g[..., None], -1)
    d = sel.reshape(n, c, h2, w2, 2, 2).transpose(0, 1, 2, 4, 3, 5).reshape(n, c, 2 * h2, 2 * w2)
    return np.where(act > 0, d, 0.0)


def forward(params, x, cin, bf16=True):
    """Outputs (n, 4) and the cache of the backward pass."""
    p = unflatten(params, cin)
    W = {k: (bf16_round(v) if (bf16 and k.startswith("w")) else v) for k, v in p.items()}
    x = np.asarray(x, np.float64)
    cache = {"x": x, "W": W}
    h = x
    for i in range(1, 4):
        a = np.maximum(_conv(h, W[f"w{i}"], W[f"b{i}"]), 0.0)
        q, arg = _pool(a)
        cache[f"h{i}"], cache[f"a{i}"], cache[f"arg{i}"] = h, a, arg
        h = q
    a4 = np.maximum(_conv(h, W["w4"], W["b4"]), 0.0)
    n, c = a4.shape[:2]
    flat = a4.reshape(n, c, -1)
    arg4 = np.argmax(flat, axis=-1)
    g = np.take_along_axis(flat, arg4[..., None], -1)[..., 0]
    cache.update(h4=h, a4=a4, arg4=arg4, g=g)
    out = g @ W["w5"].T + W["b5"]
    return out, cache


def loss_and_dout(out, labels, pos_weight, dir_weight):
    """Loss and its gradient with respect to the outputs (the kernel's k_loss)."""
    out = np.asarray(out, np.float64)
    lab = np.asarray(labels, np.float64)
    n = len(out)
    y = lab[:, 0]
    z = out[:, 0]
    w = np.where(y > 0.5, pos_weight, 1.0)
    bce = np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z)))
    sig = 1.0 / (1.0 + np.exp(-z))
    d = np.zeros_like(out)
    d[:, 0] = w * (sig - y) / n
    li = w * bce
    pos = y > 0.5
    dv = out[:, 1:4]
    t = lab[:, 1:4]
    nn = (dv * dv).sum(1) + 1e-12
    inv = 1.0 / np.sqrt(nn)
    dot = (dv * t).sum(1)
    li = li + np.where(pos, dir_weight * (1.0 - dot * inv), 0.0)
    grad_d = -dir_weight / n * inv[:, None] * (t - (dot / nn)[:, None] * dv)
    d[:, 1:4] = np.where(pos[:, None], grad_d, 0.0)
    return li.sum() / n, d


def gradients(params, x, labels, cin, pos_weight=1.0, dir_weight=1.0, bf16=True):
    """Loss and the flat gradient (the kernels' tm_pnet_gradients)."""
    out, c = forward(params, x, cin, bf16)
    loss, dout = loss_and_dout(out, labels, pos_weight, dir_weight)
    W = c["W"]
    gr = {"w5": dout.T @ c["g"], "b5": dout.sum(0)}
    dg = dout @ W["w5"]
    a4 = c["a4"]
    n, ch = a4.shape[:2]
    da4 = np.zeros((n, ch, a4.shape[2] * a4.shape[3]))
    np.put_along_axis(da4, c["arg4"][..., None], dg[..., None], -1)
    da = np.where(a4 > 0, da4.reshape(a4.shape), 0.0)
    gr["w4"], gr["b4"] = _conv_wgrad(c["h4"], da)
    dh = _conv_dgrad(da, W["w4"])
    for i in (3, 2, 1):
        da = _pool_bwd(dh, c[f"arg{i}"], c[f"a{i}"])
        gr[f"w{i}"], gr[f"b{i}"] = _conv_wgrad(c[f"h{i}"], da)
        if i > 1:
            dh = _conv_dgrad(da, W[f"w{i}"])
    return loss, flatten(gr, cin)


def loss_only(params, x, labels, cin, pos_weight=1.0, dir_weight=1.0, bf16=False):
    out, _ = forward(params, x, cin, bf16)
    return loss_and_dout(out, labels, pos_weight, dir_weight)[0]
