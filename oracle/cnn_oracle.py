"""CPU restatement (numpy, float64) of the learned short-range network.

Test infrastructure only: the tests and the smoke check compare the device
network's forward pass, gradients and Adam update with these functions.  The
network has no counterpart in the reference, so this file is its own
specification:

* input: a batch of volumes X0[B, Z, Y, X, C_IN] of mesh features;
* three valid 3x3x3 convolutions to 16 channels, each followed by
  GELU(z) = z/2 (1 + erf(z/sqrt 2)); a volume shrinks by 2 cells per axis
  per layer (the device evaluates a whole periodic mesh by padding it by 3);
* a per-node linear head 16 -> 3 (the short-range acceleration field);
* the head is read at each particle by trilinear interpolation between the
  8 mesh nodes around it (the CIC weights of the PM gather);
* loss = sum_p w_p |pred_p - target_p|^2 / sum_p w_p;
* Adam (Kingma & Ba 2015) with bias correction.

Tap t = (dz*3 + dy)*3 + dx reads input node o + (dx, dy, dz) for output node
o.  The flat parameter vector is [W1 (27,16,C_IN), b1 (16), W2 (27,16,16),
b2, W3 (27,16,16), b3, Wh (3,16), bh (3)].
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

C_HID = 16
N_OUT = 3


def param_shapes(c_in: int):
    return [(27, C_HID, c_in), (C_HID,), (27, C_HID, C_HID), (C_HID,), (27, C_HID, C_HID), (C_HID,),
            (N_OUT, C_HID), (N_OUT,)]


def n_params(c_in: int) -> int:
    return int(sum(np.prod(s) for s in param_shapes(c_in)))


def unflatten(p, c_in: int):
    out, o = [], 0
    for s in param_shapes(c_in):
        k = int(np.prod(s))
        out.append(np.asarray(p[o:o + k], dtype=np.float64).reshape(s))
        o += k
    return out


def flatten(parts):
    return np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in parts])


def init_params(c_in: int, seed: int = 0):
    """He-style initialisation (normal, std sqrt(2 / fan_in)); zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for s in param_shapes(c_in):
        if len(s) == 1:
            parts.append(np.zeros(s))
        else:
            fan_in = s[-1] * (27 if len(s) == 3 else 1)
            parts.append(rng.normal(0.0, np.sqrt(2.0 / fan_in), s))
    return flatten(parts)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def taps():
    return [(t % 3, (t // 3) % 3, t // 9) for t in range(27)]  # (dx, dy, dz)


def conv_valid(x, w, b):
    """x[B,Z,Y,X,Ci], w[27,Co,Ci], b[Co] -> z[B,Z-2,Y-2,X-2,Co]."""
    B, Z, Y, X, _ = x.shape
    z = np.zeros((B, Z - 2, Y - 2, X - 2, w.shape[1])) + b
    for t, (dx, dy, dz) in enumerate(taps()):
        z += x[:, dz:dz + Z - 2, dy:dy + Y - 2, dx:dx + X - 2, :] @ w[t].T
    return z


def conv_valid_backward(x, w, dz):
    """Gradients of conv_valid: (dx, dw, db)."""
    B, Zo, Yo, Xo, Co = dz.shape
    dx_ = np.zeros_like(x)
    dw = np.zeros_like(w)
    flat = dz.reshape(-1, Co)
    for t, (ox, oy, oz) in enumerate(taps()):
        xs = x[:, oz:oz + Zo, oy:oy + Yo, ox:ox + Xo, :]
        dw[t] = flat.T @ xs.reshape(-1, x.shape[-1])
        dx_[:, oz:oz + Zo, oy:oy + Yo, ox:ox + Xo, :] += dz @ w[t]
    return dx_, dw, flat.sum(0)


def forward(params, x0, bf16_activations: bool = False):
    """Forward pass; `bf16_activations` rounds each layer's GELU output to
    bfloat16 as the device stores it between layers."""
    w1, b1, w2, b2, w3, b3, wh, bh = unflatten(params, x0.shape[-1])
    act = (lambda z: to_bf16(gelu(z))) if bf16_activations else gelu
    z1 = conv_valid(x0, w1, b1)
    a1 = act(z1)
    z2 = conv_valid(a1, w2, b2)
    a2 = act(z2)
    z3 = conv_valid(a2, w3, b3)
    a3 = act(z3)
    out = a3 @ wh.T + bh
    return dict(z1=z1, a1=a1, z2=z2, a2=a2, z3=z3, a3=a3, out=out)


def _corners(s):
    i0 = np.floor(s).astype(np.int64)
    f = s - i0
    return i0, f


def interpolate(out, pb, ps):
    """Trilinear read of out[B,Z,Y,X,3] at local node coordinates ps[n,(x,y,z)] of volume pb[n]."""
    i0, f = _corners(ps)
    pred = np.zeros((len(pb), out.shape[-1]))
    for c in range(8):
        ox, oy, oz = c & 1, (c >> 1) & 1, c >> 2
        wgt = ((f[:, 0] if ox else 1 - f[:, 0]) * (f[:, 1] if oy else 1 - f[:, 1]) *
               (f[:, 2] if oz else 1 - f[:, 2]))
        pred += wgt[:, None] * out[pb, i0[:, 2] + oz, i0[:, 1] + oy, i0[:, 0] + ox]
    return pred


def loss_and_grads(params, x0, pb, ps, target, weight):
    """Loss and d loss / d params for one batch."""
    c_in = x0.shape[-1]
    w1, b1, w2, b2, w3, b3, wh, bh = unflatten(params, c_in)
    f = forward(params, x0)
    pred = interpolate(f["out"], pb, ps)
    wsum = weight.sum()
    diff = pred - target
    loss = float((weight[:, None] * diff * diff).sum() / wsum)
    dpred = 2.0 * weight[:, None] * diff / wsum
    dout = np.zeros_like(f["out"])
    i0, fr = _corners(ps)
    for c in range(8):
        ox, oy, oz = c & 1, (c >> 1) & 1, c >> 2
        wgt = ((fr[:, 0] if ox else 1 - fr[:, 0]) * (fr[:, 1] if oy else 1 - fr[:, 1]) *
               (fr[:, 2] if oz else 1 - fr[:, 2]))
        np.add.at(dout, (pb, i0[:, 2] + oz, i0[:, 1] + oy, i0[:, 0] + ox), wgt[:, None] * dpred)
    dflat = dout.reshape(-1, N_OUT)
    dwh = dflat.T @ f["a3"].reshape(-1, C_HID)
    dbh = dflat.sum(0)
    dz3 = (dout @ wh) * gelu_grad(f["z3"])
    da2, dw3, db3 = conv_valid_backward(f["a2"], w3, dz3)
    dz2 = da2 * gelu_grad(f["z2"])
    da1, dw2, db2 = conv_valid_backward(f["a1"], w2, dz2)
    dz1 = da1 * gelu_grad(f["z1"])
    _, dw1, db1 = conv_valid_backward(x0, w1, dz1)
    return loss, flatten([dw1, db1, dw2, db2, dw3, db3, dwh, dbh])


def adam(params, grad, m, v, step, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (step counts from 1); returns new (params, m, v)."""
    m = beta1 * m + (1.0 - beta1) * grad
    v = beta2 * v + (1.0 - beta2) * grad * grad
    mh = m / (1.0 - beta1 ** step)
    vh = v / (1.0 - beta2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v


def to_bf16(x):
    """Round float64 values to the nearest bfloat16 (ties to even), as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)
