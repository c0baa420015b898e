"""Float64 oracle of the learned multigrid smoother -- TEST INFRASTRUCTURE ONLY.

The reference's learned V-cycle smoother (``zoomy_jax/gnn_blueprint/
vcycle_structured_gnn.py`` :74-122 apply, :145-200 V-cycle;
``graph_mp_multibranch.py`` :9-16 the tanh message-passing layer;
``train_vcycle_structured_poisson.py`` :168-306 Adam training) is a local
learned operator applied to the residual on each level.  On a Cartesian grid
the B200 path uses a convolutional two-level U-Net for that operator; this
module restates that network in float64 numpy (forward, loss and the manual
backward pass) so the CUDA forward/backward/Adam kernels can be checked
against it, and a finite-difference test pins the restated backward itself.

Network (weights rounded to bf16 exactly as the device rounds them; all
arithmetic float64 here):

  s   = sqrt(mean r^2)                         per image
  c   = (cx_w + cx_e + cy_s + cy_n) / 4        cell coefficient
  in  = [r / s, c / cmax]
  e1  = tanh(conv(in, W0) + b0)                2 -> c1
  e2  = tanh(conv(e1, W1) + b1)                c1 -> c1
  m1  = tanh(conv(pool(e2), W2) + b2)          c1 -> c2 (2x2 average pool)
  m2  = tanh(conv(m1, W3) + b3)                c2 -> c2
  o1  = tanh(conv([up(m2), e2], W4) + b4)      c2 + c1 -> c1 (nearest upsample)
  out = conv(o1, W5) + b5                      c1 -> 1
  y   = s dx^2 / c * out

``conv`` is a 3x3 cross-correlation with zero padding; weights are
``[Cout][Cin][3][3]``.  Loss over a batch of patches with Dirichlet walls:
``mean_b |r_b - A_b y_b|^2 / |r_b|^2``.

``bf16_inputs=True`` mirrors the tensor-core engine: the input of every
convolution of the forward pass and of every data-gradient convolution of the
backward pass is rounded to bf16 (the MMA operands), while the weight
gradients are formed from the unrounded float32 values (the CUDA-core
weight-gradient kernel reads those).
"""
from __future__ import annotations

import numpy as np


def layer_shapes(c1, c2):
    """(cin, cout) of the six convolutions."""
    return [(2, c1), (c1, c1), (c1, c2), (c2, c2), (c1 + c2, c1), (c1, 1)]


def param_counts(c1, c2):
    nw = sum(ci * co * 9 for ci, co in layer_shapes(c1, c2))
    nb = sum(co for _, co in layer_shapes(c1, c2))
    return nw, nb


def bf16_round(w):
    """float -> nearest bf16 (ties to even) -> float64."""
    a = np.asarray(w, dtype=np.float32).copy()
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split(flat_w, flat_b, c1, c2):
    """Flat concatenated weights/biases -> per-layer arrays."""
    Ws, bs = [], []
    ow = ob = 0
    for ci, co in layer_shapes(c1, c2):
        Ws.append(np.asarray(flat_w[ow:ow + co * ci * 9], dtype=np.float64).reshape(co, ci, 3, 3))
        bs.append(np.asarray(flat_b[ob:ob + co], dtype=np.float64))
        ow += co * ci * 9
        ob += co
    return Ws, bs


def conv(x, W, b=None):
    """x (Cin, B, H, W) -> (Cout, B, H, W); zero padding, cross-correlation."""
    cin, B, H, Wd = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    out = np.zeros((W.shape[0], B, H, Wd))
    for dy in range(3):
        for dx in range(3):
            out += np.einsum("oi,ibhw->obhw", W[:, :, dy, dx], xp[:, :, dy:dy + H, dx:dx + Wd])
    if b is not None:
        out += b[:, None, None, None]
    return out


def conv_back(x, W, g, bf16_inputs=False):
    """Gradients of conv(x, W, b) for the output gradient g: (dx, dW, db).
    With ``bf16_inputs`` the data gradient is formed from g rounded to bf16."""
    cin, B, H, Wd = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    gd = bf16_round(g) if bf16_inputs else g
    dW = np.zeros_like(W)
    dxp = np.zeros_like(xp)
    for dy in range(3):
        for dx in range(3):
            dW[:, :, dy, dx] = np.einsum("obhw,ibhw->oi", g, xp[:, :, dy:dy + H, dx:dx + Wd])
            dxp[:, :, dy:dy + H, dx:dx + Wd] += np.einsum("oi,obhw->ibhw", W[:, :, dy, dx], gd)
    return dxp[:, :, 1:-1, 1:-1], dW, g.sum(axis=(1, 2, 3))


def pool(x):
    C, B, H, W = x.shape
    return x.reshape(C, B, H // 2, 2, W // 2, 2).mean(axis=(3, 5))


def up(x):
    return np.repeat(np.repeat(x, 2, axis=2), 2, axis=3)


def cell_coefficient(cx, cy):
    """cx (B, H+1, W), cy (B, H, W+1) -> (B, H, W)."""
    return 0.25 * (cx[:, :-1] + cx[:, 1:] + cy[:, :, :-1] + cy[:, :, 1:])


def apply_batch(cx, cy, x, dx):
    """A x per image (Dirichlet ghost -x); x (B, H, W)."""
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
    xp[:, 0, :] = -xp[:, 1, :]
    xp[:, -1, :] = -xp[:, -2, :]
    xp[:, :, 0] = -xp[:, :, 1]
    xp[:, :, -1] = -xp[:, :, -2]
    xc = xp[:, 1:-1, 1:-1]
    return (cx[:, 1:] * (xc - xp[:, 2:, 1:-1]) + cx[:, :-1] * (xc - xp[:, :-2, 1:-1])
            + cy[:, :, 1:] * (xc - xp[:, 1:-1, 2:]) + cy[:, :, :-1] * (xc - xp[:, 1:-1, :-2])) / dx ** 2


def forward(Ws, bs, r, cx, cy, dx, cmax, bf16_inputs=False):
    """r (B, H, W) -> (y (B, H, W), cache).  Ws must already be bf16-rounded."""
    rnd = bf16_round if bf16_inputs else (lambda a: a)
    B = r.shape[0]
    s = np.sqrt(np.mean(r.reshape(B, -1) ** 2, axis=1))
    s = np.maximum(s, 1e-30)
    c = cell_coefficient(cx, cy)
    x_in = np.stack([r / s[:, None, None], c / cmax])
    e1 = np.tanh(conv(rnd(x_in), Ws[0], bs[0]))
    e2 = np.tanh(conv(rnd(e1), Ws[1], bs[1]))
    p = pool(e2)
    m1 = np.tanh(conv(rnd(p), Ws[2], bs[2]))
    m2 = np.tanh(conv(rnd(m1), Ws[3], bs[3]))
    u = up(m2)
    cat = np.concatenate([u, e2])
    o1 = np.tanh(conv(rnd(cat), Ws[4], bs[4]))
    out = conv(rnd(o1), Ws[5], bs[5])[0]
    scale = s[:, None, None] * dx ** 2 / c
    y = scale * out
    cache = dict(x_in=x_in, e1=e1, e2=e2, p=p, m1=m1, m2=m2, u=u, cat=cat, o1=o1,
                 out=out, scale=scale, s=s)
    return y, cache


def loss_and_grads(Ws, bs, r, cx, cy, dx, cmax, bf16_inputs=False, target=None):
    """Loss and its gradients (dWs, dbs).  Without ``target``: the residual
    loss ``mean_b |r - A y|^2 / |r|^2``; with the exact errors ``target``
    (``A e = r``): the energy-norm loss ``mean_b (d . A d) / (e . A e)``,
    ``d = e - y``.  Images with a denominator <= 1e-30 are left out."""
    B = r.shape[0]
    q = bf16_inputs
    y, k = forward(Ws, bs, r, cx, cy, dx, cmax, bf16_inputs=q)
    if target is None:
        res = r - apply_batch(cx, cy, y, dx)
        Ares = apply_batch(cx, cy, res, dx)
        num = np.sum(res.reshape(B, -1) ** 2, axis=1)
        den = np.sum(r.reshape(B, -1) ** 2, axis=1)
    else:
        res = target - y
        Ares = apply_batch(cx, cy, res, dx)
        num = np.sum((res * Ares).reshape(B, -1), axis=1)
        den = np.sum((target * apply_batch(cx, cy, target, dx)).reshape(B, -1), axis=1)
    ok = den > 1e-30
    dsafe = np.where(ok, den, 1.0)
    loss = float(np.sum(np.where(ok, num / dsafe, 0.0)) / B)
    dy = np.where(ok[:, None, None], -2.0 * Ares / (B * dsafe[:, None, None]), 0.0)
    d_out = (dy * k["scale"])[None]
    dWs = [None] * 6
    dbs = [None] * 6
    d_o1, dWs[5], dbs[5] = conv_back(k["o1"], Ws[5], d_out, q)
    d_o1 = d_o1 * (1.0 - k["o1"] ** 2)
    d_cat, dWs[4], dbs[4] = conv_back(k["cat"], Ws[4], d_o1, q)
    c2 = Ws[3].shape[0]
    d_u, d_e2_skip = d_cat[:c2], d_cat[c2:]
    C, Bb, H, W = d_u.shape
    d_m2 = d_u.reshape(C, Bb, H // 2, 2, W // 2, 2).sum(axis=(3, 5))
    d_m2 = d_m2 * (1.0 - k["m2"] ** 2)
    d_m1, dWs[3], dbs[3] = conv_back(k["m1"], Ws[3], d_m2, q)
    d_m1 = d_m1 * (1.0 - k["m1"] ** 2)
    d_p, dWs[2], dbs[2] = conv_back(k["p"], Ws[2], d_m1, q)
    d_e2 = up(d_p) / 4.0 + d_e2_skip
    d_e2 = d_e2 * (1.0 - k["e2"] ** 2)
    d_e1, dWs[1], dbs[1] = conv_back(k["e1"], Ws[1], d_e2, q)
    d_e1 = d_e1 * (1.0 - k["e1"] ** 2)
    _, dWs[0], dbs[0] = conv_back(k["x_in"], Ws[0], d_e1)
    return loss, dWs, dbs


def smoother_apply(Ws, bs, f, x, cx, cy, dx, cmax, bf16_inputs=False):
    """One learned smoothing on a single grid: x + S(f - A x).
    cx (H+1, W), cy (H, W+1); x may be None (zero start)."""
    x0 = np.zeros_like(f) if x is None else x
    r = f - apply_batch(cx[None], cy[None], x0[None], dx)[0]
    y, _ = forward(Ws, bs, r[None], cx[None], cy[None], dx, cmax, bf16_inputs=bf16_inputs)
    return x0 + y[0]
