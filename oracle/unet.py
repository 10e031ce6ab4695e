"""CPU oracle of the learned pressure preconditioner (test infrastructure only).

The reference has no learned part: its pressure solve is BiCGSTAB with an FFT
preconditioner (projection_3d.py:756-791).  The learned form replaces the
preconditioner of the flexible CG with a small 3-D convolutional U-Net; this
module restates that network in float64 numpy so that the device kernels'
forward pass and gradients can be checked against it:

* layout: activations are (Z, Y, X, C) with the channel innermost;
* conv: 3x3x3, zero padding, weights W[tap][cin][cout] with
  tap = (dz+1)*9 + (dy+1)*3 + (dx+1), plus a bias per output channel;
* levels: 4, each coarser level ceil(n/2) per axis; down = 2x2x2 average
  with a fixed 1/8 (cells past an odd edge count as zero); up = nearest
  (every fine cell takes its parent's value), concatenated before the skip;
* channels 16 / 32 / 48 / 64; the input is the residual in channel 0 of 16
  (channels 1-15 zero); the output is a 1x1 head 16 -> 1 without activation;
* ``rnd=True`` rounds to bfloat16 wherever the device stores bfloat16
  (activations, their gradients, the conv weights), so the comparison with
  the device is limited only by fp32 accumulation order.
"""
from __future__ import annotations

import numpy as np

# (name, cin, cout, level, input)
LAYERS = (
    ("enc0a", 16, 16, 0), ("enc0b", 16, 16, 0),
    ("enc1a", 16, 32, 1), ("enc1b", 32, 32, 1),
    ("enc2a", 32, 48, 2), ("enc2b", 48, 48, 2),
    ("enc3a", 48, 64, 3), ("enc3b", 64, 64, 3),
    ("dec2", 112, 48, 2), ("dec1", 80, 32, 1), ("dec0", 48, 16, 0),
)
HEAD_C = 16
N_LEVELS = 4


def param_layout():
    """Offsets of every layer's W[27][cin][cout] and bias[cout] in the flat
    parameter vector, then the head's w[16] and b[1]."""
    off = 0
    out = []
    for name, cin, cout, _lv in LAYERS:
        w = off
        off += 27 * cin * cout
        b = off
        off += cout
        out.append((name, cin, cout, w, b))
    head_w = off
    off += HEAD_C
    head_b = off
    off += 1
    return out, head_w, head_b, off


def n_params():
    return param_layout()[3]


def level_dims(nz, ny, nx):
    dims = [(nz, ny, nx)]
    for _ in range(N_LEVELS - 1):
        z, y, x = dims[-1]
        dims.append(((z + 1) // 2, (y + 1) // 2, (x + 1) // 2))
    return dims


def init_params(seed=0):
    """He-uniform conv weights, zero biases, small head (float32 values)."""
    rng = np.random.default_rng(seed)
    lay, hw, hb, n = param_layout()
    p = np.zeros(n, dtype=np.float64)
    for _name, cin, cout, w, _b in lay:
        lim = np.sqrt(6.0 / (27 * cin))
        p[w:w + 27 * cin * cout] = rng.uniform(-lim, lim, 27 * cin * cout)
    p[hw:hw + HEAD_C] = rng.uniform(-0.25, 0.25, HEAD_C)
    return p.astype(np.float32).astype(np.float64)


def bf16(a, on=True):
    """Round float64 values to bfloat16 (via float32, nearest-even), as the
    device's __float2bfloat16_rn does after an fp32 result."""
    if not on:
        return np.asarray(a, dtype=np.float64)
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(a, on=True):
    return np.asarray(a, dtype=np.float32).astype(np.float64) if on else a


def _taps():
    return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def conv(x, W, b):
    """3x3x3 zero-padded convolution: out[p] = b + sum_t x[p + off(t)] @ W[t]."""
    Z, Y, X, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((Z, Y, X, W.shape[2]))
    for t, (dz, dy, dx) in enumerate(_taps()):
        out += xp[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X] @ W[t]
    if b is not None:
        out += b
    return out


def conv_bwd_data(g, W):
    """dX[q] = sum_t g[q - off(t)] @ W[t]^T (the adjoint of ``conv``)."""
    Z, Y, X, _ = g.shape
    gp = np.pad(g, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((Z, Y, X, W.shape[1]))
    for t, (dz, dy, dx) in enumerate(_taps()):
        out += gp[1 - dz:1 - dz + Z, 1 - dy:1 - dy + Y, 1 - dx:1 - dx + X] @ W[t].T
    return out


def conv_bwd_weight(x, g):
    """dW[t] = sum_p x[p + off(t)]^T g[p];  db = sum_p g[p]."""
    Z, Y, X, cin = x.shape
    cout = g.shape[3]
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    gm = g.reshape(-1, cout)
    dW = np.zeros((27, cin, cout))
    for t, (dz, dy, dx) in enumerate(_taps()):
        xs = xp[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X].reshape(-1, cin)
        dW[t] = xs.T @ gm
    return dW, gm.sum(axis=0)


def pool(f, cdims):
    Z, Y, X, C = f.shape
    cz, cy, cx = cdims
    fp = np.zeros((2 * cz, 2 * cy, 2 * cx, C))
    fp[:Z, :Y, :X] = f
    return fp.reshape(cz, 2, cy, 2, cx, 2, C).sum(axis=(1, 3, 5)) * 0.125


def up(a, fdims):
    Z, Y, X = fdims
    u = np.repeat(np.repeat(np.repeat(a, 2, axis=0), 2, axis=1), 2, axis=2)
    return u[:Z, :Y, :X]


def up_adjoint(g, cdims):
    """Sum of every coarse cell's children (the adjoint of ``up``)."""
    Z, Y, X, C = g.shape
    cz, cy, cx = cdims
    gp = np.zeros((2 * cz, 2 * cy, 2 * cx, C))
    gp[:Z, :Y, :X] = g
    return gp.reshape(cz, 2, cy, 2, cx, 2, C).sum(axis=(1, 3, 5))


def _unpack(params, rnd):
    lay, hw, hb, _ = param_layout()
    Ws, bs = [], []
    for _name, cin, cout, w, b in lay:
        Ws.append(bf16(params[w:w + 27 * cin * cout], rnd).reshape(27, cin, cout))
        bs.append(f32(params[b:b + cout], rnd))
    return Ws, bs, f32(params[hw:hw + HEAD_C], rnd), f32(params[hb], rnd)


def forward(params, r, rnd=True):
    """z = N(r) for r of shape (Z, Y, X); returns z and the activations."""
    Ws, bs, wh, bh = _unpack(params, rnd)
    dims = level_dims(*r.shape)
    A = {}
    x0 = np.zeros(r.shape + (16,))
    x0[..., 0] = bf16(f32(r, rnd), rnd)
    A["x0"] = x0

    def cr(name, x, li):
        y = conv(x, Ws[li], bs[li])
        A[name] = bf16(np.maximum(y, 0.0), rnd)
        return A[name]

    e0 = cr("e0", x0, 0)
    e0b = cr("e0b", e0, 1)
    A["d1"] = d1 = bf16(pool(e0b, dims[1]), rnd)
    e1 = cr("e1", d1, 2)
    e1b = cr("e1b", e1, 3)
    A["d2"] = d2 = bf16(pool(e1b, dims[2]), rnd)
    e2 = cr("e2", d2, 4)
    e2b = cr("e2b", e2, 5)
    A["d3"] = d3 = bf16(pool(e2b, dims[3]), rnd)
    e3 = cr("e3", d3, 6)
    e3b = cr("e3b", e3, 7)
    A["c2"] = c2 = np.concatenate([up(e3b, dims[2]), e2b], axis=3)
    u2 = cr("u2", c2, 8)
    A["c1"] = c1 = np.concatenate([up(u2, dims[1]), e1b], axis=3)
    u1 = cr("u1", c1, 9)
    A["c0"] = c0 = np.concatenate([up(u1, dims[0]), e0b], axis=3)
    u0 = cr("u0", c0, 10)
    z = f32(u0 @ wh + bh, rnd)
    return z, A


def backward(params, A, dz, rnd=True, scale=None):
    """Gradient of sum(dz * z) with respect to the flat parameters.

    With ``scale`` (a dict) also records, per layer, the norm of the same
    weight gradient taken over absolute values (sum_p |x| |g|): the size of
    the terms before they cancel, against which a rounding error in the
    terms is measured."""
    Ws, _bs, wh, _bh = _unpack(params, rnd)
    lay, hw, hb, n = param_layout()
    dims = level_dims(*dz.shape)
    grad = np.zeros(n)

    def put(li, x, g):
        dW, db = conv_bwd_weight(x, g)
        _name, cin, cout, w, b = lay[li]
        grad[w:w + 27 * cin * cout] = dW.ravel()
        grad[b:b + cout] = db
        if scale is not None:
            aW, ab = conv_bwd_weight(np.abs(x), np.abs(g))
            scale[_name + ".W"] = float(np.linalg.norm(aW))
            scale[_name + ".b"] = float(np.linalg.norm(ab))

    m = lambda a: (a > 0).astype(np.float64)  # noqa: E731
    u0 = A["u0"]
    grad[hw:hw + HEAD_C] = (u0 * dz[..., None]).reshape(-1, HEAD_C).sum(axis=0)
    grad[hb] = dz.sum()
    if scale is not None:
        scale["head"] = float(np.linalg.norm(np.append(
            (np.abs(u0) * np.abs(dz)[..., None]).reshape(-1, HEAD_C).sum(axis=0),
            np.abs(dz).sum())))
    g_u0 = bf16(dz[..., None] * wh, rnd) * m(u0)
    put(10, A["c0"], g_u0)
    g_c0 = bf16(conv_bwd_data(g_u0, Ws[10]) * m(A["c0"]), rnd)
    g_u1 = bf16(up_adjoint(g_c0[..., :32], dims[1]), rnd)
    g_e0b = g_c0[..., 32:]
    put(9, A["c1"], g_u1)
    g_c1 = bf16(conv_bwd_data(g_u1, Ws[9]) * m(A["c1"]), rnd)
    g_u2 = bf16(up_adjoint(g_c1[..., :48], dims[2]), rnd)
    g_e1b = g_c1[..., 48:]
    put(8, A["c2"], g_u2)
    g_c2 = bf16(conv_bwd_data(g_u2, Ws[8]) * m(A["c2"]), rnd)
    g_e3b = bf16(up_adjoint(g_c2[..., :64], dims[3]), rnd)
    g_e2b = g_c2[..., 64:]

    def enc(li_b, li_a, g_xb, xa_name, xin_name, g_skip_prev, fine_name):
        # block: xa = relu(conv(xin)), xb = relu(conv(xa)); xin = pool(fine)
        put(li_b, A[xa_name], g_xb)
        g_xa = bf16(conv_bwd_data(g_xb, Ws[li_b]) * m(A[xa_name]), rnd)
        put(li_a, A[xin_name], g_xa)
        if fine_name is None:
            return None
        g_in = bf16(conv_bwd_data(g_xa, Ws[li_a]), rnd)
        fine = A[fine_name]
        fd = fine.shape[:3]
        return bf16((g_skip_prev + up(g_in, fd) * 0.125) * m(fine), rnd)

    g_e2b = enc(7, 6, g_e3b, "e3", "d3", g_e2b, "e2b")
    g_e1b = enc(5, 4, g_e2b, "e2", "d2", g_e1b, "e1b")
    g_e0b = enc(3, 2, g_e1b, "e1", "d1", g_e0b, "e0b")
    enc(1, 0, g_e0b, "e0", "x0", None, None)
    return grad


def loss_and_grad(params, r, tau, rnd=True, scale=None):
    """Mean squared error of N(r) against tau and its parameter gradient."""
    z, A = forward(params, r, rnd)
    n = z.size
    d = z - tau
    dz = f32(2.0 * d / n, rnd)
    return float((d * d).sum() / n), backward(params, A, dz, rnd, scale), z
