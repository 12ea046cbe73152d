"""ORACLE -- test infrastructure only: float64 numpy restatement of the
learned denoiser of the fine density (forward pass, loss, weight gradient,
Adam step).  Never imported by the product path.

The denoiser has no counterpart in the reference (Vlasov.jl solves with the
deposited fine density as it is, deposit_smoothed! at src/accelerator.jl:531);
this file is the mathematical definition the CUDA kernels are checked
against, and its own gradient is pinned by finite differences of its own loss
(tests/test_oracle_denoiser.py, with the rounding off).

Network: four 3^3 convolutions, 1 -> 16 -> 16 -> 16 -> 3 channels, ReLU after
the first three, no biases, zero padding.  The three outputs are a flux
F = f(s x) and out = x + div F~ / s, F~ the flux with no flow through the
grid's faces (F~a = 0 on the last plane of axis a and before the first), so
that sum(out) = sum(x).  Weights of
layer l are stored flat as [27][cin][cout], tap = da + 3 db + 9 dc reading the
input at (i + da - 1, j + db - 1, k + dc - 1).  The passes use the weights
rounded to BF16 (nearest, ties to even); the gradient of the master weights is
the gradient with respect to the rounded ones (straight-through).

Volumes are numpy arrays of shape (nz, ny, nx) (x fastest, as the grids).
"""
from __future__ import annotations

import numpy as np

LAYERS = ((1, 16), (16, 16), (16, 16), (16, 3))
WEIGHT_COUNT = sum(27 * a * b for a, b in LAYERS)  # 15,552


def bf16_round(w):
    """Nearest BF16 value of float32 w, ties to even, as float32."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def split(w):
    """Flat weights -> list of (27, cin, cout) arrays."""
    out, o = [], 0
    for a, b in LAYERS:
        out.append(np.asarray(w[o:o + 27 * a * b], dtype=np.float64).reshape(27, a, b))
        o += 27 * a * b
    return out


def _shifted(x, tap):
    """x[k + dc - 1, j + db - 1, i + da - 1, :] with zeros outside; x is (nz, ny, nx, c)."""
    da, db, dc = tap % 3, (tap // 3) % 3, tap // 9
    p = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    nz, ny, nx = x.shape[:3]
    return p[dc:dc + nz, db:db + ny, da:da + nx, :]


def conv(x, w):
    """y[v, co] = sum_tap sum_ci w[tap, ci, co] x[v + tap - 1, ci]."""
    y = np.zeros(x.shape[:3] + (w.shape[2],))
    for tap in range(27):
        y += _shifted(x, tap) @ w[tap]
    return y


def conv_input_grad(g, w):
    """d/dx of sum(g * conv(x, w)): the correlation with the flipped kernel."""
    out = np.zeros(g.shape[:3] + (w.shape[1],))
    for tap in range(27):
        out += _shifted(g, 26 - tap) @ w[tap].T
    return out


def conv_weight_grad(x, g):
    """d/dw of sum(g * conv(x, w)): gw[tap, ci, co] = sum_v x[v + tap - 1, ci] g[v, co]."""
    cin, cout = x.shape[3], g.shape[3]
    gw = np.zeros((27, cin, cout))
    gf = g.reshape(-1, cout)
    for tap in range(27):
        gw[tap] = _shifted(x, tap).reshape(-1, cin).T @ gf
    return gw


def divergence(F):
    """div F~ of a (nz, ny, nx, 3) flux (channel a along axis x, y, z)."""
    out = np.zeros(F.shape[:3])
    for a, ax in ((0, 2), (1, 1), (2, 0)):
        f = np.moveaxis(F[..., a], ax, 0).copy()
        f[-1] = 0.0
        d = f.copy()
        d[1:] -= f[:-1]
        out += np.moveaxis(d, 0, ax)
    return out


def divergence_adjoint(g):
    """The adjoint of divergence(): G[u, a] = g[u] - g[u + e_a], 0 on the last plane."""
    G = np.zeros(g.shape + (3,))
    for a, ax in ((0, 2), (1, 1), (2, 0)):
        gg = np.moveaxis(g, ax, 0)
        d = np.zeros_like(gg)
        d[:-1] = gg[:-1] - gg[1:]
        G[..., a] = np.moveaxis(d, 0, ax)
    return G


def forward(x, weights, scale, rounding=True):
    """Activations of every layer (inputs included; the last is the flux F)
    and out = x + div F~ / scale.  rounding=False uses the weights as given
    (float64), for finite differences."""
    ws = split(bf16_round(weights) if rounding else weights)
    a = [scale * np.asarray(x, dtype=np.float64)[..., None]]
    for l, w in enumerate(ws):
        z = conv(a[-1], w)
        a.append(np.maximum(z, 0.0) if l < 3 else z)
    return a, np.asarray(x, dtype=np.float64) + divergence(a[-1]) / scale


def loss_and_grad(x, target, weights, scale, rounding=True):
    """loss = mean over voxels of (scale (out - target))^2 and its gradient
    with respect to the weights (flat, straight-through the BF16 rounding)."""
    ws = split(bf16_round(weights) if rounding else weights)
    a, out = forward(x, weights, scale, rounding)
    d = scale * (out - np.asarray(target, dtype=np.float64))
    nvox = d.size
    loss = float(np.sum(d * d) / nvox)
    g = divergence_adjoint(2.0 * d / nvox)
    grads = [None] * 4
    for l in range(3, -1, -1):
        grads[l] = conv_weight_grad(a[l], g)
        if l:
            g = conv_input_grad(g, ws[l]) * (a[l] > 0)
    return loss, np.concatenate([gr.ravel() for gr in grads])


def adam(w, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step with bias correction (step counts from 1); returns (w, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w, m, v


def active_tiles(x, tile=8):
    """Tiles of `tile`^3 voxels within one tile of a tile holding a nonzero input."""
    nz, ny, nx = x.shape
    tz, ty, tx = -(-nz // tile), -(-ny // tile), -(-nx // tile)
    flags = np.zeros((tz, ty, tx), dtype=bool)
    for c in range(tz):
        for b in range(ty):
            for a in range(tx):
                flags[c, b, a] = np.any(x[c * tile:(c + 1) * tile, b * tile:(b + 1) * tile, a * tile:(a + 1) * tile])
    p = np.pad(flags, 1)
    on = np.zeros_like(flags)
    for dc in range(3):
        for db in range(3):
            for da in range(3):
                on |= p[dc:dc + tz, db:db + ty, da:da + tx]
    return int(on.sum())
