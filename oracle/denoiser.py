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
F = f(s x) and out = x + div F^ / s, F~ the flux with no flow through the
grid's faces (F~a = 0 on the last plane of axis a and before the first) and
F^ that flux limited so that no voxel gives more than it holds: the face
flux p = F~a[u] leaves its donor (u + e_a when p > 0, u when p < 0); a donor
with charge c = s x and outflow O = sum of its |p| scales them all by
lam = 1 (O <= c), c / O (O > c > 0), 0 (c <= 0).  So sum(out) = sum(x) and
out >= min(x, 0).  Weights of
layer l are stored flat as [27][cin][cout], tap = da + 3 db + 9 dc reading the
input at (i + da - 1, j + db - 1, k + dc - 1).  The passes use the weights
rounded to BF16 (nearest, ties to even); the gradient of the master weights is
the gradient with respect to the rounded ones (straight-through).

The network is evaluated on the active tiles of 8^3 voxels: a tile is
flagged when its largest |x| exceeds TILE_THRESHOLD times the volume's, the
active tiles are the flagged ones and their neighbours, and every layer's
activations (the input included) are zero outside them.

Volumes are numpy arrays of shape (nz, ny, nx) (x fastest, as the grids).
"""
from __future__ import annotations

import numpy as np

LAYERS = ((1, 16), (16, 16), (16, 16), (16, 3))
TILE = 8
TILE_THRESHOLD = np.float32(1e-3)
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


AXES = ((0, 2), (1, 1), (2, 0))   # flux channel -> array axis (x, y, z)


def _shift(arr, ax, k):
    """arr at index + k along axis ax, zero outside."""
    out = np.zeros_like(arr)
    n = arr.shape[ax]
    src, dst = [slice(None)] * arr.ndim, [slice(None)] * arr.ndim
    if k > 0:
        src[ax], dst[ax] = slice(k, n), slice(0, n - k)
    else:
        src[ax], dst[ax] = slice(0, n + k), slice(-k, n)
    out[tuple(dst)] = arr[tuple(src)]
    return out


def face_flux(F):
    """F~: the flux with the last plane of each channel's axis zeroed."""
    Ft = np.array(F, dtype=np.float64)
    for a, ax in AXES:
        sl = [slice(None)] * 3
        sl[ax] = -1
        Ft[tuple(sl) + (a,)] = 0.0
    return Ft


def limiter(Ft, c):
    """(lam, O) of every voxel as a donor, for face fluxes Ft and charges c."""
    O = np.zeros(c.shape)
    for a, ax in AXES:
        p = Ft[..., a]
        O += np.maximum(-p, 0.0) + _shift(np.maximum(p, 0.0), ax, -1)
    safe = np.where(O > 0, O, 1.0)
    lam = np.where(O <= c, 1.0, np.where(c > 0, c / safe, 0.0))
    return lam, O


def _donor(arr, p, ax):
    """arr at the donor of each face flux p (index + 1 along ax when p > 0)."""
    return np.where(p > 0, _shift(arr, ax, 1), arr)


def limited_flux(Ft, lam):
    Fh = np.empty_like(Ft)
    for a, ax in AXES:
        p = Ft[..., a]
        Fh[..., a] = p * _donor(lam, p, ax)
    return Fh


def limited_flux_adjoint(G, Ft, lam, O, c):
    """dL/dF~ from G = dL/dF^ (lam, O functions of F~, c held)."""
    T = np.zeros(c.shape)
    for a, ax in AXES:
        p, Ga = Ft[..., a], G[..., a]
        T += np.where(p < 0, Ga * p, 0.0) + _shift(np.where(p > 0, Ga * p, 0.0), ax, -1)
    out = np.zeros_like(Ft)
    for a, ax in AXES:
        p, Ga = Ft[..., a], G[..., a]
        ld, Od, cd, Td = (_donor(z, p, ax) for z in (lam, O, c, T))
        lim = (Od > cd) & (cd > 0) & (p != 0)
        out[..., a] = ld * Ga - np.where(lim, ld / np.where(lim, Od, 1.0) * np.sign(p) * Td, 0.0)
    return out


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


def forward(x, weights, scale, rounding=True, details=False):
    """Activations of every layer (inputs included; the last is the flux F)
    and out = x + div F^ / scale (with the limiter's (Ft, lam, O) when
    `details`).  rounding=False uses the weights as given (float64), for
    finite differences."""
    ws = split(bf16_round(weights) if rounding else weights)
    M = voxel_mask(x)[..., None]
    x = np.asarray(x, dtype=np.float64)
    a = [scale * x[..., None] * M]
    for l, w in enumerate(ws):
        z = conv(a[-1], w) * M
        a.append(np.maximum(z, 0.0) if l < 3 else z)
    Ft = face_flux(a[-1])
    lam, O = limiter(Ft, scale * x)
    out = x + divergence(limited_flux(Ft, lam)) / scale
    return (a, out, (Ft, lam, O)) if details else (a, out)


def loss_and_grad(x, target, weights, scale, rounding=True):
    """loss = mean over voxels of (scale (out - target))^2 and its gradient
    with respect to the weights (flat, straight-through the BF16 rounding)."""
    ws = split(bf16_round(weights) if rounding else weights)
    a, out, (Ft, lam, O) = forward(x, weights, scale, rounding, details=True)
    d = scale * (out - np.asarray(target, dtype=np.float64))
    nvox = d.size
    loss = float(np.sum(d * d) / nvox)
    G = divergence_adjoint(2.0 * d / nvox)
    g = face_flux(limited_flux_adjoint(G, Ft, lam, O, scale * np.asarray(x, dtype=np.float64)))
    g = g * voxel_mask(x)[..., None]
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


def active_map(x, tile=TILE, threshold=TILE_THRESHOLD):
    """Boolean map of the active tiles (tz, ty, tx)."""
    ax = np.abs(np.asarray(x, dtype=np.float32))
    nz, ny, nx = ax.shape
    tz, ty, tx = -(-nz // tile), -(-ny // tile), -(-nx // tile)
    tmax = np.zeros((tz, ty, tx), dtype=np.float32)
    for c in range(tz):
        for b in range(ty):
            for a in range(tx):
                blk = ax[c * tile:(c + 1) * tile, b * tile:(b + 1) * tile, a * tile:(a + 1) * tile]
                tmax[c, b, a] = blk.max() if blk.size else 0.0
    tau = np.float32(threshold) * tmax.max()
    flags = (tmax > tau) & (tmax > 0)
    p = np.pad(flags, 1)
    on = np.zeros_like(flags)
    for dc in range(3):
        for db in range(3):
            for da in range(3):
                on |= p[dc:dc + tz, db:db + ty, da:da + tx]
    return on


def voxel_mask(x, tile=TILE, threshold=TILE_THRESHOLD):
    on = active_map(x, tile, threshold)
    nz, ny, nx = np.shape(x)
    m = np.repeat(np.repeat(np.repeat(on, tile, 0), tile, 1), tile, 2)
    return m[:nz, :ny, :nx]


def active_tiles(x, tile=TILE, threshold=TILE_THRESHOLD):
    """Number of active tiles."""
    return int(active_map(x, tile, threshold).sum())
