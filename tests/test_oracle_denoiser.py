"""The denoiser's oracle pinned on its own: the weight gradient against
central finite differences of the loss, the input gradient of one layer
against its definition, BF16 rounding against torch's, the tile skip as an
exact identity.  CPU only."""
import numpy as np
import torch

from oracle import denoiser as D


def _case(rng, n=(5, 6, 7)):
    x = np.zeros(n)
    x[1:4, 2:5, 1:6] = rng.random((3, 3, 5))
    t = x + 0.1 * rng.standard_normal(n) * (x > 0)
    w = 0.3 * rng.standard_normal(D.WEIGHT_COUNT)
    return x, t, w


def test_weight_count():
    assert D.WEIGHT_COUNT == 15552


def test_divergence_adds_no_charge_and_has_its_adjoint():
    rng = np.random.default_rng(3)
    F = rng.standard_normal((4, 5, 6, 3))
    g = rng.standard_normal((4, 5, 6))
    assert abs(np.sum(D.divergence(F))) < 1e-12
    assert abs(np.sum(g * D.divergence(F)) - np.sum(D.divergence_adjoint(g) * F)) < 1e-10


def test_weight_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    x, t, w = _case(rng)
    w[-27 * 16 * 3:] *= 4.0                  # strong fluxes: the limiter acts
    scale = 2.0
    _, _, (Ft, lam, O) = D.forward(x, w, scale, rounding=False, details=True)
    assert np.sum((lam > 0) & (lam < 1)) > 5 and np.sum((lam == 0) & (O > 0)) > 5
    _, g = D.loss_and_grad(x, t, w, scale, rounding=False)
    offs = np.cumsum([0] + [27 * a * b for a, b in D.LAYERS])
    picks = np.concatenate([rng.integers(offs[l], offs[l + 1], 12) for l in range(4)])
    h = 1e-6
    for i in picks:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (D.loss_and_grad(x, t, wp, scale, rounding=False)[0]
              - D.loss_and_grad(x, t, wm, scale, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, np.max(np.abs(g))), (i, fd, g[i])


def test_input_gradient_is_the_adjoint():
    rng = np.random.default_rng(7)
    x = rng.standard_normal((4, 5, 6, 3))
    g = rng.standard_normal((4, 5, 6, 2))
    w = rng.standard_normal((27, 3, 2))
    lhs = np.sum(g * D.conv(x, w))
    rhs = np.sum(x * D.conv_input_grad(g, w))
    assert abs(lhs - rhs) < 1e-9 * abs(lhs)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(9)
    w = (rng.standard_normal(10000) * 10.0 ** rng.integers(-6, 4, 10000)).astype(np.float32)
    ref = torch.from_numpy(w).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(D.bf16_round(w), ref)


def test_limiter_keeps_the_density_nonnegative():
    rng = np.random.default_rng(13)
    x, _, w = _case(rng, (12, 12, 12))
    w[-27 * 16 * 3:] *= 20.0
    _, out, (_, lam, _) = D.forward(x, w, 3.0, details=True)
    assert np.min(lam) < 0.5                      # it had work to do
    assert np.min(out) >= -1e-12 and abs(out.sum() - x.sum()) < 1e-9 * x.sum()


def test_empty_space_stays_empty():
    rng = np.random.default_rng(11)
    x, _, w = _case(rng, (20, 20, 20))
    x[:] = 0
    x[2:5, 3:6, 2:4] = 1.0
    _, out = D.forward(x, w, 1.5)
    # the flux reaches four voxels, its divergence five: beyond them out = x = 0
    far = np.ones_like(x, dtype=bool)
    far[0:10, 0:11, 0:9] = False
    assert np.all(out[far] == 0)
    assert abs(out.sum() - x.sum()) < 1e-9 * x.sum()
    assert D.active_tiles(x) == 8          # tile (0,0,0) and its neighbours in a 3^3 tile grid


def test_committed_network_loads():
    """The trained network in the package: the right count, BF16 values,
    a positive input scale; on a small noisy blob it conserves the charge
    and makes no negative density."""
    from conftest import load_package
    DN = load_package().denoiser
    w, scale, meta = DN.load_weights()
    assert w.shape == (D.WEIGHT_COUNT,) and scale > 0 and meta["low"] * 10 == meta["high"]
    assert np.array_equal(w, D.bf16_round(w))
    rng = np.random.default_rng(17)
    x = np.zeros((16, 16, 16))
    x[4:12, 4:12, 4:12] = rng.poisson(30.0, (8, 8, 8)) / (30.0 * scale)
    _, out = D.forward(x, w, scale)
    assert np.min(out) >= -1e-12 and abs(out.sum() - x.sum()) < 1e-9 * x.sum()


def test_faint_tiles_pass_through():
    """A speck below the tile threshold (1e-3 of the peak) is left as it is;
    one above it is denoised like the rest."""
    rng = np.random.default_rng(19)
    x, _, w = _case(rng, (24, 24, 40))
    w[-27 * 16 * 3:] *= 4.0
    x[20, 20, 35] = 1e-5 * x.max()
    _, out = D.forward(x, w, 2.0)
    assert out[20, 20, 35] == x[20, 20, 35] and np.all(out[16:, 16:, 32:][x[16:, 16:, 32:] == 0] == 0)
    assert D.active_tiles(x) == D.active_tiles(np.where(x > 1e-5, x, 0))
    x[20, 20, 35] = 1e-2 * x.max()
    _, out = D.forward(x, w, 2.0)
    assert out[20, 20, 35] != x[20, 20, 35]
