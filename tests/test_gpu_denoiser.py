"""The learned denoiser on the GPU: its forward pass (the 16 -> 16 layers on
the tensor cores, the others on the CUDA cores), loss, weight gradient and
Adam step against the float64 oracle (oracle/denoiser.py); the tile
skip; the network in the step, with its charge check and fallback; training
on the GPU beating the plain deposit on held-out data; the committed
network's gain at 8e6 against 8e7 particles.

Tolerances: the kernels compute in float32 (on the tensor cores: exact
products of the BF16 weights with BF16 heads and tails of the activations,
summed in float32) against the oracle's float64, with the same BF16
weights: outputs to 2e-5 of their largest value, gradients to 1e-4
(relative L2 per layer)."""
import numpy as np
import pytest

from conftest import load_package
from oracle import denoiser as D

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib
DN = vb.denoiser


def _blob_volume(rng, shape=(20, 27, 49), box=((3, 12), (6, 18), (9, 25))):
    """A smooth blob with Poisson-like noise inside `box`, zero elsewhere
    (ragged sizes, inactive tiles at the far corner)."""
    x = np.zeros(shape)
    (z0, z1), (y0, y1), (x0, x1) = box
    zz, yy, xx = np.meshgrid(np.arange(z0, z1), np.arange(y0, y1), np.arange(x0, x1), indexing="ij")
    c = np.array([(z0 + z1) / 2, (y0 + y1) / 2, (x0 + x1) / 2])
    r2 = ((zz - c[0]) / (z1 - z0)) ** 2 + ((yy - c[1]) / (y1 - y0)) ** 2 + ((xx - c[2]) / (x1 - x0)) ** 2
    smooth = 0.004 * np.exp(-8 * r2)
    x[z0:z1, y0:y1, x0:x1] = rng.poisson(smooth * 2e4) / 2e4
    t = np.zeros(shape)
    t[z0:z1, y0:y1, x0:x1] = smooth
    return x.astype(np.float32), t.astype(np.float32)


def _tensors(*arrays):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda() for a in arrays]


def test_weight_count(cuda_device):
    assert L.lib().vlb_dn_weight_count() == D.WEIGHT_COUNT == DN.WEIGHT_COUNT


def test_forward_matches_oracle(cuda_device):
    rng = np.random.default_rng(1)
    x, _ = _blob_volume(rng)
    w = DN.init_weights(3, flux_gain=0.5)
    scale = 1.0 / 0.004
    net = DN.Network(x.shape)
    try:
        xt, wt = _tensors(x, w)
        out = net.forward(xt, wt, scale).cpu().numpy()
        _, ref = D.forward(x, w, scale)
        assert np.max(np.abs(out - ref)) <= 2e-5 * np.max(np.abs(ref))
        assert np.max(np.abs(out - x)) > 1e-3 * np.max(x)        # the network did something
        assert abs(out.astype(np.float64).sum() - x.astype(np.float64).sum()) <= 1e-5 * x.sum()
        assert net.active_tiles() == D.active_tiles(x)
        assert net.active_tiles() < np.prod([-(-n // 8) for n in x.shape])  # some tiles skipped
        assert net.status() == 0
    finally:
        net.close()


def test_faint_tiles_match_oracle(cuda_device):
    """Specks below and above the tile threshold, far from the blob."""
    rng = np.random.default_rng(21)
    x, t = _blob_volume(rng)
    x[17, 22, 44] = 1e-5 * x.max()
    x[2, 24, 40] = 3e-2 * x.max()
    w = DN.init_weights(3, flux_gain=0.5)
    net = DN.Network(x.shape)
    try:
        xt, wt = _tensors(x, w)
        out = net.forward(xt, wt, 250.0).cpu().numpy()
        _, ref = D.forward(x, w, 250.0)
        assert np.max(np.abs(out - ref)) <= 2e-5 * np.max(np.abs(ref))
        assert out[17, 22, 44] == x[17, 22, 44] and out[2, 24, 40] != x[2, 24, 40]
        assert net.active_tiles() == D.active_tiles(x)
    finally:
        net.close()


def test_gradient_matches_oracle(cuda_device):
    import torch
    rng = np.random.default_rng(2)
    x, t = _blob_volume(rng)
    w = DN.init_weights(4, flux_gain=0.5)
    scale = 1.0 / 0.004
    net = DN.Network(x.shape)
    try:
        xt, tt, wt = _tensors(x, t, w)
        g = torch.empty_like(wt)
        loss = net.gradient(xt, tt, wt, scale, g, want_loss=True)
        ref_loss, ref_g = D.loss_and_grad(x, t, w, scale)
        assert abs(loss - ref_loss) <= 1e-5 * ref_loss
        g = g.cpu().numpy()
        o = 0
        for a, b in D.LAYERS:
            m = 27 * a * b
            err = np.linalg.norm(g[o:o + m] - ref_g[o:o + m]) / np.linalg.norm(ref_g[o:o + m])
            assert err < 1e-4, (a, b, err)
            o += m
    finally:
        net.close()


def test_gradient_is_deterministic(cuda_device):
    import torch
    rng = np.random.default_rng(12)
    x, t = _blob_volume(rng)
    w = DN.init_weights(5, flux_gain=0.5)
    net = DN.Network(x.shape)
    try:
        xt, tt, wt = _tensors(x, t, w)
        g1, g2 = torch.empty_like(wt), torch.empty_like(wt)
        net.gradient(xt, tt, wt, 250.0, g1)
        net.gradient(xt, tt, wt, 250.0, g2)
        assert torch.equal(g1, g2)
    finally:
        net.close()


def test_adam_matches_oracle(cuda_device):
    rng = np.random.default_rng(6)
    n = D.WEIGHT_COUNT
    w, g = rng.standard_normal(n).astype(np.float32), rng.standard_normal(n).astype(np.float32)
    m, v = (0.1 * rng.standard_normal(n)).astype(np.float32), rng.random(n).astype(np.float32)
    net = DN.Network((8, 8, 8))
    try:
        wt, gt, mt, vt = _tensors(w, g, m, v)
        net.adam(wt, gt, mt, vt, 1e-3, 7)
        f64 = [a.astype(np.float64) for a in (w, g, m, v)]
        rw, rm, rv = D.adam(*f64, 1e-3, 7)
        # float32 moments with float32 constants (0.999f is 0.999 to 1.3e-8)
        assert np.allclose(wt.cpu().numpy(), rw, rtol=0, atol=1e-6)
        assert np.allclose(mt.cpu().numpy(), rm, rtol=1e-5, atol=1e-7)
        assert np.allclose(vt.cpu().numpy(), rv, rtol=1e-5, atol=1e-7)
    finally:
        net.close()


def test_empty_volume_stays_empty(cuda_device):
    import torch
    net = DN.Network((16, 16, 24))
    try:
        x = torch.zeros((16, 16, 24), device="cuda")
        w, = _tensors(DN.init_weights(0))
        out = net.forward(x, w, 1.0)
        assert net.active_tiles() == 0 and torch.count_nonzero(out).item() == 0
    finally:
        net.close()


def test_bad_arguments_are_refused(cuda_device):
    import ctypes as C
    h = C.c_void_p()
    assert L.lib().vlb_dn_create(0, 4, 4, 0, C.byref(h)) == L.VLB_ERR_ARG
    net = DN.Network((8, 8, 8))
    try:
        x, w = _tensors(np.zeros((8, 8, 8)), DN.init_weights(0))
        assert L.lib().vlb_dn_forward(net._h, x.data_ptr(), 0.0, w.data_ptr(), x.data_ptr(), None) == L.VLB_ERR_ARG
        assert L.lib().vlb_dn_adam(net._h, w.data_ptr(), w.data_ptr(), w.data_ptr(), w.data_ptr(), 1e-3, 0,
                                   None) == L.VLB_ERR_ARG
    finally:
        net.close()


# ------------------------------------------------------------- in the step
def _sim(npart=40_000, impact=10.0, seed=-1):
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    proj = vb.xenon_projectile(x0=-20.0, impact=impact)
    return vb.Simulation(p, vb.thomas_fermi_profile(), projectile=proj, fixed_point=True, seed=seed)


def test_step_uses_the_network(cuda_device):
    """Fixed-point deposits are bit-identical, so the denoised step's fine
    density is the network applied to the plain step's, renormalised to the
    deposit's charge."""
    a, b = _sim(), _sim()
    w = DN.init_weights(8, flux_gain=0.5)
    scale = 250.0
    DN.attach(b, w, scale)
    try:
        da, db = a.step(), b.step()
        assert da.denoised == 0 and db.denoised == 1 and db.status == 0
        rho_a = a.accelerator.grid(L.VLB_GRID_RHO_FINE)
        rho_b = b.accelerator.grid(L.VLB_GRID_RHO_FINE)
        _, ref = D.forward(rho_a, w, scale)
        ref *= rho_a.astype(np.float64).sum() / ref.sum()        # charge kept (uniform interior duals)
        assert np.max(np.abs(rho_b - ref)) <= 2e-5 * np.max(np.abs(ref))
        assert not np.array_equal(rho_a, rho_b)
        # the graph-captured steps keep using it
        for _ in range(3):
            assert b.step().denoised == 1
    finally:
        a.accelerator.close()
        b.accelerator.close()


def test_step_falls_back_to_the_deposit(cuda_device):
    """Weights of +-1e30 overflow the activations (inf, then NaN): the
    prediction's charge is not the deposit's and the step keeps the deposit."""
    a, b = _sim(), _sim()
    w = np.where(np.arange(D.WEIGHT_COUNT) % 2 == 0, 1e30, -1e30).astype(np.float32)
    DN.attach(b, w, 250.0)
    try:
        da, db = a.step(), b.step()
        assert db.denoised == 0 and db.status == 0
        assert np.array_equal(a.accelerator.grid(L.VLB_GRID_RHO_FINE), b.accelerator.grid(L.VLB_GRID_RHO_FINE))
        assert abs(da.kinetic - db.kinetic) < 1e-6 * da.kinetic      # the coarse deposit's float32 atomics
        # a sane network set again takes over; clearing it restores the plain step
        DN.attach(b, DN.init_weights(9), 250.0)
        assert b.step().denoised == 1
        DN.detach(b)
        assert b.step().denoised == 0
    finally:
        a.accelerator.close()
        b.accelerator.close()


def test_denoise_without_network_is_refused(cuda_device):
    s = _sim(npart=5000)
    try:
        s.denoise = True
        with pytest.raises(L.VlbError):
            s.step()
    finally:
        s.accelerator.close()


def test_training_on_the_gpu_beats_the_deposit(cuda_device):
    """Pairs from runs of 5e4 and 5e5 particles (58^3 grids), a short
    training by the library's kernels, held-out pairs from other seeds."""
    import torch
    def pairs(seed_lo, seed_hi, steps=24, every=4):
        lo, hi = _sim(50_000, 20.0, seed_lo), _sim(500_000, 20.0, seed_hi)
        try:
            x, _ = DN.collect(lo, steps, every)
            t, _ = DN.collect(hi, steps, every)
        finally:
            lo.accelerator.close()
            hi.accelerator.close()
        return x, t
    x, t = pairs(-31, -32)
    hx, ht = pairs(-33, -34)
    w, scale, hist = DN.train(x, t, steps=400, batch=2, lr=1e-3, warmup=40, log_every=50, log=None)
    assert hist[-1][1] < hist[0][1]
    plain, learned = DN.errors(hx, ht, w, scale)
    assert np.mean(learned) < 0.97 * np.mean(plain), (plain, learned)
    torch.cuda.synchronize()


def test_committed_network_gains_at_8e6(cuda_device):
    """The committed network (trained at b = 30 and 60 a0) on the headline
    grid at b = 45 a0: the 8e6-particle density it gives is closer to the
    8e7-particle run's than the 8e6 deposit is."""
    import torch
    w, scale, _ = DN.load_weights()
    lo = DN.make_run(8_000_000, 45.0, -41)
    hi = DN.make_run(80_000_000, 45.0, -42)
    try:
        x, _ = DN.collect(lo, 24, 8)
        t, _ = DN.collect(hi, 24, 8)
    finally:
        lo.accelerator.close()
        hi.accelerator.close()
    plain, learned = DN.errors(x, t, w, scale)
    assert np.all(learned < 0.8 * plain), (plain, learned)
    torch.cuda.synchronize()
