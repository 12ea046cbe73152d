"""The film on the device (vlb_film_*): the frames of the reference's movie
(scripts/xenon.jl:370-410) -- the fine density averaged over the two planes
around z = 0, the projectile's x and y, q(<8 a0) around it and the count
within 35 a0 of the origin -- taken by the steps that ask for one, inside
the captured step.

Bars: the frame equals Float32.((rho[:, :, iz1] + rho[:, :, iz2]) ./ 2) of
the step's fine density bit for bit; the scalars equal the step's projectile
and q(<8) exactly and the count equals the count over the downloaded cloud
in float64 positions (x0 + (k - 1) h + delta, the kernel's formula)."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


def _sim(npart=40_000, seed=-1, fixed_point=False):
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    proj = vb.xenon_projectile(x0=-20.0, impact=10.0)
    return vb.Simulation(p, vb.thomas_fermi_profile(), projectile=proj, seed=seed, fixed_point=fixed_point)


def _inside(sim, radius):
    k, d, _, _ = sim.accelerator.download()
    x = sim.x0 + (k.astype(np.float64) - 1) * sim.h + d.astype(np.float64)
    return int(np.count_nonzero(x[0] * x[0] + x[1] * x[1] + x[2] * x[2] < radius * radius))


def test_film_frames_match_the_step(cuda_device):
    sim = _sim()
    acc = sim.accelerator
    try:
        assert sim.use_graph
        sim.film(3)
        n = sim.params.nfine
        expect = []
        for s in range(1, 6):
            frame = s in (1, 2, 4)   # step 1 runs eagerly, the others replay the captured step
            d = sim.step(film=frame)
            assert d.status == 0
            if frame:
                rho = acc.grid(L.VLB_GRID_RHO_FINE)        # [k][j][i]
                sl = (rho[n - 1] + rho[n]) / np.float32(2)
                assert sl.dtype == np.float32
                expect.append((sl, sim.projectile.position[0], sim.projectile.position[1], d.enclosed_charge,
                               _inside(sim, 35.0)))
        assert acc.film_frames() == (3, 3)
        f = sim.film_frames()
        assert f.taken == 3 and f.frames.shape == (3, sim.meshes.fine.n, sim.meshes.fine.n)
        for i, (sl, px, py, q, inside) in enumerate(expect):
            assert np.array_equal(f.frames[i], sl)
            assert f.proj_x[i] == px and f.proj_y[i] == py
            assert f.q_capture[i] == q
            assert f.q_net[i] == sim.jellium.nions - sim.weight * inside
        assert 0 < expect[0][4] <= sim.params.nparticles and np.max(expect[0][0]) > 0
        # past the capacity: counted, not stored
        sim.step(film=True)
        assert acc.film_frames() == (4, 3)
    finally:
        acc.close()


def test_a_reserved_film_changes_no_step(cuda_device):
    """The film's kernels run as no-ops in the steps that take no frame:
    two fixed-point runs, one with a film reserved, stay bit-identical."""
    a, b = _sim(fixed_point=True), _sim(fixed_point=True)
    try:
        b.film(2)
        for s in range(4):
            x, y = a.step(), b.step(film=(s == 2))
            assert (x.kinetic, x.escaped, x.enclosed_charge, x.outcount) == (y.kinetic, y.escaped,
                                                                              y.enclosed_charge, y.outcount)
        for u, v in zip(a.accelerator.download(), b.accelerator.download()):
            assert np.array_equal(u, v)
        assert b.accelerator.film_frames() == (1, 1)
    finally:
        a.accelerator.close()
        b.accelerator.close()


def test_film_arguments_are_checked(cuda_device):
    sim = _sim(npart=10_000)
    acc = sim.accelerator
    try:
        with pytest.raises(L.VlbError):
            sim.step(film=True)                    # no film reserved
        with pytest.raises(L.VlbError):
            acc.film_reserve(0, 27, 28, 35.0)
        with pytest.raises(L.VlbError):
            acc.film_reserve(2, 27, sim.meshes.fine.n, 35.0)
        sim.film(2)
        with pytest.raises(L.VlbError):
            acc.film_download(1, 2)
        # first + count beyond int32: refused, not wrapped round
        big = 2 ** 31 - 1
        assert L.lib().vlb_film_download(acc.handle, big, big, None, None) == L.VLB_ERR_ARG
        assert L.lib().vlb_film_download(acc.handle, 1, big, None, None) == L.VLB_ERR_ARG
        acc.film_clear()
        with pytest.raises(L.VlbError):
            acc.film_frames()
    finally:
        acc.close()
