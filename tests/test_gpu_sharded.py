"""The sharded step on the GPU: two library contexts on one B200 as two
shards of the cloud (their buffers summed between the phases in this
process; no kernel waits on the other context), against one context with
the whole cloud; and ShardedSimulation on a single rank against
Simulation."""
import copy

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib
SH = vb.sharded


def _setup(npart=30_000, nfine=28):
    p = vb.SimulationParameters.for_grid(nfine, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    proj = vb.xenon_projectile(x0=-12.0, impact=4.0)
    full = vb.Simulation(p, vb.thomas_fermi_profile(), projectile=proj, fixed_point=True, use_graph=False)
    return p, full


def _positions(acc, x0, h):
    k, d, _, _ = acc.download()
    return vb.unpack_positions(k, d, x0, h)


def test_two_shards_on_one_gpu_reproduce_the_whole_cloud(cuda_device):
    p, full = _setup()
    npart = p.nparticles
    k, d, pk, pd = full.accelerator.download()       # the primed cloud
    accs, backends = [], []
    for r in range(2):
        a, b = SH.shard_range(npart, r, 2)
        acc = vb.DeviceAccelerator(full.meshes, full.smoothing, b - a, full.weight, cuda_device)
        acc.upload(k[:, a:b], d[:, a:b], pk[:, a:b], pd[:, a:b])
        accs.append(acc)
        backends.append(SH.LibraryShard(acc, L.VLB_DEPOSIT_FIXED64, cuda_device))
    try:
        stepper = SH.ShardedStepper(backends, SH.LocalComm(), npart)
        proj = copy.deepcopy(full.projectile)
        params = full._params(advance=True, push=True, capture=8.0)
        params.use_graph = 0
        for _ in range(3):
            ds = stepper.step(proj, params)
            df = full.step()
            assert ds.status == 0 and df.status == 0
            assert ds.nout == df.nout and ds.outcount == df.outcount
            assert abs(ds.kinetic - df.kinetic) < 1e-6 * df.kinetic
            assert abs(ds.enclosed_charge - df.enclosed_charge) <= 2 * full.weight
            assert np.allclose(proj.position, full.projectile.position, rtol=0, atol=1e-9)
        # the fine density of a shard after the sum and renormalisation is the
        # whole cloud's, to the float32 scatter noise of the coarse deposit
        # carried through three steps (about 1e-6)
        rf = accs[0].grid(L.VLB_GRID_RHO_FINE).astype(np.float64)
        rg = full.accelerator.grid(L.VLB_GRID_RHO_FINE).astype(np.float64)
        assert np.linalg.norm(rf - rg) <= 1e-5 * np.linalg.norm(rg)
        # the same cloud: each coordinate, sorted, differs by at most the
        # largest per-particle difference (sorting is 1-Lipschitz in max norm)
        pos_s = np.concatenate([_positions(a, full.x0, full.h) for a in accs])
        pos_f = _positions(full.accelerator, full.x0, full.h)
        for c in range(3):
            assert np.max(np.abs(np.sort(pos_s[:, c]) - np.sort(pos_f[:, c]))) < 1e-4
    finally:
        for a in accs:
            a.close()
        full.accelerator.close()


def test_single_rank_sharded_simulation_is_the_simulation(cuda_device):
    npart = 20_000
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    a = vb.Simulation(p, vb.thomas_fermi_profile(), projectile=vb.xenon_projectile(x0=-12.0, impact=4.0),
                      fixed_point=True, use_graph=True)
    b = SH.ShardedSimulation(p, vb.thomas_fermi_profile(), comm=SH.LocalComm(), device=cuda_device,
                             projectile=vb.xenon_projectile(x0=-12.0, impact=4.0), fixed_point=True,
                             sampling="slice")
    try:
        for _ in range(3):
            da, db = a.step(), b.step()
            assert da.outcount == db.outcount and da.nout == db.nout
            assert abs(da.kinetic - db.kinetic) < 1e-6 * da.kinetic
            assert abs(da.enclosed_charge - db.enclosed_charge) <= 2 * a.weight
        assert np.allclose(a.projectile.position, b.projectile.position, rtol=0, atol=1e-9)
    finally:
        a.accelerator.close()
        b.close()


def test_phases_out_of_order_are_refused(cuda_device):
    p, full = _setup(npart=5000)
    try:
        params = full._params(advance=True, push=True, capture=8.0)
        with pytest.raises(L.VlbError):
            full.accelerator.step_fields(params, p.nparticles)
        with pytest.raises(L.VlbError):
            full.accelerator.step_advance(full.projectile, params)
        full.accelerator.step_deposit(full.projectile, params)
        with pytest.raises(L.VlbError):                 # fewer particles than this shard
            full.accelerator.step_fields(params, p.nparticles - 1)
    finally:
        full.accelerator.close()
