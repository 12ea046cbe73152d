"""The sharded step (vlasov_b200.sharded) on two CPU ranks over gloo, against
the unsharded step.

Each rank runs the oracle's device-semantics step of its slice of the cloud
in the library's three phases; between them the ranks sum the raw fine
density, the coarse density, the deposit-window count and the projectile's
reaction sums with torch.distributed (gloo).  Every particle, the projectile
and the summed diagnostics must come out as the single-rank step gives them
(float64 sums in another order: to rounding)."""
import socket
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT, load_package

NFINE, NPART, NSTEPS = 16, 6000, 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(vb, orc):
    p = vb.SimulationParameters.for_grid(NFINE, rcluster=78.0, rbox=235.0, nparticles=NPART, dt=0.5)
    meshes = vb.build_meshes(NFINE, p.ninner, p.nouter, 78.0, 235.0)
    sm = vb.gaussian_smoothing(meshes.fine.axis)
    w = 196.0 / NPART
    pos, mom = vb.sample_thomas_fermi(vb.thomas_fermi_profile(), NPART, w, seed=-1)
    kn = meshes.fine.axis.knots
    x0, h = float(kn[0]), float((kn[-1] - kn[0]) / (len(kn) - 1))
    k, d = vb.pack_positions(pos, x0, h)
    pk, pd = vb.pack_positions(pos - 0.5 * mom / w, x0, h)
    jel = vb.Jellium.of(196.0)
    params = vb._lib.StepParams()
    params.dt, params.rcmax = 0.5, 100.0
    params.jellium_nions, params.jellium_radius = jel.nions, jel.radius
    params.capture_radius = 8.0
    params.advance_projectile, params.push = 1, 1

    def oracle_step():
        return orc.DeviceSemanticsStep(meshes, sm, w, jel, 0.5, 100.0, vb.xenon_projectile(x0=-12.0, impact=4.0))

    return (k, d, pk, pd), oracle_step, params, (x0, h)


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    vb = load_package()
    from oracle import oracle as orc
    from sharded_oracle import OracleShard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        (k, d, pk, pd), oracle_step, params, _ = _case(vb, orc)
        a, b = vb.sharded.shard_range(NPART, rank, world)
        O = oracle_step()
        backend = OracleShard(orc, O, k[:, a:b], d[:, a:b], pk[:, a:b], pd[:, a:b], np.arange(a, b))
        stepper = vb.sharded.ShardedStepper(backend, vb.sharded.TorchComm(), NPART)
        diags = [stepper.step(None, params) for _ in range(NSTEPS)]
        last = diags[-1]
        np.savez(f"{out_dir}/rank{rank}.npz", k=backend.k, d=backend.d, pk=backend.pk, pd=backend.pd,
                 ids=backend.ids, proj=O.proj.position,
                 diag=np.array([last.kinetic, last.escaped, *last.angular, last.enclosed_charge, last.outcount]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_unsharded_step(orc, tmp_path):
    vb = load_package()
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")

    (k, d, pk, pd), oracle_step, params, (x0, h) = _case(vb, orc)
    O = oracle_step()
    ids = np.arange(NPART)
    for _ in range(NSTEPS):
        k, d, pk, pd, diag, _ = O.step(k, d, pk, pd)
        ids = ids[O.perm]
    q = O.enclosed_charge(k, d, 8.0)
    ref = np.array([*diag, q, O.outcount])
    pos_ref = vb.unpack_positions(k, d, x0, h)[np.argsort(ids)]
    prev_ref = vb.unpack_positions(pk, pd, x0, h)[np.argsort(ids)]

    shards = [np.load(tmp_path / f"rank{r}.npz") for r in range(2)]
    sid = np.concatenate([s["ids"] for s in shards])
    order = np.argsort(sid)
    assert np.array_equal(sid[order], np.arange(NPART))   # every particle once
    pos = np.concatenate([vb.unpack_positions(s["k"], s["d"], x0, h) for s in shards])[order]
    prev = np.concatenate([vb.unpack_positions(s["pk"], s["pd"], x0, h) for s in shards])[order]
    assert np.max(np.abs(pos - pos_ref)) < 1e-5
    assert np.max(np.abs(prev - prev_ref)) < 1e-5
    for s in shards:                                      # the projectile is the same on every rank
        assert np.allclose(s["proj"], O.proj.position, rtol=0, atol=1e-9)
    # the diagnostics are the sums over the ranks of the local ones
    for s in shards:
        assert np.allclose(s["diag"][:5], ref[:5], rtol=1e-9, atol=1e-12)
        assert abs(s["diag"][5] - ref[5]) <= 1e-9 * max(1.0, abs(ref[5]))
        assert s["diag"][6] == ref[6]


def test_shard_ranges_cover_the_cloud():
    vb = load_package()
    for n, size in ((10, 3), (8_000_000, 8), (7, 7), (5, 8)):
        spans = [vb.sharded.shard_range(n, r, size) for r in range(size)]
        assert spans[0][0] == 0 and spans[-1][1] == n
        assert all(spans[i][1] == spans[i + 1][0] for i in range(size - 1))
        assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1
