"""Batched runs (vlb_batch_*), launch shapes (vlb_set_tuning) and the
autotuner, on the GPU.

A batch step must give each run what its own step gives (the same kernels
on the same data; the float32 atomics of the coarse deposit order their
sums differently from run to run, hence the tolerances of the graph test);
launch shapes must change no result; the autotuner must leave the run where
it found it."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib
SW = vb.sweep

RUNS = [SW.Collision("Xe25+ b=5", 25.0, 131.3, 5.0, 15_000, -1, v=0.40),
        SW.Collision("Ar8+ b=10", 8.0, 40.0, 10.0, 30_000, -2, energy_kev=100.0),
        SW.Collision("p b=0", 1.0, 1.0, 0.0, 8_000, -3, energy_kev=100.0)]


def _build(device):
    # close starts: the projectiles begin near the cluster so that they matter
    sims = SW.build(RUNS, nfine=28, device=device, fixed_point=True)
    for c, s in zip(RUNS, sims):
        s.projectile = c.projectile(x0=-15.0)
    return sims


def _close(sims):
    for s in sims:
        s.accelerator.close()


def test_batch_step_gives_each_run_its_own_step(cuda_device):
    a, b = _build(cuda_device), _build(cuda_device)
    batch = SW.Batch(a)
    try:
        for _ in range(4):
            da = batch.step()
            db = [s.step() for s in b]
            for x, y, sa, sb in zip(da, db, a, b):
                assert x.status == 0 and y.status == 0
                assert x.outcount == y.outcount and x.nout == y.nout and x.noccupied == y.noccupied
                assert abs(x.kinetic - y.kinetic) < 1e-6 * y.kinetic
                assert abs(x.enclosed_charge - y.enclosed_charge) <= 2 * sa.weight
                assert np.allclose(sa.projectile.position, sb.projectile.position, rtol=0, atol=1e-9)
        for sa, sb in zip(a, b):
            ka, dka, pka, _ = sa.accelerator.download()
            kb, dkb, pkb, _ = sb.accelerator.download()
            assert np.array_equal(pka, pkb)                 # the same sort order
            assert np.mean(np.all(ka == kb, axis=0)) > 0.9999 and np.max(np.abs(dka - dkb)) < 1e-4
    finally:
        batch.close()
        _close(a)
        _close(b)


def test_batches_refuse_bad_contexts(cuda_device):
    sims = _build(cuda_device)[:1]
    try:
        import ctypes as C
        h = sims[0].accelerator.handle.value
        out = C.c_void_p()
        assert L.lib().vlb_batch_create((C.c_void_p * 2)(h, h), 2, C.byref(out)) == L.VLB_ERR_ARG
        assert L.lib().vlb_batch_create((C.c_void_p * 1)(h), 0, C.byref(out)) == L.VLB_ERR_ARG
    finally:
        _close(sims)


def test_batch_and_sharded_steps_refuse_film_frames(cuda_device):
    import ctypes as C
    sims = _build(cuda_device)[:2]
    batch = SW.Batch(sims)
    try:
        for s in sims:
            s.film(4)
        params = sims[0]._params(advance=True, push=True, capture=8.0, film=True)
        projs = (L.ProjectileDesc * 2)(*[s.projectile.to_desc() for s in sims])
        res = (L.StepResult * 2)()
        assert L.lib().vlb_batch_step(batch._h, projs, C.byref(params), res) == L.VLB_ERR_ARG
        assert b"film" in L.lib().vlb_last_error()
        p0 = sims[0].projectile.to_desc()
        assert L.lib().vlb_step_deposit(sims[0].accelerator.handle, C.byref(p0), C.byref(params)) == L.VLB_ERR_ARG
        # the refusals left the runs as they were: a plain batch step runs
        assert all(d.status == 0 for d in batch.step())
        assert sims[0].accelerator.film_frames() == (0, 0)
    finally:
        batch.close()
        _close(sims)


def test_launch_shapes_change_no_result(cuda_device):
    a, b = _build(cuda_device)[:2], _build(cuda_device)[:2]
    try:
        for s in b:
            s.accelerator.set_tuning(chunk=64, field_ctas_per_sm=2, cic_ctas_per_sm=8, push_ctas_per_sm=16,
                                     move_ctas_per_sm=4, field_tensor_cores=1)
            assert s.accelerator.tuning()["chunk"] == 64 and s.accelerator.tuning()["field_tensor_cores"] == 1
        for _ in range(3):
            for sa, sb in zip(a, b):
                x, y = sa.step(), sb.step()
                assert x.outcount == y.outcount and x.nout == y.nout
                assert abs(x.kinetic - y.kinetic) < 1e-6 * x.kinetic
        with pytest.raises(L.VlbError):
            b[0].accelerator.set_tuning(chunk=48)
        with pytest.raises(L.VlbError):
            b[0].accelerator.set_tuning(push_ctas_per_sm=0)
        with pytest.raises(ValueError):
            b[0].accelerator.set_tuning(tile=3)
    finally:
        _close(a)
        _close(b)


def test_autotune_restores_the_run(cuda_device):
    sims = _build(cuda_device)[1:2]
    sim = sims[0]
    try:
        before = sim.snapshot()
        search = {"chunk": ((64, 128), ("deposit_coarse", "forces", "sort")),
                  "field_ctas_per_sm": ((2, 3), ("forces",))}
        best = vb.autotune.tune(sim, steps=1, warmup=1, search=search)
        assert best["chunk"] in (64, 128) and best["field_ctas_per_sm"] in (2, 3)
        assert sim.accelerator.tuning() == best
        after = sim.snapshot()
        for x, y in zip(before[0], after[0]):
            assert np.array_equal(x, y)
        for x, y in zip(before[1], after[1]):
            assert np.array_equal(x, y)
        assert sim.step().status == 0
    finally:
        _close(sims)
