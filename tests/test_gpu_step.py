"""The fused step (vlb_step) against the oracle's device-semantics step, on the
same primed cloud; CUDA-graph replay against eager execution; the priming."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


def make_sim(npart=20_000, nfine=28, fixed=False, graph=True, x0=-20.0, impact=10.0):
    p = vb.SimulationParameters.for_grid(nfine, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    proj = vb.xenon_projectile(x0=x0, impact=impact)
    return vb.Simulation(p, vb.thomas_fermi_profile(), projectile=proj, fixed_point=fixed, use_graph=graph)


def oracle_for(sim, orc):
    proj = vb.Projectile(sim.projectile.mass, sim.projectile.charge, sim.projectile.softening,
                         sim.projectile.initial_energy, sim.projectile.position.copy(),
                         sim.projectile.previous.copy(), sim.projectile.velocity.copy())
    return orc.DeviceSemanticsStep(sim.meshes, sim.smoothing, sim.weight, sim.jellium, sim.params.dt,
                                   sim.params.rcmax, proj)


@pytest.mark.parametrize("fixed", [False, True])
def test_steps_follow_the_oracle(orc, cuda_device, fixed):
    sim = make_sim(fixed=fixed)
    O = oracle_for(sim, orc)
    k, d, pk, pdl = sim.accelerator.download()
    for step in range(3):
        diag = sim.step()
        k, d, pk, pdl, rdiag, F = O.step(k, d, pk, pdl)
        gk, gd, gpk, gpd = sim.accelerator.download()
        # the sort order is the same stable order on both sides
        assert np.array_equal(gpk, pk)
        same_k = np.mean(np.all(gk == k, axis=0))
        assert same_k > 0.9999
        pos_g = vb.unpack_positions(gk, gd, sim.x0, sim.h)
        pos_o = vb.unpack_positions(k, d, sim.x0, sim.h)
        assert np.max(np.abs(pos_g - pos_o)) < 1e-4
        assert abs(diag.kinetic - rdiag[0]) < 1e-4 * rdiag[0]
        assert np.allclose(sim.projectile.position, O.proj.position, rtol=0, atol=1e-9)
        assert diag.outcount == O.outcount and diag.nout == O.nout
        q = O.enclosed_charge(k, d, 8.0)
        assert abs(diag.enclosed_charge - q) <= 2 * sim.weight


def test_graph_replay_matches_eager(cuda_device):
    a = make_sim(fixed=True, graph=False)
    b = make_sim(fixed=True, graph=True)
    for _ in range(4):
        da, db = a.step(), b.step()
        assert da.outcount == db.outcount and da.nout == db.nout and da.noccupied == db.noccupied
        assert abs(da.kinetic - db.kinetic) < 1e-6 * da.kinetic
    ka, dka, *_ = a.accelerator.download()
    kb, dkb, *_ = b.accelerator.download()
    assert np.mean(np.all(ka == kb, axis=0)) > 0.9999
    assert np.max(np.abs(dka - dkb)) < 1e-4
    assert np.allclose(a.projectile.position, b.projectile.position, atol=1e-9)


def test_priming_matches_the_oracle(orc, cuda_device):
    """prime_leapfrog! (src/simulation.jl:233-277): forces at q(-dt/2) with the
    projectile fused in, then the Fortran's dt/M back step."""
    sim = make_sim(npart=8000)
    p = sim.params
    pos, mom = vb.sample_thomas_fermi(vb.thomas_fermi_profile(), p.nparticles, sim.weight)
    M, dt = sim.mass, p.dt
    half = pos - (dt / (2 * M)) * mom
    k, d = vb.pack_positions(half, sim.x0, sim.h)
    pk, pdl = vb.pack_positions(pos, sim.x0, sim.h)
    O = oracle_for(sim, orc)
    O.proj.position = np.array([-20.0, 10.0, 0.0])
    k, d, pk, pdl = O.sort(k, d, pk, pdl)
    force, _ = O.forces(k, d)
    q0 = vb.unpack_positions(pk, pdl, sim.x0, sim.h)
    hp = vb.unpack_positions(k, d, sim.x0, sim.h)
    back = -q0 + 2 * hp + (dt / M) * force.astype(np.float32).astype(np.float64).T
    gk, gd, gpk, gpd = sim.accelerator.download()
    gpos = vb.unpack_positions(gk, gd, sim.x0, sim.h)
    gprev = vb.unpack_positions(gpk, gpd, sim.x0, sim.h)
    assert np.max(np.abs(gpos - q0)) < 1e-6
    assert np.max(np.abs(gprev - back)) < 1e-4


def test_capture_of_a_slow_projectile_is_a_charge(cuda_device):
    sim = make_sim(npart=10_000, x0=0.0, impact=0.0)
    d = sim.step()
    assert 0 <= d.enclosed_charge <= 196
    assert d.noccupied > 100 and d.status == 0
    assert abs(d.enclosed_charge - sim.enclosed_charge(8.0)) < 1e-12


def test_upload_after_graph_steps_rebuilds_the_cell_keys(cuda_device):
    """The captured step takes its cell keys from the previous step's push; a
    cloud uploaded after graph steps must go through the eager step, which
    computes them, and give what a fresh context gives (to the noise of the
    float32 atomics of the coarse deposit, as in the graph test above; stale
    keys would scramble the sort instead)."""
    a = make_sim(fixed=True, graph=False)
    snap = a.accelerator.download()
    proj0 = (a.projectile.position.copy(), a.projectile.previous.copy(), a.projectile.velocity.copy())
    b = make_sim(fixed=True, graph=True)
    for _ in range(3):
        b.step()
    b.accelerator.upload(*snap)
    b.projectile.position, b.projectile.previous, b.projectile.velocity = (x.copy() for x in proj0)
    for _ in range(2):
        da, db = a.step(), b.step()
        assert da.outcount == db.outcount and da.nout == db.nout and da.noccupied == db.noccupied
        assert abs(da.kinetic - db.kinetic) < 1e-6 * da.kinetic
    ka, dka, pka, pdka = a.accelerator.download()
    kb, dkb, pkb, pdkb = b.accelerator.download()
    # the same stable sort order: the previous positions are the same records
    assert np.array_equal(pka, pkb) and np.max(np.abs(pdka - pdkb)) < 1e-5
    assert np.mean(np.all(ka == kb, axis=0)) > 0.9999 and np.max(np.abs(dka - dkb)) < 1e-5


def test_fixed_point_runs_are_bit_identical(cuda_device):
    """With the fixed-point deposits (fine and coarse) and the order-fixed
    reductions (reaction sums, diagnostics), the step does not depend on the
    order in which CTAs take their work: two runs of the same cloud agree
    bit for bit, state and scalars, graph replays included."""
    a = make_sim(npart=30_000, fixed=True, x0=-15.0, impact=5.0)
    b = make_sim(npart=30_000, fixed=True, x0=-15.0, impact=5.0)
    try:
        for _ in range(6):
            da, db = a.step(), b.step()
            assert (da.kinetic, da.escaped, da.angular, da.enclosed_charge, da.nout, da.outcount) == \
                   (db.kinetic, db.escaped, db.angular, db.enclosed_charge, db.nout, db.outcount)
            assert np.array_equal(a.projectile.position, b.projectile.position)
        for x, y in zip(a.accelerator.download(), b.accelerator.download()):
            assert np.array_equal(x, y)
        for w in (L.VLB_GRID_RHO_FINE, L.VLB_GRID_RHO_COARSE, L.VLB_GRID_CSOL_FINE):
            assert np.array_equal(a.accelerator.grid(w), b.accelerator.grid(w))
    finally:
        a.accelerator.close()
        b.accelerator.close()
