"""The energy budget on the device (step!(sim; energy=true),
src/simulation.jl:382-396): the interaction sums against the oracle's
interaction_energy (src/energy.jl:19-43, float64 on the host's positions)
with the same coefficients, in its three regimes (smoothed fine potential
inside the host margin, coarse spline, nothing outside both), on a cloud
that has moved since its sort; the step's two sums; the budget.

Tolerance: the device's 10^3 sums are FP32 and its table columns come from
the float32 offsets, the oracle's are float64: relative 2e-5 on the sums."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


def make_sim(npart=60_000, fixed=True):
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    return vb.Simulation(p, vb.thomas_fermi_profile(), projectile=vb.xenon_projectile(x0=-20.0, impact=8.0),
                         fixed_point=fixed)


def oracle_energy(orc, sim, positions, which):
    acc = sim.accelerator
    gf, gc = ((L.VLB_GRID_CSOL_FINE, L.VLB_GRID_CSOL_COARSE) if which == "total"
              else (L.VLB_GRID_CSOL_HARTREE_FINE, L.VLB_GRID_CSOL_HARTREE_COARSE))
    cf = acc.grid(gf).astype(np.float64).ravel()
    cc = acc.grid(gc).astype(np.float64).ravel()
    F, C = orc.Level(sim.meshes.fine), orc.Level(sim.meshes.coarse)
    S = orc.Smoothing(sim.smoothing)
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    return orc.lib().orc_interaction_energy(F.ref(), C.ref(), S.ref(), len(pos), orc.pd(pos), orc.pd(cf),
                                            orc.pd(cc), sim.weight, 0.0)


def test_interaction_energy_in_its_three_regimes(orc, cuda_device):
    """A twentieth of the cloud moved onto the coarse grid (85..220 a0) and
    beyond both grids (300 a0), the rest inside: the three regimes."""
    sim = make_sim()
    acc = sim.accelerator
    try:
        sim.step()
        pos, prev = sim.positions()
        rng = np.random.default_rng(4)
        n = len(pos)
        far = rng.choice(n, n // 20, replace=False)
        u = rng.standard_normal((len(far), 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        r = np.where(np.arange(len(far)) % 5 == 0, 300.0, rng.uniform(85.0, 220.0, len(far)))
        pos[far] = u * r[:, None]
        k, d = vb.pack_positions(pos, sim.x0, sim.h)
        pk, pd = vb.pack_positions(prev, sim.x0, sim.h)
        acc.upload(k, d, pk, pd)
        with pytest.raises(L.VlbError):          # an upload drops the work items
            acc.interaction_energy()
        acc.sort()
        e_dev = acc.interaction_energy(L.VLB_ENERGY_TOTAL)
        e_ref = oracle_energy(orc, sim, vb.unpack_positions(k, d, sim.x0, sim.h), "total")
        assert abs(e_dev - e_ref) <= 2e-5 * abs(e_ref), (e_dev, e_ref)
    finally:
        acc.close()


def test_energy_after_a_push_uses_the_moved_cloud(orc, cuda_device):
    """The step's interaction sum is taken after its push, on the work items
    of the sort before it: it must equal the oracle's on the new positions."""
    sim = make_sim()
    acc = sim.accelerator
    try:
        for _ in range(2):
            sim.step()
        before, _ = sim.positions()
        d = sim.step(energy=True)
        after, _ = sim.positions()
        assert d.status == 0 and d.interaction != 0 and d.hartree != 0
        e_ref = oracle_energy(orc, sim, after, "total")
        assert abs(d.interaction - e_ref) <= 2e-5 * abs(e_ref), (d.interaction, e_ref)
        h_ref = 0.5 * oracle_energy(orc, sim, before, "hartree")
        assert abs(d.hartree - h_ref) <= 2e-5 * abs(h_ref), (d.hartree, h_ref)
        # the stand-alone sum on the same cloud and coefficients is the step's
        assert acc.interaction_energy(L.VLB_ENERGY_TOTAL) == d.interaction
        b = sim.energy_budget(d)
        assert b.meanfield == d.interaction - 2 * d.hartree
        assert abs(b.total - (b.ions + b.kinetic + b.hartree + b.meanfield)) < 1e-9 * abs(b.total)
        # a plain step reports no sums; the graph-captured energy steps agree with eager ones
        assert sim.step().interaction == 0.0
    finally:
        acc.close()


def test_energy_steps_replay_like_eager_steps(cuda_device):
    a, b = make_sim(), make_sim()
    b.use_graph = False
    try:
        for _ in range(3):
            da, db = a.step(energy=True), b.step(energy=True)
            assert da.interaction == db.interaction and da.hartree == db.hartree
    finally:
        a.accelerator.close()
        b.accelerator.close()


def test_isolated_cluster_conserves_its_energy(cuda_device):
    """The reference's validation observable (src/energy.jl:1-7): without a
    projectile the total stays put while its parts swing with the cluster's
    breathing (measured: +-0.06 Ha on -23.1 Ha over 300 steps, Hartree
    swinging by 3.4 Ha, at 2e5 particles on 58^3)."""
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=200_000, dt=0.5)
    sim = vb.Simulation(p, vb.thomas_fermi_profile(), projectile=None, fixed_point=True)
    try:
        budgets = []
        for s in range(150):
            d = sim.step(energy=(s % 10 == 0))
            assert d.status == 0
            if s % 10 == 0:
                budgets.append(sim.energy_budget(d))
        total = np.array([b.total for b in budgets])
        hartree = np.array([b.hartree for b in budgets])
        assert np.ptp(total) < 0.15
        assert np.ptp(hartree) > 5 * np.ptp(total)
    finally:
        sim.accelerator.close()
