"""The sort of a step's cloud: the single-pass placement of a cloud still in
its last sort's order against the stable cellsort! (src/sorting.jl:163-204).

After a step the cloud is in the previous sort's order and the push has
written every particle's new cell; when every particle is within one cell
of its old one per axis, the sort places the particles from counts per
(old cell, direction) in one pass (step result sort_path = 1).  A particle
that moved further makes the step take the radix passes (sort_path = 2).
Both must give cellsort!'s permutation, occupied list, bounds and
out-of-stencil list bit for bit: here on the 58^3 grid with a close
projectile, after a step with a twenty-fold dt that sends particles several
cells (and the steps after it, whose cloud keeps those velocities), and at
the headline size (8e6 particles, 130^3)."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


def _forces_only_sort_matches_cellsort(orc, sim):
    """The next sort, through a forces-only fused step, against cellsort! of
    the cloud as the step found it; returns that step's sort path."""
    acc = sim.accelerator
    k, d, pk, pd = acc.download()
    r = acc.fused_step(sim.projectile, sim._params(advance=False, push=False, capture=0.0))
    assert r.status == 0
    perm, occ, bnd, out = acc.sort_products()
    nk = sim.meshes.fine.axis.nknots
    rperm, rocc, rbnd, _ = orc.cellsort(k, nk)
    assert np.array_equal(perm, rperm)
    assert np.array_equal(occ, rocc) and np.array_equal(bnd, rbnd)
    assert np.array_equal(out, orc.outside(np.ascontiguousarray(k[:, rperm]), sim.meshes.fine.n))
    gk, gd, gpk, gpd = acc.download()
    assert np.array_equal(gk, k[:, rperm]) and np.array_equal(gpd.view(np.uint32), pd[:, rperm].view(np.uint32))
    return r.sort_path


def _step_sorted_as_cellsort(orc, sim):
    """One step (a graph replay when the step's parameters are unchanged),
    checked through the previous positions it leaves: the push writes them
    in the order of the step's sort, so they are the cloud as the step found
    it, permuted by cellsort!.  Returns the step's sort path."""
    acc = sim.accelerator
    k, d, _, _ = acc.download()
    path = sim.step().sort_path
    _, _, pk, pd = acc.download()
    rperm, _, _, _ = orc.cellsort(k, sim.meshes.fine.axis.nknots)
    assert np.array_equal(pk, k[:, rperm])
    assert np.array_equal(pd.view(np.uint32), d[:, rperm].view(np.uint32))
    return path


@pytest.mark.parametrize("use_graph", [False, True], ids=["eager", "graph"])
def test_step_sorts_take_the_single_pass_placement(orc, cuda_device, use_graph):
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=60_000, dt=0.5)
    sim = vb.Simulation(p, vb.thomas_fermi_profile(), projectile=vb.xenon_projectile(x0=-8.0, impact=3.0),
                        fixed_point=True, use_graph=use_graph)
    try:
        paths = [sim.step().sort_path for _ in range(4)]
        assert paths[0] in (0, 1) and paths[1:] == [1, 1, 1], paths
        assert _forces_only_sort_matches_cellsort(orc, sim) == 1
        # a step twenty times longer: particles jump several cells
        sim.params.dt = 10.0
        d = sim.step()
        assert d.status == 0
        sim.params.dt = 0.5
        assert _forces_only_sort_matches_cellsort(orc, sim) == 2
        # a forces-only step writes no cell keys, so the step after it sorts
        # with the radix passes alone (path 0); the cloud keeps the long
        # step's velocities, so later steps may still send particles several
        # cells: each sort is exact whichever path it takes
        assert sim.step().sort_path == 0
        # the steps after it, replayed from a graph when use_graph: both the
        # single-pass placement and its fallback (a captured step runs the radix
        # passes in a conditional node) must give cellsort!'s order
        seen = {_step_sorted_as_cellsort(orc, sim) for _ in range(4)}
        assert seen <= {1, 2}
        sim.params.dt = 10.0
        assert _step_sorted_as_cellsort(orc, sim) in (0, 1, 2)
        seen |= {_step_sorted_as_cellsort(orc, sim) for _ in range(3)}
        assert 2 in seen, seen
        sim.params.dt = 0.5
        assert _forces_only_sort_matches_cellsort(orc, sim) in (1, 2)
    finally:
        sim.accelerator.close()


def test_step_sort_at_8e6_on_130_cubed(orc, cuda_device):
    p = vb.SimulationParameters.for_grid(64, rcluster=78.0, rbox=235.0, nparticles=8_000_000, dt=0.5)
    sim = vb.Simulation(p, vb.thomas_fermi_profile(), projectile=vb.xenon_projectile(x0=-15.0, impact=10.0),
                        precision=L.VLB_POISSON_3XTF32)
    try:
        assert [sim.step().sort_path for _ in range(3)][1:] == [1, 1]
        assert _forces_only_sort_matches_cellsort(orc, sim) == 1
    finally:
        sim.accelerator.close()
