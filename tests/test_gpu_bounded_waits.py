"""The sort's bounded waits, made to run out on purpose.

Each tile of the sort's decoupled look-back scan waits for its predecessors
to publish their sums, and gives up after a bounded number of polls
(vlb_tuning.scan_wait_polls; the reference's analogue is its argument and
state errors, src/accelerator.jl:262-268, 583-586).  A tile that gives up
sets VLB_STATUS_SCAN_TIMEOUT and sums its predecessors' inputs itself, so
the scan's result, and every index the sort hands on, stays exact.  With
scan_wait_polls = -1 every tile after the first gives up at once: the step
must return VLB_ERR_TIMEOUT with the status bit set and the very results of
a clean step (fixed-point deposit: a step is a function of its input), and
the context must stay usable and close cleanly.  Nothing waits forever and
nothing reads out of range, so this faults nothing."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


def _sim(npart=40_000):
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    proj = vb.xenon_projectile(x0=-15.0, impact=5.0)
    return vb.Simulation(p, vb.thomas_fermi_profile(), projectile=proj, fixed_point=True)


@pytest.mark.parametrize("use_graph", [False, True], ids=["eager", "graph"])
def test_a_look_back_wait_that_gives_up_is_flagged_and_the_sort_stays_exact(cuda_device, use_graph):
    sim = _sim()
    sim.use_graph = use_graph
    acc = sim.accelerator
    try:
        snap = sim.snapshot()
        clean = [sim.step() for _ in range(3)]
        clean_cloud = acc.download()
        clean_proj = sim.projectile.position.copy()
        sim.restore(snap)
        # step 1 with every look-back wait giving up at once, through the C ABI
        acc.set_tuning(scan_wait_polls=-1)
        assert acc.tuning()["scan_wait_polls"] == -1
        desc = sim.projectile.to_desc()
        params = sim._params(advance=True, push=True, capture=sim.capture_radius)
        res = L.StepResult()
        rc = L.lib().vlb_step(acc.handle, C.byref(desc), C.byref(params), C.byref(res))
        assert rc == L.VLB_ERR_TIMEOUT
        assert res.status & L.VLB_STATUS_SCAN_TIMEOUT
        assert b"scan" in L.lib().vlb_last_error()
        assert (res.kinetic, res.enclosed_charge, res.outcount, res.nout, res.noccupied) == (
            clean[0].kinetic, clean[0].enclosed_charge, clean[0].outcount, clean[0].nout, clean[0].noccupied)
        sim.projectile.from_desc(desc)
        # a second forced step, then the default limit again
        res2 = L.StepResult()
        desc = sim.projectile.to_desc()
        assert L.lib().vlb_step(acc.handle, C.byref(desc), C.byref(params), C.byref(res2)) == L.VLB_ERR_TIMEOUT
        sim.projectile.from_desc(desc)
        assert res2.kinetic == clean[1].kinetic and res2.outcount == clean[1].outcount
        acc.set_tuning(scan_wait_polls=0)
        d3 = sim.step()
        assert d3.status == 0 and d3.kinetic == clean[2].kinetic
        for x, y in zip(acc.download(), clean_cloud):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
        assert np.array_equal(sim.projectile.position, clean_proj)
        with pytest.raises(L.VlbError):
            acc.set_tuning(scan_wait_polls=-2)
    finally:
        acc.close()  # the context closes cleanly after the timeouts


def test_a_small_poll_limit_changes_no_result(cuda_device):
    """A limit of one poll: some waits run out (whether any does depends on
    timing), and the sort is exact either way."""
    sim = _sim(60_000)
    acc = sim.accelerator
    try:
        snap = sim.snapshot()
        acc.sort()
        perm_clean, occ_clean, bnd_clean, _ = acc.sort_products()
        sim.restore(snap)
        acc.set_tuning(scan_wait_polls=1)
        nocc, outc = C.c_int32(), C.c_int32()
        rc = L.lib().vlb_sort(acc.handle, C.byref(nocc), C.byref(outc))
        assert rc in (L.VLB_OK, L.VLB_ERR_TIMEOUT)
        assert nocc.value == len(occ_clean)
        perm, occ, bnd, _ = acc.sort_products()
        assert np.array_equal(perm, perm_clean) and np.array_equal(occ, occ_clean) and np.array_equal(bnd, bnd_clean)
    finally:
        acc.close()
