"""The sort of a step that pushes moves only the positions; the previous
positions stay where they were and the push reads them through the sort's
permutation (writing them in slot order).  Whatever reads the cloud between
the sort and the push gets them moved first.  Here the phases of a step run
one at a time with a download after the deposit phase: the download must be
the cloud permuted by the sort, previous positions included, and the step
must end where the same step run whole ends on a twin context (fixed-point
deposits: the two runs are bit-identical)."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()


def _sim():
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=60_000, dt=0.5)
    return vb.Simulation(p, vb.thomas_fermi_profile(), projectile=vb.xenon_projectile(x0=-8.0, impact=3.0),
                         fixed_point=True, use_graph=False)


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def test_download_between_the_sort_and_the_push(cuda_device):
    a, b = _sim(), _sim()
    try:
        for _ in range(2):
            a.step()
            b.step()
        acc = a.accelerator
        k, d, pk, pd = acc.download()
        params = a._params(advance=True, push=True, capture=a.capture_radius)
        acc.step_deposit(a.projectile, params)
        perm = acc.sort_products()[0]
        k2, d2, pk2, pd2 = acc.download()
        for after, before in ((k2, k), (d2, d), (pk2, pk), (pd2, pd)):
            assert np.array_equal(_bits(after), _bits(before[:, perm]))
        acc.step_fields(params, a.params.nparticles)
        acc.step_advance(a.projectile, params)
        b.step()
        for x, y in zip(a.accelerator.download(), b.accelerator.download()):
            assert np.array_equal(_bits(x), _bits(y))
        assert np.array_equal(a.projectile.position, b.projectile.position)
    finally:
        a.accelerator.close()
        b.accelerator.close()
