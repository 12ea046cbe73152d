"""Smoothing tables wider than 1,024 columns: the sort then writes no packed
table columns (they are 10 bits an axis), and the fine deposit and the
gather compute each particle's columns from delta themselves.  The same
bars as the parity tests of the packed path, on a seeded 40k cloud whose
tables have 1,101 columns."""
import numpy as np
import pytest

from conftest import load_package
from test_gpu_parity import Case, oracle_sorted, rel_l2

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


@pytest.fixture(scope="module")
def wide(orc, cuda_device):
    return Case(orc, nbdt=1100)


@pytest.fixture(scope="module")
def acc(wide):
    assert wide.sm.nbdt + 1 > 1024
    a = vb.DeviceAccelerator(wide.meshes, wide.sm, wide.p.nparticles, wide.w)
    yield a
    a.close()


def test_fine_deposit_with_wide_tables(wide, acc):
    acc.upload(wide.k, wide.d, wide.pk, wide.pd)
    acc.sort()
    nout, q = acc.deposit_smoothed(wide.w)
    rho = acc.grid(L.VLB_GRID_RHO_FINE)
    k, d, _, _ = oracle_sorted(wide)
    c, O = wide.O.c, wide.O
    cols, rnout = wide.orc.columns(k, d, c["x0f"], c["hf"], c["lo"], c["hi"], c["spacing"], c["nbdt"])
    assert nout == rnout                                   # exact
    qr = wide.orc.lib().orc_deposit_sorted(O.F.ref(), O.S.ref(), k.shape[1], wide.orc.pi(np.ascontiguousarray(cols)),
                                           wide.orc.pi(O.occ), wide.orc.pi(O.bnd), len(O.occ), rnout, wide.w,
                                           wide.orc.pd(O.rhof))
    assert rel_l2(rho, O.rhof) < 2e-6                      # float32 sums vs float64
    assert abs(q - qr) < 1e-5 * abs(qr)


def test_tensor_core_forces_with_wide_tables(wide, acc):
    O = wide.O
    k, d, _, _ = oracle_sorted(wide)
    O.forces(k, d)
    acc.set_tuning(field_tensor_cores=1)
    acc.upload(wide.k, wide.d, wide.pk, wide.pd)
    acc.sort()
    acc.set_grid(L.VLB_GRID_CSOL_FINE, O.csolf.astype(np.float32))
    acc.set_grid(L.VLB_GRID_CSOL_COARSE, O.csolc.astype(np.float32))
    O.csolf = acc.grid(L.VLB_GRID_CSOL_FINE).astype(np.float64).ravel()
    O.csolc = acc.grid(L.VLB_GRID_CSOL_COARSE).astype(np.float64).ravel()
    N = k.shape[1]
    force = np.empty((3, N))
    red = np.zeros(4)
    pr = wide.orc.projectile_struct(O.proj, softening=L.VLB_SOFTENING_DEVICE)
    outc = wide.orc.lib().orc_forces_device(O.F.ref(), O.Cl.ref(), O.S.ref(), N, wide.orc.pi(k), wide.orc.pf(d),
                                            wide.orc.pi(O.occ), wide.orc.pi(O.bnd), len(O.occ), wide.orc.pd(O.csolf),
                                            wide.orc.pd(O.csolc), wide.w, O.c["x0"], O.c["h"],
                                            __import__("ctypes").byref(pr), wide.orc.pd(force), wide.orc.pd(red))
    gred, goutc = acc.forces(O.proj)
    f = acc.force()
    assert goutc == outc
    out = wide.orc.outside(k, wide.meshes.fine.n)
    inside = np.ones(N, bool)
    inside[out] = False
    assert rel_l2(f[:, inside], force[:, inside]) < 2e-5
    assert np.all(np.isfinite(f))
    assert rel_l2(gred[:3], red[:3]) < 1e-4
