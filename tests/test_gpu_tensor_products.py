"""The split-precision tensor-core mode products (3xTF32 and BF16x3) against
the float64 oracle and the FP32 CUDA-core products.

Each field (phi on both levels from poisson!, csol from
spline_coefficients!, csol after effective_potential!) is compared with the
oracle's float64 solve of the same float32 density.  The bar for 3xTF32 is
the FP32 path's, relative L2 below 2e-5; BF16x3 (heads and tails of 8
significant bits, the dropped terms of order 2^-16) is held to 2e-4.  The
measured errors of every precision are printed (run with -s to see them).
Sizes: the test geometry (n = 58 / 56, rows of 2 mod 4 and 0 mod 4 floats)
and the benchmark's (n = 130 / 128)."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib
PRECISIONS = (("fp32", L.VLB_POISSON_FP32), ("3xtf32", L.VLB_POISSON_3XTF32), ("bf16x3", L.VLB_POISSON_BF16X3))
BAR = {"fp32": 2e-5, "3xtf32": 2e-5, "bf16x3": 2e-4}


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def blob_density(meshes, seed):
    """A smooth cluster-like density on both levels: a displaced Gaussian
    ball plus a weaker second one and small noise, float32."""
    rng = np.random.default_rng(seed)
    out = []
    for mesh in (meshes.fine, meshes.coarse):
        x = np.asarray(mesh.axis.colloc)
        X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
        r2 = (X - 3.0) ** 2 + (Y + 2.0) ** 2 + (Z - 1.0) ** 2
        r2b = (X + 20.0) ** 2 + Y ** 2 + (Z + 10.0) ** 2
        rho = 0.004 * np.exp(-r2 / (2 * 15.0 ** 2)) + 0.001 * np.exp(-r2b / (2 * 6.0 ** 2))
        rho *= 1 + 0.01 * rng.standard_normal(rho.shape)
        # the grids are stored i fastest: transpose the (i, j, k) array to (k, j, i)
        out.append(np.ascontiguousarray(rho.transpose(2, 1, 0)).astype(np.float32))
    return out


@pytest.fixture(scope="module", params=[28, 64], ids=["n58", "n130"])
def setup(request, orc, cuda_device):
    nfine = request.param
    p = vb.SimulationParameters.for_grid(nfine, rcluster=78.0, rbox=235.0, nparticles=1000, dt=0.5)
    meshes = vb.build_meshes(nfine, p.ninner, p.nouter, 78.0, 235.0)
    sm = vb.gaussian_smoothing(meshes.fine.axis)
    acc = vb.DeviceAccelerator(meshes, sm, 1000, 0.196)
    F, Cl = orc.Level(meshes.fine), orc.Level(meshes.coarse)
    yield nfine, meshes, acc, F, Cl
    acc.close()


def test_tensor_core_poisson_matches_the_oracle(setup, orc):
    nfine, meshes, acc, F, Cl = setup
    rf, rc = blob_density(meshes, 3)
    acc.set_grid(L.VLB_GRID_RHO_FINE, rf)
    acc.set_grid(L.VLB_GRID_RHO_COARSE, rc)
    rf64, rc64 = rf.astype(np.float64).ravel(), rc.astype(np.float64).ravel()
    phf, phc = np.zeros_like(rf64), np.zeros_like(rc64)
    orc.lib().orc_poisson(F.ref(), Cl.ref(), orc.pd(rf64), orc.pd(rc64), orc.pd(phf), orc.pd(phc))
    errs = {}
    for name, prec in PRECISIONS:
        acc.poisson(prec)
        errs[name] = (rel_l2(acc.grid(L.VLB_GRID_PHI_FINE), phf), rel_l2(acc.grid(L.VLB_GRID_PHI_COARSE), phc))
    print(f"\n[n={2 * nfine + 2}] phi rel L2 vs float64 oracle (fine, coarse): " +
          "; ".join(f"{k} {v[0]:.2e}, {v[1]:.2e}" for k, v in errs.items()))
    for name, _ in PRECISIONS:
        assert max(errs[name]) < BAR[name], (name, errs[name])


def test_tensor_core_coefficients_and_mean_field(setup, orc):
    nfine, meshes, acc, F, Cl = setup
    rf, rc = blob_density(meshes, 5)
    jel = vb.Jellium.of(196.0)
    for lev, wrho, wphi, wcs, Lv, rho in ((0, L.VLB_GRID_RHO_FINE, L.VLB_GRID_PHI_FINE, L.VLB_GRID_CSOL_FINE, F, rf),
                                          (1, L.VLB_GRID_RHO_COARSE, L.VLB_GRID_PHI_COARSE, L.VLB_GRID_CSOL_COARSE,
                                           Cl, rc)):
        acc.set_grid(wrho, rho)
        # a smooth potential-like field as phi
        phi = (rho.astype(np.float64) * 50.0 + 0.3).astype(np.float32)
        acc.set_grid(wphi, phi)
        phi64 = phi.astype(np.float64).ravel()
        c = np.zeros_like(phi64)
        orc.lib().orc_spline_coefficients(Lv.ref(), orc.pd(phi64), orc.pd(c))
        c_mf = c.copy()
        orc.lib().orc_effective_potential(Lv.ref(), orc.pd(c_mf), orc.pd(rho.astype(np.float64).ravel()), jel.nions,
                                          jel.radius)
        res = {}
        for name, prec in PRECISIONS:
            acc.set_precision(prec)
            acc.spline_coefficients(lev)
            e1 = rel_l2(acc.grid(wcs), c)
            acc.effective_potential(lev, jel)
            e2 = rel_l2(acc.grid(wcs), c_mf)
            res[name] = (e1, e2)
        acc.set_precision(L.VLB_POISSON_FP32)
        print(f"\n[n={2 * nfine + 2} level {lev}] csol rel L2 (coefficients, + mean field): " +
              "; ".join(f"{k} {v[0]:.2e}, {v[1]:.2e}" for k, v in res.items()))
        for name, _ in PRECISIONS:
            assert max(res[name]) < BAR[name], (name, res[name])


def test_unknown_precision_is_refused(setup):
    _, _, acc, _, _ = setup
    with pytest.raises(L.VlbError):
        acc.poisson(7)
    with pytest.raises(L.VlbError):
        acc.set_precision(-1)


def test_step_with_tensor_core_products_follows_the_fp32_step(cuda_device):
    """The same 5 fused steps with the three precisions stay within float32
    noise of each other (positions, kinetic energy)."""
    npart = 50_000
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    out = []
    for prec in (L.VLB_POISSON_FP32, L.VLB_POISSON_3XTF32, L.VLB_POISSON_BF16X3):
        sim = vb.Simulation(p, vb.thomas_fermi_profile(), projectile=vb.xenon_projectile(x0=-10.0, impact=5.0),
                            device=cuda_device, precision=prec, fixed_point=True)
        diags = sim.run(5)
        pos, _ = sim.positions()
        out.append((pos, diags))
        sim.accelerator.close()
    (p1, d1), (p2, d2), (p3, d3) = out
    assert np.max(np.abs(p1 - p2)) < 1e-3
    assert abs(d1[-1].kinetic - d2[-1].kinetic) < 1e-5 * abs(d1[-1].kinetic)
    assert np.max(np.abs(p1 - p3)) < 1e-3
    assert abs(d1[-1].kinetic - d3[-1].kinetic) < 1e-4 * abs(d1[-1].kinetic)
    assert all(x.status == 0 for x in d1 + d2 + d3)
