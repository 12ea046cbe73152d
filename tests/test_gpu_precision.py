"""The precision form of the step on the benchmark's grids (130^3): the
potential and the forces with the mode products in FP32, 3xTF32 and BF16x3,
each against a float64 tensor solve of the same densities.

The densities are those of a fixed-point step of 2e6 particles.  The float64
solve (the oracle: phi on both levels, then csol = S^-1 (phi + V_xc + V_jel))
is rounded to float32 and handed to the same gather, so that the force
errors are those of the solve alone.  Bars: potential relative L2 2e-5
(FP32, 3xTF32) and 2e-4 (BF16x3); forces 2e-4 (FP32, 3xTF32) and 1e-2
(BF16x3).  The forces come from csol = S^-1 (phi + V), and the rows of S^-1
(values to Hermite coefficients) have large entries of alternating sign: the
cancellation multiplies a product's rounding by ~1e3, which BF16x3's 2^-16
heads and tails do not survive as well as FP32's 2^-24.  The measured errors
are printed (run with -s)."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib
PRECISIONS = (("fp32", L.VLB_POISSON_FP32), ("3xtf32", L.VLB_POISSON_3XTF32), ("bf16x3", L.VLB_POISSON_BF16X3))
PHI_BAR = {"fp32": 2e-5, "3xtf32": 2e-5, "bf16x3": 2e-4}
FORCE_BAR = {"fp32": 2e-4, "3xtf32": 2e-4, "bf16x3": 1e-2}


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_field_errors_against_a_float64_solve(orc, cuda_device):
    sim = vb.denoiser.make_run(2_000_000, 45.0, -3, precision=L.VLB_POISSON_FP32, fixed_point=True)
    acc = sim.accelerator
    try:
        sim.projectile.position[0] = -20.0          # close enough for its forces to matter
        sim.projectile.previous[0] = -20.2
        sim.step()
        rf, rc = acc.grid(L.VLB_GRID_RHO_FINE), acc.grid(L.VLB_GRID_RHO_COARSE)
        F, Cl = orc.Level(sim.meshes.fine), orc.Level(sim.meshes.coarse)
        rf64, rc64 = rf.astype(np.float64).ravel(), rc.astype(np.float64).ravel()
        phf, phc = np.zeros_like(rf64), np.zeros_like(rc64)
        lib = orc.lib()
        lib.orc_poisson(F.ref(), Cl.ref(), orc.pd(rf64), orc.pd(rc64), orc.pd(phf), orc.pd(phc))
        csf, csc = np.zeros_like(phf), np.zeros_like(phc)
        lib.orc_spline_coefficients(F.ref(), orc.pd(phf), orc.pd(csf))
        lib.orc_spline_coefficients(Cl.ref(), orc.pd(phc), orc.pd(csc))
        jel = sim.jellium
        lib.orc_effective_potential(F.ref(), orc.pd(csf), orc.pd(rf64), jel.nions, jel.radius)
        lib.orc_effective_potential(Cl.ref(), orc.pd(csc), orc.pd(rc64), jel.nions, jel.radius)

        acc.sort()
        acc.set_grid(L.VLB_GRID_CSOL_FINE, csf.astype(np.float32))
        acc.set_grid(L.VLB_GRID_CSOL_COARSE, csc.astype(np.float32))
        acc.forces(sim.projectile)
        f64 = acc.force().astype(np.float64)
        assert np.all(np.isfinite(f64))

        res = {}
        for name, prec in PRECISIONS:
            acc.set_grid(L.VLB_GRID_RHO_FINE, rf)
            acc.set_grid(L.VLB_GRID_RHO_COARSE, rc)
            acc.poisson(prec)
            e_phi = (rel_l2(acc.grid(L.VLB_GRID_PHI_FINE), phf), rel_l2(acc.grid(L.VLB_GRID_PHI_COARSE), phc))
            for lev in (0, 1):
                acc.spline_coefficients(lev)
                acc.effective_potential(lev, jel)
            e_cs = (rel_l2(acc.grid(L.VLB_GRID_CSOL_FINE), csf), rel_l2(acc.grid(L.VLB_GRID_CSOL_COARSE), csc))
            acc.forces(sim.projectile)
            e_f = rel_l2(acc.force(), f64)
            res[name] = (e_phi, e_cs, e_f)
        print("\n[130^3, 2e6 particles] rel L2 vs the float64 solve: " + "; ".join(
            f"{k}: phi {v[0][0]:.2e}/{v[0][1]:.2e}, csol {v[1][0]:.2e}/{v[1][1]:.2e}, forces {v[2]:.2e}"
            for k, v in res.items()))
        for name, _ in PRECISIONS:
            e_phi, e_cs, e_f = res[name]
            assert max(e_phi) < PHI_BAR[name], (name, e_phi)
            assert e_f < FORCE_BAR[name], (name, e_f)
    finally:
        acc.close()
