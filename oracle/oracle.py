"""ORACLE -- test infrastructure only.

ctypes binding of oracle/liboracle.so (vlasov_oracle.cpp), the float64 CPU
restatement of the reference's per-step loop, plus whole-step drivers in the
two semantics the reference has:

* ``DeviceSemanticsStep``: the resident device path (src/simulation.jl:472-531)
  on the packed float32 cloud, continuous arithmetic in float64;
* ``HostStep``: the CPU path (src/simulation.jl:309-352) on float64 positions,
  the reference's CPU run of the small crossing (nfine = 28, 1e5 particles)
  and the CPU baseline.

Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline and
reference arms) import this module.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

P_D = C.POINTER(C.c_double)
P_F = C.POINTER(C.c_float)
P_I = C.POINTER(C.c_int32)


class OrcLevel(C.Structure):
    _fields_ = [("nk", C.c_int32), ("n", C.c_int32), ("knots", P_D), ("colloc", P_D), ("sinv", P_D),
                ("lap", P_D), ("M", P_D), ("Minv", P_D), ("invlsum", P_D), ("dual", P_D), ("dlen", P_D),
                ("loc_x0", C.c_double), ("loc_invw", C.c_double), ("loc_ncell", C.c_int32),
                ("loc_cells", P_I)]


class OrcSmoothing(C.Structure):
    _fields_ = [("nbdt", C.c_int32), ("spacing", C.c_double), ("overlap", P_D), ("gradient", P_D),
                ("nodes", P_D)]


class OrcProjectile(C.Structure):
    _fields_ = [("pos", C.c_double * 3), ("prev", C.c_double * 3), ("vel", C.c_double * 3),
                ("charge", C.c_double), ("mass", C.c_double), ("gauss_sigma", C.c_double),
                ("ball_radius", C.c_double), ("active", C.c_int32), ("softening", C.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} missing: build it with vlasov.jl_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        ll, i32, dbl, f32 = C.c_longlong, C.c_int32, C.c_double, C.c_float
        pl, ps, pp = C.POINTER(OrcLevel), C.POINTER(OrcSmoothing), C.POINTER(OrcProjectile)
        sig = {
            "orc_num_threads": (C.c_int, []),
            "orc_set_threads": (None, [C.c_int]),
            "orc_mode_product": (None, [P_D, P_D, P_D, C.c_int, ll]),
            "orc_spline_coefficients": (None, [pl, P_D, P_D]),
            "orc_total_charge": (dbl, [pl, P_D]),
            "orc_tensor_solve": (None, [pl, P_D, P_D]),
            "orc_multipole": (None, [pl, P_D, P_D]),
            "orc_poisson": (None, [pl, pl, P_D, P_D, P_D, P_D]),
            "orc_effective_potential": (None, [pl, P_D, P_D, dbl, dbl]),
            "orc_spline_field": (C.c_int, [pl, P_D, dbl, dbl, dbl, P_D]),
            "orc_spline_potential": (C.c_int, [pl, P_D, dbl, dbl, dbl, P_D]),
            "orc_gaussian_force_kernel": (dbl, [dbl, dbl]),
            "orc_cellsort": (C.c_int, [ll, P_I, i32, P_I, P_I, P_I, P_I]),
            "orc_outside": (ll, [ll, P_I, i32, P_I]),
            "orc_columns": (ll, [ll, P_I, P_F, f32, f32, f32, f32, f32, i32, i32, P_I]),
            "orc_deposit_sorted": (dbl, [pl, ps, ll, P_I, P_I, P_I, i32, ll, dbl, P_D]),
            "orc_deposit_sorted_raw": (dbl, [pl, ps, ll, P_I, P_I, P_I, i32, P_D]),
            "orc_deposit_cic_device": (None, [pl, ll, P_I, P_F, f32, f32, dbl, P_D]),
            "orc_forces_device": (ll, [pl, pl, ps, ll, P_I, P_F, P_I, P_I, i32, P_D, P_D, dbl, dbl, dbl, pp,
                                       P_D, P_D]),
            "orc_projectile_force_device": (None, [pp, dbl, dbl, dbl, P_D, P_D, P_D, P_D]),
            "orc_projectile_step": (None, [pp, P_D, dbl]),
            "orc_verlet_packed": (None, [ll, P_I, P_F, P_I, P_F, P_F, f32, f32, f32, dbl, f32, dbl, P_D]),
            "orc_enclosed_charge_packed": (dbl, [ll, P_I, P_F, dbl, dbl, dbl, P_D, dbl]),
            "orc_deposit_smoothed_host": (ll, [pl, ps, ll, P_D, dbl, P_D]),
            "orc_deposit_cic_host": (ll, [pl, ll, P_D, dbl, P_D]),
            "orc_forces_host": (ll, [pl, pl, ps, ll, P_D, P_D, P_D, dbl, ll, P_D]),
            "orc_interaction_energy": (dbl, [pl, pl, ps, ll, P_D, P_D, P_D, dbl, dbl]),
            "orc_projectile_forces_host": (None, [ll, P_D, P_D, pp, dbl, dbl, dbl, P_D, P_D, P_D]),
            "orc_verlet_host": (None, [ll, P_D, P_D, P_D, dbl, dbl, dbl, P_D]),
            "orc_enclosed_charge_host": (dbl, [ll, P_D, dbl, P_D, dbl]),
            "orc_sample_thomas_fermi": (None, [P_D, i32, P_D, i32, dbl, ll, dbl, i32, i32, P_D, P_D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def pd(a):
    return _p(a, C.c_double)


def pf(a):
    return _p(a, C.c_float)


def pi(a):
    return _p(a, C.c_int32)


class Level:
    """float64 tables of one mesh level, kept alive for the C structs."""

    def __init__(self, mesh):
        ax = mesh.axis
        self.mesh = mesh
        self.n = ax.nbasis
        self.keep = {
            "knots": np.ascontiguousarray(ax.knots), "colloc": np.ascontiguousarray(ax.colloc),
            "sinv": np.ascontiguousarray(mesh.cm.Sinv), "lap": np.ascontiguousarray(mesh.laplacian),
            "M": np.ascontiguousarray(mesh.op.M), "Minv": np.ascontiguousarray(mesh.op.Minv),
            "invlsum": np.ascontiguousarray(mesh.invlsum), "dual": np.ascontiguousarray(np.concatenate(mesh.duals)),
            "dlen": np.ascontiguousarray(mesh.dlen),
            "cells": np.ascontiguousarray(mesh.locator.cell, dtype=np.int32),
        }
        k = self.keep
        s = OrcLevel()
        s.nk, s.n = ax.nknots, ax.nbasis
        s.knots, s.colloc, s.sinv, s.lap = pd(k["knots"]), pd(k["colloc"]), pd(k["sinv"]), pd(k["lap"])
        s.M, s.Minv, s.invlsum, s.dual, s.dlen = pd(k["M"]), pd(k["Minv"]), pd(k["invlsum"]), pd(k["dual"]), pd(
            k["dlen"])
        s.loc_x0, s.loc_invw = mesh.locator.x0, mesh.locator.invwidth
        s.loc_ncell, s.loc_cells = len(k["cells"]), pi(k["cells"])
        self.s = s

    def ref(self):
        return C.byref(self.s)


class Smoothing:
    def __init__(self, sm):
        self.sm = sm
        self.keep = [np.ascontiguousarray(t.T) for t in (sm.overlap, sm.gradient, sm.nodes)]
        s = OrcSmoothing()
        s.nbdt, s.spacing = sm.nbdt, sm.spacing
        s.overlap, s.gradient, s.nodes = (pd(a) for a in self.keep)
        self.s = s

    def ref(self):
        return C.byref(self.s)


SOFTENING_DEVICE = 0  # the reference's device path: Gaussian in the stencil, ball in the tail
SOFTENING_BALL = 1    # its CPU path: the ball everywhere (src/projectile.jl:203-232)


def projectile_struct(proj, active=True, softening=SOFTENING_DEVICE) -> OrcProjectile:
    p = OrcProjectile()
    p.softening = softening
    if proj is None:
        p.active = 0
        p.gauss_sigma = p.ball_radius = 1.0
        p.mass = 1.0
        return p
    for i in range(3):
        p.pos[i], p.prev[i], p.vel[i] = proj.position[i], proj.previous[i], proj.velocity[i]
    p.charge, p.mass = proj.charge, proj.mass
    p.gauss_sigma = p.ball_radius = proj.softening.scale
    p.active = int(active)
    return p


# -------------------------------------------------------------- functions
def sample_thomas_fermi(profile, npart: int, weight: float, seed: int = -1, consistent: bool = False):
    """(positions, momenta) float64 (npart, 3) of the seeded ran2 stream
    (src/initial.jl:94-113), drawn by the oracle alone."""
    q = np.ascontiguousarray(profile.quantiles, dtype=np.float64)
    r = np.ascontiguousarray(profile.density, dtype=np.float64)
    pos, mom = np.empty((npart, 3)), np.empty((npart, 3))
    lib().orc_sample_thomas_fermi(pd(q), len(q), pd(r), len(r), float(profile.rmax), int(npart), float(weight),
                                  int(seed), int(consistent), pd(pos), pd(mom))
    return pos, mom


def cellsort(k: np.ndarray, nk: int):
    """Stable counting sort of a (3, N) knot array: perm, occupied, bounds, keys."""
    N = k.shape[1]
    k = np.ascontiguousarray(k, dtype=np.int32)
    keys = np.empty(N, np.int32)
    perm = np.empty(N, np.int32)
    occ = np.empty(nk ** 3, np.int32)
    bnd = np.empty(nk ** 3 + 1, np.int32)
    g = lib().orc_cellsort(N, pi(k), nk, pi(keys), pi(perm), pi(occ), pi(bnd))
    return perm, occ[:g].copy(), bnd[:g + 1].copy(), keys


def outside(k_sorted: np.ndarray, n: int) -> np.ndarray:
    N = k_sorted.shape[1]
    out = np.empty(N, np.int32)
    c = lib().orc_outside(N, pi(np.ascontiguousarray(k_sorted, dtype=np.int32)), n, pi(out))
    return out[:c].copy()


def columns(k, d, x0f, hf, lo, hi, spacing, nbdt):
    N = k.shape[1]
    cols = np.empty((3, N), np.int32)
    nout = lib().orc_columns(N, pi(np.ascontiguousarray(k, np.int32)), pf(np.ascontiguousarray(d, np.float32)),
                             x0f, hf, lo, hi, spacing, nbdt, nbdt + 1, pi(cols))
    return cols, nout


def mode_product(A: np.ndarray, src: np.ndarray) -> np.ndarray:
    n = A.shape[0]
    src = np.ascontiguousarray(src, dtype=np.float64).ravel()
    m = src.size // n
    dest = np.empty(src.size)
    lib().orc_mode_product(pd(dest), pd(np.ascontiguousarray(A)), pd(src), n, m)
    return dest


def fixed_fine_constants(fine_mesh, sm):
    """The Float32 constants the reference's device kernels see
    (src/accelerator.jl:516-529)."""
    knots = fine_mesh.axis.knots
    x0 = float(knots[0])
    h = float((knots[-1] - knots[0]) / (len(knots) - 1))
    half = sm.spacing / 2
    f32 = np.float32
    return dict(x0=x0, h=h, x0f=f32(x0), hf=f32(h), lo=f32(knots[1] + half), hi=f32(knots[-2] - half),
                spacing=f32(sm.spacing), nbdt=sm.nbdt)


# --------------------------------------------------------- whole steps
class DeviceSemanticsStep:
    """The reference's resident device step on a packed cloud: the same
    discrete choices as its Float32 kernels, every continuous quantity in
    float64.  State: k, d, pk, pd as (3, N) int32/float32 arrays."""

    def __init__(self, meshes, sm, weight, jellium, dt, rcmax, projectile=None, softening=SOFTENING_DEVICE):
        self.F, self.Cl = Level(meshes.fine), Level(meshes.coarse)
        self.S = Smoothing(sm)
        self.meshes, self.sm = meshes, sm
        self.w, self.jel, self.dt, self.rcmax = weight, jellium, dt, rcmax
        self.proj = projectile
        self.softening = softening
        self.c = fixed_fine_constants(meshes.fine, sm)
        nf, nc = self.F.n, self.Cl.n
        self.rhof = np.zeros(nf ** 3)
        self.rhoc = np.zeros(nc ** 3)
        self.phif = np.zeros(nf ** 3)
        self.phic = np.zeros(nc ** 3)
        self.csolf = np.zeros(nf ** 3)
        self.csolc = np.zeros(nc ** 3)
        self.force = None

    def sort(self, k, d, pk, pdl):
        nk = self.meshes.fine.axis.nknots
        perm, occ, bnd, keys = cellsort(k, nk)
        k, d, pk, pdl = (np.ascontiguousarray(a[:, perm]) for a in (k, d, pk, pdl))
        self.perm, self.occ, self.bnd = perm, occ, bnd
        self.outlist = outside(k, self.F.n)
        return k, d, pk, pdl

    def forces(self, k, d):
        """Deposit, Poisson, coefficients, mean field, forces on a sorted cloud."""
        c, N = self.c, k.shape[1]
        cols, nout = columns(k, d, c["x0f"], c["hf"], c["lo"], c["hi"], c["spacing"], c["nbdt"])
        self.nout = nout
        ki = np.ascontiguousarray(k, np.int32)
        df = np.ascontiguousarray(d, np.float32)
        self.q_raw = lib().orc_deposit_sorted(self.F.ref(), self.S.ref(), N, pi(np.ascontiguousarray(cols)),
                                              pi(self.occ), pi(self.bnd), len(self.occ), nout, self.w,
                                              pd(self.rhof))
        lib().orc_deposit_cic_device(self.Cl.ref(), N, pi(ki), pf(df), c["x0f"], c["hf"], self.w, pd(self.rhoc))
        lib().orc_poisson(self.F.ref(), self.Cl.ref(), pd(self.rhof), pd(self.rhoc), pd(self.phif), pd(self.phic))
        lib().orc_spline_coefficients(self.F.ref(), pd(self.phif), pd(self.csolf))
        lib().orc_spline_coefficients(self.Cl.ref(), pd(self.phic), pd(self.csolc))
        lib().orc_effective_potential(self.F.ref(), pd(self.csolf), pd(self.rhof), self.jel.nions, self.jel.radius)
        lib().orc_effective_potential(self.Cl.ref(), pd(self.csolc), pd(self.rhoc), self.jel.nions,
                                      self.jel.radius)
        force = np.empty((3, N))
        red = np.zeros(4)
        pr = projectile_struct(self.proj, softening=self.softening)
        self.outcount = lib().orc_forces_device(self.F.ref(), self.Cl.ref(), self.S.ref(), N, pi(ki), pf(df),
                                                pi(self.occ), pi(self.bnd), len(self.occ), pd(self.csolf),
                                                pd(self.csolc), self.w, c["x0"], c["h"], C.byref(pr), pd(force),
                                                pd(red))
        self.force, self.red = force, red
        return force, red

    def projectile_force(self):
        F = np.zeros(3)
        ee, ej = np.zeros(1), np.zeros(1)
        pr = projectile_struct(self.proj, softening=self.softening)
        lib().orc_projectile_force_device(C.byref(pr), self.w, self.jel.nions, self.jel.radius, pd(self.red),
                                          pd(F), pd(ee), pd(ej))
        return F

    def advance_projectile(self):
        F = self.projectile_force()
        pr = projectile_struct(self.proj, softening=self.softening)
        lib().orc_projectile_step(C.byref(pr), pd(F), self.dt)
        self.proj.position = np.array(pr.pos[:])
        self.proj.previous = np.array(pr.prev[:])
        self.proj.velocity = np.array(pr.vel[:])
        return F

    def push(self, k, d, pk, pdl, force32):
        c, N = self.c, k.shape[1]
        M = self.w
        k, d, pk, pdl = (np.ascontiguousarray(a) for a in (k, d, pk, pdl))
        diag = np.zeros(5)
        lib().orc_verlet_packed(N, pi(k), pf(d), pi(pk), pf(pdl), pf(np.ascontiguousarray(force32, np.float32)),
                                np.float32(self.dt * self.dt / M), c["hf"], c["x0f"], M / (2 * self.dt),
                                np.float32(self.rcmax ** 2), 1 / (2 * M), pd(diag))
        return k, d, pk, pdl, diag

    def step(self, k, d, pk, pdl, advance=True, push=True):
        k, d, pk, pdl = self.sort(k, d, pk, pdl)
        force, red = self.forces(k, d)
        F = self.advance_projectile() if (advance and self.proj is not None) else None
        diag = None
        if push:
            k, d, pk, pdl, diag = self.push(k, d, pk, pdl, force.astype(np.float32))
        return k, d, pk, pdl, diag, F

    def enclosed_charge(self, k, d, radius):
        c = self.c
        P = np.ascontiguousarray(self.proj.position, dtype=np.float64)
        return lib().orc_enclosed_charge_packed(k.shape[1], pi(np.ascontiguousarray(k, np.int32)),
                                                pf(np.ascontiguousarray(d, np.float32)), c["x0"], c["h"], self.w,
                                                pd(P), radius)


class HostStep:
    """The reference's CPU step (src/simulation.jl:309-352, 382-396) on float64
    positions (N, 3): host deposits, Poisson, mean field, forces! with its
    margin test, projectile_forces! with ball softening, chunked Verlet."""

    def __init__(self, meshes, sm, weight, jellium, dt, rcmax, projectile=None):
        self.F, self.Cl = Level(meshes.fine), Level(meshes.coarse)
        self.S = Smoothing(sm)
        self.meshes, self.sm = meshes, sm
        self.w, self.jel, self.dt, self.rcmax = weight, jellium, dt, rcmax
        self.proj = projectile
        nf, nc = self.F.n, self.Cl.n
        self.rhof, self.rhoc = np.zeros(nf ** 3), np.zeros(nc ** 3)
        self.phif, self.phic = np.zeros(nf ** 3), np.zeros(nc ** 3)
        self.csolf, self.csolc = np.zeros(nf ** 3), np.zeros(nc ** 3)

    def update_forces(self, pos, advance=True):
        N = len(pos)
        pos = np.ascontiguousarray(pos)
        self.nout = lib().orc_deposit_smoothed_host(self.F.ref(), self.S.ref(), N, pd(pos), self.w, pd(self.rhof))
        lib().orc_deposit_cic_host(self.Cl.ref(), N, pd(pos), self.w, pd(self.rhoc))
        lib().orc_poisson(self.F.ref(), self.Cl.ref(), pd(self.rhof), pd(self.rhoc), pd(self.phif), pd(self.phic))
        lib().orc_spline_coefficients(self.F.ref(), pd(self.phif), pd(self.csolf))
        lib().orc_spline_coefficients(self.Cl.ref(), pd(self.phic), pd(self.csolc))
        lib().orc_effective_potential(self.F.ref(), pd(self.csolf), pd(self.rhof), self.jel.nions, self.jel.radius)
        lib().orc_effective_potential(self.Cl.ref(), pd(self.csolc), pd(self.rhoc), self.jel.nions,
                                      self.jel.radius)
        force = np.empty((N, 3))
        self.noutf = lib().orc_forces_host(self.F.ref(), self.Cl.ref(), self.S.ref(), N, pd(pos), pd(self.csolf),
                                           pd(self.csolc), self.w, 0, pd(force))
        F = None
        if advance and self.proj is not None:
            F = np.zeros(3)
            ee, ej = np.zeros(1), np.zeros(1)
            pr = projectile_struct(self.proj)
            lib().orc_projectile_forces_host(N, pd(pos), pd(force), C.byref(pr), self.w, self.jel.nions,
                                             self.jel.radius, pd(F), pd(ee), pd(ej))
            lib().orc_projectile_step(C.byref(pr), pd(F), self.dt)
            self.proj.position = np.array(pr.pos[:])
            self.proj.previous = np.array(pr.prev[:])
            self.proj.velocity = np.array(pr.vel[:])
        return force, F

    def prime(self, pos, mom, consistent=False):
        """prime_leapfrog! (src/simulation.jl:233-277): the forces at the half
        step back q(-dt/2) = q0 - dt/(2M) p, without the projectile (it is
        neither advanced nor felt while priming, src/simulation.jl:242-246,
        343), then q(-dt) = -q0 + 2 q(-dt/2) + c F with the Fortran's c = dt/M
        (src/particles.jl:441-469), or dt^2/4M when `consistent`.  Returns
        (pos, prev)."""
        M, dt = self.w, self.dt
        pos = np.array(pos, dtype=np.float64)  # a copy: step() advances its arrays in place
        half = pos - (dt / (2 * M)) * mom
        force, _ = self.update_forces(half, advance=False)
        coef = dt * dt / (4 * M) if consistent else dt / M
        return pos, -pos + 2 * half + coef * force

    def step(self, pos, prev):
        """One step; pos and prev are advanced in place (float64 C-contiguous
        arrays) and returned."""
        force, _ = self.update_forces(pos)
        diag = np.zeros(5)
        pos, prev = np.ascontiguousarray(pos), np.ascontiguousarray(prev)
        lib().orc_verlet_host(len(pos), pd(pos), pd(prev), pd(force), self.dt, self.w, self.rcmax, pd(diag))
        return pos, prev, diag

    def enclosed_charge(self, pos, radius):
        P = np.ascontiguousarray(self.proj.position, dtype=np.float64)
        return lib().orc_enclosed_charge_host(len(pos), pd(np.ascontiguousarray(pos)), self.w, pd(P), radius)
