"""Host side of the drop-in: the reference's simulation driver and device
accelerator, over the C ABI.

Names and argument meanings follow the reference (the Julia `!` dropped):

* SimulationParameters ............ src/simulation.jl:26-38
* Jellium, xc constants ........... src/meanfield.jl:28-36
* BallSoftening, GaussianSoftening,
  Projectile ...................... src/projectile.jl:41-168
* RadialProfile, read_radial_profile,
  sample_thomas_fermi ............. src/initial.jl:131-203
* DeviceAccelerator ............... src/accelerator.jl:126-331 (+ DeviceMesh,
  src/devicemesh.jl:21-81): one handle on the library's context, with the
  calls the reference's resident step makes on it
* Simulation, step, run, sync_host  src/simulation.jl:128-552 (the resident,
  packed device path)

The product path runs on the GPU only; constructing a DeviceAccelerator
without the built library, or without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib as L
from .tables import GaussianSmoothing, NestedMeshes, SplineMesh, build_meshes, gaussian_smoothing, grids

WIGNER_SEITZ_NA = 4.0
ELECTRON_MASS = 1.0
DATA_DIR = Path(__file__).resolve().parent / "data"


# ---------------------------------------------------------------- physics
@dataclass
class SimulationParameters:
    nfine: int = 28
    ninner: int = 14
    nouter: int = 14
    rcluster: float = 50.0
    rbox: float = 150.0
    nions: float = 196.0
    nelectrons: float = 196.0
    nparticles: int = 20_000
    nsteps: int = 10
    dt: float = 1.0
    rcmax: float = 100.0

    @staticmethod
    def for_grid(nfine: int, **kw) -> "SimulationParameters":
        """The coarse subdivision the reference's scripts derive from nfine
        (scripts/xenon.jl:162-167)."""
        ninner, nouter = grids(nfine)
        return SimulationParameters(nfine=nfine, ninner=ninner, nouter=nouter, **kw)


@dataclass
class Jellium:
    nions: float
    radius: float

    @staticmethod
    def of(nions: float, rs: float = WIGNER_SEITZ_NA) -> "Jellium":
        return Jellium(float(nions), float(rs) * math.cbrt(float(nions)))


@dataclass
class BallSoftening:
    radius: float

    @property
    def scale(self):
        return self.radius


@dataclass
class GaussianSoftening:
    sigma: float

    @property
    def scale(self):
        return self.sigma


@dataclass
class Projectile:
    """Incident ion (src/projectile.jl:141-168).  With softening_mode
    VLB_SOFTENING_DEVICE (the default) the fused force path uses a Gaussian of
    width scale(softening) and out-of-stencil particles see the ball of the
    same radius, as the reference's device path does; with VLB_SOFTENING_BALL
    every particle sees the ball, as its CPU path does
    (src/projectile.jl:203-232)."""
    mass: float
    charge: float
    softening: object
    initial_energy: float
    position: np.ndarray
    previous: np.ndarray
    velocity: np.ndarray
    softening_mode: int = L.VLB_SOFTENING_DEVICE

    @staticmethod
    def make(*, mass, charge, energy, impact=0.0, x0, dt, softening) -> "Projectile":
        v = np.array([math.sqrt(2 * energy / mass), 0.0, 0.0])
        pos = np.array([float(x0), float(impact), 0.0])
        return Projectile(float(mass), float(charge), softening, float(energy), pos, pos - dt * v, v)

    def kinetic_energy(self):
        return self.mass * float(np.sum(self.velocity ** 2)) / 2

    def energy_loss(self):
        return self.initial_energy - self.kinetic_energy()

    def to_desc(self) -> L.ProjectileDesc:
        d = L.ProjectileDesc()
        for i in range(3):
            d.position[i] = self.position[i]
            d.previous[i] = self.previous[i]
            d.velocity[i] = self.velocity[i]
        d.charge = self.charge
        d.mass = self.mass
        d.sigma = self.softening.scale
        d.ball_radius = self.softening.scale
        d.active = 1
        d.softening = self.softening_mode
        return d

    def from_desc(self, d: L.ProjectileDesc):
        self.position = np.array(d.position[:])
        self.previous = np.array(d.previous[:])
        self.velocity = np.array(d.velocity[:])


def xenon_projectile(*, v=0.40, impact=45.0, x0=-70.0, dt=0.5, charge=25.0, mass=131.3 * 1836.154,
                     radius=5.0) -> Projectile:
    """The Xe25+ ion of scripts/xenon.jl:337-340 (energy = m v^2 / 2)."""
    return Projectile.make(mass=mass, charge=charge, energy=0.5 * mass * v ** 2, impact=impact, x0=x0, dt=dt,
                           softening=BallSoftening(radius))


# ----------------------------------------------------------- sampling
@dataclass
class RadialProfile:
    quantiles: np.ndarray
    density: np.ndarray
    rmax: float


def read_radial_profile(hm1_path, rhoinit_path) -> RadialProfile:
    """hm1.dat / rhoinit.dat format (src/initial.jl:143-158)."""
    with open(hm1_path) as f:
        n = int(f.readline())
        q = np.array([float(f.readline().replace("D", "E").replace("d", "e")) for _ in range(n)])
    with open(rhoinit_path) as f:
        n = int(f.readline())
        rmax = float(f.readline())
        rho = np.array([float(f.readline().replace("D", "E").replace("d", "e")) for _ in range(n)])
    return RadialProfile(q, rho, rmax)


def thomas_fermi_profile() -> RadialProfile:
    """The Na196 Thomas-Fermi profile the reference's runs read
    (ref/fortran/data/hm1.dat, rhoinit.dat), shipped as a fixture."""
    z = np.load(DATA_DIR / "na196_profile.npz")
    return RadialProfile(z["quantiles"], z["density"], float(z["rmax"]))


def uniform_sphere_profile(nions: float = 196.0, rs: float = WIGNER_SEITZ_NA, nq: int = 1001) -> RadialProfile:
    """Uniform ball of the jellium radius and bulk density 3/(4 pi rs^3): the
    analytic RadialProfile of test/runtests.jl:981-986 at the cluster's size."""
    R = rs * math.cbrt(nions)
    rho0 = 3 / (4 * math.pi * rs ** 3)
    q = np.array([R * math.cbrt((j - 1) / (nq - 1)) for j in range(1, nq + 1)])
    return RadialProfile(q, np.full(nq, rho0), R)


def sample_thomas_fermi(profile: RadialProfile, npart: int, weight: float, seed: int = -1,
                        consistent: bool = False):
    """(positions, momenta) float64 (npart, 3), ran2(seed) stream."""
    pos = np.empty((npart, 3))
    mom = np.empty((npart, 3))
    q = np.ascontiguousarray(profile.quantiles, dtype=np.float64)
    r = np.ascontiguousarray(profile.density, dtype=np.float64)
    L.check(L.lib().vlb_sample_thomas_fermi(L.pd(q), len(q), L.pd(r), len(r), float(profile.rmax), npart,
                                            float(weight), int(seed), int(consistent), L.pd(pos), L.pd(mom)))
    return pos, mom


class ThomasFermiStream:
    """The seeded Thomas-Fermi cloud (src/initial.jl:94-113) drawn a chunk at
    a time: consecutive draws give the particles of sample_thomas_fermi's
    one-shot cloud in order, bit for bit (vlb_sampler)."""

    def __init__(self, profile: RadialProfile, weight: float, seed: int = -1, consistent: bool = False):
        self._q = np.ascontiguousarray(profile.quantiles, dtype=np.float64)
        self._r = np.ascontiguousarray(profile.density, dtype=np.float64)
        h = C.c_void_p()
        L.check(L.lib().vlb_sampler_create(L.pd(self._q), len(self._q), L.pd(self._r), len(self._r),
                                           float(profile.rmax), float(weight), int(seed), int(consistent),
                                           C.byref(h)))
        self._h = h

    def draw(self, n: int):
        """(positions, momenta) float64 (n, 3) of the next n particles."""
        pos, mom = np.empty((n, 3)), np.empty((n, 3))
        L.check(L.lib().vlb_sampler_draw(self._h, int(n), L.pd(pos), L.pd(mom)))
        return pos, mom

    def skip(self, n: int):
        L.check(L.lib().vlb_sampler_draw(self._h, int(n), None, None))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().vlb_sampler_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


STREAM_CHUNK = 1 << 20  # particles per chunk of a streamed construction (about 150 MB of host arrays)


def stream_half_step_cloud(acc: "DeviceAccelerator", stream: ThomasFermiStream, lo: int, hi: int, M: float,
                           dt: float, chunk: int = STREAM_CHUNK):
    """The first half of prime_leapfrog! (src/simulation.jl:233-277) for the
    particles [lo, hi) of a cloud drawn from `stream` (the particles before lo
    are drawn and dropped): each chunk's current position q0 and its half
    step back q0 - dt/(2M) p, packed into the slots [0, hi - lo) of `acc`
    chunk by chunk, so that no whole host copy of the cloud exists."""
    if lo:
        for a in range(0, lo, chunk):
            stream.skip(min(chunk, lo - a))
    for a in range(lo, hi, chunk):
        n = min(chunk, hi - a)
        pos, mom = stream.draw(n)
        k, d = pack_positions(pos - (dt / (2 * M)) * mom, acc.x0, acc.h)
        pk, pd = pack_positions(pos, acc.x0, acc.h)
        del pos, mom
        acc.upload_range(a - lo, k, d, pk, pd)


def prime_back_chunked(acc: "DeviceAccelerator", M: float, dt: float, consistent: bool = False,
                       chunk: int = STREAM_CHUNK):
    """The second half of prime_leapfrog!, after the forces at the half step:
    per chunk of slots, q(-dt) = -q0 + 2 q(-dt/2) + c F with the Fortran's
    c = dt/M (dt^2/4M when `consistent`), then (q0, q(-dt)) as the record."""
    coef = dt * dt / (4 * M) if consistent else dt / M
    for a in range(0, acc.npart, chunk):
        n = min(chunk, acc.npart - a)
        k, d, pk, pd = acc.download_range(a, n)
        f = acc.force_range(a, n).astype(np.float64).T
        q0 = unpack_positions(pk, pd, acc.x0, acc.h)
        hp = unpack_positions(k, d, acc.x0, acc.h)
        back = -q0 + 2 * hp + coef * f
        k, d = pack_positions(q0, acc.x0, acc.h)
        pk, pd = pack_positions(back, acc.x0, acc.h)
        acc.upload_range(a, k, d, pk, pd)


def ran2(seed: int, n: int, consistent: bool = False) -> np.ndarray:
    out = np.empty(n, dtype=np.float32)
    L.check(L.lib().vlb_ran2(seed, int(consistent), n, L.pf(out)))
    return out


def pack_positions(pos: np.ndarray, x0: float, h: float):
    """(k, delta) SoA (3, N) of float64 positions (src/particles.jl:135-149)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n = len(pos)
    k = np.empty((3, n), dtype=np.int32)
    d = np.empty((3, n), dtype=np.float32)
    L.check(L.lib().vlb_pack_positions(n, L.pd(pos), x0, h, L.pi(k), L.pf(d)))
    return k, d


def unpack_positions(k: np.ndarray, d: np.ndarray, x0: float, h: float) -> np.ndarray:
    k = np.ascontiguousarray(k, dtype=np.int32)
    d = np.ascontiguousarray(d, dtype=np.float32)
    n = k.shape[1]
    out = np.empty((n, 3))
    L.check(L.lib().vlb_unpack_positions(n, L.pi(k), L.pf(d), x0, h, L.pd(out)))
    return out


# ------------------------------------------------------- the accelerator
def _level_desc(m: SplineMesh, keep: list) -> L.LevelDesc:
    def arr(a, dt=np.float64):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a

    d = L.LevelDesc()
    d.nknots = m.axis.nknots
    d.knots = L.pd(arr(m.axis.knots))
    d.colloc = L.pd(arr(m.axis.colloc))
    d.sinv = L.pd(arr(m.cm.Sinv))
    d.laplacian = L.pd(arr(m.laplacian))
    d.eigvec = L.pd(arr(m.op.M))
    d.eigvec_inv = L.pd(arr(m.op.Minv))
    d.eigval = L.pd(arr(m.op.lam))
    d.dual_moments = L.pd(arr(np.concatenate(m.duals)))
    d.dual_lengths = L.pd(arr(m.dlen))
    d.locate_x0 = m.locator.x0
    d.locate_invwidth = m.locator.invwidth
    d.locate_ncells = len(m.locator.cell)
    d.locate_cells = L.pi(arr(m.locator.cell, np.int32))
    return d


class DeviceAccelerator:
    """The device half of the resident step: DeviceAccelerator + the two
    DeviceMesh mirrors of the reference, behind one library context."""

    def __init__(self, meshes: NestedMeshes, sm: GaussianSmoothing, npart: int, weight: float, device: int = 0):
        keep: list = []
        cfg = L.Config()
        cfg.npart = int(npart)
        cfg.weight = float(weight)
        cfg.fine = _level_desc(meshes.fine, keep)
        cfg.coarse = _level_desc(meshes.coarse, keep)
        s = L.SmoothingDesc()
        s.nbdt = sm.nbdt
        s.spacing = sm.spacing
        for name, tab in (("overlap", sm.overlap), ("gradient", sm.gradient), ("nodes", sm.nodes)):
            a = np.ascontiguousarray(tab.T, dtype=np.float64)
            keep.append(a)
            setattr(s, name, L.pd(a))
        cfg.smoothing = s
        cfg.device = device
        handle = C.c_void_p()
        L.check(L.lib().vlb_create(C.byref(cfg), C.byref(handle)))
        self._h = handle
        self.device = int(device)
        self.npart = int(npart)
        self.weight = float(weight)
        self.meshes = meshes
        self.smoothing = sm
        knots = meshes.fine.axis.knots
        self.x0 = float(knots[0])
        self.h = float((knots[-1] - knots[0]) / (len(knots) - 1))
        self.nf = meshes.fine.n
        self.nc = meshes.coarse.n

    # handle lifetime
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().vlb_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # --- cloud transfer (upload!/download!, src/accelerator.jl:48-68)
    def upload_range(self, first: int, k, d, pk, pd):
        """Slots [first, first + count) from (3, count) arrays."""
        arrs = [np.ascontiguousarray(a, dtype=t) for a, t in
                ((k, np.int32), (d, np.float32), (pk, np.int32), (pd, np.float32))]
        count = arrs[0].shape[1]
        for a in arrs:
            if a.shape != (3, count):
                raise ValueError("particle arrays must share one (3, count) shape")
        L.check(L.lib().vlb_upload_particles_range(self._h, int(first), int(count), L.pi(arrs[0]), L.pf(arrs[1]),
                                                   L.pi(arrs[2]), L.pf(arrs[3])))

    def download_range(self, first: int, count: int):
        k = np.empty((3, count), np.int32)
        d = np.empty((3, count), np.float32)
        pk = np.empty((3, count), np.int32)
        pd = np.empty((3, count), np.float32)
        L.check(L.lib().vlb_download_particles_range(self._h, int(first), int(count), L.pi(k), L.pf(d), L.pi(pk),
                                                     L.pf(pd)))
        return k, d, pk, pd

    def force_range(self, first: int, count: int) -> np.ndarray:
        f = np.empty((3, count), np.float32)
        L.check(L.lib().vlb_get_forces_range(self._h, int(first), int(count), L.pf(f)))
        return f

    def upload(self, k, d, pk, pd):
        arrs = [np.ascontiguousarray(a, dtype=t) for a, t in
                ((k, np.int32), (d, np.float32), (pk, np.int32), (pd, np.float32))]
        for a in arrs:
            if a.shape != (3, self.npart):
                raise ValueError(f"particle arrays must be (3, {self.npart})")
        L.check(L.lib().vlb_upload_particles(self._h, L.pi(arrs[0]), L.pf(arrs[1]), L.pi(arrs[2]), L.pf(arrs[3])))

    def download(self):
        k = np.empty((3, self.npart), np.int32)
        d = np.empty((3, self.npart), np.float32)
        pk = np.empty((3, self.npart), np.int32)
        pd = np.empty((3, self.npart), np.float32)
        L.check(L.lib().vlb_download_particles(self._h, L.pi(k), L.pf(d), L.pi(pk), L.pf(pd)))
        return k, d, pk, pd

    # --- the calls of the resident step
    def sort(self):
        nocc = C.c_int32()
        nout = C.c_int32()
        L.check(L.lib().vlb_sort(self._h, C.byref(nocc), C.byref(nout)))
        self._nocc, self._outc = nocc.value, nout.value
        return nocc.value, nout.value

    def sort_products(self):
        """perm, occupied cells, bounds and out-of-stencil slots of the last sort."""
        n_occ, n_out = C.c_int32(), C.c_int32()
        L.check(L.lib().vlb_get_sort_sizes(self._h, C.byref(n_occ), C.byref(n_out)))
        nocc, outc = n_occ.value, n_out.value
        perm = np.empty(self.npart, np.int32)
        occ = np.empty(max(nocc, 1), np.int32)
        bnd = np.empty(nocc + 1, np.int32)
        out = np.empty(max(outc, 1), np.int32)
        L.check(L.lib().vlb_get_sort(self._h, L.pi(perm), L.pi(occ), L.pi(bnd), L.pi(out)))
        return perm, occ[:nocc], bnd, out[:outc]

    def deposit_smoothed(self, charge: float, fixed_point: bool = False):
        nout = C.c_int32()
        q = C.c_double()
        mode = L.VLB_DEPOSIT_FIXED64 if fixed_point else L.VLB_DEPOSIT_FLOAT32
        L.check(L.lib().vlb_deposit_fine(self._h, charge, mode, C.byref(nout), C.byref(q)))
        return nout.value, q.value

    def deposit_cic(self, charge: float):
        L.check(L.lib().vlb_deposit_coarse(self._h, charge))

    def poisson(self, precision: int = L.VLB_POISSON_FP32):
        """poisson!(phi, rho, meshes); precision VLB_POISSON_FP32 (CUDA cores),
        VLB_POISSON_3XTF32 or VLB_POISSON_BF16X3 (split-precision tensor cores).  Later coefficient
        conversions use the same precision."""
        L.check(L.lib().vlb_poisson(self._h, precision))

    def set_precision(self, precision: int):
        L.check(L.lib().vlb_set_precision(self._h, precision))

    def spline_coefficients(self, level: int):
        L.check(L.lib().vlb_coefficients(self._h, level))

    def effective_potential(self, level: int, jel: Jellium):
        L.check(L.lib().vlb_mean_field(self._h, level, jel.nions, jel.radius))

    def forces(self, projectile: Projectile | None):
        red = np.zeros(4)
        outc = C.c_int32()
        desc = projectile.to_desc() if projectile is not None else None
        L.check(L.lib().vlb_forces(self._h, C.byref(desc) if desc is not None else None, L.pd(red),
                                   C.byref(outc)))
        return red, outc.value

    def projectile_forces(self, projectile: Projectile, jel: Jellium):
        F = np.zeros(3)
        ee, ej = C.c_double(), C.c_double()
        desc = projectile.to_desc()
        L.check(L.lib().vlb_projectile_forces(self._h, C.byref(desc), jel.nions, jel.radius, L.pd(F),
                                              C.byref(ee), C.byref(ej)))
        return F, ee.value, ej.value

    def push(self, dt: float, rcmax: float = math.inf):
        diag = np.zeros(5)
        L.check(L.lib().vlb_push(self._h, dt, rcmax, L.pd(diag)))
        return dict(kinetic=diag[0], escaped=diag[1], angular=tuple(diag[2:]))

    def fused_step(self, projectile: Projectile | None, params: L.StepParams) -> L.StepResult:
        res = L.StepResult()
        desc = projectile.to_desc() if projectile is not None else None
        L.check(L.lib().vlb_step(self._h, C.byref(desc) if desc is not None else None, C.byref(params),
                                 C.byref(res)))
        if projectile is not None:
            projectile.from_desc(desc)
        self._nocc, self._outc = res.noccupied, res.outcount
        return res

    # -- the step in three phases, for a cloud sharded over several contexts
    def exchange(self, deposit_mode: int) -> L.Exchange:
        """Device addresses of the buffers the shards sum between phases."""
        x = L.Exchange()
        L.check(L.lib().vlb_exchange_buffers(self._h, deposit_mode, C.byref(x)))
        return x

    def step_deposit(self, projectile: Projectile | None, params: L.StepParams):
        desc = projectile.to_desc() if projectile is not None else None
        L.check(L.lib().vlb_step_deposit(self._h, C.byref(desc) if desc is not None else None, C.byref(params)))

    def step_fields(self, params: L.StepParams, npart_global: int):
        L.check(L.lib().vlb_step_fields(self._h, C.byref(params), int(npart_global)))

    def step_advance(self, projectile: Projectile | None, params: L.StepParams) -> L.StepResult:
        res = L.StepResult()
        desc = projectile.to_desc() if projectile is not None else None
        L.check(L.lib().vlb_step_advance(self._h, C.byref(desc) if desc is not None else None, C.byref(params),
                                         C.byref(res)))
        if projectile is not None:
            projectile.from_desc(desc)
        self._nocc, self._outc = res.noccupied, res.outcount
        return res

    def grid(self, which: int) -> np.ndarray:
        n = self.nf if which % 2 == 0 else self.nc
        out = np.empty((n, n, n), np.float32)  # [k][j][i]: i fastest
        L.check(L.lib().vlb_get_grid(self._h, which, L.pf(out)))
        return out

    def set_grid(self, which: int, values: np.ndarray):
        n = self.nf if which % 2 == 0 else self.nc
        a = np.ascontiguousarray(values, dtype=np.float32).reshape(n, n, n)
        L.check(L.lib().vlb_set_grid(self._h, which, L.pf(a)))

    def force(self) -> np.ndarray:
        out = np.empty((3, self.npart), np.float32)
        L.check(L.lib().vlb_get_forces(self._h, L.pf(out)))
        return out

    def set_force(self, f: np.ndarray):
        a = np.ascontiguousarray(f, dtype=np.float32)
        L.check(L.lib().vlb_set_forces(self._h, L.pf(a)))

    def enclosed_charge(self, position, radius: float) -> float:
        P = np.ascontiguousarray(position, dtype=np.float64)
        q = C.c_double()
        L.check(L.lib().vlb_enclosed_charge(self._h, L.pd(P), radius, C.byref(q)))
        return q.value

    # -- launch shapes (vlb_set_tuning)
    def tuning(self) -> dict:
        t = L.Tuning()
        L.check(L.lib().vlb_get_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        """Changes some launch shapes (field_tensor_cores, chunk,
        field_ctas_per_sm, cic_ctas_per_sm, push_ctas_per_sm,
        move_ctas_per_sm)."""
        cur = self.tuning()
        unknown = set(kw) - set(cur)
        if unknown:
            raise ValueError(f"unknown launch shapes {sorted(unknown)}")
        cur.update(kw)
        t = L.Tuning(**cur)
        L.check(L.lib().vlb_set_tuning(self._h, C.byref(t)))

    def launch_count(self) -> int:
        n = C.c_int64()
        L.check(L.lib().vlb_launch_count(self._h, C.byref(n)))
        return n.value

    def profile(self, on: bool):
        L.check(L.lib().vlb_profile(self._h, int(on)))

    # -- the film (vlb_film_*): density slices and capture scalars on the device
    def film_reserve(self, capacity: int, iz1: int, iz2: int, radius: float):
        L.check(L.lib().vlb_film_reserve(self._h, int(capacity), int(iz1), int(iz2), float(radius)))

    def film_frames(self) -> tuple[int, int]:
        """(taken, stored) frames since the reservation."""
        taken, stored = C.c_int32(), C.c_int32()
        L.check(L.lib().vlb_film_frames(self._h, C.byref(taken), C.byref(stored)))
        return taken.value, stored.value

    def film_download(self, first: int = 0, count: int | None = None):
        """(frames (count, n, n) float32 [j][i], scalars (count, 4) float64)."""
        if count is None:
            count = self.film_frames()[1] - first
        frames = np.empty((count, self.nf, self.nf), np.float32)
        scalars = np.empty((count, 4), np.float64)
        L.check(L.lib().vlb_film_download(self._h, int(first), int(count), L.pf(frames), L.pd(scalars)))
        return frames, scalars

    def film_clear(self):
        L.check(L.lib().vlb_film_clear(self._h))

    def interaction_energy(self, coefficients: int = L.VLB_ENERGY_TOTAL) -> float:
        """sum w phi over the cloud as it is (interaction_energy, src/energy.jl:19-43)."""
        out = C.c_double()
        L.check(L.lib().vlb_interaction_energy(self._h, int(coefficients), C.byref(out)))
        return out.value

    def stage_times(self) -> dict:
        n = L.lib().vlb_stage_count()
        ms = np.zeros(12)
        L.check(L.lib().vlb_stage_times(self._h, L.pd(ms), 12))
        return {L.lib().vlb_stage_name(i).decode(): ms[i] for i in range(n) if i != 9}

    def stream_handle(self) -> int:
        s = C.c_void_p()
        L.check(L.lib().vlb_stream(self._h, C.byref(s)))
        return s.value or 0


# ----------------------------------------------------------- simulation
@dataclass
class StepDiagnostics:
    kinetic: float
    escaped: float
    angular: tuple
    enclosed_charge: float
    nout: int
    outcount: int
    noccupied: int
    projectile_force: tuple
    total_charge: float
    status: int = 0
    denoised: int = 0            # 1: the step's fine density came from the learned denoiser
    hartree: float = 0.0         # energy steps: 1/2 sum w phi_H at the step's positions
    interaction: float = 0.0     # energy steps: sum w phi at the advanced positions
    sort_path: int = 0           # 1: single-pass placement, 2: placement given up for radix, 0: radix alone


@dataclass
class EnergyBudget:
    """The energy of the system after a step (EnergyBudget,
    src/energy.jl:69-79): total = ions + kinetic + hartree + meanfield, the
    mean field by difference, meanfield = interaction - 2 hartree
    (energy_budget, src/energy.jl:111-117)."""
    total: float
    kinetic: float
    hartree: float
    meanfield: float
    ions: float
    escaped: float

    @staticmethod
    def of(jellium: "Jellium", d: "StepDiagnostics") -> "EnergyBudget":
        meanfield = d.interaction - 2 * d.hartree
        ions = 3 * jellium.nions ** 2 / (5 * jellium.radius)   # ion_self_energy, src/energy.jl:51
        return EnergyBudget(ions + d.kinetic + d.hartree + meanfield, d.kinetic, d.hartree, meanfield, ions,
                            d.escaped)


@dataclass
class Film:
    """Frames of the reference's movie (scripts/xenon.jl:370-410), as arrays:
    frames (count, n, n) float32 [j][i], the projectile's x and y, q(<capture
    radius) around it and the net charge nions - w #{|r| < radius}; `taken`
    counts the frames asked for (more than stored when the film was full)."""
    frames: np.ndarray
    proj_x: np.ndarray
    proj_y: np.ndarray
    q_capture: np.ndarray
    q_net: np.ndarray
    taken: int


class Simulation:
    """The reference's resident device simulation (src/simulation.jl:171-216,
    472-531): meshes and tables built once on the host in float64, the packed
    cloud sampled with ran2 and primed, then every step on the GPU."""

    def __init__(self, p: SimulationParameters, profile: RadialProfile, *, projectile: Projectile | None = None,
                 seed: int = -1, consistent_startup: bool = False, device: int = 0,
                 fixed_point: bool = False, use_graph: bool = True, capture_radius: float = 8.0,
                 precision: int = L.VLB_POISSON_FP32, softening_mode: int | None = None,
                 stream_chunk: int = STREAM_CHUNK):
        """softening_mode: VLB_SOFTENING_DEVICE (the reference's device path)
        or VLB_SOFTENING_BALL (its CPU path); None keeps the projectile's.
        stream_chunk > 0: the cloud is drawn, packed, uploaded and primed
        stream_chunk particles at a time (the same cloud as a one-shot draw,
        with a bounded host peak); 0: drawn whole on the host."""
        self.params = p
        self.meshes = build_meshes(p.nfine, p.ninner, p.nouter, p.rcluster, p.rbox)
        self.smoothing = gaussian_smoothing(self.meshes.fine.axis)
        self.jellium = Jellium.of(p.nions)
        self.weight = p.nelectrons / p.nparticles
        self.projectile = projectile
        if projectile is not None and softening_mode is not None:
            if softening_mode not in (L.VLB_SOFTENING_DEVICE, L.VLB_SOFTENING_BALL):
                raise ValueError("softening_mode must be VLB_SOFTENING_DEVICE or VLB_SOFTENING_BALL")
            projectile.softening_mode = softening_mode
        self.fixed_point = fixed_point
        self.precision = precision
        self.use_graph = use_graph
        self.capture_radius = capture_radius
        self.denoise = False       # set by denoiser.attach()
        self.accelerator = DeviceAccelerator(self.meshes, self.smoothing, p.nparticles, self.weight, device)
        self.x0, self.h = self.accelerator.x0, self.accelerator.h
        self.steps_done = 0
        if stream_chunk > 0:
            stream = ThomasFermiStream(profile, self.weight, seed=seed)
            try:
                stream_half_step_cloud(self.accelerator, stream, 0, p.nparticles, self.mass, p.dt, stream_chunk)
            finally:
                stream.close()
            self._prime_forces()
            prime_back_chunked(self.accelerator, self.mass, p.dt, consistent_startup, stream_chunk)
        else:
            positions, momenta = sample_thomas_fermi(profile, p.nparticles, self.weight, seed=seed)
            self.prime_leapfrog(positions, momenta, consistent=consistent_startup)

    @property
    def mass(self):
        return ELECTRON_MASS * self.weight

    def _params(self, *, advance: bool, push: bool, capture: float, energy: bool = False,
                film: bool = False) -> L.StepParams:
        sp = L.StepParams()
        sp.dt = self.params.dt
        sp.rcmax = self.params.rcmax
        sp.jellium_nions = self.jellium.nions
        sp.jellium_radius = self.jellium.radius
        sp.capture_radius = capture
        sp.deposit_mode = L.VLB_DEPOSIT_FIXED64 if self.fixed_point else L.VLB_DEPOSIT_FLOAT32
        sp.advance_projectile = int(advance)
        sp.push = int(push)
        sp.use_graph = int(self.use_graph and push)
        sp.poisson_precision = self.precision
        sp.denoise = int(self.denoise and push)
        sp.energy = int(energy and push)
        sp.film = int(film and push)
        return sp

    def prime_leapfrog(self, positions, momenta, consistent: bool = False):
        """Two-stage priming (src/simulation.jl:233-277), with the Fortran's
        dt/M coefficient unless `consistent`.  The forces at q(-dt/2) carry the
        projectile's reaction on the device path (its forces! fuses the
        projectile, src/simulation.jl:521) and not on the CPU path (there the
        reaction comes with advance_projectile!, skipped while priming,
        src/simulation.jl:343, 454-460)."""
        M, dt = self.mass, self.params.dt
        half = positions - (dt / (2 * M)) * momenta
        k, d = pack_positions(half, self.x0, self.h)
        pk, pd = pack_positions(positions, self.x0, self.h)
        acc = self.accelerator
        acc.upload(k, d, pk, pd)
        self._prime_forces()
        k, d, pk, pd = acc.download()
        f = acc.force().astype(np.float64).T
        q0 = unpack_positions(pk, pd, self.x0, self.h)
        hp = unpack_positions(k, d, self.x0, self.h)
        coef = dt * dt / (4 * M) if consistent else dt / M
        back = -q0 + 2 * hp + coef * f
        k, d = pack_positions(q0, self.x0, self.h)
        pk, pd = pack_positions(back, self.x0, self.h)
        acc.upload(k, d, pk, pd)

    def _prime_forces(self):
        """The forces at the half step back, on the uploaded (q(-dt/2), q0)
        records: a forces-only step, the projectile not advanced."""
        pr = self.projectile
        if pr is not None and pr.softening_mode == L.VLB_SOFTENING_BALL:
            pr = None
        self.accelerator.fused_step(pr, self._params(advance=False, push=False, capture=0.0))

    def step(self, energy: bool = False, film: bool = False) -> StepDiagnostics:
        """step!(sim; energy) on the device.  With energy, the diagnostics
        carry the budget's two sums (EnergyBudget.of(sim.jellium, d) is the
        reference's return value).  With film, the step appends a frame to
        the film reserved by film()."""
        r = self.accelerator.fused_step(self.projectile, self._params(advance=True, push=True,
                                                                      capture=self.capture_radius, energy=energy,
                                                                      film=film))
        self.steps_done += 1
        return StepDiagnostics(r.kinetic, r.escaped, tuple(r.angular), r.enclosed_charge, r.nout, r.outcount,
                               r.noccupied, tuple(r.projectile_force), r.total_charge, r.status, r.denoised,
                               r.hartree, r.interaction, r.sort_path)

    def film(self, capacity: int, radius: float = 35.0):
        """Reserves `capacity` frames of the reference's movie
        (scripts/xenon.jl:370-410): the fine density averaged over the two
        planes around z = 0 and the capture scalars, taken on the device by
        the steps run with film=True."""
        n = self.params.nfine
        self.accelerator.film_reserve(capacity, n - 1, n, radius)

    def film_frames(self) -> "Film":
        """The frames taken so far (a download; the film stays reserved)."""
        frames, sc = self.accelerator.film_download()
        taken, _ = self.accelerator.film_frames()
        return Film(frames, sc[:, 0].copy(), sc[:, 1].copy(), self.weight * sc[:, 2],
                    self.jellium.nions - self.weight * sc[:, 3], taken)

    def energy_budget(self, d: StepDiagnostics) -> EnergyBudget:
        """The EnergyBudget of a step run with energy=True."""
        return EnergyBudget.of(self.jellium, d)

    def run(self, nsteps: int | None = None, callback=None):
        nsteps = self.params.nsteps if nsteps is None else nsteps
        out = []
        for i in range(1, nsteps + 1):
            d = self.step()
            out.append(d)
            if callback is not None:
                callback(i, d)
        return out

    def snapshot(self):
        """The state a step changes: the cloud and the projectile."""
        pr = self.projectile
        proj = None if pr is None else (pr.position.copy(), pr.previous.copy(), pr.velocity.copy())
        return self.accelerator.download(), proj, self.steps_done

    def restore(self, snap):
        cloud, proj, steps = snap
        self.accelerator.upload(*cloud)
        if proj is not None:
            self.projectile.position, self.projectile.previous, self.projectile.velocity = (x.copy() for x in proj)
        self.steps_done = steps

    def positions(self):
        k, d, pk, pd = self.accelerator.download()
        return unpack_positions(k, d, self.x0, self.h), unpack_positions(pk, pd, self.x0, self.h)

    def enclosed_charge(self, radius: float = 8.0) -> float:
        P = self.projectile.position if self.projectile is not None else np.zeros(3)
        return self.accelerator.enclosed_charge(P, radius)

    def sync_host(self) -> dict:
        acc = self.accelerator
        return {name: acc.grid(w) for name, w in (("rho_fine", L.VLB_GRID_RHO_FINE),
                                                   ("rho_coarse", L.VLB_GRID_RHO_COARSE),
                                                   ("phi_fine", L.VLB_GRID_PHI_FINE),
                                                   ("phi_coarse", L.VLB_GRID_PHI_COARSE),
                                                   ("csol_fine", L.VLB_GRID_CSOL_FINE),
                                                   ("csol_coarse", L.VLB_GRID_CSOL_COARSE))}
