"""The step of a cloud sharded over several ranks, one GPU each.

The particles are independent units, coupled only through the fields they
make.  Each rank holds a slice of the cloud and runs the step's three phases
(vlb_step_deposit / vlb_step_fields / vlb_step_advance); between them the
ranks sum, in place:

  after the deposit : the raw fine density (int64 fixed point, or float32),
                      the coarse density (the same) and the count of particles outside
                      the fine deposit window;
  after the forces  : the projectile's four reaction sums.

Everything else -- the charge renormalisation with the whole cloud's count,
the nested Poisson solve, the mean field, the projectile's step -- is
computed identically on every rank from identical sums.  The reference runs
one device (src/simulation.jl:472-531); on one rank this is its step.

The orchestration is written against two small interfaces so that the same
code runs on GPUs (the library's contexts, NCCL through torch.distributed)
and, for testing, on CPU ranks:

  backend: step_deposit(projectile, params), step_fields(params, npart_global),
           step_advance(projectile, params) -> result with the step's local
           sums; deposit_buffers() and reaction_buffer() -> the tensors to sum;
           stream() -> a context manager ordering the sums on the work stream;
           synchronize() -> wait for the work stream;
           tensor(values) -> a float64 tensor where comm can sum it.
  comm:    all_reduce_sum(tensor) in place over the ranks.

A rank may drive several backends (several contexts, one per GPU of the
process, or several on one GPU): their buffers are summed in the process
first, then over the ranks, and the sum is copied back to each.
"""
from __future__ import annotations

import contextlib
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import simulation as S


# ---------------------------------------------------------------- comms
class TorchComm:
    """Sum over the ranks of a torch.distributed process group (NCCL for
    device tensors, gloo for host tensors)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def all_reduce_sum(self, t):
        if self.size > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)


class LocalComm:
    """One rank: the sums are the values."""
    rank, size = 0, 1

    def all_reduce_sum(self, t):
        pass


def device_tensor(ptr: int, count: int, dtype, device: int):
    """A torch tensor over `count` elements of device memory owned by the
    library (no copy, no ownership)."""
    import torch
    typestr = {torch.float32: "<f4", torch.float64: "<f8", torch.int64: "<i8"}[dtype]

    class _View:
        __cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr, "data": (int(ptr), False),
                                    "version": 3, "strides": None}

    with torch.cuda.device(device):
        return torch.as_tensor(_View(), device=f"cuda:{device}")


# -------------------------------------------------------------- backends
class LibraryShard:
    """One rank's context of the B200 library."""

    def __init__(self, acc: S.DeviceAccelerator, deposit_mode: int, device: int):
        import torch
        self.acc, self.device = acc, device
        x = acc.exchange(deposit_mode)
        fine_dtype = torch.int64 if x.rho_fine_dtype == L.VLB_DTYPE_INT64 else torch.float32
        coarse_dtype = torch.int64 if x.rho_coarse_dtype == L.VLB_DTYPE_INT64 else torch.float32
        self._deposit = [device_tensor(x.rho_fine, x.rho_fine_count, fine_dtype, device),
                         device_tensor(x.rho_coarse, x.rho_coarse_count, coarse_dtype, device),
                         device_tensor(x.scalars, x.scalars_count, torch.float64, device)]
        self._reaction = device_tensor(x.reaction, x.reaction_count, torch.float64, device)
        self._stream = torch.cuda.ExternalStream(x.stream, device=torch.device("cuda", device))

    def stream(self):
        import torch
        return torch.cuda.stream(self._stream)

    def synchronize(self):
        self._stream.synchronize()

    def tensor(self, values):
        import torch
        return torch.tensor(values, dtype=torch.float64, device=f"cuda:{self.device}")

    def deposit_buffers(self):
        return self._deposit

    def reaction_buffer(self):
        return self._reaction

    def step_deposit(self, projectile, params):
        self.acc.step_deposit(projectile, params)

    def step_fields(self, params, npart_global):
        self.acc.step_fields(params, npart_global)

    def step_advance(self, projectile, params):
        return self.acc.step_advance(projectile, params)


@dataclass
class ShardedDiagnostics:
    """The step's diagnostics summed over the ranks."""
    kinetic: float
    escaped: float
    angular: tuple
    enclosed_charge: float
    nout: int
    outcount: int
    projectile_force: tuple
    status: int
    hartree: float = 0.0        # energy steps: the energy budget's sums over the ranks
    interaction: float = 0.0


class ShardedStepper:
    """The three phases and the two exchanges of one step, for this rank's
    backend (or list of backends, each with its own projectile copy)."""

    def __init__(self, backends, comm, npart_global: int):
        self.backends = list(backends) if isinstance(backends, (list, tuple)) else [backends]
        self.comm, self.npart_global = comm, int(npart_global)

    def _sum(self, buffers):
        """Sums, in place, the i-th tensor of every backend's list."""
        bs = self.backends
        if len(bs) > 1:
            for b in bs:
                b.synchronize()
        for i in range(len(buffers[0])):
            ts = [lst[i] for lst in buffers]
            head = ts[0]
            with bs[0].stream():
                for t in ts[1:]:
                    head.add_(t.to(head.device))
                self.comm.all_reduce_sum(head)
            if len(ts) > 1:
                bs[0].synchronize()
                for t in ts[1:]:
                    t.copy_(head.to(t.device))
        if len(bs) > 1:
            for b in bs:
                b.synchronize()
            _synchronize_all(bs)

    def step(self, projectiles, params) -> ShardedDiagnostics:
        bs = self.backends
        projs = projectiles if isinstance(projectiles, (list, tuple)) else [projectiles] * len(bs)
        for b, p in zip(bs, projs):
            b.step_deposit(p, params)
        self._sum([b.deposit_buffers() for b in bs])
        for b in bs:
            b.step_fields(params, self.npart_global)
        self._sum([[b.reaction_buffer()] for b in bs])
        rs = [b.step_advance(p, params) for b, p in zip(bs, projs)]
        local = [0.0] * 11
        for r in rs:
            vals = [r.kinetic, r.escaped, *r.angular, r.enclosed_charge, float(r.nout), float(r.outcount),
                    float(r.status != 0), getattr(r, "hartree", 0.0), getattr(r, "interaction", 0.0)]
            local = [x + y for x, y in zip(local, vals)]
        t = bs[0].tensor(local)
        self.comm.all_reduce_sum(t)
        g = [float(v) for v in t.tolist()]
        return ShardedDiagnostics(g[0], g[1], tuple(g[2:5]), g[5], int(round(g[6])), int(round(g[7])),
                                  tuple(rs[0].projectile_force), int(g[8] != 0), g[9], g[10])


def _synchronize_all(backends):
    """The copies of _sum ran on torch's current streams: wait for them
    before the backends' streams run the next phase."""
    try:
        import torch
        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except ImportError:  # host backends without torch's CUDA
        pass


# ------------------------------------------------------------ simulation
def shard_range(npart_global: int, rank: int, size: int):
    """Contiguous slice [a, b) of rank `rank`: the first npart % size ranks
    take one particle more."""
    base, extra = divmod(int(npart_global), size)
    a = rank * base + min(rank, extra)
    return a, a + base + (1 if rank < extra else 0)


class ShardedSimulation:
    """Simulation (src/simulation.jl:171-216, 472-531) of one rank's slice of
    the cloud, on this rank's GPU.

    sampling="slice": every rank draws the Ran2(seed) cloud in order and
    keeps its slice -- the single-GPU cloud exactly, at the cost of drawing
    the particles before the slice on every rank.  sampling="per-rank": rank
    r draws its own slice from Ran2(seed - r) -- the same distribution, drawn
    once.  Either way the draw is streamed (stream_chunk particles at a time,
    packed and uploaded chunk by chunk, the priming's second half chunked as
    well), so that a rank's host holds a few chunks and never its slice;
    stream_chunk = 0 draws the slice whole."""

    def __init__(self, p: S.SimulationParameters, profile: S.RadialProfile, *, comm, device: int = 0,
                 projectile: S.Projectile | None = None, seed: int = -1, fixed_point: bool = True,
                 precision: int = L.VLB_POISSON_FP32, sampling: str = "per-rank", capture_radius: float = 8.0,
                 stream_chunk: int = S.STREAM_CHUNK):
        self.params, self.comm, self.device = p, comm, device
        self.meshes = S.build_meshes(p.nfine, p.ninner, p.nouter, p.rcluster, p.rbox)
        self.smoothing = S.gaussian_smoothing(self.meshes.fine.axis)
        self.jellium = S.Jellium.of(p.nions)
        self.npart_global = int(p.nparticles)
        self.weight = p.nelectrons / p.nparticles
        self.projectile = projectile
        self.fixed_point, self.precision, self.capture_radius = fixed_point, precision, capture_radius
        a, b = shard_range(self.npart_global, comm.rank, comm.size)
        self.slice = (a, b)
        if sampling not in ("slice", "per-rank"):
            raise ValueError(f"unknown sampling {sampling!r}")
        self.accelerator = S.DeviceAccelerator(self.meshes, self.smoothing, b - a, self.weight, device)
        self.x0, self.h = self.accelerator.x0, self.accelerator.h
        self.stepper = ShardedStepper(LibraryShard(self.accelerator, self._deposit_mode(), device), comm,
                                      self.npart_global)
        if stream_chunk > 0:
            stream = S.ThomasFermiStream(profile, self.weight, seed=seed if sampling == "slice" else seed - comm.rank)
            lo, hi = (a, b) if sampling == "slice" else (0, b - a)
            try:
                S.stream_half_step_cloud(self.accelerator, stream, lo, hi, self.mass, p.dt, stream_chunk)
            finally:
                stream.close()
            self._prime_forces()
            S.prime_back_chunked(self.accelerator, self.mass, p.dt, False, stream_chunk)
        else:
            if sampling == "slice":
                pos, mom = S.sample_thomas_fermi(profile, self.npart_global, self.weight, seed=seed)
                pos, mom = pos[a:b].copy(), mom[a:b].copy()
            else:
                pos, mom = S.sample_thomas_fermi(profile, b - a, self.weight, seed=seed - comm.rank)
            self.prime_leapfrog(pos, mom)

    @property
    def mass(self):
        return S.ELECTRON_MASS * self.weight

    def _deposit_mode(self):
        return L.VLB_DEPOSIT_FIXED64 if self.fixed_point else L.VLB_DEPOSIT_FLOAT32

    def _params(self, *, advance: bool, push: bool, capture: float, energy: bool = False) -> L.StepParams:
        sp = L.StepParams()
        sp.dt = self.params.dt
        sp.rcmax = self.params.rcmax
        sp.jellium_nions = self.jellium.nions
        sp.jellium_radius = self.jellium.radius
        sp.capture_radius = capture
        sp.deposit_mode = self._deposit_mode()
        sp.advance_projectile = int(advance)
        sp.push = int(push)
        sp.use_graph = 0
        sp.poisson_precision = self.precision
        sp.energy = int(energy and push)
        return sp

    def prime_leapfrog(self, positions, momenta):
        """prime_leapfrog! (src/simulation.jl:233-277) with the forces of the
        whole cloud; the Fortran's dt/M coefficient."""
        M, dt = self.mass, self.params.dt
        half = positions - (dt / (2 * M)) * momenta
        k, d = S.pack_positions(half, self.x0, self.h)
        pk, pd = S.pack_positions(positions, self.x0, self.h)
        acc = self.accelerator
        acc.upload(k, d, pk, pd)
        self._prime_forces()
        k, d, pk, pd = acc.download()
        f = acc.force().astype(np.float64).T
        q0 = S.unpack_positions(pk, pd, self.x0, self.h)
        hp = S.unpack_positions(k, d, self.x0, self.h)
        back = -q0 + 2 * hp + (dt / M) * f
        k, d = S.pack_positions(q0, self.x0, self.h)
        pk, pd = S.pack_positions(back, self.x0, self.h)
        acc.upload(k, d, pk, pd)

    def _prime_forces(self):
        """The forces of the whole cloud at the half step back (a forces-only
        sharded step): with the projectile's reaction on the device path,
        without it on the CPU path (see Simulation._prime_forces)."""
        pr = self.projectile
        if pr is not None and pr.softening_mode == L.VLB_SOFTENING_BALL:
            pr = None
        self.stepper.step(pr, self._params(advance=False, push=False, capture=0.0))

    def step(self, energy: bool = False) -> ShardedDiagnostics:
        """With energy, the diagnostics carry the budget's two sums over the
        whole cloud (S.EnergyBudget.of(sim.jellium, d))."""
        return self.stepper.step(self.projectile,
                                 self._params(advance=True, push=True, capture=self.capture_radius, energy=energy))

    def close(self):
        self.accelerator.close()
