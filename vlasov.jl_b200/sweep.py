"""A sweep of collisions advanced together on one GPU.

Each collision is a run of its own (its cloud, its seed, its projectile, its
library context); vlb_batch_step advances all of them by one step, each on
its own stream, the whole batch step captured once as one CUDA graph.  The
clouds can be of very different sizes: while the large runs' kernels fill
the GPU, the small runs' kernels run beside them instead of leaving SMs idle
between dependent launches.  Launch shapes can be tuned per run
(vlasov_b200.autotune).

The reference runs one collision per process (scripts/xenon.jl); the sweep
below (Xe25+ 500 keV at five impact parameters, Ar8+ 100 keV, protons at
100 keV) is the batch workload, on 98^3 grids.

    python -c 'import __graft_entry__ as g; g.load().sweep.main()' --steps 700 [--tune] [--scale 0.1]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import sys
import time
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import simulation as S

AMU = 1836.154               # mass unit of the reference's projectiles (scripts/xenon.jl:337)
HARTREE_KEV = 0.0272113862   # keV per hartree


@dataclass
class Collision:
    name: str
    charge: float
    mass_amu: float
    impact: float
    npart: int
    seed: int
    v: float | None = None             # a.u.; or
    energy_kev: float | None = None

    def projectile(self, x0: float = -70.0, dt: float = 0.5) -> S.Projectile:
        mass = self.mass_amu * AMU
        energy = 0.5 * mass * self.v ** 2 if self.v is not None else self.energy_kev / HARTREE_KEV
        return S.Projectile.make(mass=mass, charge=self.charge, energy=energy, impact=self.impact, x0=x0, dt=dt,
                                 softening=S.BallSoftening(5.0))


# Xe25+ at the reference's v = 0.40 (500 keV); Ar8+ and protons from their energies.
SWEEP = [
    Collision("Xe25+ b=0", 25.0, 131.3, 0.0, 1_000_000, -1, v=0.40),
    Collision("Xe25+ b=15", 25.0, 131.3, 15.0, 2_000_000, -2, v=0.40),
    Collision("Xe25+ b=30", 25.0, 131.3, 30.0, 4_000_000, -3, v=0.40),
    Collision("Xe25+ b=45", 25.0, 131.3, 45.0, 8_000_000, -4, v=0.40),
    Collision("Xe25+ b=60", 25.0, 131.3, 60.0, 8_000_000, -5, v=0.40),
    Collision("Ar8+ b=30", 8.0, 40.0, 30.0, 3_000_000, -6, energy_kev=100.0),
    Collision("p b=0", 1.0, 1.0, 0.0, 500_000, -7, energy_kev=100.0),
    Collision("p b=30", 1.0, 1.0, 30.0, 500_000, -8, energy_kev=100.0),
]


def build(collisions, *, nfine: int = 48, device: int = 0, scale: float = 1.0, fixed_point: bool = False,
          precision: int = L.VLB_POISSON_3XTF32, profile=None):
    """One primed Simulation per collision (particle counts times `scale`)."""
    prof = S.thomas_fermi_profile() if profile is None else profile
    sims = []
    for c in collisions:
        n = max(1000, int(round(c.npart * scale)))
        p = S.SimulationParameters.for_grid(nfine, rcluster=78.0, rbox=235.0, nparticles=n, dt=0.5)
        sims.append(S.Simulation(p, prof, projectile=c.projectile(), seed=c.seed, device=device,
                                 fixed_point=fixed_point, precision=precision))
    return sims


class Batch:
    """vlb_batch over the contexts of several Simulations (one device)."""

    def __init__(self, sims):
        self.sims = list(sims)
        n = len(self.sims)
        handles = (C.c_void_p * n)(*[s.accelerator.handle.value for s in self.sims])
        self._h = C.c_void_p()
        L.check(L.lib().vlb_batch_create(handles, n, C.byref(self._h)))

    def step(self, *, capture: float = 8.0, use_graph: bool = True):
        sims = self.sims
        n = len(sims)
        params = sims[0]._params(advance=True, push=True, capture=capture)
        params.use_graph = int(use_graph)
        projs = (L.ProjectileDesc * n)(*[s.projectile.to_desc() for s in sims])
        res = (L.StepResult * n)()
        L.check(L.lib().vlb_batch_step(self._h, projs, C.byref(params), res))
        out = []
        for i, s in enumerate(sims):
            s.projectile.from_desc(projs[i])
            s.steps_done += 1
            r = res[i]
            out.append(S.StepDiagnostics(r.kinetic, r.escaped, tuple(r.angular), r.enclosed_charge, r.nout,
                                         r.outcount, r.noccupied, tuple(r.projectile_force), r.total_charge,
                                         r.status, r.denoised, r.hartree, r.interaction, r.sort_path))
        return out

    def close(self):
        if self._h:
            L.lib().vlb_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_batch(sims, nsteps: int, *, use_graph: bool = True):
    """All runs together, nsteps batch steps; the capture curves and the
    wall time (every step returns its scalars, as a run does)."""
    b = Batch(sims)
    q = np.zeros((len(sims), nsteps))
    try:
        t0 = time.perf_counter()
        for s in range(nsteps):
            for i, d in enumerate(b.step(use_graph=use_graph)):
                if d.status:
                    raise RuntimeError(f"device status {d.status} in run {i} at step {s + 1}")
                q[i, s] = d.enclosed_charge
        wall = time.perf_counter() - t0
    finally:
        b.close()
    return {"q8": q, "wall_s": wall}


def run_sequential(sims, nsteps: int):
    """Each run alone, one after the other (its own captured step)."""
    q = np.zeros((len(sims), nsteps))
    walls = []
    for i, sim in enumerate(sims):
        t0 = time.perf_counter()
        for s in range(nsteps):
            d = sim.step()
            if d.status:
                raise RuntimeError(f"device status {d.status} in run {i} at step {s + 1}")
            q[i, s] = d.enclosed_charge
        walls.append(time.perf_counter() - t0)
    return {"q8": q, "wall_s": sum(walls), "wall_per_run_s": walls}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--steps", type=int, default=700)
    ap.add_argument("--nfine", type=int, default=48)
    ap.add_argument("--scale", type=float, default=1.0, help="multiply every particle count")
    ap.add_argument("--tune", action="store_true", help="autotune each run's launch shapes first")
    ap.add_argument("--cache", default=None, help="JSON cache of tuned shapes")
    ap.add_argument("--sequential", action="store_true", help="also time the runs one after another")
    ap.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    from . import autotune
    sims = build(SWEEP, nfine=a.nfine, scale=a.scale)
    total = sum(s.params.nparticles for s in sims)
    tuning = {}
    if a.tune:
        for c, s in zip(SWEEP, sims):
            tuning[c.name] = autotune.tune_cached(s, a.cache)
    snaps = [s.snapshot() for s in sims]
    out = {"collisions": [c.name for c in SWEEP], "npart": [s.params.nparticles for s in sims],
           "nfine": a.nfine, "steps": a.steps, "tuning": tuning}
    r = run_batch(sims, a.steps)
    out["batch_wall_s"] = r["wall_s"]
    out["batch_particle_steps_per_s"] = total * a.steps / r["wall_s"]
    out["batch_final_q8"] = r["q8"][:, -1].tolist()
    print(f"batch of {len(sims)} runs, {total:.3g} particles: {1000 * r['wall_s'] / a.steps:.2f} ms per step, "
          f"{out['batch_particle_steps_per_s']:.3g} particle-steps/s")
    if a.sequential:
        for s, snap in zip(sims, snaps):
            s.restore(snap)
        r2 = run_sequential(sims, a.steps)
        out["sequential_wall_s"] = r2["wall_s"]
        out["sequential_particle_steps_per_s"] = total * a.steps / r2["wall_s"]
        out["sequential_final_q8"] = r2["q8"][:, -1].tolist()
        out["speedup"] = r2["wall_s"] / r["wall_s"]
        print(f"one after another: {1000 * r2['wall_s'] / a.steps:.2f} ms per step of all runs, "
              f"{out['sequential_particle_steps_per_s']:.3g} particle-steps/s; batch speed-up {out['speedup']:.2f}")
    for name, q in zip(out["collisions"], out["batch_final_q8"]):
        print(f"  {name:12s} q(<8 a0) after {a.steps} steps: {q:.3f}")
    for s in sims:
        s.accelerator.close()
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f)
    return out


if __name__ == "__main__":
    main()
