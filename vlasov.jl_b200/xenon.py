"""The Na196 + Xe25+ collision of scripts/xenon.jl, run on the B200 library.

Same setup as the reference's script (scripts/xenon.jl:293-420): Na196 cluster
sampled from the Thomas-Fermi profile with Ran2(-1), rcluster = 78, rbox = 235,
dt = 0.5, Xe25+ of mass 131.3*1836.154 at v = 0.40 from x = -70 with b = 45
and a ball softening of radius 5, ceil(140 / (v dt)) = 700 steps.  It prints
the reference's table -- q(<8 a0) and the out-of-stencil count every 50 steps
-- and the charge carried away.  With --film N the movie's frames (the
density slice at z = 0 and the capture scalars, scripts/xenon.jl:370-410) are
taken on the device and written as arrays; rendering them (GLMakie/Cairo in
the reference) is not done here.

    python -c 'import __graft_entry__ as g; g.load().xenon.main()' --particules 8000000 --nfine 64

(from the repository root; the package directory is imported as vlasov_b200).
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time


def run(npart: int = 8_000_000, nfine: int = 64, *, every: int = 50, fixed_point: bool = False,
        uniform: bool = False, nsteps: int | None = None, device: int = 0, seed: int = -1, quiet: bool = False,
        precision: str = "fp32", energy_every: int = 0, isolated: bool = False, film_stride: int = 0,
        film_out: str | None = None, softening: str = "device"):
    """Runs the crossing; returns a dict with the capture curve (q(<8) and
    outcount after every step), the final charge and the timing, and with
    energy_every > 0 the energy budget of every energy_every-th step
    (run!(sim; energy_every), src/simulation.jl:419-440).  isolated: the
    cluster alone, no projectile (the budget's conservation test).
    film_stride > 0: the movie's frames (scripts/xenon.jl:370-410) at step 1
    and every film_stride-th step, taken on the device and written to
    film_out (.npz: frames, times_fs, proj_x, proj_y, q_capture, q_net).
    softening: "device" (the reference's device path: a Gaussian of width 5
    for stencil particles, the ball for the rest) or "ball" (its CPU path:
    the ball of radius 5 for every particle)."""
    import numpy as np
    from . import simulation as S

    dt, v, x0 = 0.5, 0.40, -70.0
    total = math.ceil((abs(x0) + 70.0) / (v * dt))
    nsteps = total if nsteps is None else nsteps
    p = S.SimulationParameters.for_grid(nfine, rcluster=78.0, rbox=235.0, nparticles=npart, dt=dt)
    prof = S.uniform_sphere_profile() if uniform else S.thomas_fermi_profile()
    t0 = time.time()
    from . import _lib as L
    prec = {"fp32": L.VLB_POISSON_FP32, "3xtf32": L.VLB_POISSON_3XTF32, "bf16x3": L.VLB_POISSON_BF16X3}[precision]
    proj = None if isolated else S.xenon_projectile(v=v, x0=x0, dt=dt)
    soft = {"device": L.VLB_SOFTENING_DEVICE, "ball": L.VLB_SOFTENING_BALL}[softening]
    sim = S.Simulation(p, prof, projectile=proj, seed=seed, fixed_point=fixed_point, device=device,
                       precision=prec, softening_mode=soft)
    built = time.time() - t0
    if not quiet:
        print(f"Na196 + Xe25+, 500 keV, b = 45 a0 | {npart:.1e} particles, grid {2 * nfine + 2}^3")
        print(f"built in {built:.1f} s\n")
        print("   step     t (fs)    x_ion (a0)   q(<8 a0)        out    ms/step")
        sys.stdout.flush()
    fs = 41.341373335  # atomic units of time per femtosecond
    q, out, xs = np.zeros(nsteps), np.zeros(nsteps, dtype=np.int64), np.zeros(nsteps)
    budgets = []
    acc = sim.accelerator
    film_steps = []
    if film_stride > 0:
        sim.film(1 + nsteps // film_stride)
    t_run = time.time()
    tprev = t_run
    for s in range(1, nsteps + 1):
        energy = energy_every > 0 and (s - 1) % energy_every == 0
        frame = film_stride > 0 and (s % film_stride == 0 or s == 1)
        d = sim.step(energy=energy, film=frame)
        if frame:
            film_steps.append(s)
        if energy:
            b = sim.energy_budget(d)
            budgets.append({"step": s, "total": b.total, "kinetic": b.kinetic, "hartree": b.hartree,
                            "meanfield": b.meanfield, "ions": b.ions, "escaped": b.escaped,
                            "ion_energy_loss": sim.projectile.energy_loss() if sim.projectile else 0.0})
        q[s - 1] = d.enclosed_charge
        out[s - 1] = d.outcount
        xs[s - 1] = sim.projectile.position[0] if sim.projectile else 0.0
        if not quiet and (s % every == 0 or s == nsteps):
            now = time.time()
            print(f"{s:7d} {s * dt / fs:10.2f} {xs[s - 1]:12.1f} {d.enclosed_charge:10.3f} "
                  f"{d.outcount:10d} {1000 * (now - tprev) / every:10.1f}")
            sys.stdout.flush()
            tprev = now
        if d.status != 0:
            raise RuntimeError(f"device status {d.status} at step {s}")
    elapsed = time.time() - t_run
    film = None
    if film_stride > 0:
        f = sim.film_frames()
        film = {"frames": len(f.frames), "q_net_final": float(f.q_net[-1]) if len(f.q_net) else None}
        if film_out:
            np.savez(film_out, frames=f.frames, times_fs=np.array(film_steps) * dt / fs, proj_x=f.proj_x,
                     proj_y=f.proj_y, q_capture=f.q_capture, q_net=f.q_net)
    acc.close()
    if not quiet:
        print(f"\n{nsteps} steps in {elapsed:.1f} s -- {1000 * elapsed / nsteps:.2f} ms/step (wall clock, "
              f"including the per-step read of the step's scalars)")
        print(f"charge carried away by the ion: {q[-1]:.3f} electrons")
    return {"npart": npart, "nfine": nfine, "nsteps": nsteps, "q8": q.tolist(), "outcount": out.tolist(),
            "x_ion": xs.tolist(), "final_q8": float(q[-1]), "final_outcount": int(out[-1]),
            "wall_s": elapsed, "built_s": built, "fixed_point": fixed_point, "uniform": uniform,
            "precision": precision, "energy": budgets, "film": film}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--particules", type=int, default=8_000_000)
    ap.add_argument("--nfine", type=int, default=64)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--fixed-point", action="store_true")
    ap.add_argument("--uniform", action="store_true", help="uniform-sphere cloud instead of Thomas-Fermi")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "3xtf32", "bf16x3"],
                    help="mode products on the CUDA cores or split-precision on the tensor cores")
    ap.add_argument("--energy-every", type=int, default=0, help="energy budget every N steps (0: none)")
    ap.add_argument("--isolated", action="store_true", help="the cluster alone, without the projectile")
    ap.add_argument("--json", default=None, help="write the capture curve here")
    ap.add_argument("--film", type=int, default=0,
                    help="take the movie's frames at step 1 and every N steps on the device (the script's N is 4)")
    ap.add_argument("--film-out", default="film.npz", help="where --film writes its frames")
    ap.add_argument("--softening", default="device", choices=["device", "ball"],
                    help="the reference's device path (Gaussian in the stencil) or its CPU path (the ball everywhere)")
    a = ap.parse_args(argv)
    if a.nfine % 2:
        ap.error("--nfine must be even")
    r = run(a.particules, a.nfine, fixed_point=a.fixed_point, uniform=a.uniform, nsteps=a.steps,
            precision=a.precision, energy_every=a.energy_every, isolated=a.isolated, film_stride=a.film,
            film_out=a.film_out if a.film else None, softening=a.softening)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(r, f)


if __name__ == "__main__":
    main()
