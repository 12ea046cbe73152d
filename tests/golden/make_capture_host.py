"""Writes capture_host_1e5.npz: the capture curve of the reference's CPU path
on the smallest crossing, the float64 restatement of update_forces! and
step! (src/simulation.jl:309-352, 382-396; oracle.HostStep) run with the
priming of prime_leapfrog! (src/simulation.jl:233-277).

Workload: Na196 Thomas-Fermi cloud of 1e5 pseudo-particles sampled with
Ran2(-1), nfine = 28 (58^3 collocation points), rcluster = 78, rbox = 235,
dt = 0.5; Xe25+ (mass 131.3 * 1836.154, v = 0.40) from x = -70 at b = 45 with
BallSoftening(5) for every particle (the CPU path's projectile_forces!,
src/projectile.jl:203-232); 700 steps.

Stored after every step: q(<8 a0) around the projectile, the particles whose
10^3 stencil leaves the fine grid (the device path's outcount criterion,
applied to the packed positions), the host path's margin count
(src/fields.jl:498-507) and the projectile's x.  A second run starts from the
same cloud rounded to the packed float32 form (k, delta) that the device
holds: the spread between the two curves is the crossing's own sensitivity
to a float32 rounding of its initial state.

Both runs use 8 OpenMP threads of the oracle.  Run from the repository root:

    python tests/golden/make_capture_host.py
"""
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

NPART, NFINE, NSTEPS, DT = 100_000, 28, 700, 0.5


def setup():
    from __graft_entry__ import load
    vb = load()
    from oracle import oracle as orc
    orc.lib().orc_set_threads(8)
    p = vb.SimulationParameters.for_grid(NFINE, rcluster=78.0, rbox=235.0, nparticles=NPART, dt=DT)
    meshes = vb.build_meshes(p.nfine, p.ninner, p.nouter, p.rcluster, p.rbox)
    sm = vb.gaussian_smoothing(meshes.fine.axis)
    w = p.nelectrons / p.nparticles
    pos, mom = vb.sample_thomas_fermi(vb.thomas_fermi_profile(), p.nparticles, w, seed=-1)
    return vb, orc, p, meshes, sm, w, pos, mom


def stencil_out(vb, pos, x0, h, nk, n):
    """Particles whose 10^3 stencil leaves the fine grid (the clamped cell's
    base 2k - 5 outside [1, n - 9], src/kernels.jl:1041-1058)."""
    k, _ = vb.pack_positions(pos, x0, h)
    kc = np.clip(k, 1, nk)
    b = 2 * kc - 5
    fits = np.all((b >= 1) & (b + 9 <= n), axis=0)
    return int(np.count_nonzero(~fits))


def run(vb, orc, p, meshes, sm, w, pos, mom, label):
    jel = vb.Jellium.of(p.nions)
    proj = vb.xenon_projectile(v=0.40, impact=45.0, x0=-70.0, dt=DT)
    st = orc.HostStep(meshes, sm, w, jel, p.dt, p.rcmax, proj)
    kn = meshes.fine.axis.knots
    x0, h, nk, n = float(kn[0]), float((kn[-1] - kn[0]) / (len(kn) - 1)), len(kn), meshes.fine.axis.nbasis
    pos, prev = st.prime(pos, mom)  # a copy of pos: the steps advance it in place
    q = np.zeros(NSTEPS)
    out = np.zeros(NSTEPS, np.int64)
    margin = np.zeros(NSTEPS, np.int64)
    xion = np.zeros(NSTEPS)
    t0 = time.time()
    for s in range(NSTEPS):
        pos, prev, _ = st.step(pos, prev)
        q[s] = st.enclosed_charge(pos, 8.0)
        out[s] = stencil_out(vb, pos, x0, h, nk, n)
        margin[s] = st.noutf
        xion[s] = proj.position[0]
        if (s + 1) % 100 == 0:
            print(f"{label}: step {s + 1}  q(<8) {q[s]:.4f}  out {out[s]}  x {xion[s]:.2f}  "
                  f"({time.time() - t0:.0f} s)", flush=True)
    return q, out, margin, xion


def main():
    vb, orc, p, meshes, sm, w, pos, mom = setup()
    q, out, margin, xion = run(vb, orc, p, meshes, sm, w, pos, mom, "float64 cloud")
    kn = meshes.fine.axis.knots
    x0, h = float(kn[0]), float((kn[-1] - kn[0]) / (len(kn) - 1))
    k, d = vb.pack_positions(pos, x0, h)
    pos32 = vb.unpack_positions(k, d, x0, h)
    q2, out2, margin2, xion2 = run(vb, orc, p, meshes, sm, w, pos32, mom, "packed cloud")
    dest = Path(__file__).resolve().parent / "capture_host_1e5.npz"
    np.savez_compressed(dest, q8=q, outcount=out, margin_out=margin, x_ion=xion,
                        q8_packed=q2, outcount_packed=out2, weight=w, nsteps=NSTEPS)
    print(f"wrote {dest}: q(<8) at step 350 / 700 = {q[349]:.4f} / {q[-1]:.4f}, out {out[349]} / {out[-1]}; "
          f"packed start: {q2[349]:.4f} / {q2[-1]:.4f}; max |dq| between the two = {np.max(np.abs(q - q2)):.4f}")


if __name__ == "__main__":
    main()
