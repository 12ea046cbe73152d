"""Writes capture_host_1e5_ensemble.npz: the CPU path's capture curve on the
smallest crossing (the workload of make_capture_host.py) under perturbations
of the size a float32 device step makes, to measure how far the crossing's
chaos spreads two runs that differ only in rounding.

Members (each 700 steps of oracle.HostStep, primed by prime_leapfrog!):
  - "rounded": the float64 run with its positions and previous positions
    rounded to the packed float32 form (k, delta) after every step, as a
    device holds them;
  - "ulp1".."ulp5": the run from the packed cloud with every delta moved by
    one float32 ulp up or down (seeded choice per particle and axis);
  - "rounded_ulp": the per-step rounding started from the "ulp1" cloud.

Stored: q8[member] (700 steps each) and the member names.  The base curve is
q8 of capture_host_1e5.npz.  Run from the repository root (8 OpenMP threads,
about a minute a member):

    python tests/golden/make_capture_ensemble.py
"""
import sys
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
import make_capture_host as M  # noqa: E402


def run(vb, orc, p, meshes, sm, w, pos, mom, label, round_each_step, x0, h):
    jel = vb.Jellium.of(p.nions)
    proj = vb.xenon_projectile(v=0.40, impact=45.0, x0=-70.0, dt=M.DT)
    st = orc.HostStep(meshes, sm, w, jel, p.dt, p.rcmax, proj)
    pos, prev = st.prime(pos, mom)
    q = np.zeros(M.NSTEPS)
    t0 = time.time()
    for s in range(M.NSTEPS):
        pos, prev, _ = st.step(pos, prev)
        if round_each_step:
            k, d = vb.pack_positions(pos, x0, h)
            pos = np.ascontiguousarray(vb.unpack_positions(k, d, x0, h))
            k, d = vb.pack_positions(prev, x0, h)
            prev = np.ascontiguousarray(vb.unpack_positions(k, d, x0, h))
        q[s] = st.enclosed_charge(pos, 8.0)
    print(f"{label}: q(<8) at 350 / 700 = {q[349]:.4f} / {q[-1]:.4f} ({time.time() - t0:.0f} s)", flush=True)
    return q


def ulp_cloud(vb, pos, x0, h, seed):
    k, d = vb.pack_positions(pos, x0, h)
    rng = np.random.default_rng(seed)
    up = rng.integers(0, 2, size=d.shape).astype(bool)
    d2 = np.where(up, np.nextafter(d, np.float32(np.inf)), np.nextafter(d, np.float32(-np.inf))).astype(np.float32)
    return np.ascontiguousarray(vb.unpack_positions(k, d2, x0, h))


def main():
    vb, orc, p, meshes, sm, w, pos, mom = M.setup()
    kn = meshes.fine.axis.knots
    x0, h = float(kn[0]), float((kn[-1] - kn[0]) / (len(kn) - 1))
    names, curves = [], []
    names.append("rounded")
    curves.append(run(vb, orc, p, meshes, sm, w, pos.copy(), mom, "rounded", True, x0, h))
    for s in range(1, 6):
        names.append(f"ulp{s}")
        curves.append(run(vb, orc, p, meshes, sm, w, ulp_cloud(vb, pos, x0, h, s), mom, f"ulp{s}", False, x0, h))
    names.append("rounded_ulp")
    curves.append(run(vb, orc, p, meshes, sm, w, ulp_cloud(vb, pos, x0, h, 1), mom, "rounded_ulp", True, x0, h))
    dest = Path(__file__).resolve().parent / "capture_host_1e5_ensemble.npz"
    np.savez_compressed(dest, q8=np.array(curves), names=np.array(names))
    base = np.load(Path(__file__).resolve().parent / "capture_host_1e5.npz")["q8"]
    for nm, c in zip(names, curves):
        d = np.abs(c - base)
        print(f"{nm}: max |dq| to 400 {d[:400].max():.4f}, after {d[400:].max():.4f}, "
              f"rms after {np.sqrt(np.mean(d[400:] ** 2)):.4f}")
    print(f"wrote {dest}")


if __name__ == "__main__":
    main()
