"""The collision in its precision forms, at large size (8e7 pseudo-particles,
~11 GB of device state, 130^3 grids):

  plain        float32 deposits with float32 atomics, FP32 mode products
               (the reference's device arithmetic);
  fixed        int64 fixed-point deposits (fine and coarse, charge scaled by
               2^40) and reductions in a fixed order, run twice: the two runs
               must agree bit for bit (every step's scalars, the projectile,
               the final cloud);
  fixed-3xtf32 and fixed-bf16x3
               the same with the mode products on the tensor cores in the
               two split precisions.

Every capture curve q(<8 a0) is compared with the plain run's, and the
plain run is repeated to show the run-to-run spread its float32 atomics
leave (which the fixed-point form removes).  The field
errors of the three mode-product precisions against a float64 tensor solve
are measured by the GPU tests (tests/test_gpu_precision.py).

    python -c 'import __graft_entry__ as g; g.load().precision_run.main()' [--npart 80000000] [--json out.json]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import time

import numpy as np

from . import _lib as L
from . import denoiser as DN

FORMS = {
    "plain": (False, L.VLB_POISSON_FP32),
    "fixed": (True, L.VLB_POISSON_FP32),
    "fixed-3xtf32": (True, L.VLB_POISSON_3XTF32),
    "fixed-bf16x3": (True, L.VLB_POISSON_BF16X3),
}


def run_form(name: str, npart: int, nsteps: int, impact: float, seed: int, device: int = 0):
    """One run: per-step scalars, the projectile track, a digest of the final
    cloud, the wall time of the steps."""
    fixed, prec = FORMS[name]
    t0 = time.perf_counter()
    sim = DN.make_run(npart, impact, seed, device=device, precision=prec, fixed_point=fixed)
    built = time.perf_counter() - t0
    rec = {k: np.zeros(nsteps) for k in ("q8", "kinetic", "escaped", "xion")}
    outcount = np.zeros(nsteps, dtype=np.int64)
    wall = 0.0
    try:
        for s in range(nsteps):
            t = time.perf_counter()
            d = sim.step()
            wall += time.perf_counter() - t
            if d.status:
                raise RuntimeError(f"{name}: device status {d.status} at step {s + 1}")
            rec["q8"][s], rec["kinetic"][s], rec["escaped"][s] = d.enclosed_charge, d.kinetic, d.escaped
            rec["xion"][s] = sim.projectile.position[0]
            outcount[s] = d.outcount
        h = hashlib.sha256()
        for a in sim.accelerator.download():
            h.update(np.ascontiguousarray(a).tobytes())
        h.update(np.ascontiguousarray(sim.projectile.position).tobytes())
    finally:
        sim.accelerator.close()
    return {"name": name, "built_s": built, "wall_s": wall, "ms_per_step": 1000 * wall / nsteps,
            "digest": h.hexdigest(), "outcount": outcount, **rec}


def compare(a, b):
    dq = a["q8"] - b["q8"]
    return {"max_dq": float(np.max(np.abs(dq))), "rms_dq": float(np.sqrt(np.mean(dq * dq))),
            "final_dq": float(dq[-1])}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--npart", type=int, default=80_000_000)
    ap.add_argument("--steps", type=int, default=704)
    ap.add_argument("--impact", type=float, default=45.0)
    ap.add_argument("--seed", type=int, default=-1)
    ap.add_argument("--json", default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    runs = {}
    for name in ("plain", "fixed", "fixed-3xtf32", "fixed-bf16x3"):
        runs[name] = run_form(name, a.npart, a.steps, a.impact, a.seed, a.device)
        print(f"{name:14s} {a.steps} steps, {runs[name]['ms_per_step']:.2f} ms/step, "
              f"final q(<8) {runs[name]['q8'][-1]:.4f}", flush=True)
    again = run_form("fixed", a.npart, a.steps, a.impact, a.seed, a.device)
    plain2 = run_form("plain", a.npart, a.steps, a.impact, a.seed, a.device)
    f1 = runs["fixed"]
    same = {k: bool(np.array_equal(f1[k], again[k])) for k in ("q8", "kinetic", "escaped", "xion", "outcount")}
    same["final_cloud"] = f1["digest"] == again["digest"]
    print(f"fixed point, two runs bit-identical: {same}", flush=True)
    spread = compare(plain2, runs["plain"])
    spread["final_cloud_identical"] = plain2["digest"] == runs["plain"]["digest"]
    print(f"plain, two runs: max |dq| {spread['max_dq']:.4f}, rms {spread['rms_dq']:.4f}, "
          f"final cloud identical {spread['final_cloud_identical']}", flush=True)
    out = {"npart": a.npart, "steps": a.steps, "impact": a.impact, "seed": a.seed, "bit_identical": same,
           "plain_run_to_run": spread, "forms": {}}
    for name, r in runs.items():
        entry = {"ms_per_step": r["ms_per_step"], "built_s": r["built_s"], "final_q8": float(r["q8"][-1]),
                 "final_outcount": int(r["outcount"][-1]), "q8": r["q8"].tolist()}
        if name != "plain":
            entry["vs_plain"] = compare(r, runs["plain"])
            print(f"{name:14s} vs plain: max |dq| {entry['vs_plain']['max_dq']:.4f}, rms "
                  f"{entry['vs_plain']['rms_dq']:.4f}, final {entry['vs_plain']['final_dq']:+.4f}", flush=True)
        out["forms"][name] = entry
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f)
    return out


if __name__ == "__main__":
    main()
