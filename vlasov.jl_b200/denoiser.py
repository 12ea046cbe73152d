"""The learned denoiser of the fine density.

A run of N pseudo-particles deposits a density whose sampling noise falls as
1/sqrt(N); the denoiser maps the deposit of an 8e6-particle run to what a run
with ten times the particles deposits at the same instant, so that 8e6
particles give the fields of 8e7.  It is a small 3-D convolutional network
(four 3^3 layers, 1-16-16-16-3 channels, ReLU, no biases, BF16 weights,
float32 arithmetic) whose three outputs are a charge flux: the density it
returns is rho + div F / s, charge moved between neighbouring voxels and
none added.

Everything runs on the GPU through the library's own kernels:

  * training pairs come from the method itself: seeded runs of the same
    collision at 8e6 and 8e7 particles, their fine densities taken every
    4 steps (collect());
  * the network is trained by vlb_dn_gradient (forward and backward passes)
    and vlb_dn_adam (train());
  * in the step (attach()), vlb_set_denoiser puts it after the fine deposit;
    the step keeps the deposit instead whenever the prediction's charge
    differs from the deposit's by more than the tolerance (1e-3 e).

The reference has no counterpart (it solves with the deposited density as
it is, deposit_smoothed! at src/accelerator.jl:531).

    python -c 'import __graft_entry__ as g; g.load().denoiser.main()' train --out weights.npz
    python -c 'import __graft_entry__ as g; g.load().denoiser.main()' evaluate --weights weights.npz
    python -c 'import __graft_entry__ as g; g.load().denoiser.main()' profile
    python -c 'import __graft_entry__ as g; g.load().denoiser.main()' floor --json floor.json
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time
from pathlib import Path

import numpy as np

from . import _lib as L
from . import simulation as S
from . import tables as T

LAYERS = ((1, 16), (16, 16), (16, 16), (16, 3))
WEIGHT_COUNT = sum(27 * a * b for a, b in LAYERS)        # 15,552
CHARGE_TOLERANCE = 1e-3                                  # electrons
DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "denoiser_xe25_130.npz"


def init_weights(seed: int = 0, flux_gain: float = 0.0) -> np.ndarray:
    """He-normal weights (fan-in 27 cin), the flux layer scaled by
    `flux_gain`: at 0 the untrained network is the identity (no flux)."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (a, b) in enumerate(LAYERS):
        std = math.sqrt(2.0 / (27 * a)) * (flux_gain if l == 3 else 1.0)
        parts.append(rng.standard_normal(27 * a * b) * std)
    return np.concatenate(parts).astype(np.float32)


def bf16_round(w: np.ndarray) -> np.ndarray:
    """The BF16 values the kernels use (nearest, ties to even), as float32."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def save_weights(path, weights: np.ndarray, scale: float, meta: dict | None = None):
    np.savez(path, weights=bf16_round(weights), scale=np.float64(scale),
             meta=np.array(json.dumps(meta or {})))


def load_weights(path=None):
    """(weights float32, input scale, metadata) of a saved network."""
    z = np.load(DEFAULT_WEIGHTS if path is None else path)
    return z["weights"].astype(np.float32), float(z["scale"]), json.loads(str(z["meta"]))


def _ptr(t) -> int:
    return t.data_ptr()


class Network:
    """The network's device workspaces over one nz x ny x nx volume
    (vlb_dn_create).  Tensors are float32 CUDA tensors on the same device;
    the kernels run on torch's current stream."""

    def __init__(self, shape, device: int = 0):
        import torch
        self.torch = torch
        self.shape = tuple(int(n) for n in shape)
        self.device = int(device)
        nz, ny, nx = self.shape
        h = C.c_void_p()
        L.check(L.lib().vlb_dn_create(nx, ny, nz, self.device, C.byref(h)))
        self._h = h

    def _stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def _check(self, *ts):
        for t in ts:
            if t.dtype != self.torch.float32 or not t.is_cuda or not t.is_contiguous():
                raise ValueError("denoiser tensors are contiguous float32 CUDA tensors")

    def forward(self, x, weights, scale: float, out=None):
        """x + div f(scale x) / scale."""
        out = self.torch.empty_like(x) if out is None else out
        self._check(x, weights, out)
        L.check(L.lib().vlb_dn_forward(self._h, _ptr(x), float(scale), _ptr(weights), _ptr(out), self._stream()))
        return out

    def gradient(self, x, target, weights, scale: float, grad, want_loss: bool = False):
        """grad = d loss / d weights; returns the loss (a sync) when asked."""
        self._check(x, target, weights, grad)
        loss = C.c_double(float("nan"))
        L.check(L.lib().vlb_dn_gradient(self._h, _ptr(x), _ptr(target), float(scale), _ptr(weights), _ptr(grad),
                                        C.byref(loss) if want_loss else None, self._stream()))
        return loss.value if want_loss else None

    def adam(self, weights, grad, m, v, lr: float, step: int):
        self._check(weights, grad, m, v)
        L.check(L.lib().vlb_dn_adam(self._h, _ptr(weights), _ptr(grad), _ptr(m), _ptr(v), float(lr), int(step),
                                    self._stream()))

    def status(self) -> int:
        """Device flags raised since the last call (VLB_STATUS_*); synchronises."""
        f = C.c_int32()
        L.check(L.lib().vlb_dn_status(self._h, C.byref(f)))
        return f.value

    def active_tiles(self) -> int:
        n = C.c_int32()
        L.check(L.lib().vlb_dn_active_tiles(self._h, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().vlb_dn_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------- in the step
def attach(sim, weights=None, scale: float | None = None, tolerance: float = CHARGE_TOLERANCE):
    """Puts the network after the fine deposit of `sim`'s steps."""
    if weights is None:
        weights, scale, _ = load_weights()
    w = np.ascontiguousarray(weights, dtype=np.float32)
    L.check(L.lib().vlb_set_denoiser(sim.accelerator.handle, L.pf(w), len(w), float(scale), float(tolerance)))
    sim.denoise = True


def detach(sim):
    L.check(L.lib().vlb_clear_denoiser(sim.accelerator.handle))
    sim.denoise = False


# ------------------------------------------------------------ the data
def make_run(npart: int, impact: float, seed: int, *, nfine: int = 64, device: int = 0,
             precision: int = L.VLB_POISSON_3XTF32, fixed_point: bool = False):
    """A primed run of the Xe25+ 500 keV collision (the headline workload's
    grids and projectile, impact parameter `impact`); the priming step uses
    the run's own deposit."""
    ninner, nouter = T.grids(nfine)
    p = S.SimulationParameters(nfine=nfine, ninner=ninner, nouter=nouter, rcluster=78.0, rbox=235.0, nions=196.0,
                               nelectrons=196.0, nparticles=int(npart), nsteps=0, dt=0.5)
    proj = S.xenon_projectile(v=0.40, impact=impact, x0=-70.0, dt=0.5)
    return S.Simulation(p, S.thomas_fermi_profile(), projectile=proj, seed=seed, device=device,
                        precision=precision, fixed_point=fixed_point)


def collect(sim, nsteps: int, every: int = 4):
    """Runs `sim` for nsteps; the fine density of every `every`-th step (as
    the step's fields saw it) into a float32 CUDA tensor [snapshots, n, n, n],
    and the capture curve q(<8 a0)."""
    import torch
    dev = torch.device("cuda", sim.accelerator.device)
    n = sim.accelerator.nf
    snaps = torch.empty((nsteps // every, n, n, n), dtype=torch.float32, device=dev)
    q = np.zeros(nsteps)
    for s in range(1, nsteps + 1):
        d = sim.step()
        if d.status:
            raise RuntimeError(f"device status {d.status} at step {s}")
        q[s - 1] = d.enclosed_charge
        if s % every == 0:
            snaps[s // every - 1].copy_(torch.from_numpy(sim.accelerator.grid(L.VLB_GRID_RHO_FINE)))
    return snaps, q


def input_scale(x) -> float:
    """1 / the mean of the nonzero voxels of x (the network is positively
    homogeneous: the scale sets the loss's units, not the function)."""
    nz = x[x > 0]
    return float(1.0 / nz.double().mean().item())


# ------------------------------------------------------------ training
def train(inputs, targets, *, steps: int = 3000, batch: int = 4, lr: float = 1e-3, warmup: int = 100,
          seed: int = 0, scale: float | None = None, log_every: int = 100, weights=None, log=print,
          time_limit: float | None = None, val_inputs=None, val_targets=None):
    """Adam on the mean squared error of the network's density against the
    targets, pairs drawn at random, linear warm-up then cosine decay of the
    learning rate; on the GPU with vlb_dn_gradient / vlb_dn_adam.  With a
    validation set, the weights of the lowest validation loss (checked every
    `log_every` steps) are returned.  Stops early after `time_limit` seconds.
    Returns (weights, scale, history of (step, train loss, val loss, s))."""
    import torch
    dev = inputs.device
    scale = input_scale(inputs) if scale is None else scale
    net = Network(inputs.shape[1:], dev.index or 0)
    w0 = init_weights(seed) if weights is None else np.asarray(weights, np.float32)
    w = torch.from_numpy(w0.copy()).to(dev)
    m, v, g, gs = (torch.zeros_like(w) for _ in range(4))
    rng = np.random.default_rng(seed)
    hist = []
    best = (math.inf, w.clone())

    def val_loss():
        if val_inputs is None:
            return float("nan")
        return float(np.mean([net.gradient(x, t, w, scale, g, want_loss=True)
                              for x, t in zip(val_inputs, val_targets)]))

    t0 = time.perf_counter()
    try:
        for it in range(1, steps + 1):
            gs.zero_()
            want = it % log_every == 0 or it == 1
            losses = []
            for _ in range(batch):
                p = int(rng.integers(len(inputs)))
                losses.append(net.gradient(inputs[p], targets[p], w, scale, g, want_loss=want))
                gs.add_(g)
            gs.div_(batch)
            ramp = min(1.0, it / warmup) if warmup > 0 else 1.0
            lr_t = lr * ramp * 0.5 * (1.0 + math.cos(math.pi * (it - 1) / steps))
            net.adam(w, gs, m, v, lr_t, it)
            if want or it == steps:
                vl = val_loss()
                if vl < best[0]:
                    best = (vl, w.clone())
                hist.append((it, float(np.nanmean([x for x in losses if x is not None] or [np.nan])), vl,
                             time.perf_counter() - t0))
                if log:
                    log(f"step {it:5d}  loss {hist[-1][1]:.4e}  val {vl:.4e}  lr {lr_t:.2e}  {hist[-1][3]:.1f} s")
                if time_limit is not None and hist[-1][3] > time_limit:
                    if log:
                        log(f"stopped at step {it}: time limit")
                    break
        torch.cuda.synchronize(dev)
    finally:
        net.close()
    wf = best[1] if val_inputs is not None and math.isfinite(best[0]) else w
    return wf.cpu().numpy(), scale, hist


def errors(inputs, targets, weights, scale: float):
    """Relative L2 errors against the targets of the deposits as they are
    and of the network's densities, one per pair."""
    import torch
    dev = inputs.device
    net = Network(inputs.shape[1:], dev.index or 0)
    w = torch.from_numpy(np.asarray(weights, np.float32)).to(dev)
    out = torch.empty_like(inputs[0])
    plain, learned = [], []
    try:
        for x, t in zip(inputs, targets):
            net.forward(x, w, scale, out)
            tn = torch.linalg.vector_norm(t.double())
            plain.append(float(torch.linalg.vector_norm((x - t).double()) / tn))
            learned.append(float(torch.linalg.vector_norm((out - t).double()) / tn))
    finally:
        net.close()
    return np.array(plain), np.array(learned)


# ------------------------------------------------------------ the CLI
TRAIN_IMPACTS = (30.0, 60.0)
LOW, HIGH = 8_000_000, 80_000_000


def _collect_pairs(impacts, nsteps, every, low, high, device, log):
    xs, ts = [], []
    for b in impacts:
        for npart, seed, dst in ((low, -11, xs), (high, -12, ts)):
            t0 = time.perf_counter()
            sim = make_run(npart, b, seed, device=device)
            snaps, _ = collect(sim, nsteps, every)
            sim.accelerator.close()
            dst.append(snaps)
            log(f"b={b:g} npart={npart:.0e}: {len(snaps)} snapshots in {time.perf_counter() - t0:.1f} s")
    import torch
    return torch.cat(xs), torch.cat(ts)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("command", choices=["train", "evaluate", "profile", "floor"])
    ap.add_argument("--steps", type=int, default=704, help="steps of each data run")
    ap.add_argument("--every", type=int, default=4)
    ap.add_argument("--low", type=int, default=LOW)
    ap.add_argument("--high", type=int, default=HIGH)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--time-limit", type=float, default=None, help="seconds of training at most")
    ap.add_argument("--weights", default=None, help="saved network (evaluate)")
    ap.add_argument("--out", default=None, help="where train saves the network")
    ap.add_argument("--impact", type=float, default=45.0, help="impact parameter of the evaluation run")
    ap.add_argument("--json", default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    log = lambda m: print(m, flush=True)  # noqa: E731
    out = {"command": a.command}
    if a.command == "train":
        xs, ts = _collect_pairs(TRAIN_IMPACTS, a.steps, a.every, a.low, a.high, a.device, log)
        # every 8th pair is kept aside for validation
        import torch
        val = torch.arange(len(xs), device=xs.device) % 8 == 7
        w, scale, hist = train(xs[~val], ts[~val], steps=a.train_steps, batch=a.batch, lr=a.lr, log=log,
                               time_limit=a.time_limit, val_inputs=xs[val], val_targets=ts[val])
        plain, learned = errors(xs[~val], ts[~val], w, scale)
        vplain, vlearned = errors(xs[val], ts[val], w, scale)
        out.update(pairs=len(xs), scale=scale, history=hist, train_err_plain=float(plain.mean()),
                   train_err_learned=float(learned.mean()), val_err_plain=float(vplain.mean()),
                   val_err_learned=float(vlearned.mean()))
        log(f"training pairs: relative L2 error {plain.mean():.4f} plain, {learned.mean():.4f} denoised; "
            f"validation {vplain.mean():.4f} plain, {vlearned.mean():.4f} denoised")
        if a.out:
            save_weights(a.out, w, scale, {"impacts": TRAIN_IMPACTS, "low": a.low, "high": a.high,
                                           "data_steps": a.steps, "every": a.every, "train_steps": a.train_steps,
                                           "batch": a.batch, "lr": a.lr})
    elif a.command == "profile":
        out.update(profile(a.weights, impact=a.impact, npart=a.low, device=a.device, log=log))
    elif a.command == "floor":
        out.update(counting_floor(a.weights, impact=a.impact, nsteps=a.steps, low=a.low, high=a.high,
                                  device=a.device, log=log))
    else:
        out.update(evaluate(a.weights, impact=a.impact, nsteps=a.steps, every=a.every, low=a.low, high=a.high,
                            device=a.device, log=log))
    if a.json:
        Path(a.json).write_text(json.dumps(out))
    return out


def profile(weights_path=None, *, impact: float = 45.0, npart: int = LOW, at=(100, 200, 300, 400), reps: int = 5,
            device: int = 0, log=print):
    """Device time of the forward pass and of the gradient (CUDA events,
    `reps` each after two warm-ups) on the fine densities of a plain run at
    the steps `at`, with the number of active tiles of each."""
    import torch
    w, scale, _ = load_weights(weights_path)
    sim = make_run(npart, impact, -21, device=device)
    snaps = []
    for s in range(1, max(at) + 1):
        if sim.step().status:
            raise RuntimeError(f"device status at step {s}")
        if s in at:
            snaps.append(torch.from_numpy(sim.accelerator.grid(L.VLB_GRID_RHO_FINE)).to(f"cuda:{device}"))
    sim.accelerator.close()
    net = Network(snaps[0].shape, device)
    wt = torch.from_numpy(w).to(snaps[0].device)
    out, grad = torch.empty_like(snaps[0]), torch.empty_like(wt)
    res = []
    try:
        for step, x in zip(at, snaps):
            for _ in range(2):
                net.forward(x, wt, scale, out)
                net.gradient(x, x, wt, scale, grad)
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record()
            for _ in range(reps):
                net.forward(x, wt, scale, out)
            e[1].record()
            for _ in range(reps):
                net.gradient(x, x, wt, scale, grad)
            e[2].record()
            e[2].synchronize()
            r = {"step": step, "active_tiles": net.active_tiles(), "forward_ms": e[0].elapsed_time(e[1]) / reps,
                 "gradient_ms": e[1].elapsed_time(e[2]) / reps}
            res.append(r)
            log(f"step {step}: {r['active_tiles']} active tiles, forward {r['forward_ms']:.3f} ms, "
                f"gradient {r['gradient_ms']:.3f} ms")
    finally:
        net.close()
    return {"profile": res}


def evaluate(weights_path=None, *, impact: float = 45.0, nsteps: int = 704, every: int = 4, low: int = LOW,
             high: int = HIGH, device: int = 0, log=print):
    """The evaluation: plain runs at `low` and `high` particles and a
    denoised run at `low` (impact parameter `impact`, not trained on), their
    capture curves and times, and the density errors on held-out pairs."""
    import torch
    w, scale, meta = load_weights(weights_path)
    res = {"impact": impact, "low": low, "high": high, "nsteps": nsteps}
    runs = {}
    for name, npart, seed, den in (("plain_high", high, -22, False), ("plain_low", low, -21, False),
                                   ("denoised_low", low, -21, True)):
        sim = make_run(npart, impact, seed, device=device)
        if den:
            attach(sim, w, scale)
        # the steps alone are timed (each returns its scalars, a sync), not the snapshots
        q = np.zeros(nsteps)
        used = 0
        wall = 0.0
        snaps = torch.empty((nsteps // every,) + (sim.accelerator.nf,) * 3, dtype=torch.float32,
                            device=torch.device("cuda", device)) if name != "denoised_low" else None
        torch.cuda.synchronize(device)
        for s in range(1, nsteps + 1):
            t0 = time.perf_counter()
            d = sim.step()
            wall += time.perf_counter() - t0
            if d.status:
                raise RuntimeError(f"{name}: device status {d.status} at step {s}")
            q[s - 1] = d.enclosed_charge
            used += d.denoised
            if snaps is not None and s % every == 0:
                snaps[s // every - 1].copy_(torch.from_numpy(sim.accelerator.grid(L.VLB_GRID_RHO_FINE)))
        runs[name] = {"q8": q, "wall_s": wall, "denoised_steps": used, "snaps": snaps}
        sim.accelerator.close()
        log(f"{name}: {nsteps} steps in {wall:.2f} s, q(<8) final {q[-1]:.4f}, denoised steps {used}")
    qh = runs["plain_high"]["q8"]
    for name in ("plain_low", "denoised_low"):
        r = runs[name]
        res[name] = {"wall_s": r["wall_s"], "ms_per_step": 1000 * r["wall_s"] / nsteps,
                     "max_dq_vs_high": float(np.max(np.abs(r["q8"] - qh))),
                     "final_q8": float(r["q8"][-1]), "denoised_steps": r["denoised_steps"]}
    res["plain_high"] = {"wall_s": runs["plain_high"]["wall_s"],
                         "ms_per_step": 1000 * runs["plain_high"]["wall_s"] / nsteps,
                         "final_q8": float(qh[-1])}
    res["time_ratio_denoised_vs_high"] = runs["denoised_low"]["wall_s"] / runs["plain_high"]["wall_s"]
    res["q8"] = {k: runs[k]["q8"].tolist() for k in runs}
    plain, learned = errors(runs["plain_low"]["snaps"], runs["plain_high"]["snaps"], w, scale)
    res["heldout_err_plain"] = float(plain.mean())
    res["heldout_err_learned"] = float(learned.mean())
    log(f"held-out pairs at b={impact:g}: relative L2 density error {plain.mean():.4f} plain, "
        f"{learned.mean():.4f} denoised")
    log(f"capture curve vs {high:.0e}: max |dq| {res['plain_low']['max_dq_vs_high']:.4f} plain, "
        f"{res['denoised_low']['max_dq_vs_high']:.4f} denoised; time ratio {res['time_ratio_denoised_vs_high']:.3f}")
    return res


def counting_floor(weights_path=None, *, impact: float = 45.0, nsteps: int = 704, low: int = LOW,
                   high: int = HIGH, high_seeds=(-22, -23), low_seeds=(-21, -24, -25), device: int = 0,
                   log=print):
    """Where the capture-curve bar stands against the curve's own counting
    noise.  q(<8 a0) is a count of pseudo-particles (enclosed_charge,
    src/projectile.jl:243-247), so two runs of the same collision with
    different seeds differ even at `high` particles.  Runs: plain at `high`
    with each of high_seeds; plain and denoised at `low` with each of
    low_seeds.  Reports max and rms |dq| over the steps between the two
    `high` runs, and of every `low` run (plain, denoised) against the first
    `high` run, with the counting noise sqrt(q w) of one curve."""
    w, scale, _ = load_weights(weights_path)
    curves = {}

    def run(name, npart, seed, den):
        sim = make_run(npart, impact, seed, device=device)
        if den:
            attach(sim, w, scale)
        q = np.zeros(nsteps)
        t0 = time.perf_counter()
        for s in range(nsteps):
            d = sim.step()
            if d.status:
                raise RuntimeError(f"{name}: device status {d.status} at step {s + 1}")
            q[s] = d.enclosed_charge
        wall = time.perf_counter() - t0
        sim.accelerator.close()
        curves[name] = q
        log(f"{name}: {nsteps} steps in {wall:.1f} s, final q(<8) {q[-1]:.4f}")

    for sd in high_seeds:
        run(f"plain {high:.0e} seed {sd}", high, sd, False)
    for sd in low_seeds:
        run(f"plain {low:.0e} seed {sd}", low, sd, False)
        run(f"denoised {low:.0e} seed {sd}", low, sd, True)
    ref_name = f"plain {high:.0e} seed {high_seeds[0]}"
    ref = curves[ref_name]
    rows = []
    for name, q in curves.items():
        if name == ref_name:
            continue
        dq = np.abs(q - ref)
        rows.append({"run": name, "vs": ref_name, "max_dq": float(dq.max()),
                     "rms_dq": float(np.sqrt(np.mean(dq ** 2))), "final_dq": float(dq[-1])})
        log(f"{name} vs {ref_name}: max |dq| {dq.max():.4f}, rms {np.sqrt(np.mean(dq ** 2)):.4f}, "
            f"final {dq[-1]:.4f}")
    qmean = float(np.mean(ref[nsteps // 2:]))
    noise = {"q_mean_second_half": qmean, "sigma_count_high": math.sqrt(qmean * 196.0 / high),
             "sigma_count_low": math.sqrt(qmean * 196.0 / low)}
    log(f"counting noise of one curve at q = {qmean:.3f}: {noise['sigma_count_high']:.4f} e at {high:.0e}, "
        f"{noise['sigma_count_low']:.4f} e at {low:.0e}")
    return {"impact": impact, "nsteps": nsteps, "rows": rows, "noise": noise,
            "q8": {k: v.tolist() for k, v in curves.items()}}


if __name__ == "__main__":
    main()
