"""Benchmark of the per-step pseudo-particle loop: the Na196 + Xe25+ (500 keV,
b = 45 a0) collision with 8e6 pseudo-particles on the 130^3 fine grid, one
fused step (sort, fine + coarse deposit, nested Poisson, mean field, smoothed
gather with the projectile, packed Verlet push) per iteration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  `value` is ms/step measured with CUDA events
on the library's stream, inputs resident in HBM (the particle state, 2 x 384 MB,
is larger than L2).  `e2e` is the same metric through the public API with the
cloud uploaded from and downloaded to pinned host memory inside the timed
region.  `--impl reference` times the CPU restatement of the reference's own
CPU path (the oracle) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

MEASURED = ROOT / "MEASURED_PEAKS.json"
GATHER_FLOP_PER_PARTICLE = 4600.0       # 2000 FMA + 300 mul/FMA per 10^3 contraction
GATHER_TC_FLOP_PER_PARTICLE = 12000.0   # 3 split products x (oy, gy) x 100 columns x 10 y x 2
# delta in, force out; the tensor-core form also reads the sort's packed table columns (4 B)
GATHER_BYTES_PER_PARTICLE = {"tcgen05": 28.0, "fp32": 24.0}
# DRAM bytes (read + write) of one gather launch per particle, from the ncu
# captures of 4e6 particles (profiles/k_field_tc_4M.md, profiles/k_field_4M.md)
GATHER_TRAFFIC_PER_PARTICLE = {"tcgen05": (65935872 + 13056512) / 4e6, "fp32": (49494784 + 7127296) / 4e6}
# read (k, d) in slot order, (pk, pd) where the step's sort left them (through perm: 4 B), the force;
# write the record and the next sort's cell key
PUSH_BYTES_PER_PARTICLE = 24 + 24 + 4 + 12 + 48 + 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--npart", type=int, default=8_000_000)
    ap.add_argument("--nfine", type=int, default=64)
    ap.add_argument("--profile", default="thomas-fermi", choices=["thomas-fermi", "uniform-sphere"])
    ap.add_argument("--deposit", default="float32", choices=["float32", "fixed64"])
    ap.add_argument("--precision", default="3xtf32", choices=["fp32", "3xtf32", "bf16x3"],
                    help="mode products on the CUDA cores (fp32) or split-precision on the tensor cores")
    ap.add_argument("--gather", default="tcgen05", choices=["tcgen05", "fp32"],
                    help="the gather's sums over y as 3xTF32 MMAs on the tensor cores, or FP32 FMAs")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=6, help="timed steps of the CPU baseline (primed, 1 warm-up)")
    ap.add_argument("--no-learned", action="store_true", help="skip the step with the learned denoiser")
    return ap.parse_args()


def load():
    from __graft_entry__ import load as _load
    return _load()


def workload(args, vb):
    ninner, nouter = vb.grids(args.nfine)
    p = vb.SimulationParameters(nfine=args.nfine, ninner=ninner, nouter=nouter, rcluster=78.0, rbox=235.0,
                                nions=196.0, nelectrons=196.0, nparticles=args.npart, nsteps=0, dt=0.5)
    prof = vb.thomas_fermi_profile() if args.profile == "thomas-fermi" else vb.uniform_sphere_profile()
    proj = vb.xenon_projectile(v=0.40, impact=45.0, x0=-70.0, dt=0.5)
    return p, prof, proj


def config_dict(args, n):
    return {"workload": "Na196 + Xe25+ 500 keV b=45 a0 collision, one fused step",
            "npart_per_gpu": args.npart, "fine_grid": f"{2 * args.nfine + 2}^3", "coarse_grid": f"{2 * args.nfine + 2}^3",
            "profile": args.profile, "deposit": args.deposit, "mode_products": args.precision, "gather": args.gather, "dt": 0.5, "projectile": "Xe25+ v=0.40 x0=-70 b=45",
            "cuda_graph": (not args.no_graph) if n == 1 else "per-phase eager (collectives between phases)",
            "l2": "inputs larger than L2 (2 x 384 MB particle state)",
            "parallelism": (f"{n} particle shards, NCCL all-reduce of the deposited grids and the projectile's "
                            "reaction sums" if n > 1 else "1 GPU")}


class ClockSampler:
    """SM clock and throttle reasons through NVML, sampled every 20 ms."""

    def __init__(self, index):
        self.samples = []
        self.stop_flag = False
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None

    def _run(self):
        nv = self.nv
        while not self.stop_flag:
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((time.time(), mhz, reasons))
            except Exception:
                pass
            time.sleep(0.02)

    def start(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()

    def stop(self):
        self.stop_flag = True
        if self.ok:
            self.t.join()

    def summary(self, t0, t1):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        inside = [s for s in self.samples if t0 <= s[0] <= t1] or self.samples[-3:]
        nv = self.nv
        names = {
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "hw_power_brake_slowdown": getattr(nv, "nvmlClocksEventReasonHwPowerBrakeSlowdown", 0x80),
        }
        seen = sorted({n for _, _, r in inside for n, bit in names.items() if r & bit})
        return {"sm_mhz": statistics.median(m for _, m, _ in inside) if inside else None,
                "sm_max_mhz": self.max_mhz, "reasons": seen, "samples": len(inside)}


def peaks():
    try:
        return json.loads(MEASURED.read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def host_reference(args, nsteps, warmup):
    """The reference's CPU step path (update_forces! + step!, src/simulation.jl:
    309-352, 382-396) as the oracle restates it (oracle.HostStep, float64,
    OpenMP over the host cores), on this workload: the oracle's own seeded
    draw of the cloud (no product library is loaded), prime_leapfrog!
    (src/simulation.jl:233-277), `warmup` untimed steps, then `nsteps` timed
    steps.  The set-up tables come from the package's pure-Python table
    builders, as the reference's host hands its own tables over.  Returns
    (ms per step, threads)."""
    from oracle import oracle as orc
    vb = load()
    p, prof, proj = workload(args, vb)
    meshes = vb.build_meshes(p.nfine, p.ninner, p.nouter, p.rcluster, p.rbox)
    sm = vb.gaussian_smoothing(meshes.fine.axis)
    w = p.nelectrons / p.nparticles
    pos, mom = orc.sample_thomas_fermi(prof, p.nparticles, w, seed=-1)
    jel = vb.Jellium.of(p.nions)
    cores = orc.lib().orc_num_threads()
    proj.softening_mode = 1  # the CPU path's ball softening (src/projectile.jl:203-232)
    st = orc.HostStep(meshes, sm, w, jel, p.dt, p.rcmax, proj)
    pos, prev = st.prime(pos, mom)
    for _ in range(warmup):
        pos, prev, _ = st.step(pos, prev)
    t0 = time.perf_counter()
    for _ in range(nsteps):
        pos, prev, _ = st.step(pos, prev)
    return (time.perf_counter() - t0) / nsteps * 1e3, cores


REFERENCE_MAX_TIMED = 60  # timed CPU steps at most: about 75 s of the 16-thread host at 8e6


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    timed = max(1, min(args.steps, REFERENCE_MAX_TIMED))
    warm = max(1, min(args.warmup, 3))
    ms, cores = host_reference(args, timed, warm)
    line = {"metric": "ms/step at 8M particles, 130^3 grid; learned vs plain at equal capture error", "value": ms, "unit": "ms/step", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ran2 Thomas-Fermi cloud)",
            "config": config_dict(args, 1), "impl": "reference",
            "cpu_baseline": {"value": ms, "unit": "ms/step", "cores": cores, "kind": "port",
                             "sample": f"{timed} primed full CPU steps of the workload after {warm} untimed ones "
                                       "(float64 restatement of the reference CPU path, OpenMP contiguous chunks, "
                                       "ball softening; at most "
                                       f"{REFERENCE_MAX_TIMED} timed steps whatever --steps asks)"},
            "e2e": {"value": ms, "unit": "ms/step", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=120))
    vb = load()
    L = vb._lib

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    p, prof, proj = workload(args, vb)
    precision = {"fp32": vb._lib.VLB_POISSON_FP32, "3xtf32": vb._lib.VLB_POISSON_3XTF32,
                 "bf16x3": vb._lib.VLB_POISSON_BF16X3}[args.precision]
    if world > 1:
        # weak scaling: npart per GPU, one cloud of world * npart particles
        # sharded over the ranks (each rank draws its own slice)
        p.nparticles = args.npart * world
        sim = vb.sharded.ShardedSimulation(p, prof, comm=vb.sharded.TorchComm(), device=local, projectile=proj,
                                           fixed_point=args.deposit == "fixed64", precision=precision,
                                           sampling="per-rank", seed=-1)
    else:
        sim = vb.Simulation(p, prof, projectile=proj, device=local, fixed_point=args.deposit == "fixed64",
                            precision=precision, use_graph=not args.no_graph, seed=-1)
    acc = sim.accelerator
    acc.set_tuning(field_tensor_cores=1 if args.gather == "tcgen05" else 0)
    ext = torch.cuda.ExternalStream(acc.stream_handle(), device=torch.device("cuda", local))
    for _ in range(max(args.warmup, 3)):
        sim.step()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.1)
    barrier()
    launches0 = acc.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall0 = time.time()
    e0.record(ext)
    for _ in range(args.steps):
        d = sim.step()
    e1.record(ext)
    e1.synchronize()
    t_wall1 = time.time()
    barrier()
    launches = acc.launch_count() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    clocks.stop()
    ms = max_over_ranks(ms)
    clk = clocks.summary(t_wall0, t_wall1)

    # per-stage device times (eager, stage events) for the roofline
    if world == 1:
        sim.use_graph = False
    acc.profile(True)
    nprof = max(3, min(args.steps, 20))
    for _ in range(nprof):
        sim.step()
    stages = {k: v / nprof for k, v in acc.stage_times().items()}
    acc.profile(False)
    if world == 1:
        sim.use_graph = not args.no_graph

    # end to end through the public API: cloud from pinned host memory, K
    # steps, cloud back to pinned host memory
    k, dd, pk, pd = acc.download()
    pins = [torch.from_numpy(a).pin_memory() for a in (k, dd, pk, pd)]
    hk, hd, hpk, hpd = (t.numpy() for t in pins)
    outs = [torch.empty_like(t).pin_memory() for t in pins]
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(ext)
    acc.upload(hk, hd, hpk, hpd)
    for _ in range(args.steps):
        sim.step()
    L.check(L.lib().vlb_download_particles(acc.handle, L.pi(outs[0].numpy()), L.pf(outs[1].numpy()),
                                           L.pi(outs[2].numpy()), L.pf(outs[3].numpy())))
    f1.record(ext)
    f1.synchronize()
    barrier()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1) / args.steps)
    cloud_bytes = 48 * args.npart
    step_h2d = 112  # vlb_projectile in
    step_d2h = 480  # the step's scalar block out

    # the same steps with the energy budget's two sums (step!(sim; energy=true))
    energy = None
    if world == 1:
        for _ in range(max(args.warmup, 3)):
            sim.step(energy=True)
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(ext)
        for _ in range(args.steps):
            de = sim.step(energy=True)
        h1.record(ext)
        h1.synchronize()
        energy_ms = h0.elapsed_time(h1) / args.steps
        b = sim.energy_budget(de)
        energy = {"ms_per_step": energy_ms, "vs_plain": energy_ms / ms, "steps": args.steps,
                  "last_budget": {"total": b.total, "kinetic": b.kinetic, "hartree": b.hartree,
                                  "meanfield": b.meanfield, "ions": b.ions}}

    # the same steps with the learned denoiser after the fine deposit
    learned = None
    if world == 1 and not args.no_learned and args.nfine == 64:
        w_dn, s_dn, meta_dn = vb.denoiser.load_weights()
        vb.denoiser.attach(sim, w_dn, s_dn)
        for _ in range(max(args.warmup, 3)):
            sim.step()
        used = 0
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(ext)
        for _ in range(args.steps):
            used += sim.step().denoised
        g1.record(ext)
        g1.synchronize()
        learned_ms = g0.elapsed_time(g1) / args.steps
        vb.denoiser.detach(sim)
        learned = {"ms_per_step": learned_ms, "vs_plain": learned_ms / ms, "denoised_steps": used,
                   "steps": args.steps, "network": "vlasov.jl_b200/data/denoiser_xe25_130.npz",
                   "trained_on": meta_dn}

    # the strict FP32 drop-in: mode products and the gather's sums on the
    # CUDA cores in FP32, the same steps timed the same way
    fp32 = None
    if world == 1:
        saved_prec = sim.precision
        sim.precision = vb._lib.VLB_POISSON_FP32
        acc.set_tuning(field_tensor_cores=0)
        for _ in range(max(args.warmup, 3)):
            sim.step()
        j0, j1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        j0.record(ext)
        for _ in range(args.steps):
            sim.step()
        j1.record(ext)
        j1.synchronize()
        fp32 = {"ms_per_step": j0.elapsed_time(j1) / args.steps, "steps": args.steps,
                "mode_products": "fp32 (CUDA cores)", "gather": "fp32 (CUDA cores)",
                "note": "the plain FP32 drop-in, timed like value (graph replays, CUDA events)"}
        sim.precision = saved_prec
        acc.set_tuning(field_tensor_cores=1 if args.gather == "tcgen05" else 0)

    pk_, how = peaks()
    fp32_peak = vb._lib.C.c_double()
    L.check(L.lib().vlb_fp32_peak(local, vb._lib.C.byref(fp32_peak)))
    t_forces = stages.get("forces_kernel", float("nan"))
    gather_kernel = ("k_field_tc (smoothed gather + projectile, sums over y as 3xTF32 tcgen05 MMAs)"
                     if args.gather == "tcgen05" else "k_field (smoothed gather + projectile, FP32 FMAs)")
    achieved = GATHER_FLOP_PER_PARTICLE * args.npart / (t_forces * 1e-3) / 1e12
    t_push = stages.get("push", float("nan"))
    push_gbs = PUSH_BYTES_PER_PARTICLE * args.npart / (t_push * 1e-3) / 1e9

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            cms, cores = host_reference(args, args.cpu_steps, 1)
            cpu = {"value": cms, "unit": "ms/step", "cores": cores, "kind": "port",
                   "sample": f"{args.cpu_steps} primed full CPU steps of the same workload after 1 untimed one "
                             "(float64 restatement of the reference CPU path, OpenMP, ball softening)"}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "ms/step", "cores": None, "kind": "port", "sample": f"failed: {ex}"}
    line = {
        "metric": "ms/step at 8M particles, 130^3 grid; learned vs plain at equal capture error", "value": ms, "unit": "ms/step", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ran2 sample of the reference's Na196 Thomas-Fermi profile)",
        "config": config_dict(args, world),
        "particle_steps_per_s": args.npart * world / (ms * 1e-3),
        "e2e": {"value": e2e_ms, "unit": "ms/step",
                "h2d_bytes_per_step": step_h2d + cloud_bytes / args.steps,
                "d2h_bytes_per_step": step_d2h + cloud_bytes / args.steps},
        "gpu_launches": int(launches),
        "roofline": {"kernel": gather_kernel, "bound": "fp32",
                     "achieved": achieved, "peak": fp32_peak.value, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak.value,
                     "traffic": GATHER_TRAFFIC_PER_PARTICLE[args.gather] * args.npart,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a 4e6-particle launch, "
                                       "scaled by the particle count (bytes per launch; the forces written "
                                       "mostly stay in L2 past the kernel's end)",
                     "flop_per_particle": GATHER_FLOP_PER_PARTICLE,
                     "note": "FP32-equivalent FLOP of the smoothed gather (the reference's operation count) over "
                             "the gather kernel's own event time (events around its launch in profiled eager steps)",
                     "kernel_ms": t_forces, "forces_stage_ms": stages.get("forces"),
                     "peak_source": "measured FP32 FMA kernel (vlb_fp32_peak), this GPU, this run",
                     "hbm_beside": {"achieved": GATHER_BYTES_PER_PARTICLE[args.gather] * args.npart
                                    / (t_forces * 1e-3) / 1e9,
                                    "peak": pk_.get("hbm_gbs"), "unit": "GB/s",
                                    "frac": GATHER_BYTES_PER_PARTICLE[args.gather] * args.npart
                                    / (t_forces * 1e-3) / 1e9 / pk_.get("hbm_gbs", 1),
                                    "note": "12 B of delta read + 12 B of force written a particle"
                                    + (" + 4 B of packed table columns read" if args.gather == "tcgen05" else "")}},
        "roofline_hbm": {"kernel": "k_push (packed Verlet, previous positions read through the sort's permutation)",
                         "bound": "hbm", "achieved": push_gbs,
                         "peak": pk_.get("hbm_gbs"), "unit": "GB/s", "frac": push_gbs / pk_.get("hbm_gbs", 1),
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({how})"},
        "stages_ms": stages,
        "clocks": clk,
        "last_step": {"q8": d.enclosed_charge, "outcount": d.outcount, "noccupied": d.noccupied},
    }
    if args.gather == "tcgen05":
        tf32_peak = pk_.get("bf16_tflops", 1590.0) / 2
        tens = GATHER_TC_FLOP_PER_PARTICLE * args.npart / (t_forces * 1e-3) / 1e12
        line["roofline"]["tensor"] = {
            "achieved": tens, "peak": tf32_peak, "unit": "TFLOP/s", "frac": tens / tf32_peak,
            "flop_per_particle": GATHER_TC_FLOP_PER_PARTICLE,
            "note": "3xTF32 products of the sums over y (3 x 2 x 100 x 10 x 2 FLOP a particle, no padding)",
            "peak_source": f"dense TF32 taken as half the bf16 figure of MEASURED_PEAKS.json ({how})"}
    if fp32:
        line["fp32_dropin"] = fp32
    if learned:
        line["learned"] = learned
    if energy:
        line["energy_step"] = energy
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    acc.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
