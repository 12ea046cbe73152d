"""The streamed construction of a cloud on the device (the partial survey
item: seeded sampling that is sliced and bounded on the host).

The Ran2(seed) cloud is drawn, packed and uploaded a chunk at a time, and
the priming's second half (src/simulation.jl:233-277) runs chunk by chunk on
ranged downloads and uploads: the result must be the one-shot construction's
cloud bit for bit, a rank's slice must be the same slots of the whole cloud,
and at 8e7 particles the construction's host peak must stay under 1 GB
(a one-shot draw holds 48 bytes a particle for positions and momenta alone,
3.8 GB at 8e7, and several times that while priming)."""
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT, load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


def _params(npart, nfine=28):
    return vb.SimulationParameters.for_grid(nfine, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)


@pytest.mark.parametrize("softening", [L.VLB_SOFTENING_DEVICE, L.VLB_SOFTENING_BALL], ids=["device", "cpu-ball"])
def test_streamed_construction_is_the_one_shot_cloud(cuda_device, softening):
    n = 100_003
    sims = []
    try:
        for chunk in (0, 4096, 1 << 20):
            sims.append(vb.Simulation(_params(n), vb.thomas_fermi_profile(), seed=-2, fixed_point=True,
                                      projectile=vb.xenon_projectile(x0=-15.0, impact=5.0),
                                      softening_mode=softening, stream_chunk=chunk))
        ref = sims[0].accelerator.download()
        for s in sims[1:]:
            for x, y in zip(s.accelerator.download(), ref):
                assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
        d = [s.step() for s in sims]
        assert d[1].kinetic == d[0].kinetic and d[2].enclosed_charge == d[0].enclosed_charge
    finally:
        for s in sims:
            s.accelerator.close()


def test_a_slice_of_the_stream_is_the_same_slots_of_the_cloud(cuda_device):
    """stream_half_step_cloud for the slice [a, b) of the cloud (a rank of
    sampling="slice") uploads exactly the one-shot half-step records [a, b)."""
    n, (a, b) = 60_000, (23_456, 41_000)
    p = _params(n)
    prof = vb.thomas_fermi_profile()
    w = p.nelectrons / n
    M, dt = vb.simulation.ELECTRON_MASS * w, p.dt
    meshes = vb.build_meshes(p.nfine, p.ninner, p.nouter, p.rcluster, p.rbox)
    sm = vb.gaussian_smoothing(meshes.fine.axis)
    whole = vb.DeviceAccelerator(meshes, sm, n, w)
    part = vb.DeviceAccelerator(meshes, sm, b - a, w)
    try:
        for acc, lo, hi in ((whole, 0, n), (part, a, b)):
            st = vb.ThomasFermiStream(prof, w, seed=-1)
            vb.stream_half_step_cloud(acc, st, lo, hi, M, dt, chunk=5000)
            st.close()
        W, P = whole.download(), part.download()
        for x, y in zip(P, W):
            assert np.array_equal(x, y[:, a:b])
        pos, mom = vb.sample_thomas_fermi(prof, n, w, seed=-1)
        k, d = vb.pack_positions(pos - (dt / (2 * M)) * mom, whole.x0, whole.h)
        assert np.array_equal(W[0], k) and np.array_equal(W[1], d)
    finally:
        whole.close()
        part.close()


def test_8e7_construction_host_peak_is_below_1_gb(cuda_device):
    """In a fresh process: the peak resident size grows by less than 1 GB
    while the 8e7-particle simulation is built and primed.  The CUDA context
    is made first, by a small context; then the kernel's high-water mark of
    the resident size is reset to the current size (writing 5 to
    /proc/self/clear_refs), so that only the construction counts."""
    code = textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {str(ROOT)!r})
        from __graft_entry__ import load
        vb = load()

        def status_kb(key):
            for line in open("/proc/self/status"):
                if line.startswith(key + ":"):
                    return int(line.split()[1])

        p = vb.SimulationParameters.for_grid(64, rcluster=78.0, rbox=235.0, nparticles=80_000_000, dt=0.5)
        m = vb.build_meshes(p.nfine, p.ninner, p.nouter, p.rcluster, p.rbox)
        small = vb.DeviceAccelerator(m, vb.gaussian_smoothing(m.fine.axis), 1000, 0.196)
        small.close()
        with open("/proc/self/clear_refs", "w") as f:
            f.write("5")
        before, hwm0 = status_kb("VmRSS"), status_kb("VmHWM")
        sim = vb.Simulation(p, vb.thomas_fermi_profile(), projectile=vb.xenon_projectile(), fixed_point=True)
        after = status_kb("VmHWM")
        d = sim.step()
        assert d.status == 0
        print("PEAK_KB", before, after, after - before, hwm0)
    """)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("PEAK_KB")][-1]
    before, after, delta, hwm0 = (int(x) for x in line.split()[1:])
    print(f"\n[8e7 construction] resident size {before / 1e6:.2f} GB before, peak {after / 1e6:.2f} GB during "
          f"(+{delta / 1e6:.3f} GB); high-water mark after the reset {hwm0 / 1e6:.2f} GB")
    assert hwm0 <= before + 100_000   # the reset took: the mark starts at the current size
    assert delta < 1_000_000  # kilobytes
