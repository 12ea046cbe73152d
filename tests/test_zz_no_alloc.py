"""The allocation-free total charge, for callers that cannot allocate device
memory: an embedding runtime whose caching pool holds the GPU's memory, a
plugin whose host forbids allocation after set-up, a loop that must not stall
on cudaMalloc.  The entry point keeps its scratch in static device memory;
here the caller (the test) owns the device inputs and the output, and the
result is checked against the charge the existing fine-deposit entry point
reports for the same density, on two calls in a row.  The file is collected
last on purpose."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


def test_total_charge_without_allocation_matches_the_deposit_entry_point(cuda_device, orc):
    import torch

    npart = 30_000
    p = vb.SimulationParameters.for_grid(28, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    meshes = vb.build_meshes(28, p.ninner, p.nouter, 78.0, 235.0)
    sm = vb.gaussian_smoothing(meshes.fine.axis)
    w = 196.0 / npart
    pos, mom = vb.sample_thomas_fermi(vb.thomas_fermi_profile(), npart, w)
    acc = vb.DeviceAccelerator(meshes, sm, npart, w)
    try:
        x0, h = acc.x0, acc.h
        k, d = vb.pack_positions(pos, x0, h)
        acc.upload(k, d, k, d)
        acc.sort()
        # existing entry point: the fixed-point deposit reports the charge of
        # its raw density; a second deposit whose renormalisation factor is
        # exactly 1 leaves that raw density in the grid
        nout, q_ref = acc.deposit_smoothed(w, fixed_point=True)
        nout2, q_ref2 = acc.deposit_smoothed(q_ref / (npart - nout), fixed_point=True)
        assert nout2 == nout and q_ref2 == q_ref
        rho = acc.grid(L.VLB_GRID_RHO_FINE)
    finally:
        acc.close()

    n = meshes.fine.n
    dev = torch.device("cuda", cuda_device)
    d_rho = torch.from_numpy(np.ascontiguousarray(rho)).to(dev)
    d_m0 = torch.from_numpy(np.ascontiguousarray(meshes.fine.duals[0])).to(dev)
    d_q = torch.empty(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    lib = L.lib()
    # the same float32 grid summed by the float64 oracle, for a tight check
    level = orc.Level(meshes.fine)  # keeps its float64 tables alive for the call
    rho64 = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    q_oracle = orc.lib().orc_total_charge(level.ref(), orc.pd(rho64))
    for _ in range(2):
        d_q.fill_(float("nan"))
        rc = lib.vlb_total_charge_noalloc(C.c_void_p(d_rho.data_ptr()), C.c_void_p(d_m0.data_ptr()), n,
                                          C.c_void_p(d_q.data_ptr()), C.c_void_p(stream))
        assert rc == L.VLB_OK, lib.vlb_last_error()
        torch.cuda.synchronize(dev)
        q = float(d_q.item())
        # against the existing entry point: the deposit's charge was summed
        # from the int64 accumulator, the grid holds it rounded to float32
        assert abs(q - q_ref) <= 1e-6 * abs(q_ref)
        assert abs(q - q_oracle) <= 1e-12 * abs(q_oracle)

    # sizes beyond the static scratch are refused with a message
    rc = lib.vlb_total_charge_noalloc(C.c_void_p(d_rho.data_ptr()), C.c_void_p(d_m0.data_ptr()), 257,
                                      C.c_void_p(d_q.data_ptr()), C.c_void_p(stream))
    assert rc == L.VLB_ERR_ARG
    assert b"256" in lib.vlb_last_error()
