"""The oracle as a shard backend of vlasov_b200.sharded.ShardedStepper: the
device-semantics step (float64) of one rank's slice, split into the same
three phases as the library, its exchange buffers as CPU torch tensors over
numpy arrays (summed with gloo).  Test infrastructure only."""
import contextlib
from types import SimpleNamespace

import numpy as np
import torch


class OracleShard:
    def __init__(self, orc, O, k, d, pk, pd, ids):
        self.orc, self.O = orc, O
        self.k, self.d, self.pk, self.pd = (np.ascontiguousarray(a) for a in (k, d, pk, pd))
        self.ids = np.asarray(ids)
        nf, nc = O.F.n, O.Cl.n
        self.raw = np.zeros(nf ** 3)
        self.rhoc = np.zeros(nc ** 3)
        self.scal = np.zeros(1)
        self.red = np.zeros(4)
        self._deposit = [torch.from_numpy(self.raw), torch.from_numpy(self.rhoc), torch.from_numpy(self.scal)]
        self._reaction = torch.from_numpy(self.red)

    def stream(self):
        return contextlib.nullcontext()

    def synchronize(self):
        pass

    def tensor(self, values):
        return torch.tensor(values, dtype=torch.float64)

    def deposit_buffers(self):
        return self._deposit

    def reaction_buffer(self):
        return self._reaction

    def step_deposit(self, projectile, params):
        orc, O = self.orc, self.O
        nk = O.meshes.fine.axis.nknots
        perm, occ, bnd, _ = orc.cellsort(self.k, nk)
        self.k, self.d, self.pk, self.pd = (np.ascontiguousarray(a[:, perm]) for a in (self.k, self.d, self.pk, self.pd))
        self.ids = self.ids[perm]
        self.occ, self.bnd = occ, bnd
        c, N = O.c, self.k.shape[1]
        cols, nout = orc.columns(self.k, self.d, c["x0f"], c["hf"], c["lo"], c["hi"], c["spacing"], c["nbdt"])
        self.nout = nout
        orc.lib().orc_deposit_sorted_raw(O.F.ref(), O.S.ref(), N, orc.pi(np.ascontiguousarray(cols)), orc.pi(occ),
                                         orc.pi(bnd), len(occ), orc.pd(self.raw))
        orc.lib().orc_deposit_cic_device(O.Cl.ref(), N, orc.pi(self.k), orc.pf(self.d), c["x0f"], c["hf"], O.w,
                                         orc.pd(self.rhoc))
        self.scal[0] = nout

    def step_fields(self, params, npart_global):
        orc, O = self.orc, self.O
        q = orc.lib().orc_total_charge(O.F.ref(), orc.pd(self.raw))
        O.rhof[:] = self.raw * ((npart_global - self.scal[0]) * O.w / q)
        O.rhoc[:] = self.rhoc
        lib = orc.lib()
        lib.orc_poisson(O.F.ref(), O.Cl.ref(), orc.pd(O.rhof), orc.pd(O.rhoc), orc.pd(O.phif), orc.pd(O.phic))
        lib.orc_spline_coefficients(O.F.ref(), orc.pd(O.phif), orc.pd(O.csolf))
        lib.orc_spline_coefficients(O.Cl.ref(), orc.pd(O.phic), orc.pd(O.csolc))
        lib.orc_effective_potential(O.F.ref(), orc.pd(O.csolf), orc.pd(O.rhof), O.jel.nions, O.jel.radius)
        lib.orc_effective_potential(O.Cl.ref(), orc.pd(O.csolc), orc.pd(O.rhoc), O.jel.nions, O.jel.radius)
        N = self.k.shape[1]
        force = np.empty((3, N))
        red = np.zeros(4)
        pr = orc.projectile_struct(O.proj)
        c = O.c
        self.outcount = lib.orc_forces_device(O.F.ref(), O.Cl.ref(), O.S.ref(), N, orc.pi(self.k), orc.pf(self.d),
                                              orc.pi(self.occ), orc.pi(self.bnd), len(self.occ), orc.pd(O.csolf),
                                              orc.pd(O.csolc), O.w, c["x0"], c["h"], orc.C.byref(pr),
                                              orc.pd(force), orc.pd(red))
        self.force = force
        self.red[:] = red

    def step_advance(self, projectile, params):
        O = self.O
        O.red = self.red.copy()
        F = O.advance_projectile() if params.advance_projectile else O.projectile_force()
        diag = np.zeros(5)
        if params.push:
            self.k, self.d, self.pk, self.pd, diag = O.push(self.k, self.d, self.pk, self.pd,
                                                            self.force.astype(np.float32))
        q = O.enclosed_charge(self.k, self.d, params.capture_radius) if params.capture_radius > 0 else 0.0
        return SimpleNamespace(kinetic=diag[0], escaped=diag[1], angular=tuple(diag[2:5]), enclosed_charge=q,
                               nout=self.nout, outcount=self.outcount, status=0,
                               projectile_force=tuple(np.asarray(F, dtype=float)))
