"""CPU slice window for the distributed-Parareal protocol tests (test infrastructure).

Restates one window of the serial oracle Parareal (oracle.orc_parareal, itself a
restatement of Parareal.h:110-171) with the same begin/fine/coarse interface as
stencilparareal_b200.parareal.WindowParareal, on dense numpy fields, so that
DistributedParareal can be exercised with gloo ranks on a machine without a GPU.
Constant diffusivity only (the predictor is the chain U_{r+1} = G(U_r)).
"""
import numpy as np
import torch

from oracle import oracle as O


class OracleWindow:
    def __init__(self, p, endTime, P, tsFine, tsCoarse, first, count, q0, coarse=O.COARSE_EULER_F64, delta=False,
                 skip=True):
        d = O.parareal_derived(O.parareal_cfg(endTime, P, tsFine, tsCoarse, 1))
        self.p, self.first, self.count = p, first, count
        self.tsF, self.tsC, self.dtF, self.dtC, self.slice = (d["tsFine"], d["tsCoarse"], d["dtFine"], d["dtCoarse"],
                                                              d["timeSliceSize"])
        self.q0 = np.asarray(q0, dtype=np.float64)
        self.coarse_kind, self.delta, self.skip = coarse, delta, skip
        self.boundary = torch.zeros(self.q0.shape, dtype=torch.float64)

    def make_recv_buffer(self):
        return torch.zeros(self.q0.shape, dtype=torch.float64)

    def G(self, q, t0, n):
        if n == 0:
            return q.copy()
        k = self.coarse_kind
        if k == O.COARSE_EULER_F64:
            return O.euler(self.p, q, t0, self.dtC, n)
        if k == O.COARSE_RK4_F64:
            return O.rk4(self.p, q, t0, self.dtC, n)
        f = O.rk4_f32 if k == O.COARSE_RK4_F32 else O.euler_f32
        return f(self.p, q.astype(np.float32), t0, self.dtC, n).astype(np.float64)

    def t0(self, r):
        return self.slice * (self.first + r)

    def lo(self, k):
        return max(0, min(k - self.first, self.count)) if self.skip else 0

    def begin(self):
        U = [self.G(self.q0, 0.0, self.tsC * self.first) if self.first else self.q0.copy()]
        Gold = []
        for r in range(self.count):
            g = self.G(U[r], self.t0(r), self.tsC)
            Gold.append(g)
            U.append(g.copy())
        self.U, self.Gold, self.F = U, Gold, [None] * self.count
        self.D = [None] * (self.count + 1)

    def fine(self, k):
        for r in range(self.lo(k), self.count):
            self.F[r] = O.rk4(self.p, self.U[r], self.t0(r), self.dtF, self.tsF)

    def coarse(self, k, inbound=None, want_defect=True):
        lo = self.lo(k)
        new0 = inbound.numpy().copy() if inbound is not None else None
        if self.delta:
            self.D[0] = (new0 - self.U[0]) if new0 is not None else np.zeros_like(self.q0)
        if new0 is not None:
            self.U[0] = new0
        defect = 0.0
        for r in range(lo, self.count):
            if self.delta:
                dr = self.D[r] if (r == 0 or r > lo) else np.zeros_like(self.q0)
                Q = self.F[r] + self.G(dr, self.t0(r), self.tsC)
            else:
                gnew = self.G(self.U[r], self.t0(r), self.tsC)
                Q = (gnew + self.F[r]) - self.Gold[r]
                self.Gold[r] = gnew
            dq = Q - self.U[r + 1]
            defect = max(defect, float(np.sqrt((dq ** 2).sum() / (Q ** 2).sum())))
            self.D[r + 1] = dq
            self.U[r + 1] = Q
        self.boundary.copy_(torch.from_numpy(self.U[self.count]))
        return defect
