"""Test infrastructure: a CPU stand-in for one part of the distributed
operator (ncihackaton2023.jl_b200/distributed.py), built on the oracle's
assembled sparse matrix.

It gives the host logic of the distributed layer (partition, halo exchange,
sums over ranks, the CG loop) something to drive without a GPU. Each step
follows the device semantics of the sf_cgd_* entry points (include/sfb200.h):
the same scalar slots, the same stopping flag, owned points only.
"""
from __future__ import annotations

import numpy as np
import torch

# scalar slots of the sf_cgd_* block
RZ, PQ, RZ_NEW, RR, BB, DONE, ITERS, TOL2 = range(8)
PART_PQ, PART_RZ, PART_RR = 10, 11, 12


class OracleSlabEngine:
    """One part: S is the global assembled matrix (scipy sparse over the free
    dofs), layout the part's SlabLayout."""

    def __init__(self, S, layout):
        self.S = S
        self.L = layout
        self.dinv = 1.0 / S.diagonal()

    def _global(self, x: torch.Tensor) -> np.ndarray:
        L = self.L
        xg = np.zeros(self.S.shape[0])
        j0, g0, cnt = L.global_levels()
        pl = L.plane
        xg[g0 * pl:(g0 + cnt) * pl] = x.numpy()[j0 * pl:(j0 + cnt) * pl]
        return xg

    def _own(self, v: torch.Tensor) -> torch.Tensor:
        return v[self.L.owned]

    def _dinv(self) -> torch.Tensor:
        return torch.from_numpy(self.dinv[self.L.owned_global()])

    def apply(self, x, y):
        yg = self.S @ self._global(x)
        y[self.L.owned] = torch.from_numpy(yg[self.L.owned_global()])

    def cgd_start(self, b, x, r, p, q, s):
        s.zero_()
        self.apply(x, q)
        ro = self._own(b) - self._own(q)
        z = self._dinv() * ro
        r[self.L.owned] = ro
        p[self.L.owned] = z
        s[RZ_NEW] = torch.dot(ro, z)
        s[RR] = torch.dot(ro, ro)
        s[BB] = torch.dot(self._own(b), self._own(b))

    def cgd_init(self, s, reltol):
        s[RZ] = s[RZ_NEW]
        s[ITERS] = 0.0
        bb = float(s[BB])
        s[TOL2] = reltol * reltol * (bb if bb > 0 else 1.0)
        s[DONE] = 2.0 if float(s[RR]) <= float(s[TOL2]) else 0.0

    def cgd_apply(self, p, q, s):
        self.apply(p, q)
        if float(s[DONE]) == 0.0:
            s[PART_PQ] = torch.dot(self._own(p), self._own(q))

    def cgd_update(self, r, q, s):
        if float(s[DONE]) != 0.0:
            return
        pq = float(s[PART_PQ])
        alpha = float(s[RZ]) / pq
        ro = self._own(r) - alpha * self._own(q)
        r[self.L.owned] = ro
        s[PQ] = pq
        s[PART_RZ] = torch.dot(ro, self._dinv() * ro)
        s[PART_RR] = torch.dot(ro, ro)

    def cgd_direction(self, x, p, r, s):
        if float(s[DONE]) == 0.0:
            s[RZ_NEW] = s[PART_RZ]
            s[RR] = s[PART_RR]
            if float(s[RR]) <= float(s[TOL2]):
                s[DONE] = 1.0
        done = float(s[DONE])
        if done >= 2.0:
            return
        alpha = float(s[RZ]) / float(s[PQ])
        beta = float(s[RZ_NEW]) / float(s[RZ])
        po = self._own(p).clone()
        x[self.L.owned] = self._own(x) + alpha * po
        if done == 0.0:
            p[self.L.owned] = self._dinv() * self._own(r) + beta * po
        s[RZ] = s[RZ_NEW]
        s[ITERS] += 1.0
        if done == 1.0:
            s[DONE] = 2.0
