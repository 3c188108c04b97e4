"""Generates the golden fixtures in this directory from the FP64 oracle.

The reference (Julia + Gridap) cannot run here, so its outputs cannot be
recorded. Each fixture is therefore produced by the numpy restatement
(oracle/sumfac_oracle.py). Before it is written, it is cross-checked against
two independent paths: the assembled sparse matrix built from full element
matrices (the stand-in for Gridap's assembled operator, as test/Demo.jl:54-57
compares), and the C restatement of the reference loops
(oracle/sumfac_ref.c). Run from the repository root:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import cref  # noqa: E402
from oracle import sumfac_oracle as O  # noqa: E402

# name: (p, quad degree, n, perturb, perturb seed, x kind, x seed, kappa seed)
CASES = {
    # Q2 on 8^3, 3-point Gauss, x ~ U[-1,1] seed 0
    "c1_q2_n8": (2, 4, 8, 0.0, 0, "uniform", 0, None),
    # the reference's Demo.jl set-up (p=4, quad degree 6) on 4^3, x = ones
    "demo_q4_deg6_n4_ones": (4, 6, 4, 0.0, 0, "ones", 0, None),
    # variable coefficient kappa = exp(g), g ~ N(0, 0.5^2) per point
    "kappa_q3_n4": (3, 6, 4, 0.0, 0, "uniform", 2, 1),
    # deformed (trilinear) cells, interior vertices moved by up to 0.2 h
    "deformed_q4_n3": (4, 8, 3, 0.2, 5, "uniform", 6, None),
    "deformed_q8_n2": (8, 16, 2, 0.2, 7, "uniform", 8, None),
    # Q1 with a 4-point rule: SQ > SB (test/Demo_StepByStep.jl uses p=1, degree 4)
    "q1_deg4_n6": (1, 4, 6, 0.0, 0, "uniform", 9, None),
    # under-integrated Q4: degree 2(p-1) = 6 -> 4 points < 5 basis functions
    "q4_deg6_n3": (4, 6, 3, 0.0, 0, "uniform", 10, None),
}


def kappa_field(seed: int, ncells: int, nq: int) -> np.ndarray:
    g = np.random.default_rng(seed).normal(0.0, 0.5, size=(ncells, nq))
    return np.exp(g)


def make(name, p, deg, n, perturb, pseed, xkind, xseed, kseed):
    m = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, m, perturb=perturb, seed=pseed)
    cq = O.cell_quantities(m, mesh)
    if xkind == "ones":
        x = np.ones(mesh.n_free)
    else:
        x = np.random.default_rng(xseed).uniform(-1.0, 1.0, mesh.n_free)
    kappa = None if kseed is None else kappa_field(kseed, mesh.cell_dof_ids.shape[0], m.SQ ** 3)
    y = O.lazy_mul(m, mesh, x, cq, kappa)
    y_sp = O.assembled_sparse(m, mesh, cq, kappa) @ x
    y_c = cref.problem_from_oracle(m, mesh, cq, kappa).mul(x)
    scale = np.abs(y).max()
    e1 = np.abs(y - y_sp).max() / scale
    e2 = np.abs(y - y_c).max() / scale
    assert e1 < 1e-13 and e2 < 1e-13, (name, e1, e2)
    d = O.diagonal(m, mesh, cq, kappa)
    out = dict(p=p, deg=deg, n=n, perturb=perturb, perturb_seed=pseed, x=x, y=y, diag=d,
               n_free=mesh.n_free, sq=m.SQ)
    if kappa is not None:
        out["kappa"] = kappa
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: n_free={mesh.n_free} |y|max={scale:.3e} sparse={e1:.1e} c={e2:.1e}")


if __name__ == "__main__":
    for k, v in CASES.items():
        make(k, *v)
