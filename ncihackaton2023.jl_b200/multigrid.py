"""Multigrid-preconditioned CG for structured meshes (sf_mg_* of the C ABI).

The reference solves with IterativeSolvers.cg! and no preconditioner
(profiling/drivers.jl:85-95). Its iteration count grows with the condition
number: thousands of iterations for a rough right-hand side at Q4, and beyond
any budget for equispaced Q8 on perturbed cells. ``Multigrid`` builds a
hierarchy of structured operators from a ``LazyMatrix`` and hands it to the
library, whose flexible CG runs one V-cycle per iteration (FP32 in the mixed
mode, FP64 otherwise) while the outer CG stays in FP64.

Hierarchy, finest first:
  * the operator's space, in Gauss-Lobatto nodes when ``basis="gll"`` (the
    default from order 5 up: equispaced high-order bases are badly conditioned
    and point-Jacobi smoothing does little on them), else in the operator's
    own equispaced nodes;
  * lower orders on the same cells, halving the order down to 1 (quadrature of
    p_l + 1 points per level);
  * then Q1 on meshes of half the cells while the partition stays even (every
    second vertex; on perturbed meshes the coarse cells are the trilinear cells
    through those vertices).
The transfer tables are 1D Lagrange interpolation matrices between the levels'
node sets; the library applies them as tensor products along the three axes.
With a variable coefficient kappa on the operator, every coarse level gets each
cell's mean of kappa (averaged again over the children of a coarse cell).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib, fem
from ._lib import lib
from .operator import LazyMatrix, SumFactorizationMap, _f64, _stream

MODES = {"mixed": _lib.SF_MG_MIXED, "f64": _lib.SF_MG_F64}


def _ascending(nodes_gridap: np.ndarray) -> np.ndarray:
    """1D nodes in ascending position from Gridap's order (v0, v1, interior)."""
    return np.sort(np.asarray(nodes_gridap, dtype=np.float64))


def _lagrange_values(nodes: np.ndarray, pts: np.ndarray) -> np.ndarray:
    """V[i, m] = value at pts[i] of the Lagrange polynomial of nodes[m]."""
    V, _ = fem.lagrange_basis(nodes, pts)
    V[np.abs(V) < 1e-15] = 0.0
    return V


def transfer_table(fine_nodes: np.ndarray, coarse_nodes: np.ndarray, ratio: int) -> np.ndarray:
    """(ratio pf + 1) x (pc + 1) table of the coarse cell's 1D basis functions at
    the fine nodes inside that cell (ratio fine cells per coarse cell), both node
    sets in ascending position on [0, 1]."""
    pf = len(fine_nodes) - 1
    pts = np.concatenate([(k + fine_nodes[:-1]) / ratio for k in range(ratio)] + [[1.0]])
    assert len(pts) == ratio * pf + 1
    return _lagrange_values(coarse_nodes, pts)


class Multigrid:
    """V-cycle preconditioned flexible CG for a structured ``LazyMatrix``.

    mode: "mixed" (FP32 V-cycle, FP64 outer CG) or "f64". basis: "gll",
    "equispaced" or "auto" (GLL from order 5 up). degree: Chebyshev smoothing
    steps per pre- and post-smoothing. h_levels: add Q1 levels on coarser
    meshes (default True) while every axis keeps at least ``min_cells`` cells.
    coarse_steps: Chebyshev steps on the coarsest level.
    """

    def __init__(self, A: LazyMatrix, mode: str = "mixed", basis: str = "auto", degree: int = 4,
                 ratio: float = 20.0, h_levels: bool = True, coarse_steps: int = 10,
                 min_cells: int = 8):
        if mode not in MODES:
            raise ValueError(f"mode must be one of {sorted(MODES)}")
        if A.gather != "structured" or A.m.D != 3:
            raise NotImplementedError("the multigrid hierarchy needs a 3D structured operator")
        p = A.m.order
        if basis == "auto":
            basis = "gll" if p >= 5 else "equispaced"
        if basis not in ("gll", "equispaced"):
            raise ValueError("basis must be 'gll', 'equispaced' or 'auto'")
        self.A, self.mode, self.basis = A, mode, basis
        fam = "gll" if basis == "gll" else "equispaced"
        nodes = (lambda q: _ascending(fem.gll_nodes(q))) if fam == "gll" else \
            (lambda q: np.linspace(0.0, 1.0, q + 1))
        # levels: (model, order, ratio to the previous level)
        levels = [(A.model, p, 1)]
        q = p
        while q > 1:
            q = max(1, q // 2)
            levels.append((A.model, q, 1))
        model = A.model
        if h_levels:
            while all(n % 2 == 0 and n // 2 >= min_cells for n in model.partition):
                model = model.coarsened()
                levels.append((model, 1, 2))
        self.levels = []
        for l, (mdl, q, _) in enumerate(levels):
            if l == 0 and fam == "equispaced":
                self.levels.append(A)
                continue
            m = SumFactorizationMap(3, (q,) * 3, (2 * q,) * 3, nodes=fam)
            V = fem.FESpace(mdl, q)
            same = l == 0 and m.quad_degree == A.m.quad_degree  # A's geometry, reused
            self.levels.append(LazyMatrix(m, V, V, fem.Measure(mdl, 2 * q),
                                          cell_quantities=A.cell_quantities if same else None))
        self.orders = [q for _, q, _ in levels]
        self.cells = [tuple(mdl.partition) for mdl, _, _ in levels]
        tables = []
        for (_, pf, _), (_, pc, r) in zip(levels[:-1], levels[1:]):
            tables.append(_f64(transfer_table(nodes(pf), nodes(pc), r)))
        self._tables = tables
        basis_tab = None
        if fam == "gll":  # levels[0]'s GLL basis functions at A's equispaced nodes
            basis_tab = _f64(_lagrange_values(nodes(p), np.linspace(0.0, 1.0, p + 1)))
        self._basis_tab = basis_tab
        self._specs = levels
        self._set_coefficients()
        ops = (C.c_void_p * len(self.levels))(*[L._h for L in self.levels])
        tab = (C.c_void_p * max(1, len(tables)))(*[t.ctypes.data for t in tables])
        for L in self.levels:  # tile shapes of the level kernels, picked once here
            L.autotune(torch.float32 if mode == "mixed" else torch.float64)
        h = C.c_void_p()
        st = lib.sf_mg_create(C.byref(h), A._h, len(self.levels), ops, tab,
                              C.c_void_p(basis_tab.ctypes.data) if basis_tab is not None else None)
        self._h = h
        if st != _lib.SF_OK:
            msg = (lib.sf_mg_last_error(h) or b"").decode()
            self.close()
            raise _lib.SumFacError(st, f"sf_mg_create: {msg}")
        self.set_option("degree", degree)
        self.set_option("ratio", ratio)
        self.set_option("coarse_steps", coarse_steps)

    def _set_coefficients(self):
        """A variable coefficient on the coarse levels: the operator's kappa itself on a
        level with its quadrature, else each cell's mean of it (averaged over the 8
        children of a coarse cell on the h-levels), constant over the level's points.
        Without kappa on the operator, none on the levels either."""
        A, levels = self.A, self._specs
        kap = A.kappa
        if kap is None:
            for L in self.levels:
                if L is not A and L.kappa is not None:
                    L.set_coefficient(None)
            return
        if not isinstance(kap, torch.Tensor):
            kap = torch.from_numpy(np.ascontiguousarray(kap))
        kap = kap.to("cuda", torch.float64)
        cell = kap.mean(dim=1)  # (ncells,), cells x fastest
        part = tuple(A.model.partition)
        for l, ((mdl, q, r), L) in enumerate(zip(levels, self.levels)):
            if L is A:
                continue
            if r == 2:  # the coarse cell's mean of its 8 children
                nx, ny, nz = part
                cell = cell.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).mean(dim=(1, 3, 5))
                cell = cell.reshape(-1).contiguous()
                part = (nx // 2, ny // 2, nz // 2)
            nq = L.m.SQ[0] ** 3
            if L.m.quad_degree == A.m.quad_degree and mdl is A.model:
                L.set_coefficient(kap)  # the same points: the operator's own kappa
            else:
                L.set_coefficient(cell[:, None].expand(-1, nq).contiguous())

    def refresh(self):
        """Follow a new coefficient on the operator (set_coefficient): the levels get
        its cell means and the library recomputes their diagonals and eigenvalue
        estimates; the hierarchy itself is kept."""
        self._set_coefficients()
        self._err(lib.sf_mg_refresh(self._h, _stream()), "sf_mg_refresh")

    def close(self):
        if getattr(self, "_h", None):
            lib.sf_mg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, st, what):
        if st != _lib.SF_OK:
            msg = (lib.sf_mg_last_error(self._h) or b"").decode()
            raise _lib.SumFacError(st, f"{what}: {msg}")

    def set_option(self, name: str, value: float):
        self._err(lib.sf_mg_set_option(self._h, name.encode(), float(value)), "sf_mg_set_option")

    def info(self, key: str) -> float:
        v = C.c_double()
        self._err(lib.sf_mg_get_info(self._h, key.encode(), C.byref(v)), "sf_mg_get_info")
        return v.value

    def lmax(self):
        return [self.info(f"lmax{l}") for l in range(len(self.levels))]

    def solve(self, b, x=None, reltol: float = 1e-10, maxiter: int = 500,
              raise_on_fail: bool = True):
        """x with ||b - A x|| <= reltol ||b|| (x: initial guess, zero by default).
        Returns (x, info) with info = {"iters", "relres", "converged"}."""
        if b.dtype != torch.float64 or not b.is_cuda or b.numel() != self.A.n:
            raise ValueError("b must be a float64 CUDA tensor of the operator's size")
        if x is None:
            x = torch.zeros_like(b)
        it, rel = C.c_int(), C.c_double()
        st = lib.sf_mg_cg(self._h, MODES[self.mode], C.c_void_p(b.data_ptr()),
                          C.c_void_p(x.data_ptr()), float(reltol), int(maxiter), C.byref(it),
                          C.byref(rel), _stream())
        if st != _lib.SF_OK and (raise_on_fail or st != _lib.SF_ERR_NOT_CONVERGED):
            self._err(st, "sf_mg_cg")
        return x, {"iters": it.value, "relres": rel.value, "converged": st == _lib.SF_OK}
