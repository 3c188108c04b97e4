"""Batched form: many independent problems, several right-hand sides each, in
one CUDA-graph launch (sf_batch_* in include/sfb200.h).

The reference applied one problem per kernel launch (test/GPU_v3.jl:79-84).
Here the problems are grouped by order. Each group is one persistent kernel
over its (problem, right-hand side, tile) work items, and the groups are
concurrent branches of one captured graph. ``autotune`` picks each group's
tile shape (cells per CTA, threads) per dtype by timing.
"""
from __future__ import annotations

import ctypes as C

from ._lib import SumFacError, lib
from .operator import LazyMatrix, _dtype_code, _stream

import torch


def _check(status, b, what):
    if status != 0:
        raw = lib.sf_batch_last_error(b)
        raise SumFacError(status, f"{what}: {lib.sf_status_string(status).decode()} "
                                  f"({raw.decode() if raw else ''})")


class Batch:
    """ops: LazyMatrix handles on which the tiled Cartesian kernel is in use.
    X[i], Y[i]: (n_i, nrhs) column-major CUDA tensors (X[i].t() contiguous)."""

    def __init__(self, ops: list[LazyMatrix], nrhs: int):
        self.ops = list(ops)
        self.nrhs = int(nrhs)
        arr = (C.c_void_p * len(self.ops))(*[op._h for op in self.ops])
        h = C.c_void_p()
        st = lib.sf_batch_create(C.byref(h), len(self.ops), arr, self.nrhs)
        if st != 0:
            raise SumFacError(st, f"sf_batch_create: {lib.sf_status_string(st).decode()}")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.sf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ngroups(self) -> int:
        n = C.c_int()
        lib.sf_batch_groups(self._h, C.byref(n))
        return n.value

    def group_kernel(self, dtype, g: int) -> str:
        return lib.sf_batch_group_kernel(self._h, _dtype_code(dtype), g).decode()

    def _ptrs(self, X, Y):
        if len(X) != len(self.ops) or len(Y) != len(self.ops):
            raise ValueError("one X and one Y per problem")
        dt = X[0].dtype
        for op, x, y in zip(self.ops, X, Y):
            if x.dtype != dt or y.dtype != dt:
                raise ValueError("all vectors must share one dtype")
            if tuple(x.shape) != (op.n, self.nrhs) or tuple(y.shape) != (op.n, self.nrhs):
                raise ValueError("X[i], Y[i] must be (n_i, nrhs)")
            if not (x.t().is_contiguous() and y.t().is_contiguous()):
                raise ValueError("X[i], Y[i] must be column-major (x.t() contiguous)")
        xs = (C.c_void_p * len(X))(*[x.data_ptr() for x in X])
        ys = (C.c_void_p * len(Y))(*[y.data_ptr() for y in Y])
        return _dtype_code(dt), xs, ys

    def apply(self, X, Y):
        """Y[i] = A_i X[i] for every problem, one graph launch on the current stream."""
        code, xs, ys = self._ptrs(X, Y)
        _check(lib.sf_batch_apply(self._h, code, xs, ys, _stream()), self._h, "sf_batch_apply")
        return Y

    def autotune(self, X, Y):
        code, xs, ys = self._ptrs(X, Y)
        _check(lib.sf_batch_autotune(self._h, code, xs, ys, _stream()), self._h, "sf_batch_autotune")
        return [self.group_kernel(X[0].dtype, g) for g in range(self.ngroups)]


def column_major(n: int, nrhs: int, dtype=torch.float64, device="cuda"):
    """An (n, nrhs) column-major tensor (its transpose is contiguous)."""
    return torch.empty(nrhs, n, dtype=dtype, device=device).t()


def apply_cost(n_cells: int, p: int, nrhs: int = 1) -> float:
    """Work estimate of one problem's batched apply: its dofs times an order factor
    (the tiled kernel's FP64 time per dof grows with p, roughly like (p + 1)),
    times the right-hand sides."""
    return float(n_cells) * p ** 3 * (p + 1) * nrhs


def shard(costs, nranks: int) -> list[list[int]]:
    """Indices of independent problems dealt to ``nranks`` ranks, balanced by cost:
    largest first, each to the currently lightest rank (ties: lowest rank). The
    problems share nothing, so each rank then runs its own Batch with no exchange.
    Deterministic, so every rank computes the same assignment."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * nranks
    out: list[list[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]

