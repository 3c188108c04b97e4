"""The reference-facing operator API: SumFactorizationMap, LazyMatrix, mul!, cg!.

This mirrors the reference's Julia interface (src/NCIHackaton2023.jl:25-35):
``SumFactorizationMap(D, fe_orders, quad_orders)``,
``get_dimensional_parameters(m)``, ``LazyMatrix(m, trial, test, dOmega)`` and
``mul!(y, A, x)``. It adds the device CG driver that the reference ran on the
host through IterativeSolvers (profiling/drivers.jl:85-95). Every operator
action runs in libsfb200.so on the GPU. There is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from . import fem
from ._lib import check, lib

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dtype_code(t) -> int:
    if t == torch.float64:
        return _lib.SF_F64
    if t == torch.float32:
        return _lib.SF_F32
    raise TypeError(f"unsupported dtype {t}; use float64 or float32")


class SumFactorizationMap:
    """Restates ``SumFactorizationMap(D, fe_orders, quad_orders)``
    (src/SumFactorizationMaps.jl:47-65) for isotropic orders: the 1D basis
    values A0 and derivatives B0 at the 1D Gauss points, the gradient table
    gradMats[d][r] = (d != r) ? A0 : B0, and dof_map. quad_orders are
    quadrature DEGREES (Gridap convention: ceil((deg+1)/2) points)."""

    def __init__(self, D: int, fe_orders, quad_orders, nodes: str = "equispaced"):
        fe_orders = tuple(fe_orders)
        quad_orders = tuple(quad_orders)
        if D not in (2, 3):
            raise NotImplementedError("this library implements D = 2 and D = 3")
        if len(set(fe_orders)) != 1 or len(set(quad_orders)) != 1:
            raise NotImplementedError("anisotropic orders are not supported (the reference's "
                                      "to_gpu(::SumFactorizationMap) is isotropic too)")
        p = int(fe_orders[0])
        if not 1 <= p <= 9:
            raise ValueError("order p must be in 1..9")
        nq = fem.quadrature_npoints(int(quad_orders[0]))
        self.D = D
        self.order = p
        self.quad_degree = int(quad_orders[0])
        self.SB = (p + 1,) * D
        self.SQ = (nq,) * D
        self.points, self.weights = fem.gauss_legendre(nq)
        # "equispaced": Gridap's Lagrangian nodes (the reference's map). "gll":
        # Gauss-Lobatto nodes, the basis of the multigrid hierarchy of a
        # high-order space (same space, better conditioned basis).
        if nodes not in ("equispaced", "gll"):
            raise ValueError("nodes must be 'equispaced' or 'gll'")
        self.node_family = nodes
        self.nodes = fem.lagrange_nodes(p) if nodes == "equispaced" else fem.gll_nodes(p)
        self.A0, self.B0 = fem.lagrange_basis(self.nodes, self.points)
        self.dof_map = fem.hex_dof_map(p, D)
        self.node_order = fem.node_order(p)

    @property
    def gradMats(self):
        return [[self.A0 if d != r else self.B0 for r in range(self.D)] for d in range(self.D)]

    def _create_handle(self):
        h = C.c_void_p()
        A0 = _f64(self.A0.T)  # column-major SQ x SB
        B0 = _f64(self.B0.T)
        dm = _i32(self.dof_map.T)  # column-major (SB^D) x D
        st = lib.sf_create(C.byref(h), self.D, self.SB[0], self.SQ[0], _ptr(A0), _ptr(B0), _ptr(dm))
        check(st, None, "sf_create")
        return h


def get_dimensional_parameters(m: SumFactorizationMap):
    """(D, SB, SQ) of the map (src/SumFactorizationMaps.jl:15-17)."""
    return m.D, m.SB, m.SQ


class LazyMatrix:
    """Matrix-free operator over the free dofs (src/LazyMatrices.jl:1-61).

    ``gather`` selects how cells find their dofs: "structured" uses the
    implicit lexicographic numbering of the Cartesian model (the tiled
    kernels). "table" uploads get_cell_dof_ids as a Gridap Table, so that any
    global numbering works; a space with a renumbered global numbering uses
    the table unless "numbered" is asked for. "numbered" keeps the structured
    (tiled) kernels for a renumbered space of a Cartesian model: vectors in the
    space's numbering are permuted into lexicographic order and back around
    each apply, and once per solve in cg (sf_set_structured_numbering)."""

    def __init__(self, m: SumFactorizationMap, trial: fem.FESpace, test: fem.FESpace,
                 dOmega: fem.Measure, gather: str = "structured", cell_quantities=None):
        if trial is not test:
            raise NotImplementedError("trial and test spaces must be the same space")
        if dOmega.degree != m.quad_degree:
            raise ValueError("measure degree differs from the map's quadrature degree")
        if test.order != m.order:
            raise ValueError("space order differs from the map's order")
        self.m = m
        self.trial = trial
        self.test = test
        self.model = test.model
        self.n = test.num_free_dofs
        if gather == "numbered":
            self.gather = "numbered"
        else:
            self.gather = "table" if test.perm is not None else gather
        self._h = m._create_handle()
        try:
            if m.D != self.model.D:
                raise ValueError("the map's dimension differs from the model's")
            if self.gather == "structured":
                part = tuple(self.model.partition) + ((0,) if m.D == 2 else ())
                no = _i32(m.node_order)
                check(lib.sf_set_structured(self._h, *part, _ptr(no)), self._h, "sf_set_structured")
            elif self.gather == "numbered":
                if m.D != 3:
                    raise NotImplementedError("gather='numbered' is 3D only")
                no = _i32(m.node_order)
                ids = _i32(test.perm if test.perm is not None else np.arange(self.n))
                check(lib.sf_set_structured_numbering(self._h, *tuple(self.model.partition),
                                                      _ptr(no), _ptr(ids)),
                      self._h, "sf_set_structured_numbering")
            elif self.gather == "table":
                t = test.get_cell_dof_ids()
                ptrs, data = _i32(t.ptrs), _i32(t.data)
                check(lib.sf_set_cells(self._h, len(t), _ptr(ptrs), _ptr(data), self.n), self._h,
                      "sf_set_cells")
            else:
                raise ValueError("gather must be 'structured', 'table' or 'numbered'")
            # cell_quantities: (fill, wq, jq, djq) of another operator on the same model
            # and quadrature (the geometry does not depend on the basis), else computed here
            fill, wq, jq, djq = (cell_quantities if cell_quantities is not None else
                                 fem.cell_quantities(self.model, m.points, m.weights))
            self.cell_quantities = (fill, wq, jq, djq)
            wq, jq, djq = _f64(wq), _f64(jq), _f64(djq)
            check(lib.sf_set_cell_quantities(self._h, 1 if fill else 0, _ptr(wq), _ptr(jq), _ptr(djq)),
                  self._h, "sf_set_cell_quantities")
        except Exception:
            self.close()
            raise
        self.kappa = None

    # -- lifetime ---------------------------------------------------------
    def close(self):
        for mg in self.__dict__.pop("_mg", {}).values():  # they borrow this handle
            mg.close()
        if getattr(self, "_h", None):
            lib.sf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- AbstractMatrix-like ---------------------------------------------
    @property
    def shape(self):
        return (self.n, self.n)

    def size(self):
        return self.shape

    def __repr__(self):
        return f"{self.n}x{self.n} LazyMatrix{{Float64}}"

    def __matmul__(self, x):
        if torch is not None and isinstance(x, torch.Tensor):
            y = torch.empty_like(x)
        else:
            y = np.empty(self.n)
        return mul(y, self, x)

    # -- extras -----------------------------------------------------------
    def set_coefficient(self, kappa):
        """kappa at every quadrature point, shape (ncells, SQ^3), or None. A float64
        CUDA tensor is copied on the device; anything else is read on the host.
        Multigrid hierarchies kept for cg(mode="mg_...") follow the new coefficient
        (Multigrid.refresh)."""
        self._set_kappa(kappa)
        for mg in self.__dict__.get("_mg", {}).values():
            mg.refresh()

    def _set_kappa(self, kappa):
        if kappa is None:
            check(lib.sf_set_coefficient(self._h, None), self._h, "sf_set_coefficient")
            self.kappa = None
            return
        if torch is not None and isinstance(kappa, torch.Tensor) and kappa.is_cuda:
            if kappa.dtype != torch.float64 or tuple(kappa.shape) != (self.model.num_cells,
                                                                     self.m.SQ[0] ** 3):
                raise ValueError("kappa must be float64 with shape (ncells, SQ^3)")
            k = kappa.contiguous()
            check(lib.sf_set_coefficient_device(self._h, C.c_void_p(k.data_ptr()), _stream()),
                  self._h, "sf_set_coefficient_device")
            self.kappa = k
            return
        k = _f64(kappa)
        if k.shape != (self.model.num_cells, self.m.SQ[0] ** 3):
            raise ValueError("kappa must have shape (ncells, SQ^3)")
        check(lib.sf_set_coefficient(self._h, _ptr(k)), self._h, "sf_set_coefficient")
        self.kappa = k

    def kappa_vjp(self, x, ybar):
        """d(ybar . A(kappa) x)/d kappa at every quadrature point, (ncells, SQ^3) FP64:
        (grad ybar)^T G (grad x) per point, recomputed by sum factorization."""
        if x.dtype != ybar.dtype or x.numel() != self.n or ybar.numel() != self.n:
            raise ValueError("x and ybar must have the operator's size and one dtype")
        kb = torch.empty(self.model.num_cells, self.m.SQ[0] ** 3, dtype=torch.float64,
                         device=x.device)
        check(lib.sf_kappa_vjp(self._h, _dtype_code(x.dtype), C.c_void_p(x.contiguous().data_ptr()),
                               C.c_void_p(ybar.contiguous().data_ptr()), C.c_void_p(kb.data_ptr()),
                               _stream()), self._h, "sf_kappa_vjp")
        return kb

    def diagonal(self, dtype=None):
        """diag(A) as a device tensor."""
        dtype = dtype or torch.float64
        d = torch.empty(self.n, dtype=dtype, device="cuda")
        check(lib.sf_diagonal(self._h, _dtype_code(dtype), C.c_void_p(d.data_ptr()), _stream()),
              self._h, "sf_diagonal")
        return d

    def evaluate_cells(self, x_cells):
        """The Map protocol for a batch of cells: y_e = evaluate!(m, x_e, wq, jq, djq)
        for every cell (src/SumFactorizationMaps.jl:78-89). x_cells: device tensor
        (ncells, SB^3) in the local dof order."""
        x_cells = x_cells.contiguous()
        y = torch.empty_like(x_cells)
        check(lib.sf_evaluate_cells(self._h, _dtype_code(x_cells.dtype), x_cells.shape[0],
                                    C.c_void_p(x_cells.data_ptr()), C.c_void_p(y.data_ptr()),
                                    _stream()), self._h, "sf_evaluate_cells")
        return y

    def set_option(self, name: str, value: float):
        check(lib.sf_set_option(self._h, name.encode(), float(value)), self._h, "sf_set_option")

    def info(self, key: str) -> float:
        v = C.c_double()
        check(lib.sf_get_info(self._h, key.encode(), C.byref(v)), self._h, "sf_get_info")
        return v.value

    def autotune(self, dtype=None):
        """Time the tiled kernel's tile-shape candidates on this mesh and keep the
        fastest (no-op when the general element kernel is in use)."""
        dtype = dtype or torch.float64
        check(lib.sf_autotune(self._h, _dtype_code(dtype), _stream()), self._h, "sf_autotune")
        return self.kernel_name(dtype)

    def kernel_name(self, dtype=None) -> str:
        dtype = dtype or torch.float64
        return lib.sf_kernel_name(self._h, _dtype_code(dtype)).decode()

    def cg_kernel_name(self) -> str:
        """The iteration cg() runs in its FP64 modes: the fused CG kernel's tile
        shape, or the unfused apply + vector kernels."""
        return lib.sf_cg_kernel_name(self._h).decode()

    def uses_tiled_kernel(self) -> bool:
        return self.info("tiled_kernel") == 1.0

    def kernels_per_apply(self) -> int:
        return int(self.info("kernels_per_apply"))

    def last_solve_info(self):
        o, i, r = C.c_int(), C.c_int(), C.c_double()
        check(lib.sf_last_solve_info(self._h, C.byref(o), C.byref(i), C.byref(r)), self._h, "info")
        return {"outer": o.value, "inner": i.value, "relres": r.value}


def mul(y, A: LazyMatrix, x):
    """LinearAlgebra.mul!(y, A, x) (src/LazyMatrices.jl:52-61): y = A x.

    Device tensors (float64 or float32, same dtype) run on the current CUDA
    stream. numpy float64 arrays go through the host-buffer entry point
    (copy in, apply, copy out)."""
    if torch is not None and isinstance(x, torch.Tensor):
        if not (x.is_cuda and y.is_cuda):
            raise TypeError("x and y must both be CUDA tensors (or both numpy arrays)")
        if x.dtype != y.dtype or x.numel() != A.n or y.numel() != A.n:
            raise ValueError("x, y must have the operator's size and the same dtype")
        if not (x.is_contiguous() and y.is_contiguous()):
            raise ValueError("x and y must be contiguous")
        check(lib.sf_apply(A._h, _dtype_code(x.dtype), C.c_void_p(x.data_ptr()),
                           C.c_void_p(y.data_ptr()), _stream()), A._h, "sf_apply")
        return y
    xa = np.asarray(x)
    if xa.dtype != np.float64 or xa.shape != (A.n,) or not xa.flags.c_contiguous:
        raise ValueError("host x must be a contiguous float64 vector of the operator's size")
    if not (isinstance(y, np.ndarray) and y.dtype == np.float64 and y.shape == (A.n,)
            and y.flags.c_contiguous):
        raise ValueError("host y must be a contiguous float64 vector of the operator's size")
    check(lib.sf_mul_host(A._h, _ptr(xa), _ptr(y)), A._h, "sf_mul_host")
    return y


def mul_multi(Y, A: LazyMatrix, X):
    """Y[:, k] = A X[:, k] for every column k of (n, nrhs) column-major device
    tensors, i.e. tensors whose transpose is contiguous (nrhs, n)."""
    if X.shape != Y.shape or X.shape[0] != A.n:
        raise ValueError("X and Y must be (n, nrhs)")
    Xt, Yt = X.t(), Y.t()
    if not (Xt.is_contiguous() and Yt.is_contiguous()):
        raise ValueError("X and Y must be column-major (X.t() contiguous)")
    check(lib.sf_apply_multi(A._h, _dtype_code(X.dtype), X.shape[1], C.c_void_p(X.data_ptr()), A.n,
                             C.c_void_p(Y.data_ptr()), A.n, _stream()), A._h, "sf_apply_multi")
    return Y


CG_MODES = {"jacobi": _lib.SF_CG_F64, "f64": _lib.SF_CG_F64, "mixed": _lib.SF_CG_MIXED,
            "plain": _lib.SF_CG_F64_PLAIN}


def cg(A: LazyMatrix, b, x=None, reltol: float = 1e-10, maxiter: int | None = None,
       mode: str = "jacobi", raise_on_fail: bool = True):
    """Solve A x = b on the device (replaces IterativeSolvers.cg! at
    profiling/drivers.jl:85-95). b: float64 CUDA tensor. Returns (x, info)
    with info = {"iters", "relres", "outer", "inner"}. mode: "jacobi" (FP64
    Jacobi CG), "plain" (FP64 CG, no preconditioner), "mixed" (FP32 apply
    and inner CG with FP64 outer refinement), or "mg_mixed" / "mg_f64" (FP64
    flexible CG preconditioned by a multigrid V-cycle in FP32 / FP64, structured
    meshes; the hierarchy is built on the first such call and kept on A)."""
    if mode in ("mg_mixed", "mg_f64"):
        from .multigrid import Multigrid
        cache = A.__dict__.setdefault("_mg", {})
        if mode not in cache:
            cache[mode] = Multigrid(A, mode=mode[3:])
        x, info = cache[mode].solve(b, x=x, reltol=reltol,
                                    maxiter=500 if maxiter is None else int(maxiter),
                                    raise_on_fail=raise_on_fail)
        info.update({"outer": 1, "inner": info["iters"]})
        return x, info
    if mode not in CG_MODES:
        raise ValueError(f"mode must be one of {sorted(CG_MODES) + ['mg_f64', 'mg_mixed']}")
    if b.dtype != torch.float64 or not b.is_cuda or b.numel() != A.n:
        raise ValueError("b must be a float64 CUDA tensor of the operator's size")
    if x is None:
        x = torch.zeros_like(b)
    maxiter = A.n if maxiter is None else int(maxiter)
    it = C.c_int()
    rel = C.c_double()
    st = lib.sf_cg(A._h, CG_MODES[mode], C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()),
                   float(reltol), maxiter, C.byref(it), C.byref(rel), _stream())
    info = A.last_solve_info()
    info["iters"] = it.value
    if st != _lib.SF_OK and (raise_on_fail or st != _lib.SF_ERR_NOT_CONVERGED):
        check(st, A._h, "sf_cg")
    info["converged"] = st == _lib.SF_OK
    return x, info


def quadrature_points(A: LazyMatrix, device=None) -> "torch.Tensor":
    """(ncells, SQ^3, 3) physical coordinates of every cell's quadrature points
    (trilinear cell map, point index i1 fastest), computed on ``device``."""
    device = device or torch.device("cuda")
    q1 = torch.as_tensor(np.asarray(A.m.points), dtype=torch.float64)
    qz, qy, qx = torch.meshgrid(q1, q1, q1, indexing="ij")
    pts = torch.stack([qx.reshape(-1), qy.reshape(-1), qz.reshape(-1)], dim=1)
    N = torch.ones(pts.shape[0], 8, dtype=torch.float64)
    for v in range(8):
        for a, bit in enumerate(((v & 1), (v >> 1) & 1, (v >> 2) & 1)):
            N[:, v] *= pts[:, a] if bit else 1.0 - pts[:, a]
    X = torch.as_tensor(A.model.vertices[A.model.cell_vertices()], dtype=torch.float64)
    return torch.einsum("qv,cvj->cqj", N.to(device), X.to(device))


def rhs(A: LazyMatrix, f) -> "torch.Tensor":
    """b_i = integral of f phi_i (homogeneous Dirichlet data) on the device, by the
    matrix-free kernel behind sf_rhs. ``f``: a (ncells, SQ^3) float64 CUDA tensor of
    values at the quadrature points, or a function mapping a (..., 3) coordinate
    tensor to values (evaluated at ``quadrature_points(A)``)."""
    if callable(f):
        f = f(quadrature_points(A))
    fq = f.contiguous()
    nq = A.m.SQ[0] ** 3
    if fq.dtype != torch.float64 or not fq.is_cuda or fq.numel() != A.model.num_cells * nq:
        raise ValueError("f at the points must be a float64 CUDA tensor of shape (ncells, SQ^3)")
    b = torch.empty(A.n, dtype=torch.float64, device=fq.device)
    check(lib.sf_rhs(A._h, C.c_void_p(fq.data_ptr()), C.c_void_p(b.data_ptr()), _stream()), A._h,
          "sf_rhs")
    return b


def assemble_rhs(m: SumFactorizationMap, V: fem.FESpace, f, chunk: int = 32768) -> np.ndarray:
    """b_i = integral of f phi_i over the mesh with homogeneous Dirichlet data (the
    linear form ``v -> int(v*f)dOmega`` of profiling/drivers.jl:20), formed on
    the host by sum factorization over the cells. f maps (..., 3) coordinates
    to values."""
    model = V.model
    SQ, SB = m.SQ[0], m.SB[0]
    fill, wq, jq, djq = fem.cell_quantities(model, m.points, m.weights)
    nc = model.num_cells
    ids = V.get_cell_dof_ids().data.reshape(nc, SB ** 3)
    A = m.A0
    b = np.zeros(V.num_free_dofs)
    for s in range(0, nc, chunk):
        e = min(nc, s + chunk)
        xq = fem.physical_quadrature_points(model, m.points, cells=slice(s, e))
        w = (wq * djq) if fill else (wq[s:e] * djq[s:e])
        F = (f(xq) * w).reshape(e - s, SQ, SQ, SQ)  # [c, qz, qy, qx]
        T = np.einsum("cZYX,Xi->cZYi", F, A)
        T = np.einsum("cZYi,Yj->cZji", T, A)
        T = np.einsum("cZji,Zk->ckji", T, A)  # tensor order, j1 fastest (hex_dof_map order)
        be = T.reshape(e - s, SB ** 3)
        idc = ids[s:e]
        mask = idc > 0
        b += np.bincount(idc[mask] - 1, weights=be[mask], minlength=V.num_free_dofs)
    return b
