"""CPU oracle for the sum-factorized Laplacian apply (TEST INFRASTRUCTURE ONLY).

This module is the parity reference of the tests. Only ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.
The product path (the CUDA library and its Python host layer) never calls it.

It is an FP64 numpy restatement of JordiManyer/NCIHackaton2023.jl. The
reference is Julia, and Julia is not installed where this runs, so the
reference itself cannot be executed. Each function cites the reference
file:line whose behaviour it restates. Arithmetic that the reference gets
from its un-vendored Gridap.jl dependency (version unpinned: there is no
[compat] entry and Manifest.toml is git-ignored) is restated from the
published finite-element definitions, and each such place is flagged:

* The 1D Lagrange basis uses equispaced nodes on [0,1], ordered (vertex 0,
  vertex 1, interior ascending), as used at src/SumFactorizationMaps.jl:34-55.
* The quadrature is Gauss-Legendre on [0,1] with ceil((degree+1)/2) points,
  as used at src/SumFactorizationMaps.jl:51. The reference's own
  test/Demo_StepByStep.jl:19,53 pins degree 4 -> 3 points.
* Cell geometry: Jt = grad(cell_map) (Jt[i,j] = dx_j/dxi_i), jq = inv(Jt),
  djq = |det Jt|, as at src/LazyMatrices.jl:35-40.

Pinning status: the known-answer tests that the reference's own test
scripts hold for this path are reproduced in tests/test_oracle.py:

* the analytic flop model equals an operation count of the restated
  step-by-step loops (test/CompareFlops.jl:146-158);
* degree 4 gives 3 quadrature points per direction
  (test/Demo_StepByStep.jl:53);
* per-cell step-by-step equals evaluate! (test/Demo_StepByStep.jl:134-135);
* the sum-factorized apply equals the assembled sparse matvec
  (test/Demo.jl:54-57).

The assembled sparse stand-in is built here from full, non-factorized element
matrices. Bit-level parity with Gridap's own output is UNPINNED, because
Gridap cannot run here.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# ----------------------------------------------------------------------------
# 1D reference element: quadrature and Lagrange basis
# ----------------------------------------------------------------------------


def quad_npoints(degree: int) -> int:
    """Number of 1D Gauss points that Gridap's ``Quadrature(SEGMENT, degree)``
    uses (src/SumFactorizationMaps.jl:51): ceil((degree+1)/2).
    test/Demo_StepByStep.jl:19,53 pins degree 4 -> SQ = 3."""
    return int(math.ceil((degree + 1) / 2.0))


def gauss_legendre_01(npts: int):
    """Gauss-Legendre rule on [0,1], points ascending, weights summing to 1.

    Computed by Golub-Welsch: the eigenvalues of the symmetric Jacobi matrix
    of the Legendre recurrence. This is deliberately a different method from
    the product's host code, which uses numpy's ``leggauss``. Each point is
    then polished by Newton steps on P_n."""
    n = npts
    if n == 1:
        return np.array([0.5]), np.array([1.0])
    k = np.arange(1, n, dtype=np.float64)
    beta = k / np.sqrt(4.0 * k * k - 1.0)
    J = np.diag(beta, 1) + np.diag(beta, -1)
    vals, vecs = np.linalg.eigh(J)
    x = vals.copy()
    for _ in range(3):  # Newton polish on P_n(x) = 0 using the three-term recurrence
        p0 = np.ones_like(x)
        p1 = x.copy()
        for m in range(2, n + 1):
            p0, p1 = p1, ((2 * m - 1) * x * p1 - (m - 1) * p0) / m
        dp = n * (x * p1 - p0) / (x * x - 1.0)
        x = x - p1 / dp
    p0 = np.ones_like(x)
    p1 = x.copy()
    for m in range(2, n + 1):
        p0, p1 = p1, ((2 * m - 1) * x * p1 - (m - 1) * p0) / m
    dp = n * (x * p1 - p0) / (x * x - 1.0)
    w = 2.0 / ((1.0 - x * x) * dp * dp)
    order = np.argsort(x)
    return 0.5 * (x[order] + 1.0), 0.5 * w[order]


def lagrange_nodes_gridap(p: int) -> np.ndarray:
    """1D Lagrangian nodes in Gridap's SEGMENT order: vertex 0, vertex 1, then
    interior nodes ascending (the node order behind ``_get_terms`` at
    src/SumFactorizationMaps.jl:34-38)."""
    if p == 0:
        return np.array([0.5])
    return np.array([0.0, 1.0] + [i / p for i in range(1, p)])


def lagrange_eval(nodes: np.ndarray, pts: np.ndarray):
    """Values and first derivatives of the Lagrange polynomials of ``nodes`` at
    ``pts``, written out directly from the product formula. Returns
    (A0, B0) with A0[i, j] = phi_j(pts[i]) and B0[i, j] = phi_j'(pts[i])
    (src/SumFactorizationMaps.jl:53-54)."""
    nb = len(nodes)
    nq = len(pts)
    A = np.zeros((nq, nb))
    B = np.zeros((nq, nb))
    for j in range(nb):
        den = 1.0
        for m in range(nb):
            if m != j:
                den *= nodes[j] - nodes[m]
        for i in range(nq):
            x = pts[i]
            val = 1.0
            for m in range(nb):
                if m != j:
                    val *= x - nodes[m]
            A[i, j] = val / den
            d = 0.0
            for l in range(nb):
                if l == j:
                    continue
                t = 1.0
                for m in range(nb):
                    if m != j and m != l:
                        t *= x - nodes[m]
                d += t
            B[i, j] = d / den
    return A, B


# ----------------------------------------------------------------------------
# SumFactorizationMap restatement
# ----------------------------------------------------------------------------


@dataclass
class OracleMap:
    """Restates ``SumFactorizationMap{D,SB,SQ}`` (src/SumFactorizationMaps.jl:2-10,47-65).

    A0, B0: (SQ, SB) basis values / derivatives at the 1D quadrature points.
    gradMats[d][r] = A0 if d != r else B0 (src/SumFactorizationMaps.jl:57-58).
    dof_map: (SB^D, D) int array; row k is the tensor index (j1..jD, 0-based,
    positions in the 1D Gridap node order) of local dof k.
    w1d: 1D weights (SQ,)."""

    D: int
    p: int
    SB: int
    SQ: int
    A0: np.ndarray
    B0: np.ndarray
    w1d: np.ndarray
    q1d: np.ndarray
    dof_map: np.ndarray

    def grad_mat(self, d: int, r: int) -> np.ndarray:
        return self.A0 if d != r else self.B0


def make_map(D: int, p: int, quad_degree: int, local_perm: np.ndarray | None = None) -> OracleMap:
    """Restates ``SumFactorizationMap(D, fe_orders, quad_orders)``
    (src/SumFactorizationMaps.jl:47-65) for isotropic orders.

    The local HEX/QUAD node order is Gridap's (unpinned here). The oracle
    uses the tensor order j1 fastest, in 1D Gridap node positions, by default.
    Passing ``local_perm`` (a permutation of range(SB^D)) reorders the local
    dofs, to exercise arbitrary Gridap local orders through ``dof_map``."""
    nq = quad_npoints(quad_degree)
    q, w = gauss_legendre_01(nq)
    nodes = lagrange_nodes_gridap(p)
    A0, B0 = lagrange_eval(nodes, q)
    SB = p + 1
    grids = np.meshgrid(*([np.arange(SB)] * D), indexing="ij")
    # tensor order with j1 fastest: flatten index = j1 + SB*j2 + SB^2*j3
    tens = np.stack([g.transpose(*range(D - 1, -1, -1)).ravel() for g in grids], axis=1)
    if local_perm is not None:
        tens = tens[np.asarray(local_perm)]
    return OracleMap(D=D, p=p, SB=SB, SQ=nq, A0=A0, B0=B0, w1d=w, q1d=q, dof_map=tens)


# ----------------------------------------------------------------------------
# Per-cell evaluation (Arrays.evaluate!), vectorised over cells
# ----------------------------------------------------------------------------


def _contract(Z: np.ndarray, M: np.ndarray, axis: int) -> np.ndarray:
    """out[..., i, ...] = sum_j M[i, j] * Z[..., j, ...] along ``axis``."""
    out = np.tensordot(Z, M, axes=([axis], [1]))  # contracted axis moves to the end
    return np.moveaxis(out, -1, axis)


def array2tensor(m: OracleMap, xe: np.ndarray) -> np.ndarray:
    """Restates ``_sumfac_array2tensor!`` (src/SumFactorizationKernels.jl:135-151):
    copy the cell vector into each of the D components. xe: (ncells, SB^D).
    Returns Z of shape (ncells, D, SB, ..., SB) indexed [c, r, jD, ..., j1]."""
    nc = xe.shape[0]
    D, SB = m.D, m.SB
    T = np.zeros((nc,) + (SB,) * D)
    idx = tuple(m.dof_map[:, D - 1 - a] for a in range(D))  # axes ordered jD..j1
    T[(slice(None),) + idx] = xe
    return np.repeat(T[:, None], D, axis=1)


def tensor2array(m: OracleMap, Z: np.ndarray) -> np.ndarray:
    """Restates ``_sumfac_tensor2array!`` (src/SumFactorizationKernels.jl:156-172):
    y[k] = sum_r Z[r, dof_map[k]]."""
    D = m.D
    S = Z.sum(axis=1)
    idx = tuple(m.dof_map[:, D - 1 - a] for a in range(D))
    return S[(slice(None),) + idx]


def dof2quad(m: OracleMap, Z: np.ndarray) -> np.ndarray:
    """Restates the vector form of ``_sumfac_dof2quad!``
    (src/SumFactorizationKernels.jl:40-65): for d = 1..D and component k,
    Z[d+1][k, i1..id, j(d+1)..jD] = sum_jd gradMats[d,k][id, jd] * Z[d][k, ...].
    Z axes: [c, k, xD, ..., x1]; direction d lives on axis 2 + (D - d)."""
    D = m.D
    for d in range(1, D + 1):
        ax = 1 + (D - d)  # axis inside the per-component array [c, xD..x1]
        comps = []
        for k in range(1, D + 1):
            comps.append(_contract(Z[:, k - 1], m.grad_mat(d, k), ax))
        Z = np.stack(comps, axis=1)
    return Z


def quad2dof(m: OracleMap, Z: np.ndarray) -> np.ndarray:
    """Restates the vector form of ``_sumfac_quad2dof!``
    (src/SumFactorizationKernels.jl:105-130): directions d = D..1, with the
    transposed gradMats[d,k]."""
    D = m.D
    for d in range(D, 0, -1):
        ax = 1 + (D - d)
        comps = []
        for k in range(1, D + 1):
            comps.append(_contract(Z[:, k - 1], m.grad_mat(d, k).T, ax))
        Z = np.stack(comps, axis=1)
    return Z


def apply_weights(m: OracleMap, Z: np.ndarray, wq: np.ndarray, jq: np.ndarray,
                  djq: np.ndarray, kappa: np.ndarray | None = None) -> np.ndarray:
    """Restates ``_sumfac_apply_weights!`` (src/SumFactorizationKernels.jl:174-216):
    at each quadrature point (linear index i1 fastest)
    Z[r] <- wq * djq * sum_k (sum_l jq[l,r] * jq[l,k]) * Z[k].

    wq, djq: (ncells, SQ^D); jq: (ncells, SQ^D, D, D) with jq[..., l, r].
    ``kappa`` (ncells, SQ^D) optionally scales the tensor at each point (the
    variable-coefficient operator -div(kappa grad u); kappa = 1 is the
    reference's operator)."""
    D, SQ = m.D, m.SQ
    nc = Z.shape[0]
    Zf = Z.reshape(nc, D, SQ ** D)  # [c, r, q] with q = i1 + SQ*i2 + ... (C order of xD..x1)
    C = np.einsum("cqlr,cqlk->cqrk", jq, jq)
    s = wq * djq
    if kappa is not None:
        s = s * kappa
    out = np.einsum("cqrk,ckq->crq", C, Zf) * s[:, None, :]
    return out.reshape(Z.shape)


def evaluate_cells(m: OracleMap, xe: np.ndarray, wq, jq, djq, kappa=None) -> np.ndarray:
    """Restates ``Arrays.evaluate!(cache, m, x, wq, jq, djq)``
    (src/SumFactorizationMaps.jl:78-89) for a batch of cells:
    array2tensor -> dof2quad -> apply_weights -> quad2dof -> tensor2array."""
    Z = array2tensor(m, xe)
    Z = dof2quad(m, Z)
    Z = apply_weights(m, Z, wq, jq, djq, kappa)
    Z = quad2dof(m, Z)
    return tensor2array(m, Z)


# ----------------------------------------------------------------------------
# Cartesian model, FE space numbering and cell quantities
# ----------------------------------------------------------------------------


@dataclass
class OracleMesh:
    """A Cartesian mesh of [0,1]^D with n^D cells (cells numbered with x
    fastest), Q_p Lagrangian dofs and Dirichlet on the whole boundary
    (profiling/drivers.jl:7-17: CartesianDiscreteModel + FESpace with
    dirichlet_tags=["boundary"]).

    cell_dof_ids: (ncells, SB^D) int64, 1-based free ids (positive) and
    negative Dirichlet ids, in the local order of ``m.dof_map``
    (the convention read at test/Demo_StepByStep.jl:62-71). The global free
    numbering here is lexicographic over the interior grid (Gridap's own
    global numbering is unpinned)."""

    D: int
    n: tuple
    p: int
    vertices: np.ndarray        # (nverts, D) coordinates (possibly perturbed)
    cell_vertices: np.ndarray   # (ncells, 2^D) vertex ids, lexicographic x fastest
    cell_dof_ids: np.ndarray
    n_free: int
    n_dir: int
    free_grid_index: np.ndarray  # free id-1 -> global grid linear index (x fastest)
    affine: bool = True          # unperturbed Cartesian cells (all cells congruent)


def cartesian_mesh(D: int, n, p: int, m: OracleMap, perturb: float = 0.0, seed: int = 0,
                   renumber_seed: int | None = None) -> OracleMesh:
    if isinstance(n, int):
        n = (n,) * D
    n = tuple(n)
    N = tuple(ni * p for ni in n)  # dof grid has N+1 points per direction
    # vertices
    vgrids = np.meshgrid(*[np.linspace(0.0, 1.0, ni + 1) for ni in n], indexing="ij")
    verts = np.stack([g.transpose(*range(D - 1, -1, -1)).ravel() for g in vgrids], axis=1)
    vshape = tuple(ni + 1 for ni in n)
    if perturb > 0.0:
        rng = np.random.default_rng(seed)
        disp = rng.uniform(-perturb, perturb, size=verts.shape)
        vidx = np.stack(np.unravel_index(np.arange(len(verts)), vshape[::-1]), axis=1)[:, ::-1]
        interior = np.all((vidx > 0) & (vidx < np.array(n)), axis=1)
        h = np.array([1.0 / ni for ni in n])
        verts = verts + disp * h[None, :] * interior[:, None]
    # cells
    cgr = np.meshgrid(*[np.arange(ni) for ni in n], indexing="ij")
    cidx = np.stack([g.transpose(*range(D - 1, -1, -1)).ravel() for g in cgr], axis=1)  # (nc, D) c1 fastest
    corner = np.stack(np.meshgrid(*([np.arange(2)] * D), indexing="ij"), -1)
    corner = corner.transpose(*range(D - 1, -1, -1), D).reshape(-1, D)  # (2^D, D) x fastest

    def vlin(idx):
        lin = np.zeros(idx.shape[:-1], dtype=np.int64)
        stride = 1
        for a in range(D):
            lin += idx[..., a] * stride
            stride *= vshape[a]
        return lin

    cell_vertices = vlin(cidx[:, None, :] + corner[None, :, :])
    # dofs: 1D Gridap position j -> lexicographic offset t(j): 0 -> 0, 1 -> p, k>=2 -> k-1
    nodes = lagrange_nodes_gridap(p)
    off = np.rint(nodes * p).astype(np.int64)
    gshape = tuple(Ni + 1 for Ni in N)
    tens = m.dof_map  # (SB^D, D)
    gidx = cidx[:, None, :] * p + off[tens][None, :, :]  # (nc, nloc, D)
    glin = np.zeros(gidx.shape[:-1], dtype=np.int64)
    stride = 1
    for a in range(D):
        glin += gidx[..., a] * stride
        stride *= gshape[a]
    # free / dirichlet numbering, lexicographic
    all_idx = np.stack(np.unravel_index(np.arange(int(np.prod(gshape))), gshape[::-1]), axis=1)[:, ::-1]
    is_free = np.all((all_idx > 0) & (all_idx < np.array(N)), axis=1)
    ids = np.zeros(len(is_free), dtype=np.int64)
    nfree = int(is_free.sum())
    ndir = len(is_free) - nfree
    free_order = np.arange(1, nfree + 1)
    if renumber_seed is not None:
        free_order = np.random.default_rng(renumber_seed).permutation(nfree) + 1
    ids[is_free] = free_order
    ids[~is_free] = -np.arange(1, ndir + 1)
    free_grid_index = np.zeros(nfree, dtype=np.int64)
    free_grid_index[ids[is_free] - 1] = np.nonzero(is_free)[0]
    return OracleMesh(D=D, n=n, p=p, vertices=verts, cell_vertices=cell_vertices,
                      cell_dof_ids=ids[glin], n_free=nfree, n_dir=ndir,
                      free_grid_index=free_grid_index, affine=perturb == 0.0)


def cell_quantities(m: OracleMap, mesh: OracleMesh):
    """Restates the LazyMatrix constructor's geometric factors
    (src/LazyMatrices.jl:34-43): at each quadrature point of each cell,
    Jt = grad(cell_map) (multilinear map through the cell's vertices),
    jq = inv(Jt), djq = |det(Jt)|, and wq = the reference quadrature weights.
    Returns wq (nc, SQ^D), jq (nc, SQ^D, D, D), djq (nc, SQ^D).

    On an unperturbed Cartesian mesh every cell has the same factors, and
    Gridap returns Fill arrays (the ``.value`` read at test/GPU_v3.jl:66-68).
    Here the first cell's factors are then broadcast (read-only views)."""
    D, SQ = m.D, m.SQ
    q = m.q1d
    # reference-cell quadrature points, linear index i1 fastest
    qg = np.meshgrid(*([q] * D), indexing="ij")
    pts = np.stack([g.transpose(*range(D - 1, -1, -1)).ravel() for g in qg], axis=1)  # (nq, D)
    wg = np.meshgrid(*([m.w1d] * D), indexing="ij")
    w = np.ones(SQ ** D)
    for g in wg:
        w = w * g.transpose(*range(D - 1, -1, -1)).ravel()
    corner = np.stack(np.meshgrid(*([np.arange(2)] * D), indexing="ij"), -1)
    corner = corner.transpose(*range(D - 1, -1, -1), D).reshape(-1, D)
    # gradients of multilinear vertex shape functions at the points: dN[q, v, i]
    nq = len(pts)
    dN = np.zeros((nq, 2 ** D, D))
    for v in range(2 ** D):
        for i in range(D):
            val = np.ones(nq)
            for a in range(D):
                t = pts[:, a]
                if a == i:
                    val = val * (1.0 if corner[v, a] == 1 else -1.0)
                else:
                    val = val * (t if corner[v, a] == 1 else 1.0 - t)
            dN[:, v, i] = val
    nc = mesh.cell_vertices.shape[0]
    cv = mesh.cell_vertices[:1] if mesh.affine else mesh.cell_vertices
    X = mesh.vertices[cv]  # (nc or 1, 2^D, D)
    Jt = np.einsum("qvi,cvj->cqij", dN, X)  # Jt[i,j] = dx_j/dxi_i
    jq = np.linalg.inv(Jt)
    djq = np.abs(np.linalg.det(Jt))
    if mesh.affine:
        return (np.broadcast_to(w, (nc, nq)), np.broadcast_to(jq, (nc,) + jq.shape[1:]),
                np.broadcast_to(djq, (nc, nq)))
    return np.broadcast_to(w, (nc, nq)).copy(), jq, djq


# ----------------------------------------------------------------------------
# LazyMatrix mul! restatement and the assembled-sparse stand-in
# ----------------------------------------------------------------------------


def gather(mesh: OracleMesh, x: np.ndarray) -> np.ndarray:
    """scatter_free_and_dirichlet_values with Dirichlet zeros
    (src/LazyMatrices.jl:53; the negative-id rule at test/Demo_StepByStep.jl:64-71)."""
    ids = mesh.cell_dof_ids
    xe = np.where(ids > 0, x[np.maximum(ids, 1) - 1], 0.0)
    return xe


def assemble(mesh: OracleMesh, ye: np.ndarray) -> np.ndarray:
    """assemble_vector! into a zeroed y, skipping negative ids
    (src/LazyMatrices.jl:57-58; test/Demo_StepByStep.jl:143-146)."""
    ids = mesh.cell_dof_ids
    y = np.zeros(mesh.n_free)
    mask = ids > 0
    np.add.at(y, ids[mask] - 1, ye[mask])
    return y


def lazy_mul(m: OracleMap, mesh: OracleMesh, x: np.ndarray, cq=None, kappa=None,
             chunk: int = 32768) -> np.ndarray:
    """Restates ``LinearAlgebra.mul!(y, A::LazyMatrix, x)`` (src/LazyMatrices.jl:52-61)."""
    if cq is None:
        cq = cell_quantities(m, mesh)
    wq, jq, djq = cq
    xe = gather(mesh, x)
    ye = np.empty_like(xe)
    nc = xe.shape[0]
    for s in range(0, nc, chunk):
        e = min(nc, s + chunk)
        ye[s:e] = evaluate_cells(m, xe[s:e], wq[s:e], jq[s:e], djq[s:e],
                                 None if kappa is None else kappa[s:e])
    return assemble(mesh, ye)


def element_matrices(m: OracleMap, cq, kappa=None) -> np.ndarray:
    """Full (non-factorized) element stiffness matrices
    K_e[a, b] = sum_q wq djq kappa (jq grad_hat phi_a) . (jq grad_hat phi_b),
    with 3D basis gradients formed explicitly at each quadrature point. This
    is an independent path to the operator that ``AffineFEOperator`` assembles
    (profiling/drivers.jl:20-22) and that test/Demo.jl:54-57 compares against."""
    D, SB, SQ = m.D, m.SB, m.SQ
    wq, jq, djq = cq
    # reference gradients: G[q, a, i] = d phi_a / d xi_i at point q (tensor indices via dof_map)
    qi = np.stack(np.unravel_index(np.arange(SQ ** D), (SQ,) * D), axis=1)[:, ::-1]  # (nq, D) i1 first
    t = m.dof_map  # (nloc, D)
    G = np.ones((SQ ** D, SB ** D, D))
    for i in range(D):
        for a in range(D):
            M = m.B0 if a == i else m.A0
            G[:, :, i] *= M[qi[:, a][:, None], t[:, a][None, :]]
    # physical gradient: g_l = sum_r jq[l, r] * G[r]
    P = np.einsum("cqlr,qar->cqal", jq, G)
    s = wq * djq
    if kappa is not None:
        s = s * kappa
    nc, nq, na, _ = P.shape
    Ke = np.empty((nc, na, na))
    for c in range(nc):  # K_e = sum_q s_q P_q P_q^T as one BLAS product per cell
        Pc = P[c].transpose(1, 0, 2).reshape(na, nq * D)
        Ke[c] = (Pc * np.repeat(s[c], D)[None, :]) @ Pc.T
    return Ke


def assembled_sparse(m: OracleMap, mesh: OracleMesh, cq=None, kappa=None):
    """scipy CSR matrix over free dofs, assembled from ``element_matrices``."""
    import scipy.sparse as sp
    if cq is None:
        cq = cell_quantities(m, mesh)
    Ke = element_matrices(m, cq, kappa)
    ids = mesh.cell_dof_ids
    nloc = ids.shape[1]
    rows = np.repeat(ids[:, :, None], nloc, axis=2)
    cols = np.repeat(ids[:, None, :], nloc, axis=1)
    mask = (rows > 0) & (cols > 0)
    A = sp.coo_matrix((Ke[mask], (rows[mask] - 1, cols[mask] - 1)),
                      shape=(mesh.n_free, mesh.n_free)).tocsr()
    return A


# ----------------------------------------------------------------------------
# Adjoint form: derivative of ybar . A(kappa) x with respect to kappa
# ----------------------------------------------------------------------------


def kappa_vjp(m: OracleMap, mesh: OracleMesh, x: np.ndarray, ybar: np.ndarray, cq=None,
              chunk: int = 32768) -> np.ndarray:
    """kappa_bar[c, q] = d(ybar . A(kappa) x)/d kappa_q
    = wq djq sum_{r,k} (sum_l jq[l,r] jq[l,k]) (grad ybar)_r (grad x)_k, with the
    reference gradients at the points from the restated ``_sumfac_dof2quad!``
    (src/SumFactorizationKernels.jl:40-65) and the metric of
    ``_sumfac_apply_weights!`` (:174-216). Returns (ncells, SQ^D)."""
    if cq is None:
        cq = cell_quantities(m, mesh)
    wq, jq, djq = cq
    D, SQ = m.D, m.SQ
    xe, ye = gather(mesh, x), gather(mesh, ybar)
    nc = xe.shape[0]
    out = np.empty((nc, SQ ** D))
    for s in range(0, nc, chunk):
        e = min(nc, s + chunk)
        gx = dof2quad(m, array2tensor(m, xe[s:e])).reshape(e - s, D, SQ ** D)
        gy = dof2quad(m, array2tensor(m, ye[s:e])).reshape(e - s, D, SQ ** D)
        C = np.einsum("cqlr,cqlk->cqrk", jq[s:e], jq[s:e])
        out[s:e] = np.einsum("crq,cqrk,ckq->cq", gy, C, gx) * wq[s:e] * djq[s:e]
    return out


def adjoint_gradient_sparse(m: OracleMap, mesh: OracleMesh, b: np.ndarray, u_obs: np.ndarray,
                            kappa: np.ndarray, cq=None):
    """J(kappa) = 0.5 ||u - u_obs||^2 with A(kappa) u = b (sparse direct solves), and
    dJ/dkappa = -kappa_vjp(u, lambda) with A lambda = u - u_obs. Returns (J, grad, u)."""
    import scipy.sparse.linalg as spla
    if cq is None:
        cq = cell_quantities(m, mesh)
    A = assembled_sparse(m, mesh, cq, kappa).tocsc()
    lu = spla.splu(A)
    u = lu.solve(b)
    r = u - u_obs
    lam = lu.solve(r)
    return 0.5 * float(r @ r), -kappa_vjp(m, mesh, u, lam, cq), u


# ----------------------------------------------------------------------------
# Right-hand side, manufactured solution, Jacobi diagonal
# ----------------------------------------------------------------------------


def physical_points(m: OracleMap, mesh: OracleMesh) -> np.ndarray:
    """Coordinates of every cell's quadrature points, (nc, SQ^D, D)."""
    D, SQ = m.D, m.SQ
    q = m.q1d
    qg = np.meshgrid(*([q] * D), indexing="ij")
    pts = np.stack([g.transpose(*range(D - 1, -1, -1)).ravel() for g in qg], axis=1)
    corner = np.stack(np.meshgrid(*([np.arange(2)] * D), indexing="ij"), -1)
    corner = corner.transpose(*range(D - 1, -1, -1), D).reshape(-1, D)
    N = np.ones((len(pts), 2 ** D))
    for v in range(2 ** D):
        for a in range(D):
            N[:, v] *= pts[:, a] if corner[v, a] == 1 else 1.0 - pts[:, a]
    X = mesh.vertices[mesh.cell_vertices]
    return np.einsum("qv,cvj->cqj", N, X)


def rhs(m: OracleMap, mesh: OracleMesh, f, cq=None) -> np.ndarray:
    """b_i = integral of f * phi_i (the ``v -> int(v*f)dOmega`` form of
    profiling/drivers.jl:20), with homogeneous Dirichlet data."""
    D, SQ = m.D, m.SQ
    if cq is None:
        cq = cell_quantities(m, mesh)
    wq, jq, djq = cq
    xq = physical_points(m, mesh)
    fq = f(xq)  # (nc, nq)
    qi = np.stack(np.unravel_index(np.arange(SQ ** D), (SQ,) * D), axis=1)[:, ::-1]
    t = m.dof_map
    Phi = np.ones((SQ ** D, m.SB ** D))
    for a in range(D):
        Phi *= m.A0[qi[:, a][:, None], t[:, a][None, :]]
    be = np.einsum("cq,qa->ca", fq * wq * djq, Phi)
    return assemble(mesh, be)


def sin_solution(xq: np.ndarray) -> np.ndarray:
    return np.prod(np.sin(np.pi * xq), axis=-1)


def sin_forcing(xq: np.ndarray) -> np.ndarray:
    D = xq.shape[-1]
    return D * np.pi ** 2 * np.prod(np.sin(np.pi * xq), axis=-1)


def free_dof_coordinates(mesh: OracleMesh) -> np.ndarray:
    """Coordinates of the free dofs (Cartesian, unperturbed grid)."""
    D, p = mesh.D, mesh.p
    gshape = tuple(ni * p + 1 for ni in mesh.n)
    idx = np.stack(np.unravel_index(mesh.free_grid_index, gshape[::-1]), axis=1)[:, ::-1]
    return idx / np.array([ni * p for ni in mesh.n], dtype=np.float64)


def diagonal(m: OracleMap, mesh: OracleMesh, cq=None, kappa=None) -> np.ndarray:
    """diag(A) over free dofs, from the explicit element matrices."""
    if cq is None:
        cq = cell_quantities(m, mesh)
    Ke = element_matrices(m, cq, kappa)
    de = np.einsum("caa->ca", Ke)
    return assemble(mesh, de)


# ----------------------------------------------------------------------------
# Conjugate gradients (IterativeSolvers.cg!, called at profiling/drivers.jl:85-95)
# ----------------------------------------------------------------------------


def cg(apply, b: np.ndarray, x0=None, reltol=math.sqrt(np.finfo(np.float64).eps), abstol=0.0,
       maxiter=None, precond=None):
    """Restates the iteration of IterativeSolvers.jl's ``cg!`` (an
    un-vendored dependency, version unpinned): the tolerance is
    max(reltol * ||r0||, abstol) and the stopping test is ||r|| <= tol,
    checked before each iteration. ``precond`` is a callable applying P^-1
    (the ``Pl`` keyword). Returns (x, iterations, ||r||/||b||)."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - apply(x) if x0 is not None else b.copy()
    maxiter = len(b) if maxiter is None else maxiter
    res = np.linalg.norm(r)
    tol = max(reltol * res, abstol)
    u = np.zeros_like(b)
    it = 0
    if precond is None:
        prev = 1.0
        while it < maxiter and res > tol:
            beta = res ** 2 / prev ** 2
            u = r + beta * u
            c = apply(u)
            alpha = res ** 2 / np.dot(u, c)
            x += alpha * u
            r -= alpha * c
            prev = res
            res = np.linalg.norm(r)
            it += 1
    else:
        rho_prev = 1.0
        while it < maxiter and res > tol:
            z = precond(r)
            rho = np.dot(z, r)
            beta = rho / rho_prev
            u = z + beta * u
            c = apply(u)
            alpha = rho / np.dot(u, c)
            x += alpha * u
            r -= alpha * c
            rho_prev = rho
            res = np.linalg.norm(r)
            it += 1
    nb = np.linalg.norm(b)
    return x, it, res / (nb if nb > 0 else 1.0)


# ----------------------------------------------------------------------------
# Flop model (src/Utils.jl:33-72) and an operation count of the restated loops
# ----------------------------------------------------------------------------


def count_manual_flops_poisson_matrix_free(ncells, D, SQ, SB, count_only_fma_ops=True,
                                           structured_mesh_opt=True):
    """Restates the reference's analytic flop model (src/Utils.jl:33-72)."""
    SQ = tuple(SQ)
    SB = tuple(SB)
    b2 = 0
    for d in range(1, D + 1):
        b2 += D * int(np.prod(SQ[:d])) * int(np.prod(SB[d - 1:]))
    if not count_only_fma_ops:
        b2 *= 2
    if not structured_mesh_opt:
        b3 = (D - 1) * D ** D + D * D
        if not count_only_fma_ops:
            b3 = 2 * b3 + D ** D + 2 * D
    else:
        b3 = 0 if count_only_fma_ops else D
    b3 *= int(np.prod(SQ))
    b4 = b2
    return ncells * (b2 + b3 + b4)


class _Counted:
    """A float that counts additions and multiplications (a stand-in for the
    GFlops.jl counter used by test/CompareFlops.jl)."""

    adds = 0
    muls = 0

    def __init__(self, v):
        self.v = float(v)

    def __add__(self, o):
        _Counted.adds += 1
        return _Counted(self.v + (o.v if isinstance(o, _Counted) else o))

    __radd__ = __add__

    def __mul__(self, o):
        _Counted.muls += 1
        return _Counted(self.v * (o.v if isinstance(o, _Counted) else o))

    __rmul__ = __mul__


def count_step_by_step_ops_2d(m: OracleMap, ncells: int, structured_mesh_opt: bool):
    """Counts the additions and multiplications of the 2D step-by-step loops of
    test/CompareFlops.jl:36-106 (B.2 forward contractions, B.3 weights, B.4
    backward contractions), executed on ``_Counted`` numbers. Returns
    (adds, muls). The analytic model must match: adds == model(fma only),
    adds + muls == model(all flops) (test/CompareFlops.jl:150-157)."""
    D, SB, SQ = 2, m.SB, m.SQ
    mats = [[m.grad_mat(d, r) for r in (1, 2)] for d in (1, 2)]
    _Counted.adds = 0
    _Counted.muls = 0
    for _ in range(ncells):
        Z1 = [[[_Counted(1.0) for _ in range(SB)] for _ in range(SB)] for _ in range(D)]
        Z2 = [[[_Counted(0.0) for _ in range(SB)] for _ in range(SQ)] for _ in range(D)]
        Z3 = [[[_Counted(0.0) for _ in range(SQ)] for _ in range(SQ)] for _ in range(D)]
        for r in range(D):
            for i1 in range(SQ):
                for j1 in range(SB):
                    for j2 in range(SB):
                        Z2[r][i1][j2] = Z2[r][i1][j2] + _Counted(mats[0][r][i1, j1]) * Z1[r][j1][j2]
        for r in range(D):
            for i1 in range(SQ):
                for i2 in range(SQ):
                    for j2 in range(SB):
                        Z3[r][i1][i2] = Z3[r][i1][i2] + _Counted(mats[1][r][i2, j2]) * Z2[r][i1][j2]
        w = _Counted(0.5)
        if structured_mesh_opt:
            for i1 in range(SQ):
                for i2 in range(SQ):
                    for r in range(D):
                        Z3[r][i1][i2] = w * Z3[r][i1][i2]
        else:
            jq = [[_Counted(2.0), _Counted(0.0)], [_Counted(0.0), _Counted(2.0)]]
            for i1 in range(SQ):
                for i2 in range(SQ):
                    change = [[None, None], [None, None]]
                    for a in range(D):       # transpose(jq) . jq: D^2 dot products of length D
                        for b in range(D):
                            acc = jq[0][a] * jq[0][b]
                            for l in range(1, D):
                                acc = acc + jq[l][a] * jq[l][b]
                            change[a][b] = acc
                    cr = [_Counted(0.0) for _ in range(D)]
                    for r in range(D):
                        for k in range(D):
                            cr[r] = cr[r] + change[r][k] * Z3[k][i1][i2]
                    for r in range(D):
                        Z3[r][i1][i2] = w * w * cr[r]
        Z2 = [[[_Counted(0.0) for _ in range(SB)] for _ in range(SQ)] for _ in range(D)]
        Z1 = [[[_Counted(0.0) for _ in range(SB)] for _ in range(SB)] for _ in range(D)]
        for r in range(D):
            for i1 in range(SQ):
                for i2 in range(SQ):
                    for j2 in range(SB):
                        Z2[r][i1][j2] = Z2[r][i1][j2] + _Counted(mats[1][r][i2, j2]) * Z3[r][i1][i2]
        for r in range(D):
            for i1 in range(SQ):
                for j1 in range(SB):
                    for j2 in range(SB):
                        Z1[r][j1][j2] = Z1[r][j1][j2] + _Counted(mats[0][r][i1, j1]) * Z2[r][i1][j2]
    return _Counted.adds, _Counted.muls
