"""Pins the FP64 oracle to the reference's own known-answer tests, and to
mathematical identities of the operator (CPU only)."""
import os

import numpy as np
import pytest

from oracle import cref
from oracle import sumfac_oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("degree,npts", [(0, 1), (1, 1), (2, 2), (3, 2), (4, 3), (6, 4), (8, 5), (16, 9)])
def test_quadrature_points_from_degree(degree, npts):
    # test/Demo_StepByStep.jl:19,53 pins degree 4 -> SQ = 3
    assert O.quad_npoints(degree) == npts


@pytest.mark.parametrize("n", [1, 2, 3, 5, 9])
def test_gauss_legendre_exactness(n):
    x, w = O.gauss_legendre_01(n)
    assert np.all(np.diff(x) > 0) and abs(w.sum() - 1) < 1e-15
    for k in range(2 * n):
        assert abs(np.dot(w, x ** k) - 1.0 / (k + 1)) < 1e-14


def test_lagrange_basis_is_nodal_and_consistent():
    for p in range(1, 9):
        nodes = O.lagrange_nodes_gridap(p)
        A, B = O.lagrange_eval(nodes, nodes)
        assert np.allclose(A, np.eye(p + 1), atol=1e-13)
        q, _ = O.gauss_legendre_01(p + 2)
        A, B = O.lagrange_eval(nodes, q)
        assert np.allclose(A.sum(1), 1.0, atol=1e-13)   # partition of unity
        assert np.allclose(B.sum(1), 0.0, atol=1e-10)
        assert np.allclose(A @ nodes, q, atol=1e-13)    # reproduces x
        assert np.allclose(B @ nodes, 1.0, atol=1e-10)


@pytest.mark.parametrize("structured", [True, False])
def test_flop_model_matches_operation_count(structured):
    # test/CompareFlops.jl:146-158: D=2, p=1, quad degree 4, 16 cells
    m = O.make_map(2, 1, 4)
    adds, muls = O.count_step_by_step_ops_2d(m, 16, structured)
    assert adds == O.count_manual_flops_poisson_matrix_free(16, 2, (3, 3), (2, 2), True, structured)
    assert adds + muls == O.count_manual_flops_poisson_matrix_free(16, 2, (3, 3), (2, 2), False,
                                                                   structured)


def test_flop_model_values():
    f = O.count_manual_flops_poisson_matrix_free
    assert f(1, 3, (3,) * 3, (3,) * 3, False, True) == 2997
    assert f(1, 3, (4,) * 3, (4,) * 3, False, True) == 9408
    assert f(1, 3, (5,) * 3, (5,) * 3, False, True) == 22875
    assert f(64 ** 3, 3, (5,) * 3, (5,) * 3, False, True) == 5_996_544_000
    assert f(1, 3, (9,) * 3, (9,) * 3, False, False) == 352107


def test_step_by_step_equals_evaluate_2d():
    """test/Demo_StepByStep.jl:53-135: the hand-written 2D loops (p=1, degree 4)
    per cell equal evaluate!(m, x, wq, jq, djq)."""
    m = O.make_map(2, 1, 4)
    mesh = O.cartesian_mesh(2, 4, 1, m)
    wq, jq, djq = O.cell_quantities(m, mesh)
    rng = np.random.default_rng(3)
    xe = rng.uniform(-1, 1, (mesh.cell_dof_ids.shape[0], 4))
    ye = O.evaluate_cells(m, xe, wq, jq, djq)
    SQ, SB, D = 3, 2, 2
    mats = [[m.grad_mat(d, r) for r in (1, 2)] for d in (1, 2)]
    for c in range(xe.shape[0]):
        Z1 = np.zeros((D, SB, SB))
        for i, (j1, j2) in enumerate(m.dof_map):
            Z1[:, j1, j2] = xe[c, i]
        Z2 = np.zeros((D, SQ, SB))
        for r in range(D):
            for i1 in range(SQ):
                for j1 in range(SB):
                    for j2 in range(SB):
                        Z2[r, i1, j2] += mats[0][r][i1, j1] * Z1[r, j1, j2]
        Z3 = np.zeros((D, SQ, SQ))
        for r in range(D):
            for i1 in range(SQ):
                for i2 in range(SQ):
                    for j2 in range(SB):
                        Z3[r, i1, i2] += mats[1][r][i2, j2] * Z2[r, i1, j2]
        for i1 in range(SQ):
            for i2 in range(SQ):
                idx = i2 * SQ + i1
                J = jq[c, idx]
                change = J.T @ J
                cr = change @ Z3[:, i1, i2]
                Z3[:, i1, i2] = wq[c, idx] * djq[c, idx] * cr
        Z2 = np.zeros((D, SQ, SB))
        for r in range(D):
            for i1 in range(SQ):
                for i2 in range(SQ):
                    for j2 in range(SB):
                        Z2[r, i1, j2] += mats[1][r][i2, j2] * Z3[r, i1, i2]
        Z1 = np.zeros((D, SB, SB))
        for r in range(D):
            for i1 in range(SQ):
                for j1 in range(SB):
                    for j2 in range(SB):
                        Z1[r, j1, j2] += mats[0][r][i1, j1] * Z2[r, i1, j2]
        yi = np.array([Z1[:, j1, j2].sum() for (j1, j2) in m.dof_map])
        assert np.allclose(yi, ye[c], rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("D,p,deg,n", [(3, 4, 6, 4), (3, 2, 4, 5), (2, 1, 4, 4), (2, 3, 6, 5),
                                       (3, 1, 2, 3), (3, 3, 4, 3)])
def test_sumfac_equals_assembled_sparse(D, p, deg, n):
    """test/Demo.jl:54-57 (x = ones, p=4, degree 6) and seeded random inputs."""
    m = O.make_map(D, p, deg)
    mesh = O.cartesian_mesh(D, n, p, m)
    A = O.assembled_sparse(m, mesh)
    for x in (np.ones(mesh.n_free), np.random.default_rng(0).uniform(-1, 1, mesh.n_free)):
        y1 = A @ x
        y2 = O.lazy_mul(m, mesh, x)
        assert np.linalg.norm(y1 - y2) < 1e-6  # the reference's own bar
        assert np.abs(y1 - y2).max() <= 1e-13 * np.abs(y1).max()


def test_local_dof_order_is_irrelevant():
    """Any Gridap local dof order (dof_map) gives the same global operator."""
    p, deg, n = 3, 6, 3
    m0 = O.make_map(3, p, deg)
    perm = np.random.default_rng(4).permutation((p + 1) ** 3)
    m1 = O.make_map(3, p, deg, local_perm=perm)
    x = np.random.default_rng(5).uniform(-1, 1, (n * p - 1) ** 3)
    y0 = O.lazy_mul(m0, O.cartesian_mesh(3, n, p, m0), x)
    y1 = O.lazy_mul(m1, O.cartesian_mesh(3, n, p, m1), x)
    assert np.abs(y0 - y1).max() <= 1e-14 * np.abs(y0).max()


@pytest.mark.parametrize("case", [("c1_q2_n8", (2, 4, 8, 0.0, 0)), ("q4_deg6_n3", (4, 6, 3, 0.0, 0)),
                                  ("deformed_q4_n3", (4, 8, 3, 0.2, 5))])
def test_c_restatement_and_golden(case):
    name, (p, deg, n, pert, ps) = case
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    m = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, m, perturb=pert, seed=ps)
    cq = O.cell_quantities(m, mesh)
    y = O.lazy_mul(m, mesh, g["x"], cq)
    assert np.abs(y - g["y"]).max() <= 1e-14 * np.abs(g["y"]).max()
    yc = cref.problem_from_oracle(m, mesh, cq).mul(g["x"])
    assert np.abs(yc - g["y"]).max() <= 1e-14 * np.abs(g["y"]).max()
    yc4 = cref.problem_from_oracle(m, mesh, cq).mul(g["x"], nthreads=4)
    # the threaded variant visits cells colour by colour: same sums, other order
    assert np.abs(yc4 - yc).max() <= 1e-14 * np.abs(g["y"]).max()


def test_energy_identity_polynomial():
    """u^T A u = int |grad u|^2 exactly for u = x(1-x)y(1-y)z(1-z) in Q2 (= 1/900)."""
    for p, n in [(2, 1), (2, 3), (3, 2)]:
        m = O.make_map(3, p, 2 * p)
        mesh = O.cartesian_mesh(3, n, p, m)
        X = O.free_dof_coordinates(mesh)
        u = np.prod(X * (1 - X), axis=1)
        y = O.lazy_mul(m, mesh, u)
        assert abs(u @ y - 1.0 / 900.0) < 1e-15


def test_spd_and_neumann_rowsums():
    m = O.make_map(3, 2, 4)
    mesh = O.cartesian_mesh(3, 3, 2, m, perturb=0.15, seed=1)
    A = O.assembled_sparse(m, mesh).toarray()
    assert np.abs(A - A.T).max() < 1e-14 * np.abs(A).max()
    np.linalg.cholesky(A)
    Ke = O.element_matrices(m, O.cell_quantities(m, mesh))
    assert np.abs(Ke.sum(axis=2)).max() < 1e-13 * np.abs(Ke).max()  # A . 1 = 0 without Dirichlet


def test_affine_scaling():
    """Scaling the domain by s scales the 3D Laplacian by s."""
    m = O.make_map(3, 3, 6)
    mesh = O.cartesian_mesh(3, 2, 3, m)
    x = np.random.default_rng(0).uniform(-1, 1, mesh.n_free)
    y1 = O.lazy_mul(m, mesh, x)
    mesh.vertices = mesh.vertices * 2.5
    y2 = O.lazy_mul(m, mesh, x)
    assert np.abs(y2 - 2.5 * y1).max() < 1e-13 * np.abs(y2).max()


def test_cg_restatement_solves():
    import scipy.sparse.linalg as spla
    m = O.make_map(3, 2, 4)
    mesh = O.cartesian_mesh(3, 4, 2, m)
    A = O.assembled_sparse(m, mesh)
    b = O.rhs(m, mesh, O.sin_forcing)
    xs = spla.spsolve(A.tocsc(), b)
    x, it, rel = O.cg(lambda v: A @ v, b, reltol=1e-12)
    assert rel <= 1e-12 and np.abs(x - xs).max() < 1e-10 * np.abs(xs).max()
    d = A.diagonal()
    x2, it2, rel2 = O.cg(lambda v: A @ v, b, reltol=1e-12, precond=lambda r: r / d)
    assert rel2 <= 1e-12 and np.abs(x2 - xs).max() < 1e-10 * np.abs(xs).max()


def test_manufactured_solution_converges():
    """CG on the manufactured u = sin(pi x) sin(pi y) sin(pi z): the nodal error
    drops at least like h^(p+1)."""
    errs = []
    for n in (2, 4):
        m = O.make_map(3, 2, 6)
        mesh = O.cartesian_mesh(3, n, 2, m)
        A = O.assembled_sparse(m, mesh)
        b = O.rhs(m, mesh, O.sin_forcing)
        x, _, _ = O.cg(lambda v: A @ v, b, reltol=1e-13)
        X = O.free_dof_coordinates(mesh)
        errs.append(np.abs(x - O.sin_solution(X)).max())
    assert errs[1] < errs[0] / 6.0


def test_kappa_vjp_is_the_derivative():
    """ybar . A(kappa) x is linear in kappa, so the VJP is exact: for any
    direction d, ybar . (A(kappa + d) - A(kappa)) x = kappa_bar . d."""
    m = O.make_map(3, 2, 4)
    mesh = O.cartesian_mesh(3, 3, 2, m, perturb=0.15, seed=2)
    cq = O.cell_quantities(m, mesh)
    rng = np.random.default_rng(0)
    nq = m.SQ ** 3
    nc = mesh.cell_dof_ids.shape[0]
    kappa = np.exp(rng.normal(0, 0.5, (nc, nq)))
    d = rng.normal(0, 1, (nc, nq))
    x = rng.uniform(-1, 1, mesh.n_free)
    yb = rng.uniform(-1, 1, mesh.n_free)
    kb = O.kappa_vjp(m, mesh, x, yb, cq)
    lhs = yb @ (O.lazy_mul(m, mesh, x, cq, kappa + d) - O.lazy_mul(m, mesh, x, cq, kappa))
    assert abs(lhs - np.sum(kb * d)) < 1e-12 * abs(lhs)


def test_adjoint_gradient_matches_finite_differences():
    m = O.make_map(3, 2, 4)
    mesh = O.cartesian_mesh(3, 3, 2, m)
    cq = O.cell_quantities(m, mesh)
    rng = np.random.default_rng(1)
    nc, nq = mesh.cell_dof_ids.shape[0], m.SQ ** 3
    kappa = np.exp(rng.normal(0, 0.5, (nc, nq)))
    kappa_true = np.exp(rng.normal(0, 0.5, (nc, nq)))
    b = O.rhs(m, mesh, O.sin_forcing, cq)
    _, _, u_obs = O.adjoint_gradient_sparse(m, mesh, b, np.zeros(mesh.n_free), kappa_true, cq)
    J, g, _ = O.adjoint_gradient_sparse(m, mesh, b, u_obs, kappa, cq)
    d = rng.normal(0, 1, (nc, nq))
    eps = 1e-6
    Jp = O.adjoint_gradient_sparse(m, mesh, b, u_obs, kappa + eps * d, cq)[0]
    Jm = O.adjoint_gradient_sparse(m, mesh, b, u_obs, kappa - eps * d, cq)[0]
    fd = (Jp - Jm) / (2 * eps)
    assert abs(fd - np.sum(g * d)) < 1e-6 * abs(fd)


def test_bench_flop_constants_match_the_reference_model():
    """The flop figures bench.py reports come from the reference's model
    (src/Utils.jl:33-72): Q4 affine (5.997 GFLOP per 64^3 apply) and Q8 deformed."""
    import bench
    f = O.count_manual_flops_poisson_matrix_free
    assert bench.Q8_DEFORMED_FLOPS_PER_CELL == f(1, 3, (9,) * 3, (9,) * 3, count_only_fma_ops=False,
                                                 structured_mesh_opt=False)
    assert abs(64 ** 3 * f(1, 3, (5,) * 3, (5,) * 3, count_only_fma_ops=False,
                           structured_mesh_opt=True) / 1e9 - 5.996544) < 1e-9
