"""Multigrid-preconditioned CG (sf_mg_*) through the C ABI.

The solution is checked against a sparse direct solve of the oracle's
assembled matrix (the stand-in for Gridap's assembled operator), and its
residual against the oracle's restatement of the reference apply. The
iteration counts are bounded: the point of the preconditioner is that they
stay small where Jacobi CG needs hundreds or thousands."""
import numpy as np
import pytest

from oracle import sumfac_oracle as O

pytestmark = pytest.mark.gpu


def _setup(sf, p, n, perturb=0.0, seed=5):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n), perturb=perturb, seed=seed)
    V = sf.FESpace(model, p)
    m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, 2 * p))
    om = O.make_map(3, p, 2 * p)
    mesh = O.cartesian_mesh(3, n, p, om, perturb=perturb, seed=seed)
    return A, om, mesh


def _check_solution(om, mesh, b, x, tol):
    import scipy.sparse.linalg as spla
    As = O.assembled_sparse(om, mesh).tocsc()
    x_ref = spla.spsolve(As, b)
    r = b - O.lazy_mul(om, mesh, x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-9
    assert np.abs(x - x_ref).max() / np.abs(x_ref).max() < tol


@pytest.mark.parametrize("mode", ["mixed", "f64"])
@pytest.mark.parametrize("rough", [False, True])
def test_mg_cartesian_q4(sf, mode, rough):
    import torch
    A, om, mesh = _setup(sf, 4, 8)
    b = (np.random.default_rng(1).uniform(-1, 1, mesh.n_free) if rough
         else O.rhs(om, mesh, O.sin_forcing))
    mg = sf.Multigrid(A, mode=mode, min_cells=4)
    assert mg.orders == [4, 2, 1, 1] and mg.cells[-1] == (4, 4, 4)
    x, info = mg.solve(torch.from_numpy(b).cuda(), reltol=1e-10)
    assert info["converged"] and info["relres"] <= 1e-10
    assert info["iters"] <= 25, info  # Jacobi CG: 28 (smooth) / 317 (rough) here
    _check_solution(om, mesh, b, x.cpu().numpy(), 1e-7)
    # a second solve on the same handle (the captured iteration is replayed)
    x2, info2 = mg.solve(torch.from_numpy(b).cuda(), reltol=1e-10)
    assert info2["iters"] == info["iters"]
    assert torch.equal(x, x2)


@pytest.mark.parametrize("mode", ["mixed", "f64"])
def test_mg_deformed_q8(sf, mode):
    """Equispaced Q8 on perturbed cells: Jacobi CG needs about 9900 iterations on
    3^3 cells; the hierarchy in Gauss-Lobatto nodes takes a few dozen at most."""
    import torch
    A, om, mesh = _setup(sf, 8, 3, perturb=0.2)
    b = O.rhs(om, mesh, O.sin_forcing)
    mg = sf.Multigrid(A, mode=mode)
    assert mg.basis == "gll" and mg.orders == [8, 4, 2, 1]
    x, info = mg.solve(torch.from_numpy(b).cuda(), reltol=1e-10, maxiter=200)
    assert info["converged"], info
    assert info["iters"] <= 40, info
    _check_solution(om, mesh, b, x.cpu().numpy(), 1e-6)


def test_mg_deformed_h_levels(sf):
    """Perturbed Q2 on 8^3 cells: p-levels, then Q1 on the coarsened meshes."""
    import torch
    A, om, mesh = _setup(sf, 2, 8, perturb=0.2, seed=2)
    b = np.random.default_rng(3).uniform(-1, 1, mesh.n_free)
    mg = sf.Multigrid(A, mode="mixed", min_cells=4, degree=2)
    assert mg.cells == [(8, 8, 8), (8, 8, 8), (4, 4, 4)]
    x, info = mg.solve(torch.from_numpy(b).cuda(), reltol=1e-10, maxiter=200)
    assert info["converged"] and info["iters"] <= 40, info
    _check_solution(om, mesh, b, x.cpu().numpy(), 1e-7)


def test_mg_initial_guess_and_cap(sf):
    import torch
    from ncihackaton2023_b200 import _lib
    A, om, mesh = _setup(sf, 3, 6)
    b = torch.from_numpy(O.rhs(om, mesh, O.sin_forcing)).cuda()
    mg = sf.Multigrid(A, mode="mixed")
    x, info = mg.solve(b, reltol=1e-12)
    x0 = x.clone()
    x1, info1 = mg.solve(b, x=x0, reltol=1e-10)  # already converged: no iteration
    assert info1["iters"] == 0 and info1["converged"]
    _, info2 = mg.solve(b, reltol=1e-14, maxiter=3, raise_on_fail=False)
    assert info2["iters"] == 3 and not info2["converged"]
    with pytest.raises(_lib.SumFacError):
        mg.solve(b, reltol=1e-14, maxiter=3)


def test_cg_mode_mg(sf):
    """sf.cg(mode="mg_mixed") builds the hierarchy once and keeps it on the operator."""
    import torch
    A, om, mesh = _setup(sf, 2, 6)
    b = torch.from_numpy(O.rhs(om, mesh, O.sin_forcing)).cuda()
    x, info = sf.cg(A, b, reltol=1e-10, mode="mg_mixed")
    assert info["converged"] and info["relres"] <= 1e-10
    mg = A._mg["mg_mixed"]
    x2, info2 = sf.cg(A, b, reltol=1e-10, mode="mg_mixed")
    assert A._mg["mg_mixed"] is mg and torch.equal(x, x2)
    _check_solution(om, mesh, b.cpu().numpy(), x.cpu().numpy(), 1e-7)
    A.close()
    assert mg._h is None


def test_mg_variable_coefficient(sf):
    """-div(kappa grad u) with a rough kappa per quadrature point (exp of N(0, 0.5^2)):
    the coarse levels take cell means of kappa; the solve is against the oracle's
    assembled matrix with the same kappa."""
    import scipy.sparse.linalg as spla
    import torch
    p, n = 3, 4
    A, om, mesh = _setup(sf, p, n)
    nq = (p + 1) ** 3
    kappa = np.exp(np.random.default_rng(4).normal(0.0, 0.5, (n ** 3, nq)))
    A.set_coefficient(torch.from_numpy(kappa).cuda())
    b = O.rhs(om, mesh, O.sin_forcing)
    x, info = sf.cg(A, torch.from_numpy(b).cuda(), reltol=1e-10, mode="mg_mixed")
    assert info["converged"] and info["iters"] <= 40, info
    As = O.assembled_sparse(om, mesh, kappa=kappa).tocsc()
    x_ref = spla.spsolve(As, b)
    xs = x.cpu().numpy()
    assert np.linalg.norm(b - As @ xs) / np.linalg.norm(b) < 1e-9
    assert np.abs(xs - x_ref).max() / np.abs(x_ref).max() < 1e-7
    # a new coefficient: the kept hierarchy follows it (sf_mg_refresh) and solves as a
    # hierarchy built for that coefficient from scratch does
    mg = A._mg["mg_mixed"]
    kappa2 = np.exp(np.random.default_rng(9).normal(0.0, 0.5, (n ** 3, nq)))
    A.set_coefficient(torch.from_numpy(kappa2).cuda())
    assert A._mg["mg_mixed"] is mg
    x2, info2 = sf.cg(A, torch.from_numpy(b).cuda(), reltol=1e-10, mode="mg_mixed")
    assert info2["converged"]
    x2_ref = spla.spsolve(O.assembled_sparse(om, mesh, kappa=kappa2).tocsc(), b)
    assert np.abs(x2.cpu().numpy() - x2_ref).max() / np.abs(x2_ref).max() < 1e-7
    fresh = sf.Multigrid(A, mode="mixed")  # (atomic sums in the applies: equal to rounding)
    np.testing.assert_allclose(fresh.lmax(), mg.lmax(), rtol=1e-9)
    x3, info3 = fresh.solve(torch.from_numpy(b).cuda(), reltol=1e-10)
    assert abs(info3["iters"] - info2["iters"]) <= 1
    fresh.close()
    # and back to the constant coefficient
    A.set_coefficient(None)
    x4, info4 = sf.cg(A, torch.from_numpy(b).cuda(), reltol=1e-10, mode="mg_mixed")
    assert info4["converged"]
    _check_solution(om, mesh, b, x4.cpu().numpy(), 1e-7)
