"""Fused FP64 CG iteration (option cg_fused = 1: one tiled kernel per
iteration, the vector updates of iteration k-1 and q = A p of iteration k,
Jacobi diagonal from a per-cell position table) against the oracle's
restatement of IterativeSolvers.cg!, and against the default unfused
iteration (apply + vector kernels) of the same handle."""
import numpy as np
import pytest
import torch

from oracle import sumfac_oracle as O

pytestmark = pytest.mark.gpu


def setup(sf, p, n, domain=(0, 1, 0, 1, 0, 1)):
    deg = 2 * p
    model = sf.CartesianDiscreteModel(domain, n)
    V = sf.FESpace(model, p)
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, deg))
    assert A.info("cg_fused") == 0.0  # off by default
    A.set_option("cg_fused", 1)
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om) if domain == (0, 1, 0, 1, 0, 1) else None
    return A, om, mesh


def true_relres(A, b, x):
    return ((b - A @ x).norm() / b.norm()).item()


@pytest.mark.parametrize("p,n", [(1, (9, 7, 8)), (2, (5, 6, 7)), (3, (5, 4, 6)), (4, (5, 4, 3)),
                                 (5, (3, 2, 3)), (6, (2, 3, 2)), (7, (2, 2, 2)), (8, (2, 2, 2))])
@pytest.mark.parametrize("mode", ["jacobi", "plain"])
def test_fused_cg_matches_oracle(sf, p, n, mode):
    A, om, mesh = setup(sf, p, n)
    assert A.info("cg_fused") == 1.0, A.cg_kernel_name()
    S = O.assembled_sparse(om, mesh)
    b = O.rhs(om, mesh, O.sin_forcing)
    pre = None if mode == "plain" else (lambda r, d=S.diagonal(): r / d)
    x_ref, it_ref, _ = O.cg(lambda v: S @ v, b, reltol=1e-10, precond=pre, maxiter=20000)
    bd = torch.from_numpy(b).cuda()
    x, info = sf.cg(A, bd, reltol=1e-10, mode=mode, maxiter=20000)
    assert info["converged"] and info["relres"] <= 1e-10
    # equispaced high orders are ill-conditioned (Q8 Jacobi: about 1600 iterations on
    # 2^3 cells), and rounding then moves the count by a few percent
    assert abs(info["iters"] - it_ref) <= (1 if p <= 4 else max(10, it_ref // 10))
    assert np.abs(x.cpu().numpy() - x_ref).max() < 1e-8 * np.abs(x_ref).max()
    # the reported residual is that of the returned x
    assert true_relres(A, bd, x) < 2e-10


@pytest.mark.parametrize("mode", ["jacobi", "plain"])
def test_fused_and_unfused_iterations_agree(sf, mode):
    """Anisotropic cells, tiles cut by the mesh boundary in every direction."""
    A, om, mesh = setup(sf, 4, (9, 7, 6), domain=(0, 2, 0, 1, 0, 0.5))
    g = torch.Generator().manual_seed(11)
    b = torch.rand(A.n, generator=g, dtype=torch.float64).cuda() - 0.5
    x_f, i_f = sf.cg(A, b, reltol=1e-11, mode=mode, maxiter=5000)
    A.set_option("cg_fused", 0)
    assert A.info("cg_fused") == 0.0 and A.cg_kernel_name().startswith("unfused")
    x_u, i_u = sf.cg(A, b, reltol=1e-11, mode=mode, maxiter=5000)
    assert i_f["converged"] and i_u["converged"]
    assert abs(i_f["iters"] - i_u["iters"]) <= 1
    assert (x_f - x_u).abs().max().item() < 1e-9 * x_u.abs().max().item()


def test_every_tile_candidate_solves(sf):
    A, om, mesh = setup(sf, 4, (9, 8, 7))
    b = torch.from_numpy(O.rhs(om, mesh, O.sin_forcing)).cuda()
    nc = int(A.info("cg_candidates"))
    assert nc >= 2
    runs = []
    for k in range(nc):
        A.set_option("cg_candidate", k)
        runs.append(sf.cg(A, b, reltol=1e-10, mode="jacobi"))
    iters = [info["iters"] for _, info in runs]
    assert max(iters) - min(iters) <= 1
    for x, info in runs[1:]:
        assert (x - runs[0][0]).abs().max().item() < 1e-9 * runs[0][0].abs().max().item()
    with pytest.raises(sf.SumFacError):
        A.set_option("cg_candidate", nc)


@pytest.mark.parametrize("maxiter", [0, 1, 2, 7])
def test_iteration_cap_returns_the_reported_iterate(sf, maxiter):
    """maxiter iterations take maxiter + 1 passes; the x returned is x_maxiter and
    the reported residual is its true residual; it matches the unfused solve."""
    A, om, mesh = setup(sf, 3, (6, 5, 4))
    b = torch.from_numpy(O.rhs(om, mesh, O.sin_forcing)).cuda()
    x, info = sf.cg(A, b, reltol=1e-14, maxiter=maxiter, raise_on_fail=False)
    assert info["iters"] == maxiter and not info["converged"]
    assert abs(true_relres(A, b, x) - info["relres"]) <= 1e-9 * max(info["relres"], 1e-3)
    A.set_option("cg_fused", 0)
    xu, iu = sf.cg(A, b, reltol=1e-14, maxiter=maxiter, raise_on_fail=False)
    assert iu["iters"] == maxiter
    assert (x - xu).abs().max().item() <= 1e-11 * max(xu.abs().max().item(), 1e-300)


def test_initial_guess_is_used(sf):
    A, om, mesh = setup(sf, 2, (6, 6, 6))
    b = torch.from_numpy(O.rhs(om, mesh, O.sin_forcing)).cuda()
    x_ref, i_ref = sf.cg(A, b, reltol=1e-12)
    # a rough start (its residual is far above ||b||): the same solution
    x0 = x_ref + 1e-3 * torch.sin(torch.arange(A.n, dtype=torch.float64, device="cuda"))
    x, info = sf.cg(A, b, x=x0.clone(), reltol=1e-12)
    assert info["converged"] and true_relres(A, b, x) < 2e-12
    assert (x - x_ref).abs().max().item() < 1e-9 * x_ref.abs().max().item()
    # starting at the solution: no iteration
    x1, i1 = sf.cg(A, b, x=x.clone(), reltol=1e-6)
    assert i1["iters"] == 0 and torch.equal(x1, x)


def test_autotune_picks_a_cg_candidate(sf):
    A, om, mesh = setup(sf, 4, (8, 8, 8))
    A.autotune(torch.float64)
    name = A.cg_kernel_name()
    assert name.startswith("cg pass"), name
    b = torch.from_numpy(O.rhs(om, mesh, O.sin_forcing)).cuda()
    x, info = sf.cg(A, b, reltol=1e-10)
    assert info["converged"] and true_relres(A, b, x) < 2e-10


def test_unsupported_operators_use_the_unfused_iteration(sf):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (3, 3, 3), perturb=0.1, seed=2)
    V = sf.FESpace(model, 2)
    m = sf.SumFactorizationMap(3, (2,) * 3, (4,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, 4))
    A.set_option("cg_fused", 1)
    assert not A.uses_tiled_kernel() and A.info("cg_fused") == 0.0
    with pytest.raises(sf.SumFacError):
        A.set_option("cg_candidate", 0)
