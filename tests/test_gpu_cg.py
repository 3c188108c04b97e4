"""Device CG (FP64 Jacobi, plain, and FP32-inner mixed precision with FP64
refinement) against the oracle's restatement of IterativeSolvers.cg!."""
import numpy as np
import pytest

from oracle import sumfac_oracle as O

pytestmark = pytest.mark.gpu


def setup(sf, p, deg, n, perturb=0.0):
    import torch
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n), perturb=perturb, seed=1)
    V = sf.FESpace(model, p)
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, deg))
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om, perturb=perturb, seed=1)
    b = O.rhs(om, mesh, O.sin_forcing)
    return A, V, om, mesh, b, torch.from_numpy(b).cuda()


@pytest.mark.parametrize("mode", ["plain", "jacobi"])
def test_cg_matches_oracle(sf, mode):
    A, V, om, mesh, b, bd = setup(sf, 2, 4, 6)
    S = O.assembled_sparse(om, mesh)
    pre = None if mode == "plain" else (lambda r, d=S.diagonal(): r / d)
    x_ref, it_ref, rel_ref = O.cg(lambda v: S @ v, b, reltol=1e-10, precond=pre)
    x, info = sf.cg(A, bd, reltol=1e-10, mode=mode)
    assert info["relres"] <= 1e-10 and info["converged"]
    assert abs(info["iters"] - it_ref) <= 1
    x = x.cpu().numpy()
    assert np.abs(x - x_ref).max() < 1e-8 * np.abs(x_ref).max()


def test_mixed_precision_reaches_fp64_residual(sf):
    import torch
    A, V, om, mesh, b, bd = setup(sf, 4, 8, 4, perturb=0.1)
    x64, i64 = sf.cg(A, bd, reltol=1e-10, mode="jacobi")
    xm, im = sf.cg(A, bd, reltol=1e-10, mode="mixed")
    assert im["relres"] <= 1e-10 and im["outer"] >= 2
    r = (bd - A @ xm).norm().item() / bd.norm().item()
    assert r <= 1e-10
    assert (xm - x64).abs().max().item() < 1e-7 * x64.abs().max().item()


def test_discretization_error_decreases(sf):
    errs = []
    for n in (2, 4, 8):
        A, V, om, mesh, b, bd = setup(sf, 2, 6, n)
        x, info = sf.cg(A, bd, reltol=1e-12, mode="jacobi")
        X = V.free_dof_coordinates()
        errs.append(np.abs(x.cpu().numpy() - O.sin_solution(X)).max())
    assert errs[1] < errs[0] / 6 and errs[2] < errs[1] / 6


def test_iteration_cap_is_reported(sf):
    A, V, om, mesh, b, bd = setup(sf, 2, 4, 6)
    with pytest.raises(sf.SumFacError) as e:
        sf.cg(A, bd, reltol=1e-14, maxiter=3)
    assert e.value.status == 5  # SF_ERR_NOT_CONVERGED
    x, info = sf.cg(A, bd, reltol=1e-14, maxiter=3, raise_on_fail=False)
    assert info["iters"] == 3 and not info["converged"]


def test_zero_rhs(sf):
    import torch
    A, V, om, mesh, b, bd = setup(sf, 2, 4, 3)
    x, info = sf.cg(A, torch.zeros_like(bd), reltol=1e-10)
    assert info["iters"] == 0 and x.abs().max().item() == 0.0


def test_deformed_q8_iterations_match_oracle(sf):
    """High-order deformed cells (equispaced Q8, kappa(A) large): the device
    Jacobi CG follows the oracle's iteration count."""
    A, V, om, mesh, b, bd = setup(sf, 8, 16, 2, perturb=0.2)
    S = O.assembled_sparse(om, mesh)
    d = S.diagonal()
    x_ref, it_ref, _ = O.cg(lambda v: S @ v, b, reltol=1e-10, precond=lambda r: r / d,
                            maxiter=20000)
    x, info = sf.cg(A, bd, reltol=1e-10, mode="jacobi", maxiter=20000)
    # kappa(A) is large, so rounding differences move the count a little
    assert info["converged"] and abs(info["iters"] - it_ref) <= max(10, it_ref // 10)
    assert np.abs(x.cpu().numpy() - x_ref).max() < 1e-6 * np.abs(x_ref).max()


@pytest.mark.parametrize("mode", ["jacobi", "mixed"])
def test_cg_is_deterministic(sf, mode):
    """The reductions add partial sums in a fixed order, so a repeated solve
    gives the same iterates bit for bit (tiled Cartesian path, Q4)."""
    import torch
    A, V, om, mesh, b, bd = setup(sf, 4, 8, 6)
    assert A.uses_tiled_kernel()
    x1, i1 = sf.cg(A, bd, reltol=1e-10, mode=mode)
    x2, i2 = sf.cg(A, bd, reltol=1e-10, mode=mode)
    assert i1["iters"] == i2["iters"] and i1["relres"] == i2["relres"]
    assert torch.equal(x1, x2)


def test_cg_tiled_and_general_paths_agree(sf):
    """The tiled kernel (fused (p, Ap) reduction) and the general kernel
    (separate reduction) drive the same Jacobi CG."""
    import torch
    A, V, om, mesh, b, bd = setup(sf, 3, 6, 5)
    assert A.uses_tiled_kernel()
    x_t, i_t = sf.cg(A, bd, reltol=1e-11, mode="jacobi")
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (5, 5, 5), perturb=0.0, seed=1)
    Vr = sf.FESpace(model, 3, renumber_seed=7)
    m = sf.SumFactorizationMap(3, (3,) * 3, (6,) * 3)
    Ag = sf.LazyMatrix(m, Vr, Vr, sf.Measure(model, 6))
    assert not Ag.uses_tiled_kernel()
    perm = torch.from_numpy(Vr.perm).cuda()  # lexicographic index -> renumbered id
    bg = torch.empty_like(bd)
    bg[perm] = bd
    x_g, i_g = sf.cg(Ag, bg, reltol=1e-11, mode="jacobi")
    assert abs(i_t["iters"] - i_g["iters"]) <= 1
    assert (x_g[perm] - x_t).abs().max().item() < 1e-9 * x_t.abs().max().item()


@pytest.mark.parametrize("mode", ["jacobi", "mixed"])
def test_jacobi_table_and_vector_agree(sf, mode):
    """On a Cartesian mesh the FP64 Jacobi CG's vector kernels read D^-1 from a table
    per position in a cell (option jacobi_table, the default); the D^-1 vector gives
    the same CG (the mixed mode reads the FP32 vector either way). Anisotropic
    cells, several orders."""
    import torch
    for p, n, dom in ((3, (7, 5, 6), (0, 2, 0, 1, 0, 0.5)), (4, (5, 6, 4), (0, 1, 0, 3, 0, 1))):
        model = sf.CartesianDiscreteModel(dom, n)
        V = sf.FESpace(model, p)
        m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
        A = sf.LazyMatrix(m, V, V, sf.Measure(model, 2 * p))
        assert A.info("jacobi_table") == 1.0
        b = torch.from_numpy(np.random.default_rng(p).uniform(-1, 1, A.n)).cuda()
        x_t, i_t = sf.cg(A, b, reltol=1e-10, mode=mode)
        A.set_option("jacobi_table", 0)
        assert A.info("jacobi_table") == 0.0
        x_v, i_v = sf.cg(A, b, reltol=1e-10, mode=mode)
        assert i_t["converged"] and i_v["converged"]
        assert abs(i_t["iters"] - i_v["iters"]) <= (1 if mode == "jacobi" else 20)
        assert (x_t - x_v).abs().max().item() < 1e-8 * x_v.abs().max().item()
