"""2D (quadrilateral Q_p) path: the tiled 2D Cartesian kernel through the C ABI
against the oracle's 2D restatement (assembled sparse matrix from full
element matrices), for every order the kernel covers, square and non-square
cells (the anisotropic variant of the kernel), several tiles per direction, FP64
and FP32, the Kronecker diagonal and Jacobi CG."""
import numpy as np
import pytest

from oracle import sumfac_oracle as O

pytestmark = pytest.mark.gpu


def _build(sf, p, deg, n):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1), n)
    V = sf.FESpace(model, p)
    m = sf.SumFactorizationMap(2, (p, p), (deg, deg))
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, deg))
    om = O.make_map(2, p, deg)
    mesh = O.cartesian_mesh(2, n, p, om)
    return A, V, om, mesh


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("n", [(5, 7), (4, 8), (70, 3)])
def test_apply_matches_oracle(sf, p, n):
    import torch
    deg = 2 * p
    A, V, om, mesh = _build(sf, p, deg, n)
    assert A.uses_tiled_kernel()
    S = O.assembled_sparse(om, mesh)
    x = np.random.default_rng(p).uniform(-1, 1, A.n)
    y_ref = S @ x
    y = (A @ torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.abs(y - y_ref).max() <= 1e-12 * np.abs(y_ref).max()
    y32 = (A @ torch.from_numpy(x).float().cuda()).double().cpu().numpy()
    assert np.abs(y32 - y_ref).max() <= 2e-5 * np.abs(y_ref).max()


def test_reference_quadrature_rule(sf):
    """The rule of the reference's 2D benchmarks: degree 2(p-1), so SQ = p < SB."""
    import torch
    p = 4
    A, V, om, mesh = _build(sf, p, 2 * (p - 1), (9, 6))
    S = O.assembled_sparse(om, mesh)
    x = np.random.default_rng(0).uniform(-1, 1, A.n)
    y = (A @ torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.abs(y - S @ x).max() <= 1e-12 * np.abs(S @ x).max()


def test_diagonal_and_cg_match_oracle(sf):
    import torch
    p, deg, n = 3, 6, (12, 9)
    A, V, om, mesh = _build(sf, p, deg, n)
    S = O.assembled_sparse(om, mesh)
    d = A.diagonal().cpu().numpy()
    assert np.abs(d - S.diagonal()).max() <= 1e-13 * np.abs(S.diagonal()).max()
    b = O.rhs(om, mesh, O.sin_forcing)
    x_ref, it_ref, _ = O.cg(lambda v: S @ v, b, reltol=1e-10, precond=lambda r: r / S.diagonal())
    x, info = sf.cg(A, torch.from_numpy(b).cuda(), reltol=1e-10, mode="jacobi")
    assert info["converged"] and abs(info["iters"] - it_ref) <= 1
    assert np.abs(x.cpu().numpy() - x_ref).max() < 1e-8 * np.abs(x_ref).max()


def test_2d_limits(sf):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1), (3, 3))
    V = sf.FESpace(model, 2)
    m = sf.SumFactorizationMap(2, (2, 2), (4, 4))
    with pytest.raises(sf.SumFacError):
        sf.LazyMatrix(m, V, V, sf.Measure(model, 4), gather="table")
    with pytest.raises(NotImplementedError):
        sf.CartesianDiscreteModel((0, 1, 0, 1), (3, 3), perturb=0.1)
