"""Parity of the CUDA apply with the FP64 oracle, through the C ABI.

Tolerances (relative to max |y|): FP64 1e-12 (the bar of the task), FP32
2e-5 (FP32 data, metric and accumulation)."""
import os

import numpy as np
import pytest

from oracle import sumfac_oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL64 = 1e-12
TOL32 = 2e-5

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def build(sf, p, deg, n, perturb=0.0, seed=0, gather="structured", renumber_seed=None):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n) if isinstance(n, int) else n,
                                      perturb=perturb, seed=seed)
    V = sf.FESpace(model, p, renumber_seed=renumber_seed)
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    return sf.LazyMatrix(m, V, V, sf.Measure(model, deg), gather=gather), V


def relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


GOLDEN_CASES = ["c1_q2_n8", "demo_q4_deg6_n4_ones", "kappa_q3_n4", "deformed_q4_n3",
                "deformed_q8_n2", "q1_deg4_n6", "q4_deg6_n3"]


@pytest.mark.parametrize("name", GOLDEN_CASES)
@pytest.mark.parametrize("gather", ["structured", "table"])
def test_apply_matches_golden(sf, name, gather):
    torch = _torch()
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    A, V = build(sf, int(g["p"]), int(g["deg"]), int(g["n"]), float(g["perturb"]),
                 int(g["perturb_seed"]), gather)
    if "kappa" in g:
        A.set_coefficient(g["kappa"])
    x = torch.from_numpy(g["x"]).cuda()
    y = (A @ x).cpu().numpy()
    assert relerr(y, g["y"]) < TOL64
    y32 = (A @ x.float()).double().cpu().numpy()
    assert relerr(y32, g["y"]) < TOL32
    d = A.diagonal().cpu().numpy()
    assert relerr(d, g["diag"]) < TOL64


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6, 7, 8, 9])
def test_all_orders(sf, p):
    torch = _torch()
    n = 3 if p <= 4 else 2
    for deg in sorted({2 * p, 2 * p + 1, 2 * p - 2} - {-1, 0}):
        A, V = build(sf, p, deg, n)
        om = O.make_map(3, p, deg)
        mesh = O.cartesian_mesh(3, n, p, om)
        x = np.random.default_rng(p).uniform(-1, 1, mesh.n_free)
        y_ref = O.lazy_mul(om, mesh, x)
        y = (A @ torch.from_numpy(x).cuda()).cpu().numpy()
        assert relerr(y, y_ref) < TOL64, (p, deg)


@pytest.mark.parametrize("p,deg", [(2, 4), (3, 6), (4, 8), (4, 6), (5, 10), (6, 12), (7, 14),
                                   (8, 16)])
def test_every_tile_candidate(sf, p, deg):
    """Every tile shape the autotuner may pick gives the oracle's result, on a
    mesh that is not a multiple of any tile (partial tiles at the far faces)."""
    torch = _torch()
    n = (5, 6, 7)
    A, V = build(sf, p, deg, n)
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om)
    x = np.random.default_rng(p).uniform(-1, 1, mesh.n_free)
    y_ref = O.lazy_mul(om, mesh, x)
    xd = torch.from_numpy(x).cuda()
    for dt, tol, key in ((torch.float64, TOL64, "f64"), (torch.float32, TOL32, "f32")):
        ncand = int(A.info(f"tile_candidates_{key}"))
        assert ncand >= 1
        for k in range(ncand):
            A.set_option(f"tile_candidate_{key}", k)
            y = (A @ xd.to(dt)).double().cpu().numpy()
            assert relerr(y, y_ref) < tol, (key, k, A.kernel_name(dt))
        name = A.autotune(dt)
        y = (A @ xd.to(dt)).double().cpu().numpy()
        assert relerr(y, y_ref) < tol, name


@pytest.mark.parametrize("p,deg,n,perturb", [(4, 8, 24, 0.0), (2, 4, 40, 0.0), (8, 16, 6, 0.2),
                                             (4, 8, 10, 0.2)])
def test_midsize_against_c_restatement(sf, p, deg, n, perturb):
    """Meshes of many tiles (Q4 on 24^3 cells: 6 x 6 x 8 tiles of the headline
    kernel) and deformed meshes against the C restatement of the reference
    loops, FP64 and FP32, with the default and the autotuned tile shape."""
    from oracle import cref
    torch = _torch()
    A, V = build(sf, p, deg, n, perturb=perturb, seed=3)
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om, perturb=perturb, seed=3)
    x = np.random.default_rng(n).uniform(-1, 1, mesh.n_free)
    y_ref = cref.mul_mesh(om, mesh, x, layers=2)
    xd = torch.from_numpy(x).cuda()
    for dt, tol in ((torch.float64, TOL64), (torch.float32, TOL32)):
        y = (A @ xd.to(dt)).double().cpu().numpy()
        assert relerr(y, y_ref) < tol, (dt, A.kernel_name(dt))
        if A.uses_tiled_kernel():
            A.autotune(dt)
            y = (A @ xd.to(dt)).double().cpu().numpy()
            assert relerr(y, y_ref) < tol, (dt, A.kernel_name(dt))


def test_renumbered_table(sf):
    torch = _torch()
    p, deg, n = 3, 6, 4
    A, V = build(sf, p, deg, n, renumber_seed=11)
    assert A.gather == "table"
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om, renumber_seed=11)
    x = np.random.default_rng(1).uniform(-1, 1, mesh.n_free)
    y_ref = O.lazy_mul(om, mesh, x)
    y = (A @ torch.from_numpy(x).cuda()).cpu().numpy()
    assert relerr(y, y_ref) < TOL64


def test_anisotropic_partition(sf):
    torch = _torch()
    p, deg, n = 2, 4, (3, 5, 2)
    A, V = build(sf, p, deg, n)
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om)
    x = np.random.default_rng(2).uniform(-1, 1, mesh.n_free)
    y = (A @ torch.from_numpy(x).cuda()).cpu().numpy()
    assert relerr(y, O.lazy_mul(om, mesh, x)) < TOL64


def test_host_buffers_mul(sf):
    g = np.load(os.path.join(GOLDEN, "c1_q2_n8.npz"))
    A, V = build(sf, 2, 4, 8)
    y = np.empty_like(g["x"])
    sf.mul(y, A, g["x"])
    assert relerr(y, g["y"]) < TOL64
    y2 = A @ g["x"]
    # the general kernel scatters with FP64 atomics: sums may differ in order
    assert relerr(y2, y) < 1e-14


@pytest.mark.parametrize("p,n", [(4, (5, 6, 11)), (2, (4, 3, 16)), (4, (3, 3, 7))])
def test_pinned_host_mul_is_pipelined_and_exact(sf, p, n):
    """With pinned host buffers sf_mul_host copies in, applies and copies out in
    groups of tile rows on three streams; the result equals the device apply."""
    torch = _torch()
    A, V = build(sf, p, 2 * p, n)
    assert A.uses_tiled_kernel()
    x = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, A.n))
    xh = x.clone().pin_memory()
    yh = torch.full_like(x, float("nan")).pin_memory()
    for _ in range(2):  # the second call reuses the streams and events
        sf.mul(yh.numpy(), A, xh.numpy())
        y_dev = A @ x.cuda()
        assert torch.equal(yh, y_dev.cpu())


def test_evaluate_cells_matches_map(sf):
    """The Map protocol: evaluate!(m, x_e, wq, jq, djq) for a batch of cells."""
    torch = _torch()
    for pert in (0.0, 0.2):
        p, deg, n = 3, 6, 3
        A, V = build(sf, p, deg, n, perturb=pert, seed=4)
        om = O.make_map(3, p, deg)
        mesh = O.cartesian_mesh(3, n, p, om, perturb=pert, seed=4)
        wq, jq, djq = O.cell_quantities(om, mesh)
        xe = np.random.default_rng(9).uniform(-1, 1, (mesh.cell_dof_ids.shape[0], (p + 1) ** 3))
        ye_ref = O.evaluate_cells(om, xe, wq, jq, djq)
        ye = A.evaluate_cells(torch.from_numpy(xe).cuda()).cpu().numpy()
        assert relerr(ye, ye_ref) < TOL64


def test_multi_rhs(sf):
    torch = _torch()
    A, V = build(sf, 2, 4, 5)
    n = V.num_free_dofs
    X = torch.rand(4, n, dtype=torch.float64, device="cuda").t()  # column-major (n, 4)
    Y = torch.empty(4, n, dtype=torch.float64, device="cuda").t()
    sf.mul_multi(Y, A, X)
    for k in range(4):
        yk = A @ X[:, k].contiguous()
        assert ((Y[:, k] - yk).abs().max() / yk.abs().max()).item() < 1e-14


def test_linearity_and_symmetry(sf):
    torch = _torch()
    A, V = build(sf, 4, 8, 6, perturb=0.2, seed=3)
    n = V.num_free_dofs
    gen = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(n, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
    z = torch.rand(n, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
    Ax, Az = A @ x, A @ z
    lin = A @ (x + 2 * z)
    assert ((lin - Ax - 2 * Az).abs().max() / lin.abs().max()).item() < 1e-13
    s1, s2 = torch.dot(z, Ax).item(), torch.dot(x, Az).item()
    assert abs(s1 - s2) < 1e-12 * abs(s1)


def test_edge_cases(sf):
    torch = _torch()
    # one Q1 cell: no free dof at all
    A, V = build(sf, 1, 2, 1)
    assert V.num_free_dofs == 0
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    assert (A @ e).numel() == 0
    # one Q1 free dof in the middle of 2^3 cells
    A, V = build(sf, 1, 2, 2)
    x = torch.ones(1, dtype=torch.float64, device="cuda")
    om = O.make_map(3, 1, 2)
    mesh = O.cartesian_mesh(3, 2, 1, om)
    assert abs((A @ x).item() - O.lazy_mul(om, mesh, np.ones(1))[0]) < 1e-15
    # one Q3 cell: only its interior dofs are free
    A, V = build(sf, 3, 6, 1)
    assert V.num_free_dofs == 8
    x = torch.ones(8, dtype=torch.float64, device="cuda")
    om = O.make_map(3, 3, 6)
    mesh = O.cartesian_mesh(3, 1, 3, om)
    assert relerr((A @ x).cpu().numpy(), O.lazy_mul(om, mesh, np.ones(8))) < TOL64


def test_errors_are_reported(sf):
    torch = _torch()
    A, V = build(sf, 2, 4, 2)
    n = V.num_free_dofs
    with pytest.raises(ValueError):
        sf.mul(torch.empty(n, device="cuda", dtype=torch.float64), A,
               torch.empty(n + 1, device="cuda", dtype=torch.float64))
    with pytest.raises(TypeError):
        A @ torch.empty(n, device="cuda", dtype=torch.float16)
    with pytest.raises(ValueError):
        A.set_coefficient(np.ones((3, 3)))
    x = torch.zeros(n, device="cuda", dtype=torch.float64)
    with pytest.raises(sf.SumFacError):
        sf.mul(x, A, x)  # aliasing is rejected by the library


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6, 7, 8])
def test_diagonal_all_orders(sf, p):
    """diag(A) (sum-factorized per element, assembled) against the assembled oracle, for
    SQ below, at and above SB, on affine and on deformed cells."""
    n = 2
    for deg, pert in ((2 * p, 0.0), (max(2 * p - 2, 1), 0.0), (2 * p + 1, 0.15)):
        A, V = build(sf, p, deg, n, pert, 4, "structured")
        om = O.make_map(3, p, deg)
        mesh = O.cartesian_mesh(3, n, p, om, perturb=pert, seed=4)
        d_ref = O.assembled_sparse(om, mesh).diagonal()
        d = A.diagonal().cpu().numpy()
        assert relerr(d, d_ref) < TOL64, (p, deg, pert)
