"""Cartesian meshes with the caller's own dof numbering (sf_set_structured_numbering,
LazyMatrix(gather="numbered")): the tiled kernels run on lexicographically permuted
vectors. Checked against the cell-to-dof table path of the same renumbered space
(itself checked against the oracle in test_gpu_apply.py) and against the lexicographic
space, whose solve a numbered solve must reproduce exactly."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import sumfac_oracle as O

pytestmark = pytest.mark.gpu


def spaces(sf, p, n, seed=5):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), n)
    m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
    dO = sf.Measure(model, 2 * p)
    Vr = sf.FESpace(model, p, renumber_seed=seed)
    Vl = sf.FESpace(model, p)
    A_num = sf.LazyMatrix(m, Vr, Vr, dO, gather="numbered")
    A_tab = sf.LazyMatrix(m, Vr, Vr, dO, gather="table")
    A_lex = sf.LazyMatrix(m, Vl, Vl, dO)
    perm = torch.from_numpy(Vr.perm).cuda()  # lexicographic index -> renumbered id
    return m, model, A_num, A_tab, A_lex, perm


@pytest.mark.parametrize("fused", [0, 1])
@pytest.mark.parametrize("p,n", [(2, (5, 4, 6)), (4, (4, 3, 5)), (3, (6, 6, 2))])
def test_numbered_apply_matches_table(sf, p, n, fused):
    """Both ways of applying through a numbering: permuting x and y around the
    lexicographic apply (0), and the tiled kernel reading and writing through it (1)."""
    m, model, A_num, A_tab, A_lex, perm = spaces(sf, p, n)
    assert A_num.info("numbered_fused") == 0.0  # a random numbering has no locality
    A_num.set_option("numbered_fused", fused)
    assert A_num.info("numbered_fused") == float(fused)
    assert A_num.uses_tiled_kernel() and not A_tab.uses_tiled_kernel()
    assert A_num.info("numbered") == 1.0 and A_tab.info("numbered") == 0.0
    x = torch.from_numpy(np.random.default_rng(p).uniform(-1, 1, A_num.n)).cuda()
    y_ref = A_tab @ x
    y = A_num @ x
    assert (y - y_ref).abs().max().item() <= 1e-12 * y_ref.abs().max().item()
    # the same as the lexicographic operator on the permuted vector: bit for bit through the
    # permutation (the same kernel); to rounding in the numbered kernel, whose tile shape can
    # differ (a vertex between tiles adds its cells' parts in another order)
    y_lex = A_lex @ x[perm]
    if fused:
        assert (y[perm] - y_lex).abs().max().item() <= 1e-13 * y_lex.abs().max().item()
    else:
        assert torch.equal(y[perm], y_lex)
    y32 = A_num @ x.float()
    assert (y32.double() - y_ref).abs().max().item() <= 2e-5 * y_ref.abs().max().item()
    # host vectors (sf_mul_host)
    yh = A_num @ x.cpu().numpy()
    assert np.array_equal(yh, y.cpu().numpy())
    # several right-hand sides
    X = torch.empty((2, A_num.n), dtype=torch.float64, device="cuda").t()  # (n, 2) column-major
    X[:, 0] = x
    X[:, 1] = -x
    Y = torch.empty_like(X)
    sf.mul_multi(Y, A_num, X)
    assert torch.equal(Y[:, 0], y) and torch.equal(Y[:, 1], -y)


def test_numbered_diagonal_and_rhs_match_table(sf):
    m, model, A_num, A_tab, A_lex, perm = spaces(sf, 3, (5, 4, 4))
    for dt in (torch.float64, torch.float32):
        d = A_num.diagonal(dt)
        d_ref = A_tab.diagonal(dt)
        assert (d.double() - d_ref.double()).abs().max().item() <= 1e-6 * d_ref.abs().max().item()
    d = A_num.diagonal()
    d_lex = A_lex.diagonal()  # assembled with atomics: equal up to the order of the sums
    assert (d[perm] - d_lex).abs().max().item() <= 1e-13 * d_lex.abs().max().item()
    X = sf.quadrature_points(A_num)
    f = 3 * np.pi ** 2 * torch.prod(torch.sin(np.pi * X), dim=-1)
    b = sf.rhs(A_num, f)
    b_ref = sf.rhs(A_tab, f)
    assert (b - b_ref).abs().max().item() <= 1e-12 * b_ref.abs().max().item()


@pytest.mark.parametrize("mode", ["jacobi", "plain", "mixed"])
def test_numbered_cg_reproduces_the_lexicographic_solve(sf, mode):
    m, model, A_num, A_tab, A_lex, perm = spaces(sf, 4, (5, 4, 6))
    om = O.make_map(3, 4, 8)
    mesh = O.cartesian_mesh(3, (5, 4, 6), 4, om)
    b_lex = torch.from_numpy(O.rhs(om, mesh, O.sin_forcing)).cuda()
    b = torch.empty_like(b_lex)
    b[perm] = b_lex
    x, info = sf.cg(A_num, b, reltol=1e-10, mode=mode)
    x_lex, info_lex = sf.cg(A_lex, b_lex, reltol=1e-10, mode=mode)
    assert info["converged"] and info["iters"] == info_lex["iters"]
    assert torch.equal(x[perm], x_lex)
    x_tab, info_tab = sf.cg(A_tab, b, reltol=1e-10, mode=mode)
    assert abs(info_tab["iters"] - info["iters"]) <= (1 if mode != "mixed" else 30)
    assert (x - x_tab).abs().max().item() < 1e-8 * x_tab.abs().max().item()


def test_numbered_rejections(sf):
    m, model, A_num, A_tab, A_lex, perm = spaces(sf, 2, (3, 3, 3))
    lib, L = sf._lib.lib, sf._lib
    b = torch.zeros(A_num.n, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    it, rel = C.c_int(), C.c_double()
    st = lib.sf_cg_noalloc(A_num._h, 0, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 1e-8,
                           10, C.byref(it), C.byref(rel), None)
    assert st == L.SF_ERR_UNSUPPORTED
    s = torch.zeros(L.SF_CGD_SCALARS, dtype=torch.float64, device="cuda")
    st = lib.sf_cgd_apply(A_num._h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()),
                          C.c_void_p(s.data_ptr()), None)
    assert st == L.SF_ERR_UNSUPPORTED
    # a free_id that is not a permutation
    bad = np.zeros(A_num.n, dtype=np.int32)
    no = np.asarray(m.node_order, dtype=np.int32)
    st = lib.sf_set_structured_numbering(A_tab._h, 3, 3, 3, no.ctypes.data_as(C.c_void_p),
                                         bad.ctypes.data_as(C.c_void_p))
    assert st == L.SF_ERR_ARG


def test_identity_numbering_equals_structured(sf):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (4, 5, 3))
    m = sf.SumFactorizationMap(3, (3,) * 3, (6,) * 3)
    V = sf.FESpace(model, 3)
    A_id = sf.LazyMatrix(m, V, V, sf.Measure(model, 6), gather="numbered")
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, 6))
    x = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, A.n)).cuda()
    assert torch.equal(A_id @ x, A @ x)


def test_cellwise_numbering_matches_table(sf):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (4, 5, 3))
    m = sf.SumFactorizationMap(3, (4,) * 3, (8,) * 3)
    V = sf.FESpace(model, 4, cellwise=True)
    A_num = sf.LazyMatrix(m, V, V, sf.Measure(model, 8), gather="numbered")
    assert A_num.info("numbered_fused") == 1.0  # a cell-by-cell numbering keeps neighbours near
    A_tab = sf.LazyMatrix(m, V, V, sf.Measure(model, 8), gather="table")
    x = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, A_num.n)).cuda()
    y_ref = A_tab @ x
    assert ((A_num @ x) - y_ref).abs().max().item() <= 1e-12 * y_ref.abs().max().item()


@pytest.mark.parametrize("fused", [0, 1])
@pytest.mark.parametrize("p,n", [(4, (4, 3, 5)), (2, (6, 5, 4)), (3, (3, 4, 3))])
def test_gridap_numbering(sf, p, n, fused):
    """The face-grouped numbering of a conforming space (vertex, edge, face and
    interior dofs in turn) through the numbered tiled path: the apply against the
    table path and the solve against the lexicographic one."""
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), n)
    m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
    dO = sf.Measure(model, 2 * p)
    Vg = sf.FESpace(model, p, numbering="gridap")
    Vl = sf.FESpace(model, p)
    A_num = sf.LazyMatrix(m, Vg, Vg, dO, gather="numbered")
    A_tab = sf.LazyMatrix(m, Vg, Vg, dO, gather="table")
    A_lex = sf.LazyMatrix(m, Vl, Vl, dO)
    A_num.set_option("numbered_fused", fused)
    perm = torch.from_numpy(Vg.perm).cuda()
    x = torch.from_numpy(np.random.default_rng(p).uniform(-1, 1, A_num.n)).cuda()
    y_ref = A_tab @ x
    y = A_num @ x
    assert (y - y_ref).abs().max().item() <= 1e-12 * y_ref.abs().max().item()
    y32 = A_num @ x.float()
    assert (y32.double() - y_ref).abs().max().item() <= 2e-5 * y_ref.abs().max().item()
    b = x
    xs, info = sf.cg(A_num, b, reltol=1e-10)
    xl, infol = sf.cg(A_lex, b[perm], reltol=1e-10)
    assert info["iters"] == infol["iters"]
    assert (xs[perm] - xl).abs().max().item() <= 1e-12 * xl.abs().max().item()
