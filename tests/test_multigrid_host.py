"""Host-side pieces of the multigrid hierarchy (CPU only, no device calls): the
Gauss-Lobatto nodes of the finest level and the 1D transfer tables that the
library applies as tensor products (sf_mg_create's `transfer` and
`basis_change` arguments)."""
import numpy as np
import pytest


def _ascending(sf, fam, q):
    return (np.sort(sf.fem.gll_nodes(q)) if fam == "gll" else np.linspace(0.0, 1.0, q + 1))


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 8])
def test_gll_nodes_in_gridap_order(sf, p):
    x = sf.fem.gll_nodes(p)
    assert len(x) == p + 1 and x[0] == 0.0 and x[1] == 1.0
    inner = x[2:]
    assert np.all(np.diff(inner) > 0) and np.all((inner > 0) & (inner < 1))
    assert np.allclose(inner + inner[::-1], 1.0, atol=1e-14)  # symmetric about 1/2
    if p >= 2:  # interior nodes: the roots of P_p' on [-1, 1], mapped to [0, 1]
        c = np.zeros(p + 1)
        c[p] = 1.0
        dP = np.polynomial.legendre.legder(c)
        assert np.abs(np.polynomial.legendre.legval(2 * inner - 1, dP)).max() < 1e-10


@pytest.mark.parametrize("fam", ["equispaced", "gll"])
@pytest.mark.parametrize("pf,pc,ratio", [(4, 2, 1), (2, 1, 1), (8, 4, 1), (5, 2, 1), (3, 1, 1),
                                         (1, 1, 2), (8, 8, 1)])
def test_transfer_table_interpolates_coarse_polynomials(sf, fam, pf, pc, ratio):
    """Row i of the (ratio pf + 1) x (pc + 1) table holds the coarse cell's basis
    functions at the i-th fine node of that cell, so the table maps the coarse
    nodal values of any polynomial of degree <= pc to its fine nodal values; its
    rows sum to one and its first and last rows pick the cell's end points."""
    T = sf.multigrid.transfer_table(_ascending(sf, fam, pf), _ascending(sf, fam, pc), ratio)
    assert T.shape == (ratio * pf + 1, pc + 1)
    fine = np.concatenate([(k + _ascending(sf, fam, pf)[:-1]) / ratio for k in range(ratio)] + [[1.0]])
    coarse = _ascending(sf, fam, pc)
    rng = np.random.default_rng(pf * 10 + pc)
    for _ in range(3):
        poly = np.polynomial.Polynomial(rng.normal(size=pc + 1))
        assert np.abs(T @ poly(coarse) - poly(fine)).max() < 1e-12
    assert np.allclose(T.sum(axis=1), 1.0, atol=1e-13)
    assert np.allclose(T[0], np.eye(pc + 1)[0]) and np.allclose(T[-1], np.eye(pc + 1)[-1])


def test_change_of_basis_table_is_invertible_interpolation(sf):
    """The Q8 change of basis (Gauss-Lobatto basis functions at the equispaced
    nodes) maps GLL nodal values to equispaced nodal values of the same
    polynomial, and is invertible."""
    p = 8
    gll, equi = np.sort(sf.fem.gll_nodes(p)), np.linspace(0.0, 1.0, p + 1)
    T = sf.multigrid._lagrange_values(gll, equi)
    poly = np.polynomial.Polynomial(np.random.default_rng(3).normal(size=p + 1))
    assert np.abs(T @ poly(gll) - poly(equi)).max() < 1e-10
    assert np.linalg.cond(T) < 1e3
