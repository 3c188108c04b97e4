"""Host-side set-up of the package against the oracle (CPU only, no device calls)."""
import numpy as np
import pytest

from oracle import sumfac_oracle as O


@pytest.mark.parametrize("p,deg", [(1, 4), (2, 4), (3, 6), (4, 6), (4, 8), (6, 12), (8, 16), (9, 18)])
def test_map_matches_oracle(sf, p, deg):
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    om = O.make_map(3, p, deg)
    D, SB, SQ = sf.get_dimensional_parameters(m)
    assert (D, SB, SQ) == (3, (p + 1,) * 3, (om.SQ,) * 3)
    assert np.allclose(m.points, om.q1d, atol=1e-15) and np.allclose(m.weights, om.w1d, atol=1e-15)
    scale = max(1.0, np.abs(om.B0).max())
    assert np.abs(m.A0 - om.A0).max() < 1e-13
    assert np.abs(m.B0 - om.B0).max() < 1e-13 * scale
    assert np.array_equal(m.dof_map - 1, om.dof_map)
    g = m.gradMats
    assert g[0][0] is m.B0 and g[0][1] is m.A0


def test_map_rejects_unsupported(sf):
    with pytest.raises(NotImplementedError):
        sf.SumFactorizationMap(4, (2,) * 4, (4,) * 4)
    with pytest.raises(NotImplementedError):
        sf.SumFactorizationMap(3, (2, 3, 2), (4, 4, 4))
    with pytest.raises(ValueError):
        sf.SumFactorizationMap(3, (10,) * 3, (20,) * 3)


@pytest.mark.parametrize("p,n,pert", [(2, 3, 0.0), (3, 2, 0.2), (1, 4, 0.0)])
def test_cell_dof_ids_and_quantities_match_oracle(sf, p, n, pert):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n), perturb=pert, seed=3)
    V = sf.FESpace(model, p)
    om = O.make_map(3, p, 2 * p)
    mesh = O.cartesian_mesh(3, n, p, om, perturb=pert, seed=3)
    t = V.get_cell_dof_ids()
    ids = t.data.reshape(model.num_cells, -1)
    assert np.array_equal(ids, mesh.cell_dof_ids)
    assert np.array_equal(t.ptrs, 1 + np.arange(model.num_cells + 1) * (p + 1) ** 3)
    assert V.num_free_dofs == mesh.n_free
    m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
    fill, wq, jq, djq = sf.cell_quantities(model, m.points, m.weights)
    owq, ojq, odjq = O.cell_quantities(om, mesh)
    assert fill == (pert == 0.0)
    sel = slice(None) if not fill else slice(0, 1)
    assert np.allclose(wq, owq[sel], rtol=1e-14, atol=0)
    assert np.allclose(djq, odjq[sel], rtol=1e-12, atol=0)
    jq_rm = np.swapaxes(jq.reshape(jq.shape[0], -1, 3, 3), -1, -2)
    assert np.allclose(jq_rm, ojq[sel], rtol=1e-12, atol=1e-12)


def test_renumbered_space_is_a_permutation(sf):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (3, 3, 3))
    V0 = sf.FESpace(model, 2)
    V1 = sf.FESpace(model, 2, renumber_seed=7)
    d0 = V0.get_cell_dof_ids().data
    d1 = V1.get_cell_dof_ids().data
    free = d0 > 0
    assert np.array_equal(d1[free], V1.perm[d0[free] - 1] + 1)
    assert np.array_equal(d1[~free], d0[~free])
    X0 = V0.free_dof_coordinates()
    X1 = V1.free_dof_coordinates()
    assert np.allclose(X1[V1.perm], X0)


def test_rhs_matches_oracle(sf):
    p, deg, n = 3, 6, 3
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n), perturb=0.1, seed=2)
    V = sf.FESpace(model, p)
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    b = sf.assemble_rhs(m, V, O.sin_forcing)
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om, perturb=0.1, seed=2)
    bo = O.rhs(om, mesh, O.sin_forcing)
    assert np.abs(b - bo).max() < 1e-13 * np.abs(bo).max()


def test_free_dof_coordinates(sf):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (2, 3, 4))
    V = sf.FESpace(model, 2)
    om = O.make_map(3, 2, 4)
    mesh = O.cartesian_mesh(3, (2, 3, 4), 2, om)
    assert np.allclose(V.free_dof_coordinates(), O.free_dof_coordinates(mesh))


def test_cellwise_numbering(sf):
    """Cell-by-cell numbering: a permutation; the first cell's free dofs come first,
    in local order; the table of the renumbered space is the permuted lexicographic one."""
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (3, 4, 2))
    V = sf.FESpace(model, 3, cellwise=True)
    L = sf.FESpace(model, 3)
    n = V.num_free_dofs
    assert np.array_equal(np.sort(V.perm), np.arange(n))
    dv = np.asarray(V.get_cell_dof_ids().data)
    dl = np.asarray(L.get_cell_dof_ids().data)
    free = dl > 0
    assert np.array_equal(dv[free], V.perm[dl[free] - 1] + 1)
    assert np.array_equal(dv[~free], dl[~free])
    first = dv[:64][dv[:64] > 0]
    assert np.array_equal(first, np.arange(1, first.size + 1))
    with pytest.raises(ValueError):
        sf.FESpace(model, 3, cellwise=True, renumber_seed=1)


def test_gridap_numbering_groups_by_face_dimension(sf):
    """Free dofs of the face-grouped numbering: a permutation; vertex dofs first in
    vertex order, then edge, face and cell-interior dofs; each cell's interior dofs
    consecutive (x fastest)."""
    import numpy as np
    p, n = 3, (3, 4, 2)
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), n)
    V = sf.FESpace(model, p, numbering="gridap")
    perm = V.perm
    nf = V.num_free_dofs
    assert np.array_equal(np.sort(perm), np.arange(nf))
    fx, fy, fz = V.free_grid
    gz, gy, gx = np.meshgrid(np.arange(1, fz + 1), np.arange(1, fy + 1), np.arange(1, fx + 1),
                             indexing="ij")
    g = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
    dim = 3 - ((g % p) == 0).sum(axis=1)
    starts = [perm[dim == d].min() for d in range(4)]
    ends = [perm[dim == d].max() for d in range(4)]
    for d in range(3):  # the groups follow each other
        assert ends[d] + 1 == starts[d + 1]
    assert starts[0] == 0 and ends[3] == nf - 1
    v = g[dim == 0] // p  # vertex dofs in vertex order (x fastest)
    vl = v[:, 0] + (n[0] + 1) * (v[:, 1] + (n[1] + 1) * v[:, 2])
    assert np.array_equal(np.argsort(perm[dim == 0]), np.argsort(vl, kind="stable"))
    c = g[dim == 3] // p  # cell c's interior dofs: a block of (p-1)^3 ids
    cid = c[:, 0] + n[0] * (c[:, 1] + n[1] * c[:, 2])
    assert np.array_equal((perm[dim == 3] - starts[3]) // (p - 1) ** 3, cid)
