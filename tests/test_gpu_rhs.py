"""Matrix-free right-hand side on the device (sf_rhs) against the oracle's
restatement of the linear form v -> int(f v) dOmega (oracle.rhs)."""
import math

import numpy as np
import pytest
import torch

from oracle import sumfac_oracle as O

pytestmark = pytest.mark.gpu


def _f_torch(X):
    return 3 * math.pi ** 2 * torch.prod(torch.sin(math.pi * X), dim=-1)


@pytest.mark.parametrize("p,deg,n,perturb,renumber", [
    (2, 4, (4, 3, 5), 0.0, None),      # structured, tiled-path geometry (separable)
    (4, 8, (3, 3, 3), 0.0, None),
    (3, 6, 3, 0.2, None),              # deformed cells: per-point weights
    (2, 6, 3, 0.1, 11),                # renumbered table gather, SQ = SB + 1
    (5, 8, 2, 0.0, None),              # SQ = SB - 1 ... SB
])
def test_rhs_matches_oracle(sf, p, deg, n, perturb, renumber):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), n if isinstance(n, tuple) else (n,) * 3,
                                      perturb=perturb, seed=3)
    V = sf.FESpace(model, p, renumber_seed=renumber)
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, deg))
    b = sf.rhs(A, _f_torch).cpu().numpy()
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om, perturb=perturb, seed=3, renumber_seed=renumber)
    b_ref = O.rhs(om, mesh, O.sin_forcing)
    assert np.abs(b - b_ref).max() <= 1e-12 * np.abs(b_ref).max()
    # the host assembly of the package agrees too
    b_host = sf.assemble_rhs(m, V, O.sin_forcing)
    assert np.abs(b - b_host).max() <= 1e-12 * np.abs(b_ref).max()


def test_rhs_of_point_values_and_errors(sf):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (3, 3, 3))
    V = sf.FESpace(model, 2)
    m = sf.SumFactorizationMap(3, (2,) * 3, (4,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, 4))
    X = sf.quadrature_points(A)
    assert X.shape == (27, 27, 3)
    ones = torch.ones(27, 27, dtype=torch.float64, device="cuda")
    b1 = sf.rhs(A, ones)  # integral of each basis function over its support
    # sum over all basis functions (free + Dirichlet) is the volume; the free part is less
    assert 0 < b1.sum().item() < 1.0
    with pytest.raises(ValueError):
        sf.rhs(A, ones[:, :5])
