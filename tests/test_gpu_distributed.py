"""Slab operators on the GPU (sf_set_structured_slab, sf_cgd_*), with every
part in one process: the halo planes between parts are copied on the device,
so nothing waits on another rank. Checked against the single-operator path
(itself checked against the oracle in test_gpu_apply.py / test_gpu_cg.py)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(sf, p, n, domain=(0, 1, 0, 1, 0, 1)):
    deg = 2 * p
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    model = sf.CartesianDiscreteModel(domain, n)
    V = sf.FESpace(model, p)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, deg))
    return m, model, V, A


def _gather(D, parts, n):
    out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    for sl, v in D.owned(parts):
        out[sl] = v
    return out


@pytest.mark.parametrize("p,n,nparts", [(4, (4, 5, 9), 3), (4, (3, 3, 8), 4), (2, (5, 4, 7), 2),
                                        (3, (4, 4, 5), 5), (4, (4, 4, 6), 1)])
def test_slab_apply_matches_single_operator(sf, p, n, nparts):
    m, model, V, A = _setup(sf, p, n)
    D = sf.distributed.DistributedLazyMatrix(m, model, nparts=nparts)
    x = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, A.n)).cuda()
    y_ref = A @ x
    ys = D.mul(D.new_vector(), D.from_global(x))
    y = _gather(D, ys, A.n)
    assert not torch.isnan(y).any()
    assert (y - y_ref).abs().max().item() <= 1e-13 * y_ref.abs().max().item()


def test_slab_halo_is_read_and_owned_only_written(sf):
    """A slab writes its owned planes only, and its result depends on the halo planes."""
    p, n = 4, (3, 3, 6)
    m, model, V, A = _setup(sf, p, n)
    D = sf.distributed.DistributedLazyMatrix(m, model, nparts=2)
    x = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, A.n)).cuda()
    xs = D.from_global(x)
    L, e = D.layouts[0], D.engines[0]
    y = torch.full_like(xs[0], 7.0)
    e.apply(xs[0], y)
    assert (y[:L.owned.start] == 7.0).all() and (y[L.owned.stop:] == 7.0).all()
    x_nohalo = xs[0].clone()
    x_nohalo[L.recv_above()] = 0
    y2 = torch.empty_like(y)
    e.apply(x_nohalo, y2)
    assert (y2[L.owned] - y[L.owned]).abs().max().item() > 0


def test_slab_diagonal_matches_single_operator(sf):
    p, n = 4, (3, 4, 7)
    m, model, V, A = _setup(sf, p, n)
    d_ref = A.diagonal()
    D = sf.distributed.DistributedLazyMatrix(m, model, nparts=3)
    parts = []
    for e in D.engines:
        d = torch.zeros(e.layout.n, dtype=torch.float64, device="cuda")
        sf._lib.check(sf._lib.lib.sf_diagonal(e._h, 0, e._p(d), e._s()), e._h, "sf_diagonal")
        parts.append(d)
    d = _gather(D, parts, A.n)
    assert (d - d_ref).abs().max().item() <= 1e-13 * d_ref.abs().max().item()


@pytest.mark.parametrize("nparts", [1, 3])
def test_distributed_cg_matches_single_operator(sf, nparts):
    p, n = 4, (4, 4, 6)
    m, model, V, A = _setup(sf, p, n, domain=(0, 2, 0, 1, 0, 1))  # anisotropic cells
    b = torch.from_numpy(np.random.default_rng(4).uniform(-1, 1, A.n)).cuda()
    x_ref, info_ref = sf.cg(A, b, reltol=1e-10, mode="jacobi")
    D = sf.distributed.DistributedLazyMatrix(m, model, nparts=nparts)
    xs, info = sf.distributed.cg(D, D.from_global(b), reltol=1e-10)
    assert info["converged"] and info["relres"] <= 1e-10
    assert abs(info["iters"] - info_ref["iters"]) <= 1
    x = _gather(D, xs, A.n)
    assert (x - x_ref).abs().max().item() < 1e-9 * x_ref.abs().max().item()


def test_slab_operator_rejects_single_operator_calls(sf):
    p, n = 2, (3, 3, 4)
    m, model, V, A = _setup(sf, p, n)
    D = sf.distributed.DistributedLazyMatrix(m, model, nparts=2)
    e = D.engines[0]
    b = torch.zeros(e.layout.n, dtype=torch.float64, device="cuda")
    st = sf._lib.lib.sf_cg(e._h, 0, e._p(b), e._p(b), 1e-10, 10, None, None, e._s())
    assert st == sf._lib.SF_ERR_UNSUPPORTED
