"""Batched form: one CUDA-graph launch of persistent per-order kernels must give,
for every problem and right-hand side, the single-problem apply's result
(and the oracle's)."""
import numpy as np
import pytest

from oracle import sumfac_oracle as O

pytestmark = pytest.mark.gpu


def make_ops(sf, specs):
    ops = []
    for n, p in specs:
        model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n))
        V = sf.FESpace(model, p)
        m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)  # p+1 Gauss points
        ops.append(sf.LazyMatrix(m, V, V, sf.Measure(model, 2 * p)))
    return ops


SPECS = [(3, 2), (5, 4), (2, 6), (4, 3), (3, 5), (6, 2), (2, 4), (7, 1), (4, 4)]


@pytest.mark.parametrize("dt_name", ["float64", "float32"])
def test_batch_matches_single_applies(sf, dt_name):
    import torch
    from ncihackaton2023_b200.batch import Batch, column_major
    dt = getattr(torch, dt_name)
    tol = 1e-13 if dt == torch.float64 else 1e-6
    nrhs = 3
    ops = make_ops(sf, SPECS)
    b = Batch(ops, nrhs)
    assert b.ngroups == len({p for _, p in SPECS})
    g = torch.Generator(device="cuda").manual_seed(0)
    X = [column_major(op.n, nrhs, dt) for op in ops]
    Y = [column_major(op.n, nrhs, dt) for op in ops]
    for x in X:
        x.copy_(torch.rand(x.shape, dtype=dt, device="cuda", generator=g) * 2 - 1)
    for rnd in range(3):
        if rnd == 1:
            b.autotune(X, Y)
        if rnd == 2:  # new buffers: the graph is captured again
            Y = [column_major(op.n, nrhs, dt) for op in ops]
        for y in Y:
            y.fill_(float("nan"))
        b.apply(X, Y)
        torch.cuda.synchronize()
        for op, x, y in zip(ops, X, Y):
            for k in range(nrhs):
                ref = op @ x[:, k].contiguous()
                err = ((y[:, k] - ref).abs().max() / ref.abs().max()).item()
                assert err < tol, (op.model.partition, op.m.order, k, err)


def test_batch_against_oracle(sf):
    import torch
    from ncihackaton2023_b200.batch import Batch, column_major
    specs = [(3, 2), (2, 5), (4, 3)]
    ops = make_ops(sf, specs)
    b = Batch(ops, 2)
    X = [column_major(op.n, 2) for op in ops]
    Y = [column_major(op.n, 2) for op in ops]
    rng = np.random.default_rng(4)
    xs = [rng.uniform(-1, 1, (op.n, 2)) for op in ops]
    for x, xn in zip(X, xs):
        x.copy_(torch.from_numpy(xn))
    b.apply(X, Y)
    for (n, p), y, xn in zip(specs, Y, xs):
        om = O.make_map(3, p, 2 * p)
        mesh = O.cartesian_mesh(3, n, p, om)
        for k in range(2):
            ref = O.lazy_mul(om, mesh, xn[:, k])
            assert np.abs(y[:, k].cpu().numpy() - ref).max() < 1e-12 * np.abs(ref).max()


def test_batch_rejects_non_cartesian(sf):
    from ncihackaton2023_b200.batch import Batch
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (3, 3, 3), perturb=0.1)
    V = sf.FESpace(model, 2)
    m = sf.SumFactorizationMap(3, (2,) * 3, (4,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, 4))
    with pytest.raises(sf.SumFacError) as e:
        Batch([A], 1)
    assert e.value.status == 4
