"""Host logic of the z-slab decomposition (distributed.py) on the CPU: the
partition, the slab index arithmetic, the halo exchange, the sums over ranks
and the distributed CG loop, with the oracle standing in for the device parts
(tests/slab_oracle.py). The multi-process case runs world_size 2 over gloo."""
import os
import socket

import numpy as np
import pytest
import torch

from oracle import sumfac_oracle as O
from slab_oracle import OracleSlabEngine


def _problem(p, deg, n):
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om)
    return om, mesh, O.assembled_sparse(om, mesh)


def test_partition_and_owners(sf):
    D = sf.distributed
    assert D.slab_partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert D.slab_partition(4, 4) == [(0, 1), (1, 2), (2, 3), (3, 4)]
    with pytest.raises(ValueError):
        D.slab_partition(3, 4)
    assert [D.parts_of_rank(5, 2, r) for r in range(2)] == [[0, 1, 2], [3, 4]]
    assert [D.owner_of(g, 5, 2) for g in range(5)] == [0, 0, 0, 1, 1]


@pytest.mark.parametrize("p,n,nparts", [(2, (3, 2, 5), 3), (3, (2, 3, 4), 4), (1, (4, 4, 6), 2)])
def test_owned_points_cover_the_mesh_once(sf, p, n, nparts):
    D = sf.distributed
    nx, ny, nz = n
    nfree = (nx * p - 1) * (ny * p - 1) * (nz * p - 1)
    count = np.zeros(nfree, dtype=int)
    xg = torch.arange(nfree, dtype=torch.float64)
    for z0, z1 in D.slab_partition(nz, nparts):
        L = D.SlabLayout(nx, ny, nz, p, z0, z1)
        assert L.n == L.plane * ((z1 - z0 + 1) * p + 1)
        count[L.owned_global()] += 1
        xs = L.from_global(xg)
        assert torch.equal(xs[L.owned], xg[L.owned_global()])
    assert (count == 1).all()


def test_local_exchange_fills_every_halo(sf):
    D = sf.distributed
    nx, ny, nz, p = 2, 3, 7, 2
    m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (nx, ny, nz))
    A = D.DistributedLazyMatrix(m, model, nparts=4, engine=lambda L: None)
    nfree = (nx * p - 1) * (ny * p - 1) * (nz * p - 1)
    xg = torch.rand(nfree, dtype=torch.float64)
    ref = A.from_global(xg)
    xs = []
    for L, r in zip(A.layouts, ref):  # keep the owned points, clear the halos
        x = torch.zeros_like(r)
        x[L.owned] = r[L.owned]
        xs.append(x)
    A.exchange(xs)
    for x, r in zip(xs, ref):
        assert torch.equal(x, r)


@pytest.mark.parametrize("nparts", [1, 2, 3])
def test_distributed_mul_matches_oracle(sf, nparts):
    p, deg, n = 2, 4, (3, 2, 5)
    om, mesh, S = _problem(p, deg, n)
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), n)
    A = sf.distributed.DistributedLazyMatrix(m, model, nparts=nparts,
                                             engine=lambda L: OracleSlabEngine(S, L))
    xg = np.random.default_rng(0).uniform(-1, 1, S.shape[0])
    xs = A.from_global(torch.from_numpy(xg))
    for L, x in zip(A.layouts, xs):  # only the owned points are known before the exchange
        x[:L.owned.start] = 0
        x[L.owned.stop:] = 0
    ys = A.mul(A.new_vector(), xs)
    y = np.zeros_like(xg)
    for sl, v in A.owned(ys):
        y[sl] = v.numpy()
    assert np.abs(y - S @ xg).max() <= 1e-13 * np.abs(S @ xg).max()


def test_distributed_cg_matches_oracle(sf):
    p, deg, n = 2, 4, (3, 3, 6)
    om, mesh, S = _problem(p, deg, n)
    b = O.rhs(om, mesh, O.sin_forcing)
    d = S.diagonal()
    x_ref, it_ref, _ = O.cg(lambda v: S @ v, b, reltol=1e-10, precond=lambda r: r / d)
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), n)
    A = sf.distributed.DistributedLazyMatrix(m, model, nparts=3,
                                             engine=lambda L: OracleSlabEngine(S, L))
    xs, info = sf.distributed.cg(A, A.from_global(torch.from_numpy(b)), reltol=1e-10,
                                 check_every=3)
    assert info["converged"] and abs(info["iters"] - it_ref) <= 1
    x = np.zeros_like(b)
    for sl, v in A.owned(xs):
        x[sl] = v.numpy()
    assert np.abs(x - x_ref).max() < 1e-8 * np.abs(x_ref).max()


# ---------------------------------------------------------------------------
# two processes over gloo
# ---------------------------------------------------------------------------


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, out_dir):
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, repo)
    sys.path.insert(0, os.path.join(repo, "tests"))
    import torch.distributed as dist
    import __graft_entry__ as g
    from oracle import sumfac_oracle as Ox
    from slab_oracle import OracleSlabEngine as Eng
    sf = g.load()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        p, deg, n = 2, 4, (2, 3, 7)
        om = Ox.make_map(3, p, deg)
        mesh = Ox.cartesian_mesh(3, n, p, om)
        S = Ox.assembled_sparse(om, mesh)
        b = Ox.rhs(om, mesh, Ox.sin_forcing)
        m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
        model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), n)
        # 3 parts on 2 ranks: rank 0 holds parts 0 and 1 (a local cut), rank 1 part 2
        A = sf.distributed.DistributedLazyMatrix(m, model, nparts=3, group=dist.group.WORLD,
                                                 engine=lambda L: Eng(S, L))
        xg = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, S.shape[0]))
        ys = A.mul(A.new_vector(), A.from_global(xg))
        xs, info = sf.distributed.cg(A, A.from_global(torch.from_numpy(b)), reltol=1e-10)
        res = {"y": [(sl.start, sl.stop, v.numpy()) for sl, v in A.owned(ys)],
               "x": [(sl.start, sl.stop, v.numpy()) for sl, v in A.owned(xs)],
               "iters": info["iters"], "relres": info["relres"], "parts": A.comm.parts}
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), res, allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_match_oracle(sf, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_gloo_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    p, deg, n = 2, 4, (2, 3, 7)
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om)
    S = O.assembled_sparse(om, mesh)
    b = O.rhs(om, mesh, O.sin_forcing)
    xg = np.random.default_rng(3).uniform(-1, 1, S.shape[0])
    d = S.diagonal()
    x_ref, it_ref, _ = O.cg(lambda v: S @ v, b, reltol=1e-10, precond=lambda r: r / d)
    y = np.full(S.shape[0], np.nan)
    x = np.full(S.shape[0], np.nan)
    res = [np.load(tmp_path / f"rank{r}.npy", allow_pickle=True).item() for r in range(world)]
    assert res[0]["parts"] == [0, 1] and res[1]["parts"] == [2]
    for r in res:
        for a, e, v in r["y"]:
            y[a:e] = v
        for a, e, v in r["x"]:
            x[a:e] = v
        assert abs(r["iters"] - it_ref) <= 1
        assert r["iters"] == res[0]["iters"] and r["relres"] == res[0]["relres"]
    assert not np.isnan(y).any() and not np.isnan(x).any()
    assert np.abs(y - S @ xg).max() <= 1e-13 * np.abs(S @ xg).max()
    assert np.abs(x - x_ref).max() < 1e-8 * np.abs(x_ref).max()


def test_batched_problems_shard_by_cost(sf):
    """The batched form's independent problems are dealt to ranks by a greedy
    cost balance (no exchange between ranks); every rank gets the same answer."""
    shard, cost = sf.batch.shard, sf.batch.apply_cost
    rng = np.random.default_rng(2024)
    specs = [(int(rng.integers(8, 41)), int(rng.integers(2, 7))) for _ in range(48)]
    costs = [cost(n ** 3, p, 4) for n, p in specs]
    for nranks in (1, 2, 3, 8):
        parts = shard(costs, nranks)
        assert sorted(i for part in parts for i in part) == list(range(48))
        loads = [sum(costs[i] for i in part) for part in parts]
        # greedy largest-first: no rank exceeds the mean by more than the largest problem
        assert max(loads) <= sum(costs) / nranks + max(costs)
        assert parts == shard(costs, nranks)
    with pytest.raises(ValueError):
        shard(costs, 0)
