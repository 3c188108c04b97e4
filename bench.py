"""Benchmark: Q4 64^3 matrix-free Laplacian apply (GDOF/s) and CG to relres
1e-10, FP64 vs mixed precision, on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one apply y = A x of the Q4 (p = 4), 5-point Gauss, 64^3-cell
unit-cube problem with homogeneous Dirichlet boundary. The GDOF/s figure
counts the 257^3 = 16,974,593 dofs of the mesh, boundary included. x is
drawn from U[-1, 1] (seed 0) and is resident in HBM. Each timed step uses the
next of 4 rotating x/y buffer pairs (1.09 GB in total, above the 126 MB L2),
so a step never starts with its inputs in L2.

With N > 1 (torchrun, one process per GPU), one problem of 64 x 64 x 64N
cells is split into N z-slabs of 64^3 cells, one per rank (weak scaling:
(256+1)^2 (256N+1) dofs in all). A step is one distributed apply: the halo
exchange of the input (NCCL point-to-point, p + 1 planes per cut) and each
rank's slab apply. The timed region is bracketed by a barrier and a device
synchronize, and the reported time is the maximum over ranks.

``--impl reference`` times the reference's CPU path on this machine's host
cores instead. Julia and Gridap are not available, so it runs the C
restatement of the reference loops (oracle/sumfac_ref.c), using all host
threads, on a bounded sample of the cells per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

P, DEG, NCELL = 4, 8, 64
N_DOF_TOTAL = (NCELL * P + 1) ** 3  # 16,974,593
METRIC = "Q4 64^3 Laplacian apply GDOF/s; CG time to relres 1e-10, mixed vs FP64, 1 B200"
WORKLOAD = "Q4 64^3 affine hex, 5-pt Gauss, homogeneous Dirichlet, FP64 apply y=Ax"
# DRAM bytes (read + write) of one apply launch on this workload, from one ncu
# capture of the kernel (dram__bytes_read.sum + dram__bytes_write.sum).
NCU_TRAFFIC_BYTES = {"tiled-cartesian": 224.9e6}  # 132.7 MB read + 92.2 MB written


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cg", action="store_true", help="skip the CG solves")
    ap.add_argument("--cg-only", action="store_true",
                    help="only the CG solves (autotuned tiles; no apply leg): for profiling")
    ap.add_argument("--cg-maxiter", type=int, default=6000,
                    help="iteration cap of each CG solve (and of the multigrid section's solve)")
    ap.add_argument("--section", choices=["batched", "adjoint", "deformed_q8", "quad2d",
                                          "table_gather", "multigrid"],
                    default=None,
                    help="run only this secondary configuration (no apply leg): for profiling")
    ap.add_argument("--deformed-cells", type=int, default=32,
                    help="cells per direction of the deformed Q8 section")
    ap.add_argument("--deformed-cg", type=int, default=1500,
                    help="CG iteration budget of the deformed Q8 section (0: no CG)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the full-size parity checks against the C restatement")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the batched, adjoint, deformed-mesh, 2D and table-gather sections")
    ap.add_argument("--tile", type=int, default=None,
                    help="force tile candidate K of the FP64 tiled kernel (skips the autotuner)")
    ap.add_argument("--cells", type=int, default=64,
                    help="cells per direction (64 is the benchmark; smaller only for profiling)")
    a = ap.parse_args()
    global NCELL, N_DOF_TOTAL, DO_PARITY
    DO_PARITY = not a.no_parity
    NCELL = a.cells
    N_DOF_TOTAL = (NCELL * P + 1) ** 3
    return a


# ----------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.15)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------


def build_problem(sf):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (NCELL,) * 3)
    V = sf.FESpace(model, P)
    m = sf.SumFactorizationMap(3, (P,) * 3, (DEG,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, DEG))
    return m, model, V, A


# count_manual_flops_poisson_matrix_free(1, 3, (9,)*3, (9,)*3, count_only_fma_ops=false,
# structured_mesh_opt=false) of src/Utils.jl:33-72: flops per deformed Q8 cell
Q8_DEFORMED_FLOPS_PER_CELL = 352107


def HBM_PEAK_GBS():
    """The measured copy bandwidth of MEASURED_PEAKS.json, else the fallback figure."""
    try:
        return float(json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return 6650.0


def roofline_entry(achieved_gbs, peaks, traffic):
    peak = peaks.get("hbm_gbs") if peaks else None
    src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    return {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved_gbs / peak, 4), "traffic": traffic, "peak_source": src}


def cpu_baseline_port(nsteps_full=3):
    """The C restatement, 1 thread (the reference's mode), on full applies."""
    from oracle import cref
    from oracle import sumfac_oracle as O
    m = O.make_map(3, P, DEG)
    mesh = O.cartesian_mesh(3, NCELL, P, m)
    cq = O.cell_quantities(m, mesh)
    prob = cref.problem_from_oracle(m, mesh, cq)
    x = np.random.default_rng(0).uniform(-1, 1, mesh.n_free)
    y = np.empty(mesh.n_free)
    prob.mul(x, y)  # warm-up (first touch)
    t0 = time.perf_counter()
    for _ in range(nsteps_full):
        prob.mul(x, y)
    t = (time.perf_counter() - t0) / nsteps_full
    return {"value": round(N_DOF_TOTAL / t / 1e9, 6), "unit": "GDOF/s", "cores": 1, "kind": "port",
            "sample": f"{nsteps_full} full Q4 64^3 applies after 1 warm-up, C restatement of the "
                      f"reference loops (oracle/sumfac_ref.c), 1 thread; {t:.3f} s per apply"}


PARITY_TOL = {"f64": 1e-12, "f32": 2e-5}  # max |y - y_ref| / max |y_ref|, as in tests/


def _relerr(y, y_ref):
    return float(np.abs(y - y_ref).max() / max(np.abs(y_ref).max(), 1e-300))


def parity_headline(sf, A, x0, y64, dev):
    """Full-size parity of the benchmark apply, outside the timed region: the FP64
    result of the timed loop (y64 = A x0) and an FP32 apply of x0 against the C
    restatement of the reference loops (oracle/sumfac_ref.c, all host threads)."""
    import torch
    from oracle import cref
    from oracle import sumfac_oracle as O
    om = O.make_map(3, P, DEG)
    mesh = O.cartesian_mesh(3, NCELL, P, om)
    x = x0.cpu().numpy()
    t0 = time.perf_counter()
    y_ref = cref.mul_mesh(om, mesh, x)
    t_ref = time.perf_counter() - t0
    y32 = torch.empty(A.n, dtype=torch.float32, device=dev)
    sf.mul(y32, A, x0.float())
    e64 = _relerr(y64.cpu().numpy(), y_ref)
    e32 = _relerr(y32.double().cpu().numpy(), y_ref)
    return {"max_rel_err_f64": e64, "max_rel_err_f32": e32,
            "pass": e64 <= PARITY_TOL["f64"] and e32 <= PARITY_TOL["f32"], "tol": PARITY_TOL,
            "checker": f"C restatement of the reference loops, {cref.max_threads()} threads, "
                       f"{t_ref:.2f} s", "x": "the timed loop's x (U[-1,1], seed 0)"}


def time_tile_candidates(A, dev, reps=20):
    """ms per apply of every tile shape of the tiled kernel (FP64 and FP32)."""
    import torch
    out = {}
    for dt, key in ((torch.float64, "f64"), (torch.float32, "f32")):
        nc = int(A.info(f"tile_candidates_{key}"))
        x = torch.zeros(A.n, dtype=dt, device=dev)
        y = torch.empty_like(x)
        for k in range(nc):
            A.set_option(f"tile_candidate_{key}", k)
            for _ in range(3):
                A @ x
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                from __graft_entry__ import load
                load().mul(y, A, x)
            e1.record()
            torch.cuda.synchronize()
            out[f"{key}: {A.kernel_name(dt)}"] = round(e0.elapsed_time(e1) / reps, 4)
    return out


def run_slabs(args, sf, rank, world, dev):
    """N > 1: one 64 x 64 x 64N problem, one z-slab of 64^3 cells per rank."""
    import torch
    import torch.distributed as dist
    nz = NCELL * world
    m = sf.SumFactorizationMap(3, (P,) * 3, (DEG,) * 3)
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, world), (NCELL, NCELL, nz))
    D = sf.distributed.DistributedLazyMatrix(m, model, nparts=world, group=dist.group.WORLD,
                                             device=dev)
    D.autotune(torch.float64)
    dist.barrier()  # the world communicator exists before the first point-to-point exchange
    L = D.layouts[0]
    n_total = (NCELL * P + 1) ** 2 * (nz * P + 1)
    rng = np.random.default_rng(rank)
    NBUF = 4
    xs, ys = [], []
    for _ in range(NBUF):
        x = D.new_vector()
        x[0][L.owned] = torch.from_numpy(rng.uniform(-1, 1, L.owned.stop - L.owned.start)).to(dev)
        xs.append(x)
        ys.append(D.new_vector())
    for i in range(max(3, args.warmup)):
        D.mul(ys[i % NBUF], xs[i % NBUF])
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        ev0.record()
        for i in range(args.steps):
            D.mul(ys[i % NBUF], xs[i % NBUF])
        ev1.record()
        torch.cuda.synchronize()
    dist.barrier()
    t = torch.tensor([ev0.elapsed_time(ev1)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = t.item() / args.steps
    value = n_total / (ms_step * 1e-3) / 1e9

    # end to end: each rank's owned x from pinned host memory, the distributed apply,
    # and its owned y back to pinned host memory, every step
    e2e = None
    if not args.no_e2e:
        own = L.owned.stop - L.owned.start
        xh = torch.empty(own, dtype=torch.float64).pin_memory()
        yh = torch.empty(own, dtype=torch.float64).pin_memory()
        xh.copy_(xs[0][0][L.owned].cpu())
        ne2e = max(5, min(50, args.steps // 40))

        def e2e_step():
            xs[0][0][L.owned].copy_(xh, non_blocking=True)
            D.mul(ys[0], xs[0])
            yh.copy_(ys[0][0][L.owned], non_blocking=True)
            torch.cuda.synchronize()
        for _ in range(3):
            e2e_step()
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ne2e):
            e2e_step()
        te = torch.tensor([(time.perf_counter() - t0) / ne2e], device=dev)
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        te2e = te.item()
        e2e = {"value": round(n_total / te2e / 1e9, 4), "unit": "GDOF/s",
               "h2d_bytes_per_step": own * 8 * world, "d2h_bytes_per_step": own * 8 * world,
               "ms_per_step": round(te2e * 1e3, 4),
               "buffers": "pinned host, each rank's owned points, distributed apply"}
    peaks = None
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    alg_bytes = n_total * 16 / world  # per rank (one launch)
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GDOF/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: owned x ~ U[-1,1] (rank r: seed r)",
        "config": {"workload": f"Q4 64x64x{nz} affine hex (64^3 cells per rank), 5-pt Gauss, "
                               "homogeneous Dirichlet, FP64 apply y=Ax",
                   "n_cells": NCELL ** 3 * world, "order": P, "quad_points": 5,
                   "n_dof_total": n_total, "kernel": "tiled-cartesian (z-slab)",
                   "tile": {"f64": D.engines[0].kernel_name(torch.float64)},
                   "l2": "4 rotating x/y buffer sets (> 126 MB L2 per rank)",
                   "parallelism": f"z-slab x{world}, halo exchange over NCCL"},
        "e2e": e2e,
        "gpu_launches": args.steps,
        "roofline": roofline_entry(alg_bytes / (ms_step * 1e-3) / 1e9, peaks, None),
        "clocks": clk.summary(),
    }
    out["roofline"]["algorithmic_bytes_per_launch"] = alg_bytes
    try:
        out["batched_sharded"] = run_batched_sharded(sf, dev, rank, world)
    except Exception as e:  # reported, not fatal; every rank takes the same steps
        out["batched_sharded"] = {"error": f"{type(e).__name__}: {e}"}
    return out


def run_batched_sharded(sf, dev, rank, world, nprob=48, nrhs=4, seed=2024, reps=10):
    """The batched draw of run_batched (48 problems, 4 right-hand sides, FP64) dealt
    to the ranks by batch.shard (largest estimated cost first, to the lightest
    rank): every rank applies its own problems in one graph launch, with no
    exchange. Time: max over ranks of the device time of `reps` launches."""
    import torch
    import torch.distributed as dist
    from ncihackaton2023_b200.batch import Batch, apply_cost, column_major, shard
    rng = np.random.default_rng(seed)
    specs = [(int(rng.integers(8, 41)), int(rng.integers(2, 7))) for _ in range(nprob)]
    mine = shard([apply_cost(n ** 3, p, nrhs) for n, p in specs], world)[rank]
    ops, X, Y = [], [], []
    for i in mine:
        n, p = specs[i]
        model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n))
        V = sf.FESpace(model, p)
        m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
        op = sf.LazyMatrix(m, V, V, sf.Measure(model, 2 * p))
        ops.append(op)
        x = column_major(op.n, nrhs, torch.float64, dev)
        g = torch.Generator(device=dev).manual_seed(seed + i)
        x.copy_(torch.rand(x.shape, dtype=torch.float64, device=dev, generator=g) * 2 - 1)
        X.append(x)
        Y.append(column_major(op.n, nrhs, torch.float64, dev))
    b = Batch(ops, nrhs) if ops else None
    if b is not None:
        b.autotune(X, Y)
        for _ in range(3):
            b.apply(X, Y)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        if b is not None:
            b.apply(X, Y)
    e1.record()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1) / reps], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dofs = sum((n * p + 1) ** 3 for n, p in specs) * nrhs
    mine_dofs = torch.tensor([float(sum((specs[i][0] * specs[i][1] + 1) ** 3 for i in mine) * nrhs)],
                             device=dev)
    dist.all_reduce(mine_dofs, op=dist.ReduceOp.MAX)
    return {"problems": nprob, "nrhs": nrhs, "ms_per_apply_max_over_ranks": round(t.item(), 4),
            "gdof_s": round(dofs / (t.item() * 1e-3) / 1e9, 2),
            "largest_rank_share": round(mine_dofs.item() / dofs, 4),
            "sharding": "batch.shard: largest cost first, to the lightest rank; no exchange"}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import __graft_entry__ as g

    sf = g.load()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        out = run_slabs(args, sf, rank, world, dev)
        dist.barrier()
        return out
    if args.section is not None:
        fn = {"batched": run_batched, "adjoint": run_adjoint, "quad2d": run_quad2d,
              "deformed_q8": lambda sf_, dev_: run_deformed(sf_, dev_, n=args.deformed_cells,
                                                            cg_iters=args.deformed_cg),
              "table_gather": run_table_gather,
              "multigrid": lambda sf_, dev_: run_multigrid(sf_, dev_, args.cg_maxiter)}
        return {args.section: fn[args.section](sf, dev)}
    m, model, V, A = build_problem(sf)
    if args.cg_only:
        A.autotune(torch.float64)
        A.autotune(torch.float32)
        return {"cg": run_cg(sf, m, model, V, A, dev, args.cg_maxiter)}
    tile_ms = {}
    if args.tile is not None:
        A.set_option("tile_candidate_f64", args.tile)
        tuned = {"f64": A.kernel_name(torch.float64), "f32": A.kernel_name(torch.float32)}
    else:
        tile_ms = time_tile_candidates(A, dev)
        tuned = {"f64": A.autotune(torch.float64), "f32": A.autotune(torch.float32)}
    n = V.num_free_dofs
    rng = np.random.default_rng(0 + rank)
    x0 = torch.from_numpy(rng.uniform(-1, 1, n)).to(dev)
    NBUF = 4
    xs = [x0.clone() for _ in range(NBUF)]
    ys = [torch.empty_like(x0) for _ in range(NBUF)]
    stream = torch.cuda.current_stream()
    for i in range(max(3, args.warmup)):
        sf.mul(ys[i % NBUF], A, xs[i % NBUF])
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for i in range(args.steps):
            sf.mul(ys[i % NBUF], A, xs[i % NBUF])
        ev1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = t.item()
    ms_step = ms / args.steps
    value = world * N_DOF_TOTAL / (ms_step * 1e-3) / 1e9
    kernel_path = "tiled-cartesian" if A.uses_tiled_kernel() else "general-element"
    parity = None
    if rank == 0 and not args.no_parity:
        log("parity of the benchmark apply")
        parity = parity_headline(sf, A, xs[0], ys[0], dev)
        log(f"parity: {parity}")

    # end to end through the public host-buffer call (mul! on host vectors)
    e2e = None
    if not args.no_e2e:
        xh = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
        yh = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
        xh[:] = x0.cpu().numpy()
        for _ in range(3):
            sf.mul(yh, A, xh)
        ne2e = max(5, min(50, args.steps // 40))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ne2e):
            sf.mul(yh, A, xh)
        te2e = (time.perf_counter() - t0) / ne2e
        if world > 1:
            t = torch.tensor([te2e], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te2e = t.item()
        e2e = {"value": round(world * N_DOF_TOTAL / te2e / 1e9, 4), "unit": "GDOF/s",
               "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8,
               "ms_per_step": round(te2e * 1e3, 4),
               "buffers": "pinned host; sf_mul_host pipelines the copies in, the apply and "
                          "the copies out over 8 groups of tile rows on three streams"}

    peaks = None
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    alg_bytes = N_DOF_TOTAL * 16
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GDOF/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: x ~ U[-1,1] seed 0 (rank r: seed r)",
        "config": {"workload": WORKLOAD, "n_cells": NCELL ** 3, "order": P, "quad_points": 5,
                   "n_dof_total": N_DOF_TOTAL, "n_free": n, "kernel": kernel_path,
                   "tile": tuned, "tile_ms": tile_ms,
                   "l2": "4 rotating x/y pairs (1.09 GB) > 126 MB L2",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": e2e,
        "parity": parity,
        "gpu_launches": args.steps * A.kernels_per_apply(),
        "roofline": roofline_entry(achieved, peaks,
                                   NCU_TRAFFIC_BYTES.get(kernel_path) if NCELL == 64 else None),
        "flops_reference_model": {"per_apply_gflop": 5.996544, "achieved_tflops":
                                  round(5.996544 / (ms_step * 1e-3) / 1e3, 3)},
    }
    out["clocks"] = clk.summary()
    out["roofline"]["algorithmic_bytes_per_launch"] = alg_bytes

    if not args.no_secondary and world == 1 and NCELL == 64:
        t_sec = time.perf_counter()
        for key, fn in (("batched", run_batched), ("adjoint", run_adjoint),
                        ("deformed_q8", run_deformed), ("quad2d", run_quad2d),
                        ("table_gather", run_table_gather)):
            if time.perf_counter() - t_sec > SECONDARY_BUDGET_S:
                out[key] = {"skipped": "secondary time budget spent"}
                continue
            log(key)
            try:
                out[key] = fn(sf, dev)
            except Exception as e:  # a failed section is reported, not fatal
                out[key] = {"error": f"{type(e).__name__}: {e}"}
            log(f"{key}: {out[key]}")
    if not args.no_cg:
        out["cg"] = run_cg(sf, m, model, V, A, dev, args.cg_maxiter)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline_port()
    out["summary"] = summarize(out)
    if world > 1:
        dist.barrier()
    return out


def summarize(out):
    """The solver and form results of the sections in a few lines (ms, iterations)."""
    def pick(d, *keys):
        for k in keys:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    def solve(d):
        if not isinstance(d, dict):
            return None
        return {k: d.get(k) for k in ("ms", "iters", "converged") if k in d}
    summ = {"apply_gdof_s": out.get("value"), "roofline_frac": pick(out, "roofline", "frac"),
            "parity_pass": pick(out, "parity", "pass")}
    cg = out.get("cg")
    if isinstance(cg, dict):
        for rhs, d in (("manufactured", cg), ("rough", cg.get("rough_rhs"))):
            summ[f"cg_{rhs}"] = {k: solve(pick(d, k)) for k in ("f64", "f64_plain", "mixed",
                                                             "mg_f64", "mg_mixed")}
    dq = out.get("deformed_q8")
    if isinstance(dq, dict):
        summ["deformed_q8"] = {"apply_ms": {k: pick(dq, k, "ms") for k in ("f64", "f32")},
                               "parity_pass": pick(dq, "parity", "pass"),
                               "mg_mixed": solve(dq.get("cg_mg_mixed")),
                               "mg_f64": solve(dq.get("cg_mg_f64")),
                               "jacobi_f64_1500_converged": pick(dq, "cg_f64", "converged")}
    bt = out.get("batched")
    if isinstance(bt, dict):
        summ["batched_ms"] = {k: pick(bt, k, "ms_graph") for k in ("f64", "f32")}
        summ["batched_parity_pass"] = all(pick(bt, k, "parity", "pass") is not False
                                          for k in ("f64", "f32"))
    return summ


CG_MAXITER = 6000
SECONDARY_BUDGET_S = 180.0
DO_PARITY = True  # full-size parity checks of the secondary sections (--no-parity: off)


def _timed_solves(sf, A, b, u_exact=None, warm=True, maxiter=CG_MAXITER, mg_modes=True):
    import torch
    res, sols = {}, {}
    for mode in ("jacobi", "mixed", "plain"):
        cg_mode = mode
        if warm:  # workspaces, diagonal
            sf.cg(A, b, reltol=1e-10, mode=cg_mode, maxiter=maxiter, raise_on_fail=False)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record()
            x, info = sf.cg(A, b, reltol=1e-10, mode=cg_mode, maxiter=maxiter,
                            raise_on_fail=False)
            e1.record()
            torch.cuda.synchronize()
        sols[mode] = x
        key = {"jacobi": "f64", "mixed": "mixed", "plain": "f64_plain"}[mode]
        ms = e0.elapsed_time(e1)
        res[key] = {"ms": round(ms, 3), "iters": info["iters"],
                    "ms_per_iter": round(ms / max(1, info["iters"]), 4),
                    "refinements": info["outer"], "relres": info["relres"],
                    "converged": info["converged"], "clocks": clk.summary()}
        log(f"cg {key}: {res[key]}")
        if u_exact is not None:
            res[key]["err_vs_exact_max"] = (x - u_exact).abs().max().item()
    for mode in ("mixed", "f64") if mg_modes else ():
        key = f"mg_{mode}"
        t0 = time.perf_counter()
        mg = sf.Multigrid(A, mode=mode)
        setup_s = time.perf_counter() - t0
        if warm:
            mg.solve(b, reltol=1e-10, maxiter=500, raise_on_fail=False)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record()
            x, info = mg.solve(b, reltol=1e-10, maxiter=500, raise_on_fail=False)
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        sols[key] = x
        res[key] = {"ms": round(ms, 3), "iters": info["iters"],
                    "ms_per_iter": round(ms / max(1, info["iters"]), 4), "relres": info["relres"],
                    "converged": info["converged"], "setup_s": round(setup_s, 2),
                    "levels": [f"Q{q} {c[0]}^3" for q, c in zip(mg.orders, mg.cells)],
                    "basis": mg.basis, "graph": mg.info("graph") == 1.0,
                    "clocks": clk.summary()}
        if u_exact is not None:
            res[key]["err_vs_exact_max"] = (x - u_exact).abs().max().item()
        res[key]["err_vs_f64_max_rel"] = ((x - sols["jacobi"]).abs().max() /
                                          sols["jacobi"].abs().max()).item()
        log(f"cg {key}: {res[key]}")
        mg.close()
        del mg
    if mg_modes:
        res["speedup_mg_mixed_vs_f64"] = round(res["f64"]["ms"] / res["mg_mixed"]["ms"], 3)
        res["speedup_mg_mixed_vs_f64_plain"] = round(res["f64_plain"]["ms"] / res["mg_mixed"]["ms"], 3)
        res["speedup_mg_mixed_vs_mg_f64"] = round(res["mg_f64"]["ms"] / res["mg_mixed"]["ms"], 3)
    res["f64"]["iteration"] = A.cg_kernel_name()
    res["mixed"]["err_vs_f64_max_rel"] = ((sols["mixed"] - sols["jacobi"]).abs().max() /
                                          sols["jacobi"].abs().max()).item()
    res["speedup_mixed_vs_f64"] = round(res["f64"]["ms"] / res["mixed"]["ms"], 3)
    res["speedup_mixed_vs_f64_plain"] = round(res["f64_plain"]["ms"] / res["mixed"]["ms"], 3)
    return res


def run_cg(sf, m, model, V, A, dev, maxiter=CG_MAXITER):
    """CG to relres 1e-10: the manufactured problem of the benchmark
    (f = 3 pi^2 sin sin sin; its right-hand side formed on the device by sf_rhs,
    and on the host by numpy as a cross-check), and a rough right-hand side
    (b ~ U[-1,1], seed 1): FP64 Jacobi CG, mixed precision (FP32 recurrence and
    apply with Jacobi, FP64 reliable updates), and FP64 CG without a
    preconditioner (the reference's cg! call, profiling/drivers.jl:87)."""
    import torch

    def f(X):  # f = 3 pi^2 sin(pi x) sin(pi y) sin(pi z) at (..., 3) device coordinates
        return 3 * np.pi ** 2 * torch.prod(torch.sin(np.pi * X), dim=-1)
    fq = f(sf.quadrature_points(A, dev))
    b = sf.rhs(A, fq)  # matrix-free right-hand side on the device
    torch.cuda.synchronize()
    rhs_ms = _events_ms(lambda: sf.rhs(A, fq), 5)
    t0 = time.perf_counter()
    b_host = sf.assemble_rhs(m, V, lambda X: 3 * np.pi ** 2 * np.prod(np.sin(np.pi * X), axis=-1))
    host_s = time.perf_counter() - t0
    rhs_info = {"device_ms": round(rhs_ms, 3), "host_numpy_s": round(host_s, 2),
                "max_rel_diff_device_vs_host": float(np.abs(b.cpu().numpy() - b_host).max() /
                                                     np.abs(b_host).max())}
    X = V.free_dof_coordinates()
    u_exact = torch.from_numpy(np.prod(np.sin(np.pi * X), axis=1)).to(dev)
    res = _timed_solves(sf, A, b, u_exact, maxiter=maxiter)
    res["preconditioner"] = "Jacobi (matrix-free diagonal)"
    res["rhs"] = rhs_info
    b_rough = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, V.num_free_dofs)).to(dev)
    res["rough_rhs"] = _timed_solves(sf, A, b_rough, maxiter=maxiter)
    return res


# ----------------------------------------------------------------------------
# secondary configurations (batched, adjoint, deformed high order)
# ----------------------------------------------------------------------------


def log(msg):
    sys.stderr.write(f"[bench {time.strftime('%H:%M:%S')}] {msg}\n")
    sys.stderr.flush()


def _events_ms(fn, reps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_batched(sf, dev, nprob=48, nrhs=4, seed=2024):
    """48 independent unit-cube problems, n^3 cells with n ~ U{8..40}, order
    p ~ U{2..6} with p+1 Gauss points, 4 right-hand sides each (x ~ U[-1,1],
    seed 2024 + problem), applied by one CUDA-graph launch (FP64 and FP32). The
    comparison is the same applies launched one problem at a time."""
    import torch
    from ncihackaton2023_b200.batch import Batch, column_major
    rng = np.random.default_rng(seed)
    specs = [(int(rng.integers(8, 41)), int(rng.integers(2, 7))) for _ in range(nprob)]
    ops = []
    for n, p in specs:
        model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n))
        V = sf.FESpace(model, p)
        m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
        ops.append(sf.LazyMatrix(m, V, V, sf.Measure(model, 2 * p)))
    dofs = sum((n * p + 1) ** 3 for n, p in specs) * nrhs
    out = {"problems": nprob, "nrhs": nrhs, "dof_total_x_rhs": dofs,
           "orders": sorted({p for _, p in specs}),
           "launch": "one CUDA graph launch per apply: one persistent kernel per order group "
                     "(problems of one order share it), the groups as concurrent graph branches"}
    oracle_meshes = []
    if DO_PARITY:
        from oracle import cref
        from oracle import sumfac_oracle as O
    for dt, key in ((torch.float64, "f64"), (torch.float32, "f32")):
        X, Y = [], []
        for i, op in enumerate(ops):
            x = column_major(op.n, nrhs, dt, dev)
            g = torch.Generator(device=dev).manual_seed(seed + i)
            x.copy_(torch.rand(x.shape, dtype=dt, device=dev, generator=g) * 2 - 1)
            X.append(x)
            Y.append(column_major(op.n, nrhs, dt, dev))
        b = Batch(ops, nrhs)
        tiles = b.autotune(X, Y)
        for _ in range(3):
            b.apply(X, Y)
        ms = _events_ms(lambda: b.apply(X, Y), 10)
        for op in ops:
            op.autotune(dt)

        def seq():
            for op, x, y in zip(ops, X, Y):
                sf.mul_multi(y, op, x)
        seq()
        ms_seq = _events_ms(seq, 3)
        vb = 8 if key == "f64" else 4
        alg = dofs * 2 * vb  # every right-hand side read and its result written once
        out[key] = {"ms_graph": round(ms, 3), "gdof_s": round(dofs / (ms * 1e-3) / 1e9, 2),
                    "ms_one_problem_at_a_time": round(ms_seq, 3),
                    "speedup_vs_sequential": round(ms_seq / ms, 3), "group_tiles": tiles,
                    "alg_bytes": alg, "achieved_gbs": round(alg / (ms * 1e-3) / 1e9, 1)}
        if DO_PARITY:
            # every problem and right-hand side of the graph launch against the C
            # restatement (the graph is run again so that Y is its result)
            b.apply(X, Y)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            worst = 0.0
            for i, (n, p) in enumerate(specs):
                if len(oracle_meshes) <= i:
                    om = O.make_map(3, p, 2 * p)
                    oracle_meshes.append((om, O.cartesian_mesh(3, n, p, om)))
                om, mesh = oracle_meshes[i]
                xi, yi = X[i].double().cpu().numpy(), Y[i].double().cpu().numpy()
                for j in range(nrhs):
                    worst = max(worst, _relerr(yi[:, j], cref.mul_mesh(om, mesh, xi[:, j])))
            out[key]["parity"] = {"max_rel_err": worst, "pass": worst <= PARITY_TOL[key],
                                  "cases": f"{nprob} problems x {nrhs} right-hand sides",
                                  "checker": f"C restatement, {cref.max_threads()} threads, "
                                             f"{time.perf_counter() - t0:.1f} s"}
        del X, Y, b
        torch.cuda.empty_cache()
    return out


def run_adjoint(sf, dev, n=32, p=3, seed=11):
    """Q3 32^3, 4-point Gauss, kappa = exp(g) with g ~ N(0, 0.5^2) per point:
    VJP kernel time, apply with kappa, and dJ/dkappa of J = 0.5||u - u_obs||^2 by
    adjoint CG (u_obs from a seeded kappa_true), checked by a central finite
    difference with step 1e-6 along a seeded direction."""
    import torch
    from ncihackaton2023_b200.adjoint import objective, objective_gradient
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n))
    V = sf.FESpace(model, p)
    m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, 2 * p))
    nc, nq = n ** 3, (p + 1) ** 3
    rng = np.random.default_rng(seed)
    kappa = torch.from_numpy(np.exp(rng.normal(0, 0.5, (nc, nq)))).to(dev)
    kappa_true = torch.from_numpy(np.exp(rng.normal(0, 0.5, (nc, nq)))).to(dev)
    b = torch.from_numpy(sf.assemble_rhs(m, V, lambda X: 3 * np.pi ** 2 *
                                         np.prod(np.sin(np.pi * X), axis=-1))).to(dev)
    x = torch.from_numpy(rng.uniform(-1, 1, A.n)).to(dev)
    yb = torch.from_numpy(rng.uniform(-1, 1, A.n)).to(dev)
    A.set_coefficient(kappa)
    y = torch.empty_like(x)
    A.kappa_vjp(x, yb)
    vjp_ms = _events_ms(lambda: A.kappa_vjp(x, yb), 20)
    apply_ms = _events_ms(lambda: sf.mul(y, A, x), 20)
    A.set_coefficient(kappa_true)
    u_obs, _ = sf.cg(A, b, reltol=1e-11, maxiter=CG_MAXITER)
    t0 = time.perf_counter()
    J, grad, u, info = objective_gradient(A, b, u_obs, kappa, reltol=1e-11)
    torch.cuda.synchronize()
    grad_s = time.perf_counter() - t0
    # a second coefficient, as the next step of an optimisation loop would set
    kappa_b = kappa * torch.exp(0.1 * torch.from_numpy(rng.normal(0, 1, (nc, nq))).to(dev))
    _, grad_b, _, _ = objective_gradient(A, b, u_obs, kappa_b, reltol=1e-11)
    # the same gradients with multigrid-preconditioned solves: at kappa the hierarchy is
    # built inside the first solve (that set-up is included); at kappa_b the kept
    # hierarchy follows the new coefficient (Multigrid.refresh, included)
    t0 = time.perf_counter()
    J_mg, grad_mg, _, info_mg = objective_gradient(A, b, u_obs, kappa, reltol=1e-11,
                                                   mode="mg_mixed", maxiter=500)
    torch.cuda.synchronize()
    grad_mg_s = time.perf_counter() - t0
    grad_mg_diff = ((grad_mg - grad).abs().max() / grad.abs().max()).item()
    t0 = time.perf_counter()
    _, grad_mg_b, _, info_mg_b = objective_gradient(A, b, u_obs, kappa_b, reltol=1e-11,
                                                    mode="mg_mixed", maxiter=500)
    torch.cuda.synchronize()
    grad_mg_next_s = time.perf_counter() - t0
    grad_mg_next_diff = ((grad_mg_b - grad_b).abs().max() / grad_b.abs().max()).item()
    for mg in A.__dict__.pop("_mg", {}).values():  # the checks below use Jacobi CG
        mg.close()
    d = torch.from_numpy(rng.normal(0, 1, (nc, nq))).to(dev)
    eps = 1e-6
    fd = (objective(A, b, u_obs, kappa + eps * d, 1e-11) -
          objective(A, b, u_obs, kappa - eps * d, 1e-11)) / (2 * eps)
    ad = torch.sum(grad * d).item()
    return {"mesh": f"{n}^3 Q{p}, {p + 1}-pt Gauss", "kappa_points": nc * nq,
            "vjp_ms": round(vjp_ms, 4), "apply_kappa_ms": round(apply_ms, 4),
            "gradient_s": round(grad_s, 4), "cg_iters": info, "J": J,
            "gradient_mg_s": round(grad_mg_s, 4), "mg_iters": info_mg,
            "gradient_mg_vs_jacobi_max_rel": grad_mg_diff,
            "gradient_mg_next_kappa_s": round(grad_mg_next_s, 4), "mg_next_iters": info_mg_b,
            "gradient_mg_next_vs_jacobi_max_rel": grad_mg_next_diff,
            "fd_directional": fd, "adjoint_directional": ad,
            "fd_rel_err": abs(fd - ad) / abs(fd)}


def run_deformed(sf, dev, n=32, p=8, seed=5, cg_iters=1500):
    """Q8 on 32^3 cells, interior vertices moved by U[-0.2h, 0.2h] (seeded),
    9-point Gauss, per-point symmetric metric (6 FP64 values) stored: FP64 and
    FP32 apply times and bytes moved, and CG to 1e-10 (FP64 and mixed)."""
    import torch
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n), perturb=0.2, seed=seed)
    V = sf.FESpace(model, p)
    m = sf.SumFactorizationMap(3, (p,) * 3, (2 * p,) * 3)
    t0 = time.perf_counter()
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, 2 * p))
    setup_s = time.perf_counter() - t0
    x = torch.from_numpy(np.random.default_rng(seed).uniform(-1, 1, A.n)).to(dev)
    y = torch.empty_like(x)
    res = {"mesh": f"{n}^3 Q{p}, {p + 1}-pt Gauss, perturbed 0.2h", "n_free": A.n,
           "setup_s": round(setup_s, 2), "kernel": A.kernel_name()}
    nq = (p + 1) ** 3
    ys_ = {}
    # the reference's flop model (src/Utils.jl:33-72) for Q8, 9 points, deformed cells
    model_gflop = n ** 3 * Q8_DEFORMED_FLOPS_PER_CELL / 1e9 if p == 8 else float("nan")
    for dt, key, vb in ((torch.float64, "f64", 8), (torch.float32, "f32", 4)):
        xx, yy = x.to(dt), y.to(dt)
        for _ in range(3):
            sf.mul(yy, A, xx)
        ms = _events_ms(lambda: sf.mul(yy, A, xx), 10)
        # the per-point metric (6 values, in the kernel's type) and x, y
        byts = n ** 3 * nq * 6 * vb + (n * p + 1) ** 3 * 2 * vb
        # reference-model flops (src/Utils.jl:33-72, deformed cells: structured_mesh_opt false)
        # against the nominal vector-pipe peak at 1965 MHz (148 SMs x 64 FP64 / 128 FP32 FMA per clock)
        tf = model_gflop / ms  # GFLOP / ms = TFLOP/s
        peak = 148 * (64 if key == "f64" else 128) * 2 * 1.965e9 / 1e12
        res[key] = {"ms": round(ms, 3), "gdof_s": round((n * p + 1) ** 3 / (ms * 1e-3) / 1e9, 2),
                    "alg_bytes": byts, "achieved_gbs": round(byts / (ms * 1e-3) / 1e9, 1),
                    "hbm_frac": round(byts / (ms * 1e-3) / 1e9 / HBM_PEAK_GBS(), 4),
                    "model_tflops": round(tf, 2), "model_tflops_frac_of_nominal_pipe":
                        round(tf / peak, 3), "nominal_pipe_tflops": round(peak, 1)}
        ys_[key] = yy.double().cpu().numpy()
    if DO_PARITY:  # the full-size applies against the C restatement (chunked geometry)
        from oracle import cref
        from oracle import sumfac_oracle as O
        om = O.make_map(3, p, 2 * p)
        mesh = O.cartesian_mesh(3, n, p, om, perturb=0.2, seed=seed)
        t0 = time.perf_counter()
        y_ref = cref.mul_mesh(om, mesh, x.cpu().numpy())
        e = {k: _relerr(v, y_ref) for k, v in ys_.items()}
        res["parity"] = {"max_rel_err_f64": e["f64"], "max_rel_err_f32": e["f32"],
                         "pass": e["f64"] <= PARITY_TOL["f64"] and e["f32"] <= PARITY_TOL["f32"],
                         "checker": f"C restatement, {cref.max_threads()} threads, "
                                    f"{time.perf_counter() - t0:.1f} s"}
        del mesh, y_ref
    b = torch.from_numpy(sf.assemble_rhs(m, V, lambda X: 3 * np.pi ** 2 *
                                         np.prod(np.sin(np.pi * X), axis=-1))).to(dev)
    log(f"deformed apply: {res}")
    # multigrid-preconditioned CG in Gauss-Lobatto nodes (FP32 V-cycle, FP64 outer CG)
    for mode in ("mixed", "f64"):
        t0 = time.perf_counter()
        mg = sf.Multigrid(A, mode=mode)
        setup_s = time.perf_counter() - t0
        mg.solve(b, reltol=1e-10, maxiter=300, raise_on_fail=False)  # warm
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        xs, info = mg.solve(b, reltol=1e-10, maxiter=300, raise_on_fail=False)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[f"cg_mg_{mode}"] = {"ms": round(ms, 2), "iters": info["iters"],
                                "relres": info["relres"], "converged": info["converged"],
                                "setup_s": round(setup_s, 2), "basis": mg.basis,
                                "levels": [f"Q{q} {c[0]}^3" for q, c in zip(mg.orders, mg.cells)]}
        if mode == "mixed":
            x_mixed = xs
        else:
            res["cg_mg_mixed"]["err_vs_mg_f64_max_rel"] = (
                (x_mixed - xs).abs().max() / xs.abs().max()).item()
            res["speedup_mg_mixed_vs_mg_f64"] = round(res["cg_mg_f64"]["ms"] /
                                                       res["cg_mg_mixed"]["ms"], 3)
        log(f"deformed cg_mg_{mode}: {res[f'cg_mg_{mode}']}")
        mg.close()
        del mg
    # Equispaced Q8 Lagrange on perturbed cells is very ill-conditioned: kappa(A)
    # is ~5e6 on 3^3 cells already and grows like h^-2, so Jacobi CG cannot reach
    # 1e-10 here in a bounded time. Report the residual it reaches after a fixed
    # iteration budget in FP64 and in mixed precision, beside the multigrid solves.
    res["cg_budget_iters"] = cg_iters
    for mode, key in ((("jacobi", "f64"), ("mixed", "mixed")) if cg_iters > 0 else ()):
        t0 = time.perf_counter()
        _, info = sf.cg(A, b, reltol=1e-10, mode=mode, maxiter=cg_iters, raise_on_fail=False)
        torch.cuda.synchronize()
        res[f"cg_{key}"] = {"s": round(time.perf_counter() - t0, 3), "iters": info["iters"],
                            "relres": info["relres"], "converged": info["converged"]}
    return res


# The reference's only published timings (test/my_plot.jl:4-7): one 2D apply on
# 1024 x 1024 cells, quadrature degree 2(p - 1), GPU sum-factorization kernel
# gpu_mul_v3! on a V100 (its operator uses the weights only, no geometric factors).
REF_2D_V100_S = {4: 0.003, 5: 0.0051, 6: 0.00805, 7: 0.014}


def run_multigrid(sf, dev, maxiter=500):
    """The multigrid CG at Q4 64^3 on the rough right-hand side (b ~ U[-1,1],
    seed 1), FP32 V-cycle: one warm solve, then one timed solve; with a small
    maxiter a fixed number of iterations (for a profiler's launch list)."""
    import torch
    m, model, V, A = build_problem(sf)
    b = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, A.n)).to(dev)
    mg = sf.Multigrid(A, mode="mixed")
    tol = 1e-10 if maxiter >= 50 else 1e-300
    mg.solve(b, reltol=tol, maxiter=maxiter, raise_on_fail=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    _, info = mg.solve(b, reltol=tol, maxiter=maxiter, raise_on_fail=False)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"ms": round(ms, 3), "iters": info["iters"],
            "ms_per_iter": round(ms / max(1, info["iters"]), 4), "converged": info["converged"],
            "levels": [f"Q{q} {c[0]}^3" for q, c in zip(mg.orders, mg.cells)]}


def run_table_gather(sf, dev, n=64, p=P, seed=7):
    """The unstructured (cell-to-dof table) gather: the Q4 64^3 problem driven by
    sf_set_cells' table (int32 per cell and local dof) through the general element
    kernel's gather and atomic scatter, with the lexicographic numbering (cells
    near in the table are near in the vectors) and with the free dofs randomly
    renumbered (no locality: the worst case), and numbered cell by cell (as a
    finite-element library numbers its spaces); and these numberings through
    sf_set_structured_numbering instead (the tiled kernel between a permutation of
    x in and of y out). FP64 and FP32 apply times and bytes moved; the tiled kernel
    does the lexicographic mesh in about 0.123 ms (FP64)."""
    import torch
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n))
    m = sf.SumFactorizationMap(3, (p,) * 3, (DEG,) * 3)
    ndof = (n * p + 1) ** 3
    ids_bytes = n ** 3 * (p + 1) ** 3 * 4
    res = {"mesh": f"{n}^3 Q{p}, {DEG}-degree Gauss", "table_bytes": ids_bytes}
    for numbering, rseed, gather in (("lexicographic", None, "table"), ("random", seed, "table"),
                                     ("random_numbered", seed, "numbered"),
                                     ("cellwise", "cellwise", "table"),
                                     ("cellwise_numbered", "cellwise", "numbered"),
                                     ("gridap", "gridap", "table"),
                                     ("gridap_numbered", "gridap", "numbered")):
        # "numbered": the same numbering through sf_set_structured_numbering (the tiled
        # kernel on permuted vectors; no table). "cellwise": free dofs numbered cell by cell
        if rseed == "cellwise":
            V = sf.FESpace(model, p, cellwise=True)
        elif rseed == "gridap":  # grouped by face dimension, as Gridap's conforming spaces
            V = sf.FESpace(model, p, numbering="gridap")
        else:
            V = sf.FESpace(model, p, renumber_seed=rseed)
        A = sf.LazyMatrix(m, V, V, sf.Measure(model, DEG), gather=gather)
        assert A.uses_tiled_kernel() == (gather == "numbered")
        x = torch.from_numpy(np.random.default_rng(seed).uniform(-1, 1, A.n)).to(dev)
        y = torch.empty_like(x)
        out = {"kernel": A.kernel_name()}
        if gather == "numbered":
            out["numbered_fused"] = A.info("numbered_fused")
        for dt, key, vb in ((torch.float64, "f64", 8), (torch.float32, "f32", 4)):
            xx, yy = x.to(dt), y.to(dt)
            for _ in range(3):
                sf.mul(yy, A, xx)
            ms = _events_ms(lambda: sf.mul(yy, A, xx), 10)
            byts = (ids_bytes if gather == "table" else 0) + ndof * 2 * vb
            out[key] = {"ms": round(ms, 3), "gdof_s": round(ndof / (ms * 1e-3) / 1e9, 2),
                        "alg_bytes": byts, "achieved_gbs": round(byts / (ms * 1e-3) / 1e9, 1)}
        A.diagonal()
        out["diagonal_ms"] = round(_events_ms(lambda: A.diagonal(), 3), 3)  # element form
        # FP64 Jacobi CG, 30 iterations (a numbered solve permutes b and x once)
        sf.cg(A, x, reltol=1e-300, maxiter=3, raise_on_fail=False)
        out["cg30_ms"] = round(_events_ms(lambda: sf.cg(A, x, reltol=1e-300, maxiter=30,
                                                        raise_on_fail=False), 2), 3)
        res[numbering] = out
        del A, x, y
    log(f"table gather apply: {res}")
    return res


def run_quad2d(sf, dev, n=1024, orders=(4, 5, 6, 7)):
    """The reference's published 2D configuration on this GPU: 1024^2 cells, Q_p,
    degree 2(p-1) quadrature, x ~ U[-1,1] (seed p), FP64 and FP32 applies of the full
    Laplacian (with geometric factors), autotuned, 2 rotating x/y pairs."""
    import torch
    out = {"mesh": f"{n}^2 unit square", "reference_hw": "V100 (published, test/my_plot.jl)",
           "note": "different hardware, and the reference's 2D kernel omits the geometric "
                   "factors; the ratio is for orientation only"}
    for p in orders:
        deg = 2 * (p - 1)
        model = sf.CartesianDiscreteModel((0, 1, 0, 1), (n, n))
        V = sf.FESpace(model, p)
        m = sf.SumFactorizationMap(2, (p, p), (deg, deg))
        A = sf.LazyMatrix(m, V, V, sf.Measure(model, deg))
        ndof = (n * p + 1) ** 2
        rec = {"dofs": ndof}
        for dt, key in ((torch.float64, "f64"), (torch.float32, "f32")):
            A.autotune(dt)
            rng = np.random.default_rng(p)
            xs = [torch.from_numpy(rng.uniform(-1, 1, A.n)).to(dev, dt) for _ in range(2)]
            ys = [torch.empty_like(xs[0]) for _ in range(2)]
            for i in range(3):
                sf.mul(ys[i % 2], A, xs[i % 2])
            k = [0]

            def step():
                sf.mul(ys[k[0] % 2], A, xs[k[0] % 2])
                k[0] += 1
            ms = _events_ms(step, 20)
            rec[key] = {"ms": round(ms, 4), "gdof_s": round(ndof / (ms * 1e-3) / 1e9, 2),
                        "tile": A.kernel_name(dt)}
        ref = REF_2D_V100_S.get(p)
        if ref:
            rec["reference_v100_ms"] = ref * 1e3
            rec["ratio_vs_reference_v100_f64"] = round(ref * 1e3 / rec["f64"]["ms"], 1)
        out[f"q{p}"] = rec
    return out


# ----------------------------------------------------------------------------
# reference arm: the reference CPU path on the host cores
# ----------------------------------------------------------------------------


def run_reference(args):
    from oracle import cref
    from oracle import sumfac_oracle as O
    m = O.make_map(3, P, DEG)
    mesh = O.cartesian_mesh(3, NCELL, P, m)
    cq = O.cell_quantities(m, mesh)
    threads = cref.max_threads()
    nc = mesh.cell_dof_ids.shape[0]
    x = np.random.default_rng(0).uniform(-1, 1, mesh.n_free)
    y = np.empty(mesh.n_free)
    # calibrate: one full apply with all threads
    full = cref.problem_from_oracle(m, mesh, cq)
    full.mul(x, y, nthreads=threads)
    t0 = time.perf_counter()
    full.mul(x, y, nthreads=threads)
    t_full = time.perf_counter() - t0
    budget = 90.0  # seconds for warm-up + timed steps
    frac = min(1.0, budget / max(1, args.steps + args.warmup) / max(t_full, 1e-9))
    # sample: whole z-layers of cells, so the colouring stays valid
    layers = max(1, int(round(frac * NCELL)))
    cells = np.arange(layers * NCELL * NCELL)
    wq, jq, djq = cq
    sub_ids = mesh.cell_dof_ids[cells]
    col, ncol = cref.cartesian_colors((NCELL, NCELL, layers))
    prob = cref.Problem(m.A0, m.B0, m.dof_map, sub_ids, mesh.n_free, False, wq[cells], jq[cells],
                        djq[cells], None, col, ncol)
    for _ in range(args.warmup):
        prob.mul(x, y, nthreads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        prob.mul(x, y, nthreads=threads)
    t = (time.perf_counter() - t0) / args.steps
    dofs = N_DOF_TOTAL * layers / NCELL
    value = dofs / t / 1e9
    sample = (f"{layers} of 64 z-layers of cells ({len(cells)} cells) per step; full apply "
              f"{t_full:.3f} s with {threads} threads")
    return {"metric": METRIC, "value": round(value, 6), "unit": "GDOF/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: x ~ U[-1,1] seed 0",
            "config": {"workload": WORKLOAD, "n_cells": NCELL ** 3, "order": P, "quad_points": 5},
            "impl": "reference",
            "cpu_baseline": {"value": round(value, 6), "unit": "GDOF/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(value, 6), "unit": "GDOF/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "Julia/Gridap absent: C restatement of src/SumFactorizationKernels.jl + "
                    "src/LazyMatrices.jl mul! loops (oracle/sumfac_ref.c), colour-parallel"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    out = run_ours(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
