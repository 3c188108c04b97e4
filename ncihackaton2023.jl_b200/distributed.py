"""One structured problem split into z-slabs over ranks (one process per GPU).

The reference solves on one process (a Gridap model, src/LazyMatrices.jl:52-61
behind IterativeSolvers.cg! at profiling/drivers.jl:85-95). Here the cells of
an nx x ny x nz Cartesian mesh are cut into contiguous z-slabs ("parts"); each
part is a slab operator (sf_set_structured_slab) whose vectors hold its owned
grid levels plus one halo level below and p above. One apply is

    halo exchange (the owned levels next to each cut go to the neighbour part)
    -> each part applies its cells and writes its owned levels.

Owner-computes: every output is computed by exactly one part, so nothing is
summed across the cut and the result does not depend on the partition. The CG
adds one sum over ranks of 1 scalar after the apply and of 2 after the update
(sf_cgd_* steps).

A process may hold several consecutive parts: halo levels between its own
parts are copied on the device, and those between processes go through
torch.distributed point-to-point (NCCL on GPUs, gloo on CPUs). The parts of a
process are driven in lock step by the host, so no kernel ever waits for
another.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import check, lib


def slab_partition(nz: int, nparts: int) -> list[tuple[int, int]]:
    """Contiguous cell ranges [z0, z1) of nearly equal size covering 0..nz."""
    if nparts < 1 or nparts > nz:
        raise ValueError("need 1 <= nparts <= nz")
    base, extra = divmod(nz, nparts)
    out, z = [], 0
    for k in range(nparts):
        z1 = z + base + (1 if k < extra else 0)
        out.append((z, z1))
        z = z1
    return out


def parts_of_rank(nparts: int, world: int, rank: int) -> list[int]:
    """The consecutive parts a rank holds (parts dealt out in contiguous blocks)."""
    if world > nparts:
        raise ValueError("more ranks than parts")
    base, extra = divmod(nparts, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def owner_of(part: int, nparts: int, world: int) -> int:
    for r in range(world):
        if part in parts_of_rank(nparts, world, r):
            return r
    raise ValueError("part out of range")


@dataclass(frozen=True)
class SlabLayout:
    """Index arithmetic of one part's vectors (see sf_set_structured_slab)."""

    nx: int
    ny: int
    nz: int
    p: int
    z0: int
    z1: int

    @property
    def plane(self) -> int:
        return (self.nx * self.p - 1) * (self.ny * self.p - 1)

    @property
    def nplanes(self) -> int:
        return (self.z1 - self.z0 + 1) * self.p + 1

    @property
    def n(self) -> int:
        return self.plane * self.nplanes

    @property
    def owned_planes(self) -> int:
        return (self.z1 - self.z0) * self.p - (1 if self.z1 == self.nz else 0)

    @property
    def owned(self) -> slice:
        return slice(self.plane, self.plane * (1 + self.owned_planes))

    def planes(self, j0: int, j1: int) -> slice:
        """Planes j0 .. j1-1 of the slab vector."""
        return slice(j0 * self.plane, j1 * self.plane)

    # halo pattern: what this part sends and where it receives
    def send_down(self) -> slice:   # levels z0 p + 1 .. z0 p + p -> upper halo of the part below
        return self.planes(1, 1 + self.p)

    def send_up(self) -> slice:     # level z1 p -> lower halo of the part above
        top = (self.z1 - self.z0) * self.p
        return self.planes(top, top + 1)

    def recv_above(self) -> slice:  # levels z1 p + 1 .. z1 p + p
        top = (self.z1 - self.z0) * self.p
        return self.planes(top + 1, top + 1 + self.p)

    def recv_below(self) -> slice:  # level z0 p
        return self.planes(0, 1)

    # global free vector <-> slab vector (lexicographic free numbering, x fastest)
    def global_levels(self) -> tuple[int, int, int]:
        """(first slab plane, first global free plane, number of planes) that exist in
        the mesh's free grid (levels 1 .. nz p - 1)."""
        lo = max(1, self.z0 * self.p)
        hi = min(self.nz * self.p - 1, (self.z1 + 1) * self.p)
        return lo - self.z0 * self.p, lo - 1, max(0, hi - lo + 1)

    def from_global(self, xg: torch.Tensor) -> torch.Tensor:
        """The slab vector of a global free vector (halo planes included)."""
        out = torch.zeros(self.n, dtype=xg.dtype, device=xg.device)
        j0, g0, cnt = self.global_levels()
        out[j0 * self.plane:(j0 + cnt) * self.plane] = xg[g0 * self.plane:(g0 + cnt) * self.plane]
        return out

    def owned_global(self) -> slice:
        """The global free indices of the owned points."""
        g0 = self.z0 * self.p  # level z0 p + 1 has free plane index z0 p
        return slice(g0 * self.plane, (g0 + self.owned_planes) * self.plane)


class SlabComm:
    """Halo exchange and sums over the parts of all ranks. ``group`` is a
    torch.distributed process group (None: this process holds every part)."""

    def __init__(self, nparts: int, group=None):
        import torch.distributed as dist
        self.dist = dist if group is not None else None
        self.group = group
        self.world = dist.get_world_size(group) if group is not None else 1
        self.rank = dist.get_rank(group) if group is not None else 0
        self.nparts = nparts
        self.parts = parts_of_rank(nparts, self.world, self.rank)

    def exchange(self, layouts: list[SlabLayout], xs: list[torch.Tensor]) -> None:
        """Fill the halo planes of every local part's vector from its neighbours."""
        parts = self.parts
        local = {g: k for k, g in enumerate(parts)}
        ops = []
        for k, g in enumerate(parts):
            L, x = layouts[k], xs[k]
            if g > 0:
                if g - 1 in local:  # neighbour below is here: copy its top owned level
                    kb = local[g - 1]
                    x[L.recv_below()] = xs[kb][layouts[kb].send_up()]
                else:
                    src = owner_of(g - 1, self.nparts, self.world)
                    ops.append(self.dist.P2POp(self.dist.isend, x[L.send_down()], src, self.group))
                    ops.append(self.dist.P2POp(self.dist.irecv, x[L.recv_below()], src, self.group))
            if g < self.nparts - 1:
                if g + 1 in local:
                    ka = local[g + 1]
                    x[L.recv_above()] = xs[ka][layouts[ka].send_down()]
                else:
                    dst = owner_of(g + 1, self.nparts, self.world)
                    ops.append(self.dist.P2POp(self.dist.isend, x[L.send_up()], dst, self.group))
                    ops.append(self.dist.P2POp(self.dist.irecv, x[L.recv_above()], dst, self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()

    def allreduce(self, views: list[torch.Tensor]) -> None:
        """views[k] (one per local part, same shape): each becomes the sum over all parts."""
        total = views[0].clone()
        for v in views[1:]:
            total += v
        if self.dist is not None and self.world > 1:
            self.dist.all_reduce(total, group=self.group)
        for v in views:
            v.copy_(total)


class _SlabEngine:
    """One part on the device: a slab operator of the C library."""

    def __init__(self, m, model, layout: SlabLayout):
        from . import fem
        from .operator import _f64, _i32, _ptr
        self.layout = layout
        self._h = m._create_handle()
        try:
            nx, ny, nz = model.partition
            no = _i32(m.node_order)
            check(lib.sf_set_structured_slab(self._h, nx, ny, nz, layout.z0, layout.z1, _ptr(no)),
                  self._h, "sf_set_structured_slab")
            fill, wq, jq, djq = fem.cell_quantities(model, m.points, m.weights)
            if not fill:
                raise ValueError("slab decomposition needs a Cartesian model (one cell shared by all)")
            wq, jq, djq = _f64(wq), _f64(jq), _f64(djq)
            check(lib.sf_set_cell_quantities(self._h, 1, _ptr(wq), _ptr(jq), _ptr(djq)), self._h,
                  "sf_set_cell_quantities")
            v = C.c_double()
            check(lib.sf_get_info(self._h, b"tiled_kernel", C.byref(v)), self._h, "sf_get_info")
            if v.value != 1.0:
                raise ValueError("slab decomposition needs the tiled Cartesian kernel")
        except Exception:
            self.close()
            raise

    def close(self):
        if getattr(self, "_h", None):
            lib.sf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr())

    def _s(self):
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def apply(self, x, y):
        from .operator import _dtype_code
        check(lib.sf_apply(self._h, _dtype_code(x.dtype), self._p(x), self._p(y), self._s()),
              self._h, "sf_apply")

    def autotune(self, dtype):
        from .operator import _dtype_code
        check(lib.sf_autotune(self._h, _dtype_code(dtype), self._s()), self._h, "sf_autotune")

    def kernel_name(self, dtype) -> str:
        from .operator import _dtype_code
        raw = lib.sf_kernel_name(self._h, _dtype_code(dtype))
        return raw.decode() if raw else ""

    def cgd_start(self, b, x, r, p, q, s):
        check(lib.sf_cgd_start(self._h, *map(self._p, (b, x, r, p, q, s)), self._s()), self._h,
              "sf_cgd_start")

    def cgd_init(self, s, reltol):
        check(lib.sf_cgd_init(self._h, self._p(s), float(reltol), self._s()), self._h,
              "sf_cgd_init")

    def cgd_apply(self, p, q, s):
        check(lib.sf_cgd_apply(self._h, *map(self._p, (p, q, s)), self._s()), self._h,
              "sf_cgd_apply")

    def cgd_update(self, r, q, s):
        check(lib.sf_cgd_update(self._h, *map(self._p, (r, q, s)), self._s()), self._h,
              "sf_cgd_update")

    def cgd_direction(self, x, p, r, s):
        check(lib.sf_cgd_direction(self._h, *map(self._p, (x, p, r, s)), self._s()), self._h,
              "sf_cgd_direction")


class DistributedLazyMatrix:
    """The operator of a Cartesian model split into ``nparts`` z-slabs.

    ``group``: the torch.distributed group of the ranks sharing the problem
    (None: this process holds every part). Vectors are lists with one slab
    vector per local part (``new_vector``, ``from_global``). ``engine``
    replaces the device slab operator (a factory ``engine(layout)``), for
    testing the host logic without a GPU."""

    def __init__(self, m, model, nparts: int | None = None, group=None, engine=None,
                 device=None):
        nx, ny, nz = model.partition
        world = 1 if group is None else torch.distributed.get_world_size(group)
        self.nparts = nparts or world
        self.comm = SlabComm(self.nparts, group)
        ranges = slab_partition(nz, self.nparts)
        p = m.order
        self.layouts = [SlabLayout(nx, ny, nz, p, *ranges[g]) for g in self.comm.parts]
        make = engine or (lambda L: _SlabEngine(m, model, L))
        self.engines = [make(L) for L in self.layouts]
        if device is None:
            device = torch.device("cpu") if engine is not None else torch.device("cuda")
        self.device = device
        self.n_global = (nx * p - 1) * (ny * p - 1) * (nz * p - 1)

    def close(self):
        for e in self.engines:
            if hasattr(e, "close"):
                e.close()

    def new_vector(self, dtype=torch.float64):
        return [torch.zeros(L.n, dtype=dtype, device=self.device) for L in self.layouts]

    def from_global(self, xg: torch.Tensor):
        return [L.from_global(xg) for L in self.layouts]

    def owned(self, xs):
        """(global slice, owned values) of every local part."""
        return [(L.owned_global(), x[L.owned]) for L, x in zip(self.layouts, xs)]

    def exchange(self, xs) -> None:
        self.comm.exchange(self.layouts, xs)

    def autotune(self, dtype=torch.float64):
        for e in self.engines:
            e.autotune(dtype)

    def mul(self, ys, xs):
        """ys = A xs (owned points), after the halo exchange of xs."""
        self.exchange(xs)
        for e, x, y in zip(self.engines, xs, ys):
            e.apply(x, y)
        return ys


def cg(A: DistributedLazyMatrix, bs, xs=None, reltol: float = 1e-10, maxiter: int = 10000,
       check_every: int = 4, raise_on_fail: bool = True):
    """Jacobi FP64 CG on the distributed operator (every rank calls it). bs, xs:
    lists of slab vectors (halo planes of bs are not read). The stopping flag is
    read every ``check_every`` iterations; iterations past convergence change
    nothing. Returns (xs, info)."""
    eng, L = A.engines, A.layouts
    if xs is None:
        xs = A.new_vector()
    rs, ps, qs = A.new_vector(), A.new_vector(), A.new_vector()
    ss = [torch.zeros(_lib.SF_CGD_SCALARS, dtype=torch.float64, device=A.device) for _ in eng]
    A.exchange(xs)
    for e, b, x, r, p, q, s in zip(eng, bs, xs, rs, ps, qs, ss):
        e.cgd_start(b, x, r, p, q, s)
    A.comm.allreduce([s[2:5] for s in ss])
    for e, s in zip(eng, ss):
        e.cgd_init(s, reltol)
    it = 0
    done = ss[0][_lib.SF_CGD_DONE].item()
    while it < maxiter and done == 0.0:
        A.exchange(ps)
        for e, p, q, s in zip(eng, ps, qs, ss):
            e.cgd_apply(p, q, s)
        A.comm.allreduce([s[10:11] for s in ss])
        for e, r, q, s in zip(eng, rs, qs, ss):
            e.cgd_update(r, q, s)
        A.comm.allreduce([s[11:13] for s in ss])
        for e, x, p, r, s in zip(eng, xs, ps, rs, ss):
            e.cgd_direction(x, p, r, s)
        it += 1
        if it % check_every == 0 or it == maxiter:
            done = ss[0][_lib.SF_CGD_DONE].item()
    s = ss[0].cpu()
    bb = float(s[_lib.SF_CGD_BB])
    nb = bb ** 0.5 if bb > 0 else 1.0
    info = {"iters": int(s[_lib.SF_CGD_ITERS]), "relres": float(s[_lib.SF_CGD_RR]) ** 0.5 / nb,
            "converged": float(s[_lib.SF_CGD_DONE]) == 2.0}
    if float(s[_lib.SF_CGD_DONE]) == 3.0:
        raise _lib.SumFacError(_lib.SF_ERR_NONFINITE, "non-finite residual in distributed CG")
    if raise_on_fail and not info["converged"]:
        raise _lib.SumFacError(_lib.SF_ERR_NOT_CONVERGED, "distributed CG reached its iteration cap")
    return xs, info
