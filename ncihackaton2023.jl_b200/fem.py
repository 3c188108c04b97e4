"""Host-side finite-element set-up: the pieces of Gridap that the reference's
hot path consumes, restated for a Python host.

In the reference, the Julia host keeps the mesh, the dof numbering and the
geometric factors (src/LazyMatrices.jl:30-50, profiling/drivers.jl:7-17), and
only the operator apply moves to the device. This module is that host side:
1D Lagrange basis and Gauss-Legendre quadrature (src/SumFactorizationMaps.jl:47-65),
a Cartesian model of [0,1]^3 with optional interior-vertex perturbation, the
Q_p dof numbering with Dirichlet dofs on the boundary, and the per-point
geometric factors (wq, jq, djq). All of this is set-up work, done once.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# ----------------------------------------------------------------------------
# 1D reference element
# ----------------------------------------------------------------------------


def quadrature_npoints(degree: int) -> int:
    """Gauss points per direction for a quadrature of the given degree:
    ceil((degree+1)/2), Gridap's rule for Quadrature(SEGMENT, degree)."""
    if degree < 0:
        raise ValueError("quadrature degree must be >= 0")
    return int(math.ceil((degree + 1) / 2.0))


def gauss_legendre(npts: int):
    """Points (ascending) and weights (sum 1) of the npts-point rule on [0,1]."""
    x, w = np.polynomial.legendre.leggauss(npts)
    return 0.5 * (x + 1.0), 0.5 * w


def lagrange_nodes(p: int) -> np.ndarray:
    """1D nodes in Gridap's SEGMENT order: vertex 0, vertex 1, interior ascending."""
    return np.array([0.0, 1.0] + [i / p for i in range(1, p)])


def gll_nodes(p: int) -> np.ndarray:
    """Gauss-Lobatto-Legendre nodes on [0, 1] in Gridap's SEGMENT order (vertex 0,
    vertex 1, interior ascending): the end points and the roots of P_p'. The
    multigrid hierarchy of an equispaced high-order space works in this basis."""
    if p == 1:
        return np.array([0.0, 1.0])
    c = np.zeros(p + 1)
    c[p] = 1.0
    inner = np.sort(np.real(np.polynomial.legendre.legroots(np.polynomial.legendre.legder(c))))
    return np.concatenate([[0.0, 1.0], 0.5 * (inner + 1.0)])


def node_order(p: int) -> np.ndarray:
    """Position 0..p along the segment of each 1D basis function (Gridap order)."""
    return np.array([0, p] + list(range(1, p)), dtype=np.int32)


def lagrange_basis(nodes: np.ndarray, pts: np.ndarray):
    """Values A[i, j] = phi_j(pts[i]) and derivatives B[i, j] = phi_j'(pts[i]) of
    the Lagrange polynomials on ``nodes``, by the barycentric formulas."""
    nodes = np.asarray(nodes, dtype=np.float64)
    pts = np.asarray(pts, dtype=np.float64)
    nb = len(nodes)
    diff = nodes[:, None] - nodes[None, :]
    np.fill_diagonal(diff, 1.0)
    lam = 1.0 / np.prod(diff, axis=1)  # barycentric weights
    A = np.zeros((len(pts), nb))
    B = np.zeros((len(pts), nb))
    for i, x in enumerate(pts):
        d = x - nodes
        hit = np.nonzero(np.abs(d) < 1e-300)[0]
        if hit.size:
            # x coincides with a node: values are a unit vector; derivative by the
            # differentiation-matrix row of that node
            m = hit[0]
            A[i, m] = 1.0
            for j in range(nb):
                if j != m:
                    B[i, j] = (lam[j] / lam[m]) / (nodes[m] - nodes[j])
            B[i, m] = -np.sum(B[i, np.arange(nb) != m])
            continue
        l = np.prod(d)
        A[i] = l * lam / d
        # phi_j'(x) = phi_j(x) * sum_{m != j} 1/(x - x_m)
        s = np.sum(1.0 / d)
        B[i] = A[i] * (s - 1.0 / d)
    return A, B


def hex_dof_map(p: int, D: int = 3) -> np.ndarray:
    """Tensor index (1-based, in the 1D Gridap basis order) of each local dof of
    a hexahedron (D = 3) or quadrilateral (D = 2), as the (SB^D, D) array
    m.dof_map of src/SumFactorizationMaps.jl:40-45. The local order used by this
    package's FE space is the tensor order with j1 fastest."""
    SB = p + 1
    k = np.arange(SB ** D)
    cols = [k % SB, (k // SB) % SB, k // (SB * SB)][:D]
    return np.stack(cols, axis=1).astype(np.int32) + 1


# ----------------------------------------------------------------------------
# Model, FE space and measure
# ----------------------------------------------------------------------------


@dataclass
class CartesianDiscreteModel:
    """[x0,x1]x[y0,y1]x[z0,z1] split into partition = (nx, ny, nz) cells, numbered
    with x fastest (profiling/drivers.jl:8-10). ``perturb`` > 0 moves every
    interior vertex by a seeded uniform displacement of at most perturb*h per
    coordinate, giving trilinear (deformed) cells."""

    domain: tuple = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    partition: tuple = (1, 1, 1)
    perturb: float = 0.0
    seed: int = 0
    vertices: np.ndarray = field(init=False, repr=False)

    @property
    def D(self) -> int:
        return len(self.partition)

    def __post_init__(self):
        if self.D == 2:
            if len(self.domain) == 6:
                self.domain = tuple(self.domain[:4])
            if self.perturb > 0.0:
                raise NotImplementedError("2D models are affine Cartesian (no perturbation)")
            nx, ny = self.partition
            X, Y = np.meshgrid(np.linspace(self.domain[0], self.domain[1], nx + 1),
                               np.linspace(self.domain[2], self.domain[3], ny + 1), indexing="xy")
            self.vertices = np.stack([X.ravel(), Y.ravel()], axis=1)
            return
        nx, ny, nz = self.partition
        xs = [np.linspace(self.domain[2 * a], self.domain[2 * a + 1], n + 1)
              for a, n in enumerate(self.partition)]
        Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        v = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
        if self.perturb > 0.0:
            h = np.array([(self.domain[2 * a + 1] - self.domain[2 * a]) / n
                          for a, n in enumerate(self.partition)])
            rng = np.random.default_rng(self.seed)
            disp = rng.uniform(-self.perturb, self.perturb, size=v.shape) * h
            iz, iy, ix = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1),
                                     indexing="ij")
            interior = ((ix > 0) & (ix < nx) & (iy > 0) & (iy < ny) & (iz > 0) & (iz < nz)).ravel()
            v = v + disp * interior[:, None]
        self.vertices = v

    @property
    def num_cells(self) -> int:
        return int(np.prod(self.partition))

    def coarsened(self) -> "CartesianDiscreteModel":
        """The model of every second vertex along each axis (half the cells; the
        partition must be even): the coarse mesh of an h-multigrid level. On a
        perturbed model its cells are the trilinear cells through those vertices."""
        if self.D != 3 or any(n % 2 for n in self.partition):
            raise ValueError("coarsening needs a 3D model with an even partition")
        c = CartesianDiscreteModel(self.domain, tuple(n // 2 for n in self.partition))
        nx, ny, nz = self.partition
        v = self.vertices.reshape(nz + 1, ny + 1, nx + 1, 3)[::2, ::2, ::2]
        c.vertices = np.ascontiguousarray(v.reshape(-1, 3))
        c.perturb = self.perturb  # deformed cells stay deformed (per-cell geometry)
        return c

    @property
    def is_affine_cartesian(self) -> bool:
        return self.perturb == 0.0

    def cell_vertices(self) -> np.ndarray:
        """(ncells, 2^D) vertex ids, corners ordered with x fastest."""
        if self.D == 2:
            nx, ny = self.partition
            c = np.arange(self.num_cells)
            cx, cy = c % nx, c // nx
            out = np.empty((self.num_cells, 4), dtype=np.int64)
            for v in range(4):
                out[:, v] = (cx + (v & 1)) + (nx + 1) * (cy + ((v >> 1) & 1))
            return out
        nx, ny, nz = self.partition
        c = np.arange(self.num_cells)
        cx, cy, cz = c % nx, (c // nx) % ny, c // (nx * ny)
        out = np.empty((self.num_cells, 8), dtype=np.int64)
        for v in range(8):
            dx, dy, dz = v & 1, (v >> 1) & 1, (v >> 2) & 1
            out[:, v] = (cx + dx) + (nx + 1) * ((cy + dy) + (ny + 1) * (cz + dz))
        return out


# Local edges and faces of a hexahedron as Gridap's HEX polytope lists them (vertices x
# fastest): edges along x, then y, then z; faces z = 0, z = 1, y = 0, y = 1, x = 0, x = 1.
# Each entry: (axis of the edge / normal axis of the face, offset of its lowest vertex).
_HEX_EDGES = [(0, (0, 0, 0)), (0, (0, 1, 0)), (0, (0, 0, 1)), (0, (0, 1, 1)),
              (1, (0, 0, 0)), (1, (1, 0, 0)), (1, (0, 0, 1)), (1, (1, 0, 1)),
              (2, (0, 0, 0)), (2, (1, 0, 0)), (2, (0, 1, 0)), (2, (1, 1, 0))]
_HEX_FACES = [(2, (0, 0, 0)), (2, (0, 0, 1)), (1, (0, 0, 0)), (1, (0, 1, 0)),
              (0, (0, 0, 0)), (0, (1, 0, 0))]


def gridap_free_numbering(model: "CartesianDiscreteModel", p: int) -> np.ndarray:
    """Free-dof numbering of a conforming Q_p space as Gridap builds it, face
    dimension by face dimension: the dofs owned by vertices (in vertex order),
    then by edges, by faces, and the cell-interior dofs (cell by cell); the
    Dirichlet dofs are left out and the free ones keep that order. Edges and
    faces carry the numbers of the grid topology, which gives each a number when
    it is first met going through the cells in order and through each cell's
    local edges / faces in the HEX order. A face's own dofs run x fastest, an
    edge's along its axis.

    Restated from the conforming-space construction of Gridap (FESpaces,
    ``_generate_face_to_own_dofs``; Geometry, the topology's face numbering). The
    reference does not pin Gridap's version and Gridap does not run here, so this
    numbering is UNPINNED: it has Gridap's structure (grouped by face dimension),
    not a verified bit-for-bit copy. Returns perm with perm[i] = the 0-based id of
    lexicographic free point i (the ``FESpace.perm`` convention)."""
    if model.D != 3:
        raise NotImplementedError("3D models only")
    n = np.array(model.partition)
    N = n * p
    V = n + 1                                   # vertices per axis
    vlin = lambda v: v[..., 0] + V[0] * (v[..., 1] + V[1] * v[..., 2])
    nc = int(np.prod(n))
    c = np.arange(nc)
    cell = np.stack([c % n[0], (c // n[0]) % n[1], c // (n[0] * n[1])], axis=1)

    def first_visit(table):
        """Topology numbers of the entities of `table`: key of each (cell, local)."""
        keys = np.stack([a * (int(np.prod(V)) + 1) + vlin(cell + np.array(off))
                         for a, off in table], axis=1).ravel()
        uniq, first = np.unique(keys, return_index=True)
        order = np.argsort(first, kind="stable")  # entity number -> index into uniq
        rank = np.empty(len(uniq), dtype=np.int64)
        rank[order] = np.arange(len(uniq))
        return uniq, rank                        # uniq sorted; rank[k] = number of uniq[k]

    # free grid points, lexicographic (x fastest)
    fz, fy, fx = np.meshgrid(*[np.arange(1, N[a]) for a in (2, 1, 0)], indexing="ij")
    g = np.stack([fx.ravel(), fy.ravel(), fz.ravel()], axis=1)
    aligned = (g % p) == 0
    dim = 3 - aligned.sum(axis=1)
    perm = np.empty(len(g), dtype=np.int64)
    base = 0
    # vertices: interior vertices in vertex order
    m = dim == 0
    vid = vlin(g[m] // p)
    iv = np.unique(vid)
    perm[m] = base + np.searchsorted(iv, vid)
    base += len(iv)
    # edges and faces: entities in topology order, own dofs in a fixed local order
    for d, table in ((1, _HEX_EDGES), (2, _HEX_FACES)):
        m = dim == d
        gd = g[m]
        al = aligned[m]
        if d == 1:
            axis = np.argmax(~al, axis=1)                # the edge's axis
        else:
            axis = np.argmax(al, axis=1)                 # the face's normal axis
        low = gd // p                                    # lowest vertex of the entity
        key = axis * (int(np.prod(V)) + 1) + vlin(low)
        uniq, rank = first_visit(table)
        number = rank[np.searchsorted(uniq, key)]
        loc = gd % p - 1                                 # 0 .. p-2 on the free axes
        if d == 1:
            local = loc[np.arange(len(gd)), axis]
            own = p - 1
        else:
            a1 = np.where(axis == 0, 1, 0)
            a2 = np.where(axis == 2, 1, 2)
            local = loc[np.arange(len(gd)), a1] + (p - 1) * loc[np.arange(len(gd)), a2]
            own = (p - 1) ** 2
        # entities with free dofs, in topology order, get consecutive blocks
        used = np.unique(number)
        perm[m] = base + np.searchsorted(used, number) * own + local
        base += len(used) * own
    # cell interiors: cells in order
    m = dim == 3
    gd = g[m]
    cidx = gd // p
    cid = cidx[:, 0] + n[0] * (cidx[:, 1] + n[1] * cidx[:, 2])
    loc = gd % p - 1
    own = (p - 1) ** 3
    perm[m] = base + cid * own + loc[:, 0] + (p - 1) * (loc[:, 1] + (p - 1) * loc[:, 2])
    return perm


@dataclass
class Table:
    """Gridap's ``Table``: CSR with 1-based ``ptrs`` (length n+1) into ``data``."""

    data: np.ndarray
    ptrs: np.ndarray

    def __len__(self):
        return len(self.ptrs) - 1

    def __getitem__(self, i):
        return self.data[self.ptrs[i] - 1:self.ptrs[i + 1] - 1]


@dataclass
class FESpace:
    """Lagrangian Q_p space on a CartesianDiscreteModel with Dirichlet dofs on the
    whole boundary (``dirichlet_tags=["boundary"]``, profiling/drivers.jl:15-16).
    Free dofs are numbered lexicographically (x fastest) over the interior dof
    grid; Dirichlet dofs get negative ids. ``renumber_seed`` applies a seeded
    random permutation to the free ids (an arbitrary global numbering, with no
    locality). ``cellwise`` numbers the free dofs instead in the order in which
    they first appear going through the cells in order, each cell in its local
    dof order: a cell-by-cell numbering such as a finite-element library gives
    its spaces (locality kept). ``numbering="gridap"`` numbers the free dofs
    grouped by face dimension, as Gridap's conforming spaces do
    (``gridap_free_numbering``)."""

    model: CartesianDiscreteModel
    order: int
    dirichlet_tags: str = "boundary"
    renumber_seed: int | None = None
    cellwise: bool = False
    numbering: str = "lexicographic"

    def __post_init__(self):
        if self.dirichlet_tags != "boundary":
            raise NotImplementedError("only dirichlet_tags='boundary' is supported")
        p = self.order
        self.grid = tuple(n * p + 1 for n in self.model.partition)
        self.free_grid = tuple(n * p - 1 for n in self.model.partition)
        self._ids = None
        self.perm = None
        if self.renumber_seed is not None and self.cellwise:
            raise ValueError("renumber_seed and cellwise are exclusive")
        if self.numbering not in ("lexicographic", "gridap"):
            raise ValueError("numbering must be 'lexicographic' or 'gridap'")
        if self.numbering == "gridap":
            if self.renumber_seed is not None or self.cellwise:
                raise ValueError("numbering='gridap' excludes renumber_seed and cellwise")
            self.perm = gridap_free_numbering(self.model, p)
            return
        if self.renumber_seed is not None:
            self.perm = (np.random.default_rng(self.renumber_seed)
                         .permutation(self.num_free_dofs).astype(np.int64))
        elif self.cellwise:
            data = np.asarray(self.get_cell_dof_ids().data)  # lexicographic ids, cell by cell
            free = data[data > 0]
            lex, first = np.unique(free, return_index=True)
            perm = np.empty(self.num_free_dofs, dtype=np.int64)
            perm[lex[np.argsort(first, kind="stable")] - 1] = np.arange(lex.size)
            self.perm = perm
            self._ids = None

    @property
    def num_free_dofs(self) -> int:
        return int(np.prod(self.free_grid))

    def grid_ids(self) -> np.ndarray:
        """Id of every point of the (N+1)^D dof grid (x fastest): 1-based free ids,
        negative Dirichlet ids."""
        axes = np.meshgrid(*[np.arange(G) for G in self.grid[::-1]], indexing="ij")[::-1]
        free = np.ones(axes[0].shape, dtype=bool)
        for g, G in zip(axes, self.grid):
            free &= (g > 0) & (g < G - 1)
        free = free.ravel()
        ids = np.zeros(free.size, dtype=np.int64)
        lex = np.arange(1, int(free.sum()) + 1)
        if self.perm is not None:
            lex = self.perm[lex - 1] + 1
        ids[free] = lex
        ids[~free] = -np.arange(1, int((~free).sum()) + 1)
        return ids

    def get_cell_dof_ids(self) -> Table:
        """The cell-to-dof Table in the local order of ``hex_dof_map(p)``."""
        if self._ids is None and self.model.D == 2:
            p, SB = self.order, self.order + 1
            nx, ny = self.model.partition
            Gx = self.grid[0]
            gids = self.grid_ids()
            c = np.arange(self.model.num_cells)
            cx, cy = c % nx, c // nx
            order = node_order(p)
            dm = hex_dof_map(p, 2) - 1
            ox, oy = order[dm[:, 0]], order[dm[:, 1]]
            lin = (cx[:, None] * p + ox[None, :]) + Gx * (cy[:, None] * p + oy[None, :])
            data = gids[lin].astype(np.int32).ravel()
            ptrs = (np.arange(self.model.num_cells + 1, dtype=np.int64) * SB ** 2 + 1).astype(np.int32)
            self._ids = Table(data=data, ptrs=ptrs)
        if self._ids is None:
            p = self.order
            SB = p + 1
            nx, ny, nz = self.model.partition
            Gx, Gy, _ = self.grid
            gids = self.grid_ids()
            c = np.arange(self.model.num_cells)
            cx, cy, cz = c % nx, (c // nx) % ny, c // (nx * ny)
            order = node_order(p)
            dm = hex_dof_map(p) - 1
            ox, oy, oz = order[dm[:, 0]], order[dm[:, 1]], order[dm[:, 2]]
            lin = ((cx[:, None] * p + ox[None, :]) + Gx * ((cy[:, None] * p + oy[None, :])
                   + Gy * (cz[:, None] * p + oz[None, :])))
            data = gids[lin].astype(np.int32).ravel()
            ptrs = (np.arange(self.model.num_cells + 1, dtype=np.int64) * SB ** 3 + 1).astype(np.int32)
            self._ids = Table(data=data, ptrs=ptrs)
        return self._ids

    def free_dof_coordinates(self) -> np.ndarray:
        """Coordinates of the free dofs in free-id order (unperturbed grid)."""
        if self.model.D == 2:
            fx, fy = self.free_grid
            Gx, Gy = self.grid
            gy, gx = np.meshgrid(np.arange(1, fy + 1), np.arange(1, fx + 1), indexing="ij")
            d = self.model.domain
            pts = np.stack([d[0] + (d[1] - d[0]) * gx.ravel() / (Gx - 1),
                            d[2] + (d[3] - d[2]) * gy.ravel() / (Gy - 1)], axis=1)
            if self.perm is not None:
                out = np.empty_like(pts)
                out[self.perm] = pts
                return out
            return pts
        fx, fy, fz = self.free_grid
        Gx, Gy, Gz = self.grid
        gz, gy, gx = np.meshgrid(np.arange(1, fz + 1), np.arange(1, fy + 1), np.arange(1, fx + 1),
                                 indexing="ij")
        d = self.model.domain
        pts = np.stack([d[0] + (d[1] - d[0]) * gx.ravel() / (Gx - 1),
                        d[2] + (d[3] - d[2]) * gy.ravel() / (Gy - 1),
                        d[4] + (d[5] - d[4]) * gz.ravel() / (Gz - 1)], axis=1)
        if self.perm is not None:
            out = np.empty_like(pts)
            out[self.perm] = pts
            return out
        return pts


def TrialFESpace(V: FESpace, g=None) -> FESpace:
    """Trial space with homogeneous Dirichlet data (the apply only ever sees
    Dirichlet zeros: src/LazyMatrices.jl:48,53)."""
    if g is not None and g != 0:
        raise NotImplementedError("the operator apply uses zero Dirichlet values")
    return V


@dataclass
class Measure:
    """Integration measure dOmega = Measure(Omega, degree) (profiling/drivers.jl:12)."""

    model: CartesianDiscreteModel
    degree: int


# ----------------------------------------------------------------------------
# Geometric factors
# ----------------------------------------------------------------------------


def _trilinear_gradients(pts: np.ndarray) -> np.ndarray:
    """dN[q, v, i]: derivative along xi_i of the trilinear vertex function v at pts[q]."""
    nq = len(pts)
    dN = np.empty((nq, 8, 3))
    for v in range(8):
        c = ((v & 1), (v >> 1) & 1, (v >> 2) & 1)
        f = [pts[:, a] if c[a] else 1.0 - pts[:, a] for a in range(3)]
        df = [1.0 if c[a] else -1.0 for a in range(3)]
        dN[:, v, 0] = df[0] * f[1] * f[2]
        dN[:, v, 1] = f[0] * df[1] * f[2]
        dN[:, v, 2] = f[0] * f[1] * df[2]
    return dN


def cell_quantities(model: CartesianDiscreteModel, q1d: np.ndarray, w1d: np.ndarray):
    """(wq, jq, djq) at the quadrature points of every cell, as the LazyMatrix
    constructor forms them (src/LazyMatrices.jl:34-43): Jt = grad(cell map),
    jq = inv(Jt), djq = |det Jt|, wq the reference weights (x fastest).

    Returns (fill, wq, jq, djq). fill is True when every cell has the same
    values (an affine Cartesian model, where Gridap returns Fill arrays); the
    arrays then hold one cell. jq is returned column-major per point
    (jq[..., l + 3 r] = jq[l, r]), the layout of the C ABI."""
    SQ = len(q1d)
    if model.D == 2:  # affine Cartesian: Jt = diag(hx, hy) at every point
        qy, qx = np.meshgrid(w1d, w1d, indexing="ij")
        w = (qx * qy).ravel()
        d = model.domain
        hx, hy = (d[1] - d[0]) / model.partition[0], (d[3] - d[2]) / model.partition[1]
        jq = np.tile(np.array([1.0 / hx, 0.0, 0.0, 1.0 / hy]), (1, SQ ** 2, 1))
        djq = np.full((1, SQ ** 2), hx * hy)
        return True, w[None, :].copy(), jq, djq
    qz, qy, qx = np.meshgrid(q1d, q1d, q1d, indexing="ij")
    pts = np.stack([qx.ravel(), qy.ravel(), qz.ravel()], axis=1)
    wz, wy, wx = np.meshgrid(w1d, w1d, w1d, indexing="ij")
    w = (wx * wy * wz).ravel()
    dN = _trilinear_gradients(pts)
    if model.is_affine_cartesian:
        X = model.vertices[model.cell_vertices()[:1]]
    else:
        X = model.vertices[model.cell_vertices()]
    Jt = np.einsum("qvi,cvj->cqij", dN, X)   # Jt[i, j] = dx_j / dxi_i
    jq = np.linalg.inv(Jt)
    djq = np.abs(np.linalg.det(Jt))
    jq_cm = np.ascontiguousarray(np.swapaxes(jq, -1, -2)).reshape(jq.shape[0], SQ ** 3, 9)
    wq = np.broadcast_to(w, (X.shape[0], SQ ** 3)).copy()
    return model.is_affine_cartesian, wq, jq_cm, djq


def physical_quadrature_points(model: CartesianDiscreteModel, q1d: np.ndarray,
                               cells: slice = slice(None)) -> np.ndarray:
    """(ncells, SQ^3, 3) coordinates of the quadrature points of ``cells``."""
    qz, qy, qx = np.meshgrid(q1d, q1d, q1d, indexing="ij")
    pts = np.stack([qx.ravel(), qy.ravel(), qz.ravel()], axis=1)
    N = np.ones((len(pts), 8))
    for v in range(8):
        c = ((v & 1), (v >> 1) & 1, (v >> 2) & 1)
        for a in range(3):
            N[:, v] *= pts[:, a] if c[a] else 1.0 - pts[:, a]
    X = model.vertices[model.cell_vertices()[cells]]
    return np.einsum("qv,cvj->cqj", N, X)
