"""ctypes front end of oracle/libsumfac_ref.so, the C restatement of the
reference CPU path (TEST INFRASTRUCTURE ONLY: the parity reference and the timed CPU
baseline; see sumfac_ref.c)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsumfac_ref.so")
_lib = None


def build(march: str | None = None, force: bool = False) -> str:
    args = ["make", "-C", HERE]
    if force:
        args.append("-B")
    if march:
        args.append(f"MARCH={march}")
    subprocess.run(args, check=True, capture_output=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        vp = C.c_void_p
        lib.sfref_mul.restype = C.c_int
        lib.sfref_mul.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int64, vp, C.c_int64, C.c_int,
                                  vp, vp, vp, vp, vp, vp, C.c_int, vp, C.c_int]
        lib.sfref_max_threads.restype = C.c_int
        _lib = lib
    return _lib


def max_threads() -> int:
    return load().sfref_max_threads()


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def cartesian_colors(n) -> tuple[np.ndarray, int]:
    """8 colours by the parity of the cell coordinates (x fastest cell order):
    cells of one colour share no dof."""
    nx, ny, nz = n
    c = np.arange(nx * ny * nz)
    col = (c % nx) % 2 + 2 * (((c // nx) % ny) % 2) + 4 * ((c // (nx * ny)) % 2)
    return col.astype(np.int32), 8


class Problem:
    """Arrays prepared once for repeated sfref_mul calls."""

    def __init__(self, A0, B0, dof_map0, cell_ids, n_free, fill, wq, jq_rowmajor, djq, kappa=None,
                 colors=None, ncolors=0):
        SQ, SB = A0.shape
        self.SB, self.SQ = SB, SQ
        self.A0 = np.ascontiguousarray(A0.T, dtype=np.float64)  # column-major SQ x SB
        self.B0 = np.ascontiguousarray(B0.T, dtype=np.float64)
        self.dof_map = np.ascontiguousarray((np.asarray(dof_map0) + 1).T, dtype=np.int32)
        self.cell_ids = np.ascontiguousarray(cell_ids, dtype=np.int32)
        self.ncells = self.cell_ids.shape[0]
        self.n_free = int(n_free)
        self.fill = 1 if fill else 0
        self.wq = np.ascontiguousarray(wq, dtype=np.float64)
        # jq per point column-major: jq[l + 3 r] = jq[l, r]
        self.jq = np.ascontiguousarray(np.swapaxes(jq_rowmajor, -1, -2), dtype=np.float64)
        self.djq = np.ascontiguousarray(djq, dtype=np.float64)
        self.kappa = None if kappa is None else np.ascontiguousarray(kappa, dtype=np.float64)
        self.colors = None if colors is None else np.ascontiguousarray(colors, dtype=np.int32)
        self.ncolors = ncolors

    def mul(self, x: np.ndarray, y: np.ndarray | None = None, nthreads: int = 1) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        if y is None:
            y = np.empty(self.n_free)
        st = load().sfref_mul(self.SB, self.SQ, _p(self.A0), _p(self.B0), _p(self.dof_map),
                              self.ncells, _p(self.cell_ids), self.n_free, self.fill, _p(self.wq),
                              _p(self.jq), _p(self.djq), _p(self.kappa), _p(x), _p(y), nthreads,
                              _p(self.colors) if nthreads > 1 else None, self.ncolors)
        if st != 0:
            raise RuntimeError(f"sfref_mul failed with {st}")
        return y


def problem_from_oracle(m, mesh, cq, kappa=None, colors=True) -> Problem:
    """Builds a Problem from sumfac_oracle objects (OracleMap, OracleMesh,
    cell quantities). Cell quantities that are equal in every cell are
    passed as a Fill."""
    wq, jq, djq = cq
    fill = jq.strides[0] == 0 or bool(np.all(jq == jq[:1]) and np.all(djq == djq[:1])
                                       and np.all(wq == wq[:1]))
    if fill:
        wq, jq, djq = wq[:1], jq[:1], djq[:1]
    col, ncol = cartesian_colors(mesh.n) if colors else (None, 0)
    return Problem(m.A0, m.B0, m.dof_map, mesh.cell_dof_ids, mesh.n_free, fill, wq, jq, djq, kappa,
                   col, ncol)


def mul_mesh(m, mesh, x: np.ndarray, nthreads: int | None = None, layers: int = 4,
             kappa: np.ndarray | None = None) -> np.ndarray:
    """y = A x on a whole 3D oracle mesh by the C restatement, with all host
    threads by default. An affine mesh without kappa passes its geometry as a
    Fill. Otherwise the cells are taken in chunks of `layers` z-layers (an even
    number, so the parity colouring of each chunk is valid), so that only one
    chunk's per-point geometry is held on the host at a time, and the chunks'
    contributions are added. This is the checker of the full-size parity runs."""
    import copy

    from oracle import sumfac_oracle as O
    nthreads = max_threads() if nthreads is None else nthreads
    x = np.ascontiguousarray(x, dtype=np.float64)
    if mesh.affine and kappa is None:
        return problem_from_oracle(m, mesh, O.cell_quantities(m, mesh)).mul(x, nthreads=nthreads)
    assert layers % 2 == 0 and mesh.D == 3
    nx, ny, nz = mesh.n
    per = nx * ny
    y = np.zeros(mesh.n_free)
    for z0 in range(0, nz, layers):
        z1 = min(nz, z0 + layers)
        cells = slice(z0 * per, z1 * per)
        sub = copy.copy(mesh)
        sub.n = (nx, ny, z1 - z0)
        sub.cell_vertices = mesh.cell_vertices[cells]
        sub.cell_dof_ids = mesh.cell_dof_ids[cells]
        wq, jq, djq = (np.ascontiguousarray(a) for a in O.cell_quantities(m, sub))
        col, ncol = cartesian_colors(sub.n)
        prob = Problem(m.A0, m.B0, m.dof_map, sub.cell_dof_ids, mesh.n_free, False, wq, jq, djq,
                       None if kappa is None else kappa[cells], col, ncol)
        y += prob.mul(x, nthreads=nthreads)
    return y
