"""Seeded synthetic triangulations in TENSUM's partitioned-mesh format.

gmsh is not available, so every mesh the solver runs on is generated here and
written in the reference's ``PARTITION/part_file_<p>.dat`` layout (format:
readme/README.md:154-202, parsed by src/read_part_mesh_file.cc:17-250).  With
one partition every vertex and cell is active and each vertex lists partition
0 as its only owner.

Two families cover the workloads:

* :func:`periodic_square` -- an N x N vertex grid on a rectangle, each quad cut
  along a seeded random diagonal, interior vertices jittered by
  U[-j h, j h]; all four sides periodic (left/right, bottom/top, 4 corners).
* :func:`annulus` -- an O-mesh around a cylinder (inner no-slip wall, outer
  far field) with geometric radial stretching and seeded diagonals; the
  angular seam shares vertices and is not a periodic boundary.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np


@dataclasses.dataclass
class TriMesh:
    """Vertices, CCW triangles, boundary faces and periodic vertex sets.

    ``bfaces`` rows are (v0, v1, tag, periodic_flag) in file order;
    ``periodic_sets`` is a list of vertex-id lists, each one periodic set
    P_i (src/grid.h:96-101).  ``on_boundary`` is the part-file d_bnd flag.
    """

    coords: np.ndarray          # (V, 2) float64
    cells: np.ndarray           # (C, 3) int64, counter-clockwise
    bfaces: np.ndarray          # (B, 4) int64
    periodic_sets: list
    on_boundary: np.ndarray     # (V,) bool
    name: str = "mesh"

    @property
    def n_vertex(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_cell(self) -> int:
        return int(self.cells.shape[0])


def _split_quads(ids: np.ndarray, diag: np.ndarray) -> np.ndarray:
    """Cut each quad a=(i,j) b=(i+1,j) c=(i+1,j+1) d=(i,j+1) into two CCW triangles.

    diag == 0 uses the a-c diagonal, diag == 1 the b-d diagonal.
    """
    a = ids[:-1, :-1]
    b = ids[1:, :-1]
    c = ids[1:, 1:]
    d = ids[:-1, 1:]
    t0 = np.where(diag[..., None] == 0, np.stack([a, b, c], -1), np.stack([a, b, d], -1))
    t1 = np.where(diag[..., None] == 0, np.stack([a, c, d], -1), np.stack([b, c, d], -1))
    # interleave so that both triangles of a quad are neighbours in the cell list
    cells = np.stack([t0, t1], axis=-2)            # (ni, nj, 2, 3)
    cells = cells.transpose(1, 0, 2, 3)             # quad order: j outer, i inner
    return cells.reshape(-1, 3).astype(np.int64)


def periodic_square(n: int, x0: float, x1: float, y0: float, y1: float, seed: int,
                    jitter: float = 0.15, name: str | None = None) -> TriMesh:
    """N x N vertex periodic grid, seeded diagonals, interior jitter of +-jitter*h."""
    if n < 3:
        raise ValueError("periodic_square needs at least 3 vertices per side")
    rng = np.random.default_rng(seed)
    hx = (x1 - x0) / (n - 1)
    hy = (y1 - y0) / (n - 1)
    i = np.arange(n)
    X, Y = np.meshgrid(x0 + i * hx, y0 + i * hy, indexing="ij")   # [i, j]
    diag = rng.integers(0, 2, size=(n - 1, n - 1))
    jit = rng.uniform(-jitter, jitter, size=(n, n, 2))
    interior = np.zeros((n, n), dtype=bool)
    interior[1:-1, 1:-1] = True
    X = X + np.where(interior, jit[..., 0] * hx, 0.0)
    Y = Y + np.where(interior, jit[..., 1] * hy, 0.0)
    # global id = j * n + i (rows of constant y)
    ids = (np.arange(n)[None, :] * n + np.arange(n)[:, None]).astype(np.int64)  # ids[i, j]
    coords = np.empty((n * n, 2))
    coords[ids.ravel(), 0] = X.ravel()
    coords[ids.ravel(), 1] = Y.ravel()
    cells = _split_quads(ids, diag)

    bf = []
    for k in range(n - 1):
        bf.append((ids[k, 0], ids[k + 1, 0], 1, 1))            # bottom
    for k in range(n - 1):
        bf.append((ids[n - 1, k], ids[n - 1, k + 1], 2, 1))    # right
    for k in range(n - 1):
        bf.append((ids[k + 1, n - 1], ids[k, n - 1], 3, 1))    # top
    for k in range(n - 1):
        bf.append((ids[0, k + 1], ids[0, k], 4, 1))            # left
    bfaces = np.array(bf, dtype=np.int64)

    sets = []
    for k in range(1, n - 1):
        sets.append([int(ids[0, k]), int(ids[n - 1, k])])      # left <-> right
    for k in range(1, n - 1):
        sets.append([int(ids[k, 0]), int(ids[k, n - 1])])      # bottom <-> top
    sets.append([int(ids[0, 0]), int(ids[n - 1, 0]), int(ids[n - 1, n - 1]), int(ids[0, n - 1])])
    on_b = np.zeros(n * n, dtype=bool)
    on_b[ids[~interior]] = True
    return TriMesh(coords, cells, bfaces, sets, on_b, name or f"square{n}")


def radial_stations(n_r: int, r0: float, r1: float, dr0: float) -> np.ndarray:
    """Geometric radial stations from r0 to r1 with first spacing dr0.

    The growth ratio q solves dr0 (q^(n_r-1) - 1)/(q - 1) = r1 - r0 (bisection),
    so both end radii are met exactly.
    """
    target = (r1 - r0) / dr0
    m = n_r - 1
    if target <= m:
        raise ValueError("first spacing too large for the requested radii")
    lo, hi = 1.0 + 1e-12, 2.0
    for _ in range(200):
        q = 0.5 * (lo + hi)
        s = (q ** m - 1.0) / (q - 1.0)
        if s > target:
            hi = q
        else:
            lo = q
    q = 0.5 * (lo + hi)
    r = r0 + dr0 * (q ** np.arange(n_r) - 1.0) / (q - 1.0)
    r[-1] = r1
    return r


def annulus(n_r: int, n_t: int, r0: float, r1: float, dr0: float, seed: int,
            wall_tag: int = 1, far_tag: int = 2, name: str | None = None) -> TriMesh:
    """O-mesh: n_r radial stations x n_t angular points, seeded diagonals."""
    rng = np.random.default_rng(seed)
    r = radial_stations(n_r, r0, r1, dr0)
    th = 2.0 * np.pi * np.arange(n_t) / n_t
    R, T = np.meshgrid(r, th, indexing="ij")          # [k, t]
    ids_core = (np.arange(n_r)[:, None] * n_t + np.arange(n_t)[None, :]).astype(np.int64)
    coords = np.stack([(R * np.cos(T)).ravel(), (R * np.sin(T)).ravel()], axis=1)
    ids = np.concatenate([ids_core, ids_core[:, :1]], axis=1)   # wrap the seam
    diag = rng.integers(0, 2, size=(n_r - 1, n_t))
    cells = _split_quads(ids, diag)
    bf = []
    for t in range(n_t):
        bf.append((ids[0, t + 1], ids[0, t], wall_tag, 0))
    for t in range(n_t):
        bf.append((ids[n_r - 1, t], ids[n_r - 1, t + 1], far_tag, 0))
    on_b = np.zeros(n_r * n_t, dtype=bool)
    on_b[ids_core[0]] = True
    on_b[ids_core[-1]] = True
    return TriMesh(coords, cells, np.array(bf, dtype=np.int64), [], on_b,
                   name or f"annulus{n_r}x{n_t}")


# ----------------------------------------------------------------------------
# part-file I/O
# ----------------------------------------------------------------------------

def write_part_file(mesh: TriMesh, case_dir: str) -> str:
    """Write PARTITION/part_file_0.dat (one partition) and return its path."""
    pdir = os.path.join(case_dir, "PARTITION")
    os.makedirs(pdir, exist_ok=True)
    path = os.path.join(pdir, "part_file_0.dat")
    V = mesh.n_vertex
    lines = ["DIMENSION 2", "PARTITIONS 1", f"NODES {V} OF {V}"]
    xy = mesh.coords
    ob = mesh.on_boundary.astype(int)
    xs = [repr(float(a)) for a in xy[:, 0]]   # shortest round-trip decimal: exact when read back
    ys = [repr(float(a)) for a in xy[:, 1]]
    lines.extend(f"{v} {xs[v]} {ys[v]} 0 1 0 {ob[v]}" for v in range(V))
    lines.append(f"PERIODIC {len(mesh.periodic_sets)}")
    for k, s in enumerate(mesh.periodic_sets):
        lines.append(f"{k} {len(s)} " + " ".join(str(v) for v in s) + " 1 0")
    B = mesh.bfaces.shape[0]
    lines.append(f"FACES {B} OF {B}")
    lines.extend(f"{f[2]} {f[0]} {f[1]} {f[3]}" for f in mesh.bfaces)
    C = mesh.n_cell
    lines.append(f"CELLS {C} OF {C}")
    lines.extend(f"{c[0]} {c[1]} {c[2]} 0" for c in mesh.cells)
    with open(path, "w") as fh:
        fh.write("\n".join(lines))
        fh.write("\n")
    return path


def read_part_file(path: str) -> TriMesh:
    """Parse a single-partition part file (active entities only)."""
    with open(path) as fh:
        tok = fh.read().split()
    p = 0

    def nxt():
        nonlocal p
        p += 1
        return tok[p - 1]

    assert nxt() == "DIMENSION" and int(nxt()) == 2
    assert nxt() == "PARTITIONS"
    npart = int(nxt())
    if npart != 1:
        raise ValueError("only single-partition files are supported on the GPU path")
    assert nxt() == "NODES"
    nv = int(nxt()); nxt(); int(nxt())
    gid = np.empty(nv, np.int64)
    coords = np.empty((nv, 2))
    on_b = np.empty(nv, bool)
    for i in range(nv):
        gid[i] = int(nxt())
        coords[i, 0] = float(nxt()); coords[i, 1] = float(nxt()); float(nxt())
        ns = int(nxt())
        for _ in range(ns):
            nxt()
        on_b[i] = bool(int(nxt()))
    g2l = {int(g): i for i, g in enumerate(gid)}
    assert nxt() == "PERIODIC"
    sets = []
    for _ in range(int(nxt())):
        nxt()
        k = int(nxt())
        sets.append([g2l[int(nxt())] for _ in range(k)])
        for _ in range(int(nxt())):
            nxt()
    assert nxt() == "FACES"
    nf = int(nxt()); nxt(); nxt()
    bf = np.empty((nf, 4), np.int64)
    for i in range(nf):
        t = int(nxt()); a = g2l[int(nxt())]; b = g2l[int(nxt())]; per = int(nxt())
        bf[i] = (a, b, t, per)
    assert nxt() == "CELLS"
    nc = int(nxt()); nxt(); nxt()
    cells = np.empty((nc, 3), np.int64)
    for i in range(nc):
        cells[i] = (g2l[int(nxt())], g2l[int(nxt())], g2l[int(nxt())])
        if int(nxt()) != 0:
            raise ValueError("ghost cells are not expected in a single-partition file")
    return TriMesh(coords, cells, bf, sets, on_b, os.path.basename(path))
