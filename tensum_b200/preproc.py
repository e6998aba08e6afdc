"""Host-side mesh preprocessing: the median-dual geometry TENSUM builds in Grid::preproc.

This is the step the reference runs once on the host before any solve
(src/grid_preproc.cc:1147-1194).  Its outputs -- the face list with dual-face
normals, boundary faces with outward normals, P1 basis normals, cell and dual
areas, periodic vertex sets -- are exactly the arrays the C ABI
``tg_create`` takes (``tg_mesh`` in include/tensum_gpu.h), so a caller that
already has a reference ``Grid`` passes its members directly and a caller
without one (the tests, the benchmark) uses :func:`preprocess`.

Every floating-point expression follows the reference's operation order so the
geometry is bit-identical to the reference's on the same part file:

* face / cell centroids: ``Vector::equ`` (src/vec.h:254-272), src/grid_preproc.cc:18-30, 156-170
* cell area and median dual area: src/grid_preproc.cc:175-211, periodic sum src/reduce_dual_area.cc:18-133
* Voronoi dual cells (``cell="voronoi"``): circumcentres with the small-face
  fix and the boundary check, src/grid_preproc.cc:38-149; dual areas by the
  polygon (shoelace) sum per cell corner, src/grid_preproc.cc:211-246
* face orientation and dual normals: src/grid_preproc.cc:252-303
* boundary-face outward normals: src/grid_preproc.cc:306-328
* P1 basis normals: src/grid_preproc.cc:330-362
* face list order (boundary faces first, then interior faces in discovery
  order) and left/right cells: src/grid_preproc.cc:373-550
* boundary-cell face marks: src/grid_preproc.cc:811-832
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .mesh import TriMesh


@dataclasses.dataclass
class Geometry:
    coords: np.ndarray        # (V, 2)
    cells: np.ndarray         # (C, 3) int64
    cell_normal: np.ndarray   # (C, 3, 2) P1 normals (unscaled, length = opposite edge)
    cell_area: np.ndarray     # (C,)
    face_vertex: np.ndarray   # (F, 2) int64, oriented
    face_type: np.ndarray     # (F,) -1 interior, else boundary tag
    face_normal: np.ndarray   # (F, 2) dual-face normal
    face_measure: np.ndarray  # (F,)
    face_lcell: np.ndarray    # (F,)
    face_rcell: np.ndarray    # (F,) -1 on boundary faces
    bface_vertex: np.ndarray  # (B, 2) oriented so the normal points out
    bface_type: np.ndarray    # (B,)
    bface_normal: np.ndarray  # (B, 2) outward, length = face length
    bface_measure: np.ndarray
    bface_lcell: np.ndarray
    bface_periodic: np.ndarray  # (B,) bool
    dcarea: np.ndarray        # (V,) dual area (periodic-summed)
    mcarea: np.ndarray        # (V,) median area (periodic-summed)
    periodic_sets: list
    # axisymmetric radii (src/grid_preproc.cc:750-777); None for a planar mesh
    vertex_radius: np.ndarray | None = None   # (V,) vertex x
    face_radius: np.ndarray | None = None     # (F,) face centre x
    cell_radius: np.ndarray | None = None     # (C,) cell centre x (dual vertex)

    @property
    def n_vertex(self):
        return self.coords.shape[0]

    @property
    def n_face(self):
        return self.face_vertex.shape[0]

    @property
    def n_bface(self):
        return self.bface_vertex.shape[0]

    @property
    def n_cell(self):
        return self.cells.shape[0]


def _build_face_list(cells: np.ndarray, bfaces: np.ndarray):
    """Face list as src/grid_preproc.cc:447-520 builds it (add_face / make_faces).

    Boundary faces keep their file order and vertex order and take the first
    cell that contains them as left cell; interior faces follow in order of
    first discovery over (cell, local edge 01, 12, 20), with vertex order from
    the discovering cell, left cell = discovering cell, right cell = the other.
    """
    C = cells.shape[0]
    he = np.stack([cells[:, [0, 1]], cells[:, [1, 2]], cells[:, [2, 0]]], axis=1).reshape(-1, 2)
    he_cell = np.repeat(np.arange(C, dtype=np.int64), 3)
    key = np.minimum(he[:, 0], he[:, 1]) * (1 << 32) + np.maximum(he[:, 0], he[:, 1])
    order = np.argsort(key, kind="stable")
    ks = key[order]
    starts = np.flatnonzero(np.r_[True, ks[1:] != ks[:-1]])
    counts = np.diff(np.r_[starts, ks.size])
    if counts.max() > 2:
        raise ValueError("non-manifold mesh: an edge has more than two cells")
    first = order[starts]                     # half-edge index of first occurrence
    second = np.where(counts == 2, order[np.minimum(starts + 1, ks.size - 1)], -1)
    ukey = ks[starts]

    bkey = np.minimum(bfaces[:, 0], bfaces[:, 1]) * (1 << 32) + np.maximum(bfaces[:, 0], bfaces[:, 1])
    pos = np.searchsorted(ukey, bkey)
    if np.any(pos >= ukey.size) or np.any(ukey[np.minimum(pos, ukey.size - 1)] != bkey):
        raise ValueError("a boundary face is not an edge of any cell")
    if np.any(counts[pos] != 1):
        raise ValueError("a boundary face has two cells")
    is_b = np.zeros(ukey.size, bool)
    is_b[pos] = True

    B = bfaces.shape[0]
    b_vertex = bfaces[:, :2].copy()
    b_lcell = he_cell[first[pos]]

    inter = np.flatnonzero(~is_b)
    inter = inter[np.argsort(first[inter], kind="stable")]
    i_vertex = he[first[inter]]
    i_lcell = he_cell[first[inter]]
    if np.any(second[inter] < 0):
        raise ValueError("an edge with one cell is not listed as a boundary face")
    i_rcell = he_cell[second[inter]]

    face_vertex = np.concatenate([b_vertex, i_vertex]).astype(np.int64)
    face_type = np.concatenate([bfaces[:, 2], -np.ones(inter.size, np.int64)])
    face_lcell = np.concatenate([b_lcell, i_lcell])
    face_rcell = np.concatenate([-np.ones(B, np.int64), i_rcell])
    return face_vertex, face_type, face_lcell, face_rcell


def _voronoi_centroids(x, y, cells, bcen, blc):
    """Cell centres of the Voronoi dual (src/grid_preproc.cc:38-149): the
    circumcentre, or the midpoint of the edge opposite a vertex whose weight
    beta vanishes (an obtuse or nearly degenerate corner); a cell whose centre
    falls on one of its boundary faces' centres takes the geometric centroid."""
    n1, n2, n3 = cells[:, 0], cells[:, 1], cells[:, 2]
    x1, y1, x2, y2, x3, y3 = x[n1], y[n1], x[n2], y[n2], x[n3], y[n3]
    pw = np.frompyfunc(math.pow, 2, 1)        # libm pow(d, 2), as the reference calls it

    def sq(d):
        return pw(d, 2.0).astype(np.float64)

    l1 = sq(x2 - x3) + sq(y2 - y3)
    l2 = sq(x3 - x1) + sq(y3 - y1)
    l3 = sq(x1 - x2) + sq(y1 - y2)
    beta1 = np.where(0.0 < l2 + l3 - l1, l2 + l3 - l1, 0.0)   # std::max(0.0, .)
    beta2 = np.where(0.0 < l3 + l1 - l2, l3 + l1 - l2, 0.0)
    beta3 = np.where(0.0 < l1 + l2 - l3, l1 + l2 - l3, 0.0)
    beta1 = np.where((beta1 < beta2 / 2.0) & (beta1 < beta3 / 2.0), 0.0, beta1)
    beta2 = np.where((beta2 < beta3 / 2.0) & (beta2 < beta1 / 2.0), 0.0, beta2)
    beta3 = np.where((beta3 < beta1 / 2.0) & (beta3 < beta2 / 2.0), 0.0, beta3)
    det = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1)
    b1 = 0.5 * ((x2 - x1) * (x2 + x1) + (y2 - y1) * (y2 + y1))
    b2 = 0.5 * ((x3 - x1) * (x3 + x1) + (y3 - y1) * (y3 + y1))
    with np.errstate(divide="ignore", invalid="ignore"):
        xc = ((y3 - y1) * b1 - (y2 - y1) * b2) / det
        yc = (-(x3 - x1) * b1 + (x2 - x1) * b2) / det
    cx = np.where(beta1 == 0.0, 0.5 * (x2 + x3), np.where(beta2 == 0.0, 0.5 * (x3 + x1),
                                                           np.where(beta3 == 0.0, 0.5 * (x1 + x2), xc)))
    cy = np.where(beta1 == 0.0, 0.5 * (y2 + y3), np.where(beta2 == 0.0, 0.5 * (y3 + y1),
                                                           np.where(beta3 == 0.0, 0.5 * (y1 + y2), yc)))
    cen = np.stack([cx, cy], 1)
    third = 1.0 / 3.0
    for i in range(bcen.shape[0]):
        c = blc[i]
        dx = bcen[i, 0] * 1.0 + cen[c, 0] * (-1.0)
        dy = bcen[i, 1] * 1.0 + cen[c, 1] * (-1.0)
        if math.sqrt(dx * dx + dy * dy + 0.0 * 0.0) < 1.0e-14:
            v0, v1, v2 = cells[c]
            cen[c, 0] = x[v0] * third + x[v1] * third + x[v2] * third
            cen[c, 1] = y[v0] * third + y[v1] * third + y[v2] * third
    return cen


def _polygon_dual_areas(x, y, cells, cen, V):
    """Dual area per vertex as the reference sums it for non-median cells
    (src/grid_preproc.cc:211-246): per cell corner n0, the polygon n0, mid(n0, n2),
    cell centre, mid(n0, n1) by the shoelace formula, added in cell and corner order."""
    C = cells.shape[0]
    areas = np.empty((C, 3))
    for j in range(3):
        n0 = cells[:, j]
        n1 = cells[:, 2] if j == 0 else cells[:, j - 1]
        n2 = cells[:, 0] if j == 2 else cells[:, j + 1]
        px = [x[n0], x[n0] * 0.5 + x[n2] * 0.5, cen[:, 0], x[n0] * 0.5 + x[n1] * 0.5, x[n0]]
        py = [y[n0], y[n0] * 0.5 + y[n2] * 0.5, cen[:, 1], y[n0] * 0.5 + y[n1] * 0.5, y[n0]]
        a = np.zeros(C)
        for k in range(4):
            a = a + (px[k] * py[k + 1] - px[k + 1] * py[k])
        if np.any(a < 0.0):
            raise ValueError("dual cell area is non-positive (src/grid_preproc.cc:237-241)")
        areas[:, j] = a * 0.5
    dc = np.zeros(V)
    np.add.at(dc, cells.reshape(-1), areas.reshape(-1))
    return dc


def preprocess(mesh: TriMesh, periodic_types=None, cell: str = "median", axisymmetric: bool = False) -> Geometry:
    """Dual-mesh preprocessing of a single-partition mesh, median or Voronoi
    dual cells (the grid section's ``cell`` entry), planar (radius 1) or
    axisymmetric (the reference's -axi: radius = x, src/grid_preproc.cc:750-777).

    ``periodic_types``: boundary tags whose BC is ``periodic``.  Faces with
    such a tag keep their part-file periodic flag; all others are marked
    non-periodic, as src/read_part_mesh_file.cc:166-170 does.
    """
    if cell not in ("median", "voronoi"):
        raise ValueError(f"unknown dual cell type {cell!r}")
    coords = np.asarray(mesh.coords, np.float64)
    cells = np.asarray(mesh.cells, np.int64)
    bfaces = np.asarray(mesh.bfaces, np.int64)
    V, C = coords.shape[0], cells.shape[0]
    x, y = coords[:, 0], coords[:, 1]

    fv, ftype, flc, frc = _build_face_list(cells, bfaces)
    if periodic_types is None:
        periodic_types = set(int(t) for t in bfaces[bfaces[:, 3] == 1, 2])
    bper = np.array([(bool(f[3]) and int(f[2]) in periodic_types) for f in bfaces], bool)

    third = 1.0 / 3.0
    # face centroids  (equ(a, b, 0.5, 0.5) = a*0.5 + b*0.5)
    def mid(v0, v1):
        return np.stack([x[v0] * 0.5 + x[v1] * 0.5, y[v0] * 0.5 + y[v1] * 0.5], 1)

    c0, c1, c2 = cells[:, 0], cells[:, 1], cells[:, 2]
    if cell == "voronoi":
        B0 = bfaces.shape[0]
        cen = _voronoi_centroids(x, y, cells, mid(bfaces[:, 0], bfaces[:, 1]), flc[:B0])
    else:
        cen = np.stack([x[c0] * third + x[c1] * third + x[c2] * third,
                        y[c0] * third + y[c1] * third + y[c2] * third], 1)

    # cell area: l1 = v1 - v0, l2 = v2 - v0, area = 0.5 * (l1.x*l2.y - l1.y*l2.x)
    l1x = x[c1] * 1.0 + x[c0] * (-1.0)
    l1y = y[c1] * 1.0 + y[c0] * (-1.0)
    l2x = x[c2] * 1.0 + x[c0] * (-1.0)
    l2y = y[c2] * 1.0 + y[c0] * (-1.0)
    area = 0.5 * (l1x * l2y - l1y * l2x)
    if np.any(area <= 0.0):
        raise ValueError("non-positive cell area (cells must be counter-clockwise)")
    # median areas: mcarea[v] += area/3 in cell order, vertices 0,1,2
    a3 = area / 3.0
    mc = np.zeros(V)
    contrib_v = cells.reshape(-1)
    contrib_a = np.repeat(a3, 3)
    # np.add.at accumulates in index order, i.e. the reference's loop order
    np.add.at(mc, contrib_v, contrib_a)
    dcv = _polygon_dual_areas(x, y, cells, cen, V) if cell == "voronoi" else None
    for s in mesh.periodic_sets:
        acc = 0.0
        for v in s:
            acc += mc[v] * 1.0
        mc[s] = acc
        if dcv is not None:
            acc = 0.0
            for v in s:
                acc += dcv[v] * 1.0
            dcv[s] = acc
    dc = mc.copy() if dcv is None else dcv

    # face orientation (src/grid_preproc.cc:256-277)
    fc = mid(fv[:, 0], fv[:, 1])
    drx = x[fv[:, 1]] * 1.0 + x[fv[:, 0]] * (-1.0)
    dry = y[fv[:, 1]] * 1.0 + y[fv[:, 0]] * (-1.0)
    nx, ny = dry, -drx
    dcfx = fc[:, 0] * 1.0 + cen[flc, 0] * (-1.0)
    dcfy = fc[:, 1] * 1.0 + cen[flc, 1] * (-1.0)
    d = dcfx * nx + dcfy * ny + 0.0 * 0.0
    flip = d < 0.0
    fv = np.where(flip[:, None], fv[:, ::-1], fv)
    fc = mid(fv[:, 0], fv[:, 1])
    # dual-face normals
    dx = fc[:, 0] * 1.0 + cen[flc, 0] * (-1.0)
    dy = fc[:, 1] * 1.0 + cen[flc, 1] * (-1.0)
    inter = ftype == -1
    rc = np.where(inter, frc, 0)
    dx = np.where(inter, dx + (cen[rc, 0] * 1.0 + fc[:, 0] * (-1.0)), dx)
    dy = np.where(inter, dy + (cen[rc, 1] * 1.0 + fc[:, 1] * (-1.0)), dy)
    fnormal = np.stack([-dy, dx], 1)
    fmeasure = np.sqrt(fnormal[:, 0] * fnormal[:, 0] + fnormal[:, 1] * fnormal[:, 1] + 0.0)
    if cell == "voronoi":
        # remove_empty_faces (src/grid_preproc.cc:633-647): dual faces of zero measure go
        keep = fmeasure > 0.0
        fv, ftype, flc, frc = fv[keep], ftype[keep], flc[keep], frc[keep]
        fnormal, fmeasure = fnormal[keep], fmeasure[keep]

    # boundary faces (copied from the face list before the flip above)
    B = bfaces.shape[0]
    bv = bfaces[:, :2].copy()
    blc = flc[:B].copy()
    bcen = mid(bv[:, 0], bv[:, 1])
    bdx = x[bv[:, 1]] * 1.0 + x[bv[:, 0]] * (-1.0)
    bdy = y[bv[:, 1]] * 1.0 + y[bv[:, 0]] * (-1.0)
    bn = np.stack([bdy, -bdx], 1)
    bmeasure = np.sqrt(bn[:, 0] * bn[:, 0] + bn[:, 1] * bn[:, 1] + 0.0)
    bd = (bcen[:, 0] * 1.0 + cen[blc, 0] * (-1.0)) * bn[:, 0] + \
         (bcen[:, 1] * 1.0 + cen[blc, 1] * (-1.0)) * bn[:, 1] + 0.0 * 0.0
    bflip = bd < 0.0
    bv = np.where(bflip[:, None], bv[:, ::-1], bv)
    bn = np.where(bflip[:, None], bn * -1.0, bn)

    # P1 normals: normal[0] = dr12, normal[1] = dr20, normal[2] = dr01
    def drn(a, b):
        return np.stack([y[a] - y[b], -(x[a] - x[b])], 1)
    cnormal = np.stack([drn(c1, c2), drn(c2, c0), drn(c0, c1)], 1)

    radii = {}
    if axisymmetric:
        radii = dict(vertex_radius=x.copy(), face_radius=mid(fv[:, 0], fv[:, 1])[:, 0].copy(),
                     cell_radius=cen[:, 0].copy())
    return Geometry(coords=coords, cells=cells, cell_normal=cnormal, cell_area=area,
                    face_vertex=fv, face_type=ftype, face_normal=fnormal, face_measure=fmeasure,
                    face_lcell=flc, face_rcell=frc,
                    bface_vertex=bv, bface_type=bfaces[:, 2].copy(), bface_normal=bn,
                    bface_measure=bmeasure, bface_lcell=blc, bface_periodic=bper,
                    dcarea=dc, mcarea=mc, periodic_sets=[list(s) for s in mesh.periodic_sets], **radii)
