"""Quasi-uniform icosahedral Voronoi C-grid meshes in MPAS conventions.

The dycore consumes the same mesh fields as an MPAS static file
(``hexcore/mesh.py`` ``Mesh`` in the reference reads them from netCDF).  These
meshes are built here, from scratch, so the GPU box needs no mesh assets:

* an icosahedron bisected ``level`` times gives the generators
  (10*4**level + 2 of them: 2562 at 4, 10242 at 5, 40962 at 6, 163842 at 7);
* a seeded jitter followed by ``lloyd`` Lloyd iterations relaxes them towards
  a centroidal Voronoi tessellation;
* the Delaunay triangulation is the convex hull of the generators, and the
  Voronoi vertices are the triangles' circumcentres;
* cells are numbered along a 3-D Hilbert curve of the generator positions
  (the space-filling-curve order the GPU kernels rely on for gather
  locality), edges by their (cell1, cell2) pair and vertices by their sorted
  cell triple, so neighbouring entities sit close in memory.

Conventions (zero-based, ``-1`` padding), as the reference's consumers use
them (``hexcore/acoustic.py:224`` edge signs, ``hexcore/diagnostics.py:49``
vertex signs, ``hexcore/diagnostics.py:64`` kites):

* ``cellsOnEdge[e] = (c1, c2)`` with ``c1 < c2``; the edge normal points from
  c1 to c2;
* ``verticesOnEdge[e] = (v1, v2)``: v2 lies to the left of the normal, so the
  tangent ``t = k x n`` points from v1 to v2;
* ``cellsOnCell/edgesOnCell`` run counter-clockwise seen from outside, and
  ``verticesOnCell[i][m]`` is the vertex between ``edgesOnCell[i][m]`` and
  ``edgesOnCell[i][m+1]``;
* ``cellsOnVertex[v]`` is counter-clockwise and ``edgesOnVertex[v][m]`` joins
  ``cellsOnVertex[v][m]`` and ``cellsOnVertex[v][m+1]``;
* ``weightsOnEdge`` are the TRiSK weights of Thuburn et al. (2009) and
  Ringler et al. (2010), with ``dvEdge(e')/dcEdge(e)`` folded in, so that the
  tangential velocity is ``v_e = sum_j weightsOnEdge[e][j] u[edgesOnEdge[e][j]]``.

All geometry is float64 (as in an MPAS static file); the dycore casts to its
FP32 working precision where the reference does.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np
from scipy.spatial import ConvexHull

EARTH_RADIUS = 6371220.0
OMEGA = 7.29212e-5
MAX_EDGES = 6
MAX_EDGES2 = 2 * MAX_EDGES


def _icosahedron() -> tuple[np.ndarray, np.ndarray]:
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = np.array(
        [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
         (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], dtype=np.float64)
    faces = np.array(
        [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
         (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
         (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
         (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int64)
    return verts / np.linalg.norm(verts, axis=1, keepdims=True), faces


def bisected_icosahedron(level: int) -> np.ndarray:
    """Unit generators of an icosahedron bisected ``level`` times."""
    if level < 0:
        raise ValueError("level must be non-negative")
    points, faces = _icosahedron()
    for _ in range(level):
        edges = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inverse = np.unique(key, axis=0, return_inverse=True)
        inverse = inverse.reshape(-1)
        mids = points[uniq[:, 0]] + points[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = points.shape[0]
        points = np.concatenate([points, mids])
        nf = faces.shape[0]
        m01 = base + inverse[:nf]
        m12 = base + inverse[nf:2 * nf]
        m20 = base + inverse[2 * nf:]
        a, b, c = faces.T
        faces = np.concatenate([
            np.stack([a, m01, m20], axis=1),
            np.stack([m01, b, m12], axis=1),
            np.stack([m20, m12, c], axis=1),
            np.stack([m01, m12, m20], axis=1),
        ])
    return points


def _delaunay(points: np.ndarray) -> np.ndarray:
    """Counter-clockwise (seen from outside) Delaunay triangles on the sphere."""
    tri = ConvexHull(points).simplices.astype(np.int64)
    a, b, c = points[tri[:, 0]], points[tri[:, 1]], points[tri[:, 2]]
    flip = np.einsum("ij,ij->i", np.cross(b - a, c - a), a) < 0.0
    tri[flip] = tri[flip][:, [0, 2, 1]]
    return tri


def _circumcentres(points: np.ndarray, tri: np.ndarray) -> np.ndarray:
    a, b, c = points[tri[:, 0]], points[tri[:, 1]], points[tri[:, 2]]
    n = np.cross(b - a, c - a)
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def _oriented_area(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """Signed area of the unit-sphere triangle (a, b, c) (Van Oosterom-Strackee)."""
    num = np.einsum("ij,ij->i", a, np.cross(b, c))
    den = 1.0 + np.einsum("ij,ij->i", a, b) + np.einsum("ij,ij->i", b, c) + np.einsum("ij,ij->i", c, a)
    return 2.0 * np.arctan2(num, den)


def _arc(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return 2.0 * np.arcsin(np.clip(0.5 * np.linalg.norm(a - b, axis=1), 0.0, 1.0))


def _lloyd_step(points: np.ndarray) -> np.ndarray:
    tri = _delaunay(points)
    cc = _circumcentres(points, tri)
    n = points.shape[0]
    acc = np.zeros_like(points)
    # Each triangle contributes, to each of its corners, the two planar
    # sub-triangles (corner, edge-midpoint, circumcentre) of that corner's
    # Voronoi cell; their area-weighted centroids average to the cell centroid.
    for k in range(3):
        p = points[tri[:, k]]
        for other in (tri[:, (k + 1) % 3], tri[:, (k + 2) % 3]):
            m = 0.5 * (p + points[other])
            area = 0.5 * np.linalg.norm(np.cross(m - p, cc - p), axis=1)
            centroid = (p + m + cc) / 3.0
            np.add.at(acc, tri[:, k], area[:, None] * centroid)
    return acc / np.linalg.norm(acc, axis=1, keepdims=True)


def _hilbert_keys(points: np.ndarray, bits: int = 16) -> np.ndarray:
    """3-D Hilbert index of each point (Skilling 2004, axes to transpose)."""
    q = np.clip(((points + 1.0) * 0.5 * ((1 << bits) - 1)).round(), 0, (1 << bits) - 1)
    x = [q[:, i].astype(np.uint64) for i in range(3)]
    m = np.uint64(1 << (bits - 1))
    big_q = m
    while big_q > 1:
        p = big_q - np.uint64(1)
        for i in range(3):
            hit = (x[i] & big_q) != 0
            if i == 0:
                x[0] = np.where(hit, x[0] ^ p, x[0])
                continue
            t = (x[0] ^ x[i]) & p
            new0 = np.where(hit, x[0] ^ p, x[0] ^ t)
            newi = np.where(hit, x[i], x[i] ^ t)
            x[0], x[i] = new0, newi
        big_q >>= np.uint64(1)
    for i in range(1, 3):
        x[i] = x[i] ^ x[i - 1]
    t = np.zeros_like(x[0])
    big_q = m
    while big_q > 1:
        t = np.where((x[2] & big_q) != 0, t ^ (big_q - np.uint64(1)), t)
        big_q >>= np.uint64(1)
    x = [xi ^ t for xi in x]
    key = np.zeros_like(x[0])
    for b in range(bits - 1, -1, -1):
        for i in range(3):
            key = (key << np.uint64(1)) | ((x[i] >> np.uint64(b)) & np.uint64(1))
    return key


@dataclass
class VoronoiMesh:
    """MPAS-convention mesh fields (float64 geometry, int64 connectivity)."""

    arrays: dict[str, Any] = field(default_factory=dict)
    level: int = 0
    lloyd: int = 0
    seed: int = 0

    def __getattr__(self, name: str) -> Any:
        arrays = self.__dict__.get("arrays")
        if arrays is not None and name in arrays:
            return arrays[name]
        raise AttributeError(name)

    @property
    def n_cells(self) -> int:
        return int(self.arrays["areaCell"].size)

    @property
    def n_edges(self) -> int:
        return int(self.arrays["dcEdge"].size)

    @property
    def n_vertices(self) -> int:
        return int(self.arrays["areaTriangle"].size)


def build_mesh(level: int, *, lloyd: int = 20, seed: int = 0,
               radius: float = EARTH_RADIUS, jitter: float = 1.0e-3) -> VoronoiMesh:
    """Build the bisected-icosahedron Voronoi mesh with ``lloyd`` iterations.

    ``jitter`` is the seeded random displacement of each generator, in units
    of the mean generator spacing, applied before the Lloyd iterations.
    """
    points = bisected_icosahedron(level)
    rng = np.random.default_rng(seed)
    spacing = np.sqrt(4.0 * np.pi / points.shape[0])
    points = points + jitter * spacing * rng.standard_normal(points.shape)
    points /= np.linalg.norm(points, axis=1, keepdims=True)
    for _ in range(lloyd):
        points = _lloyd_step(points)
    points = points[np.argsort(_hilbert_keys(points), kind="stable")]
    mesh = VoronoiMesh(arrays=_connectivity(points, radius), level=level, lloyd=lloyd, seed=seed)
    return mesh


def _connectivity(points: np.ndarray, radius: float) -> dict[str, Any]:
    n_cells = points.shape[0]
    tri = _delaunay(points)
    # Vertices in the order of their sorted cell triple.
    order = np.lexsort(np.sort(tri, axis=1).T[::-1])
    tri = tri[order]
    n_vertices = tri.shape[0]
    # Rotate each triangle so that its smallest cell comes first (keeps ccw).
    rot = np.argmin(tri, axis=1)
    idx = (rot[:, None] + np.arange(3)[None, :]) % 3
    tri = np.take_along_axis(tri, idx, axis=1)
    cc = _circumcentres(points, tri)

    # Directed half-edges a->b of every ccw triangle: the triangle lies on
    # the left of a->b and c = succ of b around a.
    a = tri.reshape(-1)
    b = tri[:, [1, 2, 0]].reshape(-1)
    c = tri[:, [2, 0, 1]].reshape(-1)
    tri_of = np.repeat(np.arange(n_vertices), 3)
    half_key = a * n_cells + b
    half_order = np.argsort(half_key)
    half_sorted = half_key[half_order]

    def half_lookup(src: np.ndarray, dst: np.ndarray) -> np.ndarray:
        pos = np.searchsorted(half_sorted, src * n_cells + dst)
        if np.any(half_sorted[np.minimum(pos, half_sorted.size - 1)] != src * n_cells + dst):
            raise RuntimeError("mesh half-edge lookup failed")
        return half_order[pos]

    # Edges: unordered Delaunay edges, c1 < c2, sorted by (c1, c2).
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    keys = np.unique(lo * n_cells + hi)
    cells_on_edge = np.stack([keys // n_cells, keys % n_cells], axis=1)
    n_edges = cells_on_edge.shape[0]

    def edge_index(x: np.ndarray, y: np.ndarray) -> np.ndarray:
        k = np.minimum(x, y) * n_cells + np.maximum(x, y)
        pos = np.searchsorted(keys, k)
        return pos

    c1, c2 = cells_on_edge[:, 0], cells_on_edge[:, 1]
    left = tri_of[half_lookup(c1, c2)]    # triangle with directed edge c1->c2
    right = tri_of[half_lookup(c2, c1)]
    vertices_on_edge = np.stack([right, left], axis=1)

    # Cells: neighbours counter-clockwise starting from the smallest index.
    degree = np.bincount(a, minlength=n_cells)
    if degree.max() > MAX_EDGES or degree.min() < 5:
        raise RuntimeError("unexpected cell degree in the icosahedral mesh")
    first = np.full(n_cells, np.iinfo(np.int64).max)
    np.minimum.at(first, a, b)
    cells_on_cell = np.full((n_cells, MAX_EDGES), -1, dtype=np.int64)
    vertices_on_cell = np.full((n_cells, MAX_EDGES), -1, dtype=np.int64)
    cur = first.copy()
    cell_ids = np.arange(n_cells)
    for m in range(MAX_EDGES):
        active = m < degree
        ci, cj = cell_ids[active], cur[active]
        h = half_lookup(ci, cj)
        cells_on_cell[ci, m] = cj
        vertices_on_cell[ci, m] = tri_of[h]
        cur[active] = c[h]
    edges_on_cell = np.full((n_cells, MAX_EDGES), -1, dtype=np.int64)
    valid = cells_on_cell >= 0
    rows = np.nonzero(valid)
    edges_on_cell[rows] = edge_index(rows[0], cells_on_cell[rows])

    cells_on_vertex = tri.copy()
    edges_on_vertex = np.stack(
        [edge_index(tri[:, m], tri[:, (m + 1) % 3]) for m in range(3)], axis=1)

    # Geometry on the unit sphere, scaled at the end.
    x_edge = points[c1] + points[c2]
    x_edge /= np.linalg.norm(x_edge, axis=1, keepdims=True)
    dc = _arc(points[c1], points[c2])
    dv = _arc(cc[vertices_on_edge[:, 0]], cc[vertices_on_edge[:, 1]])
    d = points[c2] - points[c1]
    normal = d - np.einsum("ij,ij->i", d, x_edge)[:, None] * x_edge
    normal /= np.linalg.norm(normal, axis=1, keepdims=True)
    zhat = np.array([0.0, 0.0, 1.0])
    east = np.cross(np.broadcast_to(zhat, x_edge.shape), x_edge)
    east /= np.linalg.norm(east, axis=1, keepdims=True)
    north = np.cross(x_edge, east)
    angle_edge = np.arctan2(np.einsum("ij,ij->i", normal, north),
                            np.einsum("ij,ij->i", normal, east))

    # Kites: the part of triangle v inside the Voronoi cell of each corner.
    kites = np.zeros((n_vertices, 3))
    for m in range(3):
        pc = points[tri[:, m]]
        pn = points[tri[:, (m + 1) % 3]]
        pp = points[tri[:, (m + 2) % 3]]
        mn = pc + pn
        mn /= np.linalg.norm(mn, axis=1, keepdims=True)
        mp = pc + pp
        mp /= np.linalg.norm(mp, axis=1, keepdims=True)
        kites[:, m] = _oriented_area(pc, mn, cc) + _oriented_area(pc, cc, mp)
    if np.any(kites <= 0.0):
        raise RuntimeError("non-positive kite area: the mesh has an obtuse Delaunay triangle")
    area_triangle = kites.sum(axis=1)
    area_cell = np.zeros(n_cells)
    np.add.at(area_cell, tri.reshape(-1), kites.reshape(-1))

    lat = lambda p: np.arcsin(np.clip(p[:, 2], -1.0, 1.0))  # noqa: E731
    lon = lambda p: np.mod(np.arctan2(p[:, 1], p[:, 0]), 2.0 * np.pi)  # noqa: E731

    r2 = radius * radius
    arrays: dict[str, Any] = {
        "nCells": n_cells, "nEdges": n_edges, "nVertices": n_vertices,
        "sphere_radius": radius, "on_a_sphere": True,
        "nEdgesOnCell": degree.astype(np.int64),
        "cellsOnCell": cells_on_cell, "edgesOnCell": edges_on_cell,
        "verticesOnCell": vertices_on_cell,
        "cellsOnEdge": cells_on_edge, "verticesOnEdge": vertices_on_edge,
        "cellsOnVertex": cells_on_vertex, "edgesOnVertex": edges_on_vertex,
        "xCell": radius * points[:, 0], "yCell": radius * points[:, 1],
        "zCell": radius * points[:, 2],
        "latCell": lat(points), "lonCell": lon(points),
        "xEdge": radius * x_edge[:, 0], "yEdge": radius * x_edge[:, 1],
        "zEdge": radius * x_edge[:, 2],
        "latEdge": lat(x_edge), "lonEdge": lon(x_edge),
        "xVertex": radius * cc[:, 0], "yVertex": radius * cc[:, 1],
        "zVertex": radius * cc[:, 2],
        "latVertex": lat(cc), "lonVertex": lon(cc),
        "dcEdge": radius * dc, "dvEdge": radius * dv,
        "angleEdge": angle_edge,
        "areaCell": r2 * area_cell, "areaTriangle": r2 * area_triangle,
        "kiteAreasOnVertex": r2 * kites,
        "meshDensity": np.ones(n_cells),
        "indexToCellID": np.arange(1, n_cells + 1, dtype=np.int64),
    }
    arrays["fEdge"] = 2.0 * OMEGA * np.sin(arrays["latEdge"])
    arrays["fVertex"] = 2.0 * OMEGA * np.sin(arrays["latVertex"])
    arrays["fCell"] = 2.0 * OMEGA * np.sin(arrays["latCell"])
    arrays["nominalMinDc"] = np.array(float(np.min(arrays["dcEdge"])))
    _trisk(arrays)
    # Edge normal/tangent unit vectors (not MPAS fields; used by the case
    # builder to project wind vectors onto edges).
    arrays["_edge_normal"] = normal
    arrays["_edge_tangent"] = np.cross(x_edge, normal)
    return arrays


def _kite_slot(arrays: dict[str, Any]) -> np.ndarray:
    """``kiteForCell``: the slot of cell i in cellsOnVertex[verticesOnCell[i][m]]."""
    voc = arrays["verticesOnCell"]
    cov = arrays["cellsOnVertex"]
    n_cells = voc.shape[0]
    out = np.full(voc.shape, -1, dtype=np.int64)
    valid = voc >= 0
    rows, cols = np.nonzero(valid)
    cand = cov[voc[rows, cols]]
    hit = cand == rows[:, None]
    if not np.all(hit.sum(axis=1) == 1):
        raise RuntimeError("cell missing from its vertex")
    out[rows, cols] = np.argmax(hit, axis=1)
    del n_cells
    return out


def _trisk(arrays: dict[str, Any]) -> None:
    """TRiSK ``edgesOnEdge`` / ``weightsOnEdge`` (Thuburn et al. 2009).

    For edge e and each of its cells i, the other edges of i are visited
    counter-clockwise starting after e; ``R`` accumulates the kite area of
    each vertex passed, as a fraction of the cell area, and the weight of the
    edge reached is ``s_i (1/2 - R) n_{e',i} dv(e')/dc(e)`` with ``s_i = +1``
    for cell1 and ``-1`` for cell2 and ``n_{e',i} = +1`` if i is cell1 of e'.
    """
    coe = arrays["cellsOnEdge"]
    eoc = arrays["edgesOnCell"]
    voc = arrays["verticesOnCell"]
    deg = arrays["nEdgesOnCell"]
    kites = arrays["kiteAreasOnVertex"]
    area = arrays["areaCell"]
    dc = arrays["dcEdge"]
    dv = arrays["dvEdge"]
    kite_slot = _kite_slot(arrays)
    n_edges = coe.shape[0]
    eoe = np.full((n_edges, MAX_EDGES2), -1, dtype=np.int64)
    w = np.zeros((n_edges, MAX_EDGES2))
    count = np.zeros(n_edges, dtype=np.int64)
    edges = np.arange(n_edges)
    for side, sign in ((0, 1.0), (1, -1.0)):
        cell = coe[:, side]
        n = deg[cell]
        j = np.argmax(eoc[cell] == edges[:, None], axis=1)
        if not np.all(eoc[cell, j] == edges):
            raise RuntimeError("edge missing from its cell")
        r = np.zeros(n_edges)
        for step in range(1, MAX_EDGES):
            active = step < n
            e_idx = edges[active]
            jj = (j[active] + step) % n[active]
            prev = (j[active] + step - 1) % n[active]
            cl = cell[active]
            vertex = voc[cl, prev]      # vertex between the previous edge and this one
            r[active] += kites[vertex, kite_slot[cl, prev]] / area[cl]
            other = eoc[cl, jj]
            n_sign = np.where(coe[other, 0] == cl, 1.0, -1.0)
            slot = count[active]
            eoe[e_idx, slot] = other
            w[e_idx, slot] = sign * (0.5 - r[active]) * n_sign * dv[other] / dc[e_idx]
            count[active] += 1
    arrays["nEdgesOnEdge"] = count
    arrays["edgesOnEdge"] = eoe
    arrays["weightsOnEdge"] = w
