"""MPAS mesh files (netCDF classic and 64-bit offset) to and from
``hexdyn.mesh.VoronoiMesh``.

Reads the horizontal mesh of an MPAS grid or static file with the MPAS
variable names and conventions: 1-based connectivity with 0 marking an
unused slot (stored here 0-based with -1), the ``sphere_radius`` and
``on_a_sphere`` global attributes, Coriolis parameters from the file or
from 2 Omega sin(latitude) when a grid file has none, ``nominalMinDc`` from
the file or as the smallest ``dcEdge``.  The mesh can then be renumbered
(``hexdyn.reorder``), given a vertical grid and state (``hexdyn.case``) and
stepped.  The reader is SciPy's netCDF-3 reader: netCDF-4 (HDF5) and CDF-5
files are refused with a message saying so.
"""

from __future__ import annotations

from pathlib import Path
from typing import Any

import numpy as np

from .mesh import OMEGA, VoronoiMesh

# connectivity: variable -> (entity of the rows, dimension of the slots)
_INDEX = {
    "cellsOnEdge": ("nEdges", "TWO"), "verticesOnEdge": ("nEdges", "TWO"),
    "edgesOnCell": ("nCells", "maxEdges"), "verticesOnCell": ("nCells", "maxEdges"),
    "cellsOnCell": ("nCells", "maxEdges"), "edgesOnEdge": ("nEdges", "maxEdges2"),
    "cellsOnVertex": ("nVertices", "vertexDegree"), "edgesOnVertex": ("nVertices", "vertexDegree"),
}
_COUNTS = {"nEdgesOnCell": "nCells", "nEdgesOnEdge": "nEdges"}
_IDS = {"indexToCellID": "nCells", "indexToEdgeID": "nEdges", "indexToVertexID": "nVertices"}
_REAL = {
    "xCell": ("nCells",), "yCell": ("nCells",), "zCell": ("nCells",), "latCell": ("nCells",),
    "lonCell": ("nCells",), "areaCell": ("nCells",), "meshDensity": ("nCells",),
    "xEdge": ("nEdges",), "yEdge": ("nEdges",), "zEdge": ("nEdges",), "latEdge": ("nEdges",),
    "lonEdge": ("nEdges",), "dcEdge": ("nEdges",), "dvEdge": ("nEdges",), "angleEdge": ("nEdges",),
    "weightsOnEdge": ("nEdges", "maxEdges2"),
    "xVertex": ("nVertices",), "yVertex": ("nVertices",), "zVertex": ("nVertices",),
    "latVertex": ("nVertices",), "lonVertex": ("nVertices",), "areaTriangle": ("nVertices",),
    "kiteAreasOnVertex": ("nVertices", "vertexDegree"),
}
_CORIOLIS = {"fCell": "latCell", "fEdge": "latEdge", "fVertex": "latVertex"}


def _netcdf(path: str | Path, mode: str = "r", **kw):
    from scipy.io import netcdf_file

    try:
        return netcdf_file(str(path), mode, mmap=False, **kw)
    except TypeError as exc:  # SciPy's message for a file that is not netCDF-3
        raise ValueError(f"{path}: not a netCDF classic or 64-bit-offset file ({exc}); convert netCDF-4 "
                         "or CDF-5 files with `nccopy -k 2`") from exc


def read_mesh(path: str | Path) -> VoronoiMesh:
    """The horizontal mesh of an MPAS grid/static file."""
    f = _netcdf(path)
    try:
        v = f.variables
        missing = [k for k in (*_INDEX, *_COUNTS, *_REAL) if k not in v and k != "meshDensity"]
        if missing:
            raise ValueError(f"{path}: missing MPAS mesh variables {missing}")
        arrays: dict[str, Any] = {}
        for name in _INDEX:
            arrays[name] = np.asarray(v[name][:], dtype=np.int64) - 1  # 0 (unused) -> -1
        for name in _COUNTS:
            arrays[name] = np.asarray(v[name][:], dtype=np.int64)
        for name in _IDS:
            if name in v:
                arrays[name] = np.asarray(v[name][:], dtype=np.int64)
        for name in _REAL:
            if name in v:
                arrays[name] = np.asarray(v[name][:], dtype=np.float64)
        n_cells = arrays["areaCell"].size
        arrays.setdefault("meshDensity", np.ones(n_cells))
        for fname, lat in _CORIOLIS.items():
            arrays[fname] = (np.asarray(v[fname][:], dtype=np.float64) if fname in v
                             else 2.0 * OMEGA * np.sin(arrays[lat]))
        attrs = f._attributes
        radius = float(attrs.get("sphere_radius", 6371229.0))
        sphere = attrs.get("on_a_sphere", b"YES")
        sphere = sphere.decode() if isinstance(sphere, bytes) else str(sphere)
        if sphere.strip().upper() != "YES":
            raise ValueError(f"{path}: only spherical meshes (on_a_sphere = YES) are supported")
        arrays["sphere_radius"] = radius
        arrays["on_a_sphere"] = True
        arrays["nominalMinDc"] = np.array(float(np.asarray(v["nominalMinDc"].data).reshape(-1)[0])
                                          if "nominalMinDc" in v else float(np.min(arrays["dcEdge"])))
    finally:
        f.close()
    arrays["nCells"] = n_cells
    arrays["nEdges"] = arrays["dcEdge"].size
    arrays["nVertices"] = arrays["areaTriangle"].size
    # edge normal and tangent unit vectors from angleEdge (the angle of the
    # normal from local east) at the edge's latitude and longitude
    lat, lon, ang = arrays["latEdge"], arrays["lonEdge"], arrays["angleEdge"]
    east = np.stack([-np.sin(lon), np.cos(lon), np.zeros_like(lon)], axis=1)
    north = np.stack([-np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)], axis=1)
    normal = np.cos(ang)[:, None] * east + np.sin(ang)[:, None] * north
    x_edge = np.stack([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)], axis=1)
    arrays["_edge_normal"] = normal
    arrays["_edge_tangent"] = np.cross(x_edge, normal)
    return VoronoiMesh(arrays=arrays)


def write_mesh(mesh: VoronoiMesh, path: str | Path) -> None:
    """Write the MPAS mesh variables of ``mesh`` (64-bit offset netCDF)."""
    a = mesh.arrays
    f = _netcdf(path, "w", version=2)
    try:
        dims = {"nCells": mesh.n_cells, "nEdges": mesh.n_edges, "nVertices": mesh.n_vertices,
                "maxEdges": a["edgesOnCell"].shape[1], "maxEdges2": a["edgesOnEdge"].shape[1],
                "vertexDegree": a["cellsOnVertex"].shape[1], "TWO": 2}
        for name, size in dims.items():
            f.createDimension(name, size)
        for name, shape in _INDEX.items():
            var = f.createVariable(name, "i", shape)
            var[:] = (np.asarray(a[name], dtype=np.int64) + 1).astype(np.int32)
        for name, dim in {**_COUNTS, **_IDS}.items():
            if name in a:
                var = f.createVariable(name, "i", (dim,))
                var[:] = np.asarray(a[name], dtype=np.int32)
        for name, shape in _REAL.items():
            var = f.createVariable(name, "d", shape)
            var[:] = np.asarray(a[name], dtype=np.float64)
        for fname in _CORIOLIS:
            dim = {"fCell": "nCells", "fEdge": "nEdges", "fVertex": "nVertices"}[fname]
            var = f.createVariable(fname, "d", (dim,))
            var[:] = np.asarray(a[fname], dtype=np.float64)
        var = f.createVariable("nominalMinDc", "d", ())
        var.data[()] = float(np.asarray(a["nominalMinDc"]))
        f.sphere_radius = float(a["sphere_radius"])
        f.on_a_sphere = "YES"
    finally:
        f.close()
