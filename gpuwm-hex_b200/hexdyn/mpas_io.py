"""MPAS mesh, init and restart files (netCDF classic and 64-bit offset).

Meshes to and from ``hexdyn.mesh.VoronoiMesh`` (``read_mesh``,
``write_mesh``); the native vertical grid, slope metrics, prognostic state,
base state and saved diagnostics of an init or restart file
(``read_vertical_grid``, ``read_initial_state``, ``read_restart``) as the
reference's loaders form them, and restart files of a case or of a
driver's state (``write_restart``).

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
    f = _netcdf(path, "w", version=2)
    try:
        _write_mesh_vars(f, mesh)
    finally:
        f.close()


def _write_mesh_vars(f, mesh: VoronoiMesh) -> None:
    a = mesh.arrays
    if True:  # noqa: SIM108 - one indentation level with the old body
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


# ------------------------------------------------------------ init / restart
# Vertical grid, initial state, base state and saved diagnostics of an MPAS
# init or restart file, read the way the reference's loaders read them:
# ``load_mpas_vertical_grid`` (hexcore/driver.py:1419) and
# ``load_mpas_initial_state`` (hexcore/driver.py:1582).  Fields are read in
# the logical [level][entity] layout whatever the file's dimension order.

RVORD_RGAS, RVORD_RV = 287.0, 461.6  # rvord = rv / rgas, an FP32 division


class MpasRefusal(ValueError):
    """A field the requested read needs is absent or inconsistent; ``field``
    names it."""

    def __init__(self, field: str, reason: str):
        self.field = field
        super().__init__(f"{field}: {reason}")


def _var(f, name: str):
    if name not in f.variables:
        raise MpasRefusal(name, "absent from the file")
    return f.variables[name]


def _native(a) -> np.ndarray:
    """A file array in native byte order (the file stores big-endian words)."""
    a = np.asarray(a)
    return a.astype(a.dtype.newbyteorder("="), copy=True)


def _logical(var, level_dim: str, entity_dim: str, time_index: int = 0) -> np.ndarray:
    """``var`` as a C-contiguous (level, entity) array, the Time axis taken at
    ``time_index`` (hexcore/driver.py:1275 ``_logical_netcdf_field``)."""
    dims = list(var.dimensions)
    data = _native(var.data)
    if "Time" in dims:
        data = np.take(data, time_index, axis=dims.index("Time"))
        dims.remove("Time")
    if sorted(dims) != sorted([level_dim, entity_dim]):
        raise MpasRefusal(getattr(var, "name", "?"), f"dimensions {var.dimensions} are not ({level_dim}, "
                          f"{entity_dim})")
    return np.ascontiguousarray(np.transpose(data, (dims.index(level_dim), dims.index(entity_dim))))


def _vector(var) -> np.ndarray:
    return _native(var.data).reshape(-1)


def _scalar_value(var) -> float:
    return float(np.asarray(var.data).reshape(-1)[0])


def terrain_cells(mesh: VoronoiMesh, zb: np.ndarray, zb3: np.ndarray, coef_3rd_order: float):
    """Cell-oriented slope metrics from the file's edge-sided ``zb``/``zb3``
    (native layout [nEdges][2][nVertLevelsP1]): for each active slot s of
    cell c, edge e = edgesOnCell[c][s] on side 0 when c is cellsOnEdge[e][0],
    else side 1; ``zb3`` is scaled by ``config_coef_3rd_order`` once, in the
    field's precision (hexcore/terrain.py:182 build_terrain_coupling and its
    host preparation, hexcore/rust_hostprep.py:189)."""
    eoc = np.asarray(mesh.arrays["edgesOnCell"], dtype=np.int64)
    coe = np.asarray(mesh.arrays["cellsOnEdge"], dtype=np.int64)
    counts = np.asarray(mesh.arrays["nEdgesOnCell"], dtype=np.int64)
    ne = coe.shape[0]
    if zb.shape[:2] != (ne, 2) or zb3.shape != zb.shape:
        raise MpasRefusal("zb", f"shape {zb.shape} is not (nEdges={ne}, 2, nVertLevelsP1)")
    nc, me = eoc.shape
    nl = zb.shape[2]
    active = np.arange(me)[None, :] < counts[:, None]
    safe = np.where(active, eoc, 0)
    cell = np.arange(nc)[:, None]
    first = coe[safe, 0] == cell
    if np.any(active & ~first & (coe[safe, 1] != cell)):
        raise MpasRefusal("cellsOnEdge", "a cell's edge does not list the cell")
    side = np.where(first, 0, 1)
    coef = zb.dtype.type(coef_3rd_order)
    zb_cell = np.zeros((nl, nc, me), dtype=zb.dtype)
    zb3_cell = np.zeros((nl, nc, me), dtype=zb.dtype)
    for s in range(me):
        on = np.flatnonzero(active[:, s])
        zb_cell[:, on, s] = zb[safe[on, s], side[on, s], :].T
        zb3_cell[:, on, s] = (coef * zb3[safe[on, s], side[on, s], :]).T
    return zb_cell, zb3_cell


def read_vertical_grid(path: str | Path, mesh: VoronoiMesh, *, coef_3rd_order: float = 0.25,
                       invariant_path: str | Path | None = None):
    """The native vertical metric set of an init file (and of the invariant
    stream, whose fields win where it has them): ``(VerticalGridData,
    zb_cell, zb3_cell)``.  The derived level arrays follow
    ``load_mpas_vertical_grid`` (hexcore/driver.py:1419): ``dzw = 1/rdzw``,
    ``zw`` the running sum of ``dzw`` from 0, ``zu`` the mid-points, and the
    ``rdzwp/rdzwm`` weights of the level spacing."""
    from .case import VerticalGridData

    files = [_netcdf(path)]
    try:
        if invariant_path is not None:
            files.insert(0, _netcdf(invariant_path))

        def get(name):
            for f in files:
                if name in f.variables:
                    return f.variables[name]
            raise MpasRefusal(name, "the native vertical grid is incomplete")

        zgrid = _logical(get("zgrid"), "nVertLevelsP1", "nCells")
        dt = zgrid.dtype
        zz = _logical(get("zz"), "nVertLevels", "nCells").astype(dt, copy=False)
        zxu = _logical(get("zxu"), "nVertLevels", "nEdges").astype(dt, copy=False)
        dss = _logical(get("dss"), "nVertLevels", "nCells").astype(dt, copy=False)
        rdzw, dzu, rdzu, fzm, fzp = (_vector(get(k)).astype(dt, copy=False)
                                     for k in ("rdzw", "dzu", "rdzu", "fzm", "fzp"))
        zb = _native(get("zb").data).astype(dt, copy=False)
        zb3 = _native(get("zb3").data).astype(dt, copy=False)
        cf1, cf2, cf3 = (_scalar_value(get(k)) for k in ("cf1", "cf2", "cf3"))
    finally:
        for f in files:
            f.close()
    nlev, ncells = zz.shape
    if rdzw.shape != (nlev,) or zgrid.shape != (nlev + 1, ncells):
        raise MpasRefusal("rdzw", "vertical dimensions disagree")
    dzw = np.reciprocal(rdzw)
    zw = np.empty(nlev + 1, dtype=dt)
    zw[0] = 0.0
    zw[1:] = np.cumsum(dzw, dtype=dt)
    zu = (zw[:-1] + zw[1:]) * dt.type(0.5)
    rdzwp = np.zeros(nlev, dtype=dt)
    rdzwm = np.zeros(nlev, dtype=dt)
    rdzwp[1:] = dzw[:-1] / (dzw[1:] * (dzw[1:] + dzw[:-1]))
    rdzwm[1:] = dzw[1:] / (dzw[:-1] * (dzw[1:] + dzw[:-1]))
    vertical = VerticalGridData(zw=zw, dzw=dzw, rdzw=rdzw, zu=zu, dzu=dzu, rdzu=rdzu, rdzwp=rdzwp, rdzwm=rdzwm,
                                fzp=fzp, fzm=fzm, ah=np.zeros(nlev + 1, dtype=dt), hx=np.zeros_like(zgrid),
                                zgrid=zgrid, zz=zz, zxu=zxu, dss=dss, cf1=cf1, cf2=cf2, cf3=cf3,
                                first_height_level=nlev + 1)
    zb_cell, zb3_cell = terrain_cells(mesh, zb, zb3, coef_3rd_order)
    return vertical, zb_cell, zb3_cell


def read_initial_state(path: str | Path, mesh: VoronoiMesh, vertical, *, scalar_names: tuple[str, ...] = (),
                       reference_path: str | Path | None = None, terrain=None, time_index: int = 0,
                       normal_velocity_name: str = "u"):
    """Prognostic state, base state and (when the file carries them) saved
    diagnostics of an init or restart file, as ``load_mpas_initial_state``
    (hexcore/driver.py:1582, its default non-cold-start reading) forms them:

    * ``rho_zz`` (else public ``rho / zz``), ``theta_m`` (else public
      ``theta * (1 + rvord qv)``, rvord = 461.6/287 in FP32);
    * ``ru`` (else ``(0.5 u) (rho(cell1) + rho(cell2))``), ``rw`` (else
      ``w`` times the interpolated ``rho_zz`` and ``zz``, zero at both ends,
      then the terrain correction of every active slot in slot order,
      hexcore/rust_hostprep.py:265);
    * ``rho_theta = rtheta_p + rtheta_base`` with ``rtheta_p`` from the file
      or ``theta_m (rho - rho_base) + rho_base (theta_m - theta_base)``;
    * ``rho_base``, ``rtheta_base`` (else ``rho_base theta_base``),
      ``exner_base`` and ``pressure_base`` from the reference file (default:
      the same file);
    * the saved diagnostics when ``exner``, ``rtheta_p``, ``rho_p``,
      ``pressure_p``, the normal velocity and ``w`` are all present; else
      None (the driver rebuilds them on the device from the state,
      hexcore/driver.py:2655).

    Returns ``(HostState, ReferenceStateData, HostSidecar | None)``.
    """
    from .driver import HostSidecar, HostState

    f = _netcdf(path)
    try:
        v = f.variables
        if "rho_zz" in v:
            rho = _logical(v["rho_zz"], "nVertLevels", "nCells", time_index)
        elif "rho" in v:
            rho = _logical(v["rho"], "nVertLevels", "nCells", time_index) / np.asarray(vertical.zz)
        else:
            raise MpasRefusal("rho_zz", "neither rho_zz nor public rho is present")
        dt = rho.dtype
        if "theta_m" in v:
            theta_m = _logical(v["theta_m"], "nVertLevels", "nCells", time_index).astype(dt, copy=False)
        elif "theta" in v:
            theta = _logical(v["theta"], "nVertLevels", "nCells", time_index).astype(dt, copy=False)
            qv = _logical(_var(f, "qv"), "nVertLevels", "nCells", time_index).astype(dt, copy=False)
            rvord = dt.type(RVORD_RV) / dt.type(RVORD_RGAS)
            theta_m = theta * (dt.type(1.0) + rvord * qv)
        else:
            raise MpasRefusal("theta_m", "neither theta_m nor public theta is present")

        def opt(name, lev="nVertLevels", ent="nCells"):
            return _logical(v[name], lev, ent, time_index).astype(dt, copy=False) if name in v else None

        exner, rtheta_p, rho_p, pressure_p = opt("exner"), opt("rtheta_p"), opt("rho_p"), opt("pressure_p")
        u = opt(normal_velocity_name, ent="nEdges")
        w = opt("w", lev="nVertLevelsP1")
        coe = np.asarray(mesh.arrays["cellsOnEdge"], dtype=np.int64)
        if np.any(coe < 0):
            raise MpasRefusal("cellsOnEdge", "a boundary edge in a closed-mesh state")
        if "ru" in v:
            rho_u = _logical(v["ru"], "nVertLevels", "nEdges", time_index).astype(dt, copy=False)
        elif u is not None:
            rho_u = (dt.type(0.5) * u) * (rho[:, coe[:, 0]] + rho[:, coe[:, 1]])
        else:
            raise MpasRefusal(normal_velocity_name, "neither the normal velocity nor ru is present")
        if "rw" in v:
            rho_w = _logical(v["rw"], "nVertLevelsP1", "nCells", time_index).astype(dt, copy=False)
        elif w is not None:
            rho_w = _public_rw(mesh, vertical, rho, rho_u, w, terrain)
        else:
            raise MpasRefusal("w", "neither w nor rw is present")
        scalars = [(_logical(_var(f, name), "nVertLevels", "nCells", time_index).astype(dt, copy=False))
                   for name in scalar_names]
        scalars = np.stack(scalars) if scalars else np.empty((0, *rho.shape), dtype=dt)
        time_seconds = 0.0
        if "Time" in v and np.asarray(v["Time"].data).size > time_index:
            t = float(np.asarray(v["Time"].data).reshape(-1)[time_index])
            time_seconds = t if np.isfinite(t) else 0.0
    finally:
        f.close()
    rf = _netcdf(reference_path if reference_path is not None else path)
    try:
        rv = rf.variables
        rho_base = _logical(_var(rf, "rho_base"), "nVertLevels", "nCells", time_index).astype(dt, copy=False)
        theta_base = (_logical(rv["theta_base"], "nVertLevels", "nCells", time_index).astype(dt, copy=False)
                      if "theta_base" in rv else None)
        if "rtheta_base" in rv:
            rtheta_base = _logical(rv["rtheta_base"], "nVertLevels", "nCells", time_index).astype(dt, copy=False)
        elif theta_base is not None:
            rtheta_base = rho_base * theta_base
        else:
            raise MpasRefusal("theta_base", "rtheta_base needs rtheta_base or theta_base")
        if theta_base is None:
            theta_base = rtheta_base / rho_base
        # the exact base Exner and pressure: deriving them needs the C
        # library's powf order, so the file must carry them
        exner_base = _logical(_var(rf, "exner_base"), "nVertLevels", "nCells", time_index).astype(dt, copy=False)
        pressure_base = _logical(_var(rf, "pressure_base"), "nVertLevels", "nCells",
                                 time_index).astype(dt, copy=False)
    finally:
        rf.close()
    # perturbation order of the native reader (F:5937-5947)
    rho_perturbation = rho - rho_base if rho_p is None else rho_p
    rtp = (theta_m * rho_perturbation + rho_base * (theta_m - theta_base)) if rtheta_p is None else rtheta_p
    rho_theta = rtp + rtheta_base
    state = HostState(rho=rho, rho_theta=rho_theta, rho_u=rho_u, rho_w=rho_w, scalars=scalars,
                      time_seconds=time_seconds)
    reference = ReferenceStateData(rho_base=rho_base, rho_theta_base=rtheta_base, pressure_base=pressure_base,
                                   exner_base=exner_base)
    sidecar = None
    if all(x is not None for x in (exner, rtheta_p, rho_p, pressure_p, u, w)):
        sidecar = HostSidecar(theta_m=theta_m, exner=exner, density_perturbation=rho_perturbation,
                              rho_theta_perturbation=rtp, pressure_perturbation=pressure_p,
                              normal_velocity=u, vertical_velocity=w)
    return state, reference, sidecar


def _public_rw(mesh: VoronoiMesh, vertical, rho, rho_u, w, terrain) -> np.ndarray:
    """rw from public w (atm_init_coupled_diagnostics): w times the
    interpolated rho_zz and zz, +0 at both ends, then, when the slope
    metrics are given, each active slot's terrain correction in slot order
    (hexcore/driver.py:1780-1850, hexcore/rust_hostprep.py:265)."""
    dt = rho.dtype
    nl = rho.shape[0]
    fzm, fzp = np.asarray(vertical.fzm, dtype=dt), np.asarray(vertical.fzp, dtype=dt)
    zz = np.asarray(vertical.zz, dtype=dt)
    idens = np.zeros_like(w)
    izz = np.zeros_like(w)
    for k in range(1, nl):
        idens[k] = fzm[k] * rho[k] + fzp[k] * rho[k - 1]
        izz[k] = fzm[k] * zz[k] + fzp[k] * zz[k - 1]
    rw = w * idens * izz
    rw[0] = dt.type(0.0)
    rw[-1] = dt.type(0.0)
    if terrain is None and np.max(np.abs(np.asarray(vertical.zxu)), initial=0.0) > 2.0e-14:
        raise MpasRefusal("zb", "public w to rw on a grid with terrain needs zb/zb3 (read_vertical_grid)")
    if terrain is not None:
        zb_cell, zb3_cell = terrain
        eoc = np.asarray(mesh.arrays["edgesOnCell"], dtype=np.int64)
        coe = np.asarray(mesh.arrays["cellsOnEdge"], dtype=np.int64)
        counts = np.asarray(mesh.arrays["nEdgesOnCell"], dtype=np.int64)
        nc, me = eoc.shape
        active = np.arange(me)[None, :] < counts[:, None]
        safe = np.where(active, eoc, 0)
        signs = np.where(coe[safe, 0] == np.arange(nc)[:, None], dt.type(1.0), dt.type(-1.0))
        one = dt.type(1.0)
        value = rw[1:nl].copy()
        with np.errstate(all="ignore"):
            for s in range(me):
                on = active[:, s]
                edge = safe[:, s]
                flux = fzm[1:nl, None] * rho_u[1:nl, edge] + fzp[1:nl, None] * rho_u[0:nl - 1, edge]
                slope = zb_cell[1:nl, :, s] + np.copysign(one, flux) * zb3_cell[1:nl, :, s]
                correction = signs[:, s][None, :] * slope * flux * izz[1:nl]
                value = np.where(on[None, :], value - correction, value)
        rw[1:nl] = value
    return rw


class ReferenceStateData:
    """The base state under the reference's ``DryReferenceState`` names."""

    def __init__(self, rho_base, rho_theta_base, pressure_base, exner_base):
        self.rho_base, self.rho_theta_base = rho_base, rho_theta_base
        self.pressure_base, self.exner_base = pressure_base, exner_base


def edge_sided(mesh: VoronoiMesh, zb_cell: np.ndarray, zb3_cell: np.ndarray, coef_3rd_order: float):
    """The inverse of ``terrain_cells``: edge-sided ``zb``/``zb3`` in the
    native layout [nEdges][2][nVertLevelsP1] from the cell-oriented metrics.
    ``zb3`` is divided by ``config_coef_3rd_order``, which must be a power of
    two so that the read-back product is the same word."""
    c = float(coef_3rd_order)
    if c <= 0.0 or np.frexp(c)[0] != 0.5:
        raise MpasRefusal("config_coef_3rd_order", f"{c} is not a power of two; zb3 would not round-trip")
    eoc = np.asarray(mesh.arrays["edgesOnCell"], dtype=np.int64)
    coe = np.asarray(mesh.arrays["cellsOnEdge"], dtype=np.int64)
    counts = np.asarray(mesh.arrays["nEdgesOnCell"], dtype=np.int64)
    nl, nc, me = zb_cell.shape
    zb = np.zeros((coe.shape[0], 2, nl), dtype=zb_cell.dtype)
    zb3 = np.zeros_like(zb)
    for s in range(me):
        on = np.flatnonzero(counts > s)
        e = eoc[on, s]
        side = np.where(coe[e, 0] == on, 0, 1)
        zb[e, side, :] = zb_cell[:, on, s].T
        zb3[e, side, :] = (zb3_cell[:, on, s] / zb_cell.dtype.type(c)).T
    return zb, zb3


def write_restart(path: str | Path, case: Any, sidecar: Any = None, *, state: Any = None,
                  time_seconds: float | None = None) -> None:
    """Write a restart-style MPAS file (64-bit offset netCDF) of a case: the
    mesh, the native vertical grid and slope metrics, the base state, the
    prognostic state under its native names (``rho_zz``, ``theta_m``, ``ru``,
    ``rw``, each scalar by name), the reference wind profiles, the advection
    tables and, when ``sidecar`` is given (a ``HostSidecar``, e.g. from
    ``HexDycoreDriver.get_state``), the saved diagnostics (``exner``,
    ``rtheta_p``, ``rho_p``, ``pressure_p``, ``u``, ``w``).  ``case`` has the
    attributes of ``hexdyn.case.DycoreCase``; ``state`` (e.g. the first value
    of ``HexDycoreDriver.get_state()``), when given, replaces the case's
    prognostic fields and time.  ``read_restart`` reads the file back into a
    case."""
    mesh, vg = case.mesh, case.vertical
    src = case if state is None else state
    if time_seconds is None:
        time_seconds = float(getattr(src, "time_seconds", 0.0))
    L = int(np.asarray(vg.zz).shape[0])
    f = _netcdf(path, "w", version=2)
    try:
        f.createDimension("Time", None)  # the record dimension, first as netCDF-3 requires
        _write_mesh_vars(f, mesh)
        f.createDimension("nVertLevels", L)
        f.createDimension("nVertLevelsP1", L + 1)
        adv_w = int(np.asarray(case.adv_cells_for_edge).shape[1])
        f.createDimension("nAdvCellsMax", adv_w)

        def put(name, dims, value, typ="f"):
            var = f.createVariable(name, typ, dims)
            if dims:
                var[:] = value
            else:
                var.data[()] = value

        def field(name, value, lev="nVertLevels", ent="nCells"):
            put(name, ("Time", ent, lev), np.asarray(value, dtype=np.float32).T[None])

        put("Time", ("Time",), np.array([time_seconds]), "d")
        put("zgrid", ("nCells", "nVertLevelsP1"), np.asarray(vg.zgrid, dtype=np.float32).T)
        put("zz", ("nCells", "nVertLevels"), np.asarray(vg.zz, dtype=np.float32).T)
        put("zxu", ("nEdges", "nVertLevels"), np.asarray(vg.zxu, dtype=np.float32).T)
        put("dss", ("nCells", "nVertLevels"), np.asarray(vg.dss, dtype=np.float32).T)
        for k in ("rdzw", "dzu", "rdzu", "fzm", "fzp"):
            put(k, ("nVertLevels",), np.asarray(getattr(vg, k), dtype=np.float32))
        for k in ("cf1", "cf2", "cf3"):
            put(k, (), np.float32(getattr(vg, k)))
        zb, zb3 = edge_sided(mesh, np.asarray(case.zb_cell, dtype=np.float32),
                             np.asarray(case.zb3_cell, dtype=np.float32), getattr(case, "coef_3rd_order", 0.25))
        put("zb", ("nEdges", "TWO", "nVertLevelsP1"), zb)
        put("zb3", ("nEdges", "TWO", "nVertLevelsP1"), zb3)
        field("rho_base", case.rho_base)
        field("rtheta_base", case.rho_theta_base)
        field("theta_base", np.asarray(case.rho_theta_base, np.float32) / np.asarray(case.rho_base, np.float32))
        field("exner_base", case.exner_base)
        field("pressure_base", case.pressure_base)
        field("rho_zz", src.rho)
        field("ru", src.rho_u, ent="nEdges")
        field("rw", src.rho_w, lev="nVertLevelsP1")
        names = tuple(getattr(case, "scalar_names", ())) or tuple(f"scalar{i}" for i in range(len(src.scalars)))
        for name, q in zip(names, np.asarray(src.scalars)):
            field(name, q)
        if sidecar is not None:
            field("theta_m", sidecar.theta_m)
            field("exner", sidecar.exner)
            field("rtheta_p", sidecar.rho_theta_perturbation)
            field("rho_p", sidecar.density_perturbation)
            field("pressure_p", sidecar.pressure_perturbation)
            field("u", sidecar.normal_velocity, ent="nEdges")
            field("w", sidecar.vertical_velocity, lev="nVertLevelsP1")
        else:
            rho = np.asarray(src.rho, dtype=np.float32)
            field("theta_m", np.asarray(src.rho_theta, np.float32) / rho)
        put("u_init", ("nVertLevels",), np.asarray(case.u_init, dtype=np.float32))
        put("v_init", ("nVertLevels",), np.asarray(case.v_init, dtype=np.float32))
        put("nAdvCellsForEdge", ("nEdges",), np.asarray(case.n_adv_cells_for_edge, dtype=np.int32), "i")
        put("advCellsForEdge", ("nEdges", "nAdvCellsMax"),
            (np.asarray(case.adv_cells_for_edge, dtype=np.int64) + 1).astype(np.int32), "i")
        put("adv_coefs", ("nEdges", "nAdvCellsMax"), np.asarray(case.adv_coefs, dtype=np.float64), "d")
        put("adv_coefs_3rd", ("nEdges", "nAdvCellsMax"), np.asarray(case.adv_coefs_3rd, dtype=np.float64), "d")
        f.scalar_names = " ".join(names)
        f.config_coef_3rd_order = float(getattr(case, "coef_3rd_order", 0.25))
    finally:
        f.close()


def read_restart(path: str | Path, *, scalar_names: tuple[str, ...] | None = None, grid_path: str | Path | None = None,
                 coef_3rd_order: float | None = None, time_index: int = 0):
    """An MPAS init or restart file as a case for ``hexdyn.from_case`` (the
    attributes of ``hexdyn.case.DycoreCase``) and its saved diagnostics
    (``HostSidecar`` or None; pass it as ``saved_diagnostics`` to
    ``HexDycoreDriver.from_host``).  The mesh comes from ``grid_path`` or the
    file itself; the vertical grid, slope metrics, state and base state are
    read by ``read_vertical_grid`` and ``read_initial_state``; the advection
    tables are read when the file has them (``nAdvCellsForEdge``,
    ``advCellsForEdge``, ``adv_coefs``, ``adv_coefs_3rd``) and otherwise
    formed from the mesh (``hexdyn.case.deriv_two`` and
    ``advection_stencil``); ``u_init``/``v_init`` default to zero."""
    from types import SimpleNamespace

    from . import case as casemod

    mesh = read_mesh(grid_path if grid_path is not None else path)
    f = _netcdf(path)
    try:
        attrs = f._attributes
        if scalar_names is None:
            raw = attrs.get("scalar_names", b"")
            raw = raw.decode() if isinstance(raw, bytes) else str(raw)
            scalar_names = tuple(raw.split()) if raw else tuple(
                n for n in ("qv", "qc", "qr", "qi", "qs", "qg") if n in f.variables)
        if coef_3rd_order is None:
            coef_3rd_order = float(attrs.get("config_coef_3rd_order", 0.25))
        v = f.variables
        L = int(f.dimensions["nVertLevels"])
        winds = {k: (_vector(v[k]).astype(np.float32) if k in v else np.zeros(L, dtype=np.float32))
                 for k in ("u_init", "v_init")}
        adv = None
        if all(k in v for k in ("nAdvCellsForEdge", "advCellsForEdge", "adv_coefs", "adv_coefs_3rd")):
            adv = (_native(v["adv_coefs"].data).astype(np.float64), _native(v["adv_coefs_3rd"].data).astype(np.float64),
                   _native(v["nAdvCellsForEdge"].data).astype(np.int64),
                   _native(v["advCellsForEdge"].data).astype(np.int64) - 1)
    finally:
        f.close()
    vertical, zb_cell, zb3_cell = read_vertical_grid(path, mesh, coef_3rd_order=coef_3rd_order)
    state, ref, sidecar = read_initial_state(path, mesh, vertical, scalar_names=scalar_names,
                                             terrain=(zb_cell, zb3_cell), time_index=time_index)
    if adv is None:
        d2 = casemod.deriv_two(mesh)
        adv = casemod.advection_stencil(mesh, d2)
    case = SimpleNamespace(mesh=mesh, vertical=vertical, zb_cell=zb_cell, zb3_cell=zb3_cell,
                           rho_base=ref.rho_base, rho_theta_base=ref.rho_theta_base,
                           pressure_base=ref.pressure_base, exner_base=ref.exner_base,
                           rho=state.rho, rho_theta=state.rho_theta, rho_u=state.rho_u, rho_w=state.rho_w,
                           scalars=state.scalars, scalar_names=tuple(scalar_names), adv_coefs=adv[0],
                           adv_coefs_3rd=adv[1], n_adv_cells_for_edge=adv[2], adv_cells_for_edge=adv[3],
                           u_init=winds["u_init"], v_init=winds["v_init"], coef_3rd_order=coef_3rd_order,
                           time_seconds=state.time_seconds)
    return case, sidecar
