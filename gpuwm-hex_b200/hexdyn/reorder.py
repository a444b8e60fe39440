"""Reversible renumbering of the cells, edges and vertices of a case.

A permutation of every entity-indexed array, as the reference's offline
tool does for MPAS files (``tree/tools/hex_order/hex_order.rs:1-16``): row
``i`` of a cell array in the renumbered case is row ``perm_c[i]`` of the
original, and every connectivity value (cellsOnEdge, edgesOnCell, the
advection stencil ...) is mapped to the new numbering.  The order of a
row's neighbour slots is kept, so every per-entity sum runs over the same
operands in the same order and a step of the renumbered case equals, after
the inverse permutation, the step of the original bit for bit.

``hilbert_order`` numbers cells along a 3-D Hilbert curve of their
positions, edges by their new (cell1, cell2) pair and vertices by their
sorted new cell triple, which keeps the neighbours of an entity close in
memory (the stencil gathers then hit L1/L2); ``random_order`` scrambles the
numbering (a test of the permutation, and the worst case for locality).

Arrays are handled in the flat layout of ``hexdyn.case.case_arrays``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np

# mesh arrays by the entity their rows belong to, and the entity their
# values index (None: plain data)
_MESH_ROWS = {
    "cell": {"areaCell": None, "cellsOnCell": "cell", "edgesOnCell": "edge", "verticesOnCell": "vertex",
             "fCell": None, "indexToCellID": None, "latCell": None, "lonCell": None, "meshDensity": None,
             "nEdgesOnCell": None, "xCell": None, "yCell": None, "zCell": None},
    "edge": {"_edge_normal": None, "_edge_tangent": None, "angleEdge": None, "cellsOnEdge": "cell",
             "dcEdge": None, "dvEdge": None, "edgesOnEdge": "edge", "fEdge": None, "latEdge": None,
             "lonEdge": None, "nEdgesOnEdge": None, "verticesOnEdge": "vertex", "weightsOnEdge": None,
             "xEdge": None, "yEdge": None, "zEdge": None, "indexToEdgeID": None},
    "vertex": {"areaTriangle": None, "cellsOnVertex": "cell", "edgesOnVertex": "edge", "fVertex": None,
               "kiteAreasOnVertex": None, "latVertex": None, "lonVertex": None, "xVertex": None,
               "yVertex": None, "zVertex": None, "indexToVertexID": None},
}
# other case arrays: (entity, axis of the entity, entity the values index)
_CASE = {
    "vertical.hx": ("cell", 1, None), "vertical.zgrid": ("cell", 1, None), "vertical.zz": ("cell", 1, None),
    "vertical.zxu": ("edge", 1, None), "vertical.dss": ("cell", 1, None),
    "zb_cell": ("cell", 1, None), "zb3_cell": ("cell", 1, None),
    "rho_base": ("cell", 1, None), "rho_theta_base": ("cell", 1, None), "pressure_base": ("cell", 1, None),
    "exner_base": ("cell", 1, None), "rho": ("cell", 1, None), "rho_theta": ("cell", 1, None),
    "rho_u": ("edge", 1, None), "rho_w": ("cell", 1, None), "scalars": ("cell", 2, None),
    "adv_coefs": ("edge", 0, None), "adv_coefs_3rd": ("edge", 0, None), "n_adv_cells_for_edge": ("edge", 0, None),
    "adv_cells_for_edge": ("edge", 0, "cell"),
}
# level-only or scalar arrays pass through unchanged
_PASS = ("vertical.zw", "vertical.dzw", "vertical.rdzw", "vertical.zu", "vertical.dzu", "vertical.rdzu",
         "vertical.rdzwp", "vertical.rdzwm", "vertical.fzp", "vertical.fzm", "vertical.ah", "vertical.cf1",
         "vertical.cf2", "vertical.cf3", "vertical.first_height_level", "u_init", "v_init", "coef_3rd_order",
         "scalar_names")


@dataclass(frozen=True)
class Renumbering:
    """``perm[new] = old`` for cells, edges and vertices."""

    cell: np.ndarray
    edge: np.ndarray
    vertex: np.ndarray

    def inverse(self) -> "Renumbering":
        return Renumbering(_inverse(self.cell), _inverse(self.edge), _inverse(self.vertex))

    def of(self, entity: str) -> np.ndarray:
        return {"cell": self.cell, "edge": self.edge, "vertex": self.vertex}[entity]


def _inverse(perm: np.ndarray) -> np.ndarray:
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size, dtype=perm.dtype)
    return inv


def _check(perm: np.ndarray, n: int, what: str) -> np.ndarray:
    perm = np.asarray(perm, dtype=np.int64)
    if perm.shape != (n,) or not np.array_equal(np.sort(perm), np.arange(n)):
        raise ValueError(f"the {what} permutation is not a permutation of 0..{n - 1}")
    return perm


def _remap(values: np.ndarray, new_of_old: np.ndarray) -> np.ndarray:
    """Map index values (negative: unused slot, kept) to the new numbering."""
    v = np.asarray(values)
    out = v.copy()
    used = v >= 0
    out[used] = new_of_old[v[used]]
    return out


def _sizes(arr: dict[str, Any]) -> dict[str, int]:
    return {"cell": int(np.asarray(arr["mesh.areaCell"]).size), "edge": int(np.asarray(arr["mesh.dcEdge"]).size),
            "vertex": int(np.asarray(arr["mesh.areaTriangle"]).size)}


def apply(arr: dict[str, Any], ren: Renumbering) -> dict[str, Any]:
    """The case arrays of ``arr`` renumbered by ``ren``; unknown entity-sized
    arrays are refused rather than passed through unpermuted."""
    n = _sizes(arr)
    perm = {e: _check(ren.of(e), n[e], e) for e in n}
    new_of_old = {e: _inverse(p) for e, p in perm.items()}
    out: dict[str, Any] = {}
    for key, value in arr.items():
        if key.startswith("mesh."):
            name = key[5:]
            for entity, table in _MESH_ROWS.items():
                if name in table:
                    a = np.asarray(value)[perm[entity]]
                    target = table[name]
                    out[key] = _remap(a, new_of_old[target]) if target else a
                    break
            else:
                a = np.asarray(value)
                if a.ndim > 0:
                    raise ValueError(f"no renumbering rule for mesh array {name!r} of shape {a.shape}")
                out[key] = value
        elif key in _CASE:
            entity, axis, target = _CASE[key]
            a = np.take(np.asarray(value), perm[entity], axis=axis)
            out[key] = _remap(a, new_of_old[target]) if target else a
        elif key in _PASS:
            out[key] = value
        else:
            raise ValueError(f"no renumbering rule for case array {key!r}")
    return out


def random_order(arr: dict[str, Any], seed: int = 0) -> Renumbering:
    n = _sizes(arr)
    rng = np.random.default_rng(seed)
    return Renumbering(rng.permutation(n["cell"]), rng.permutation(n["edge"]), rng.permutation(n["vertex"]))


def hilbert_order(arr: dict[str, Any], bits: int = 16) -> Renumbering:
    """Cells along a 3-D Hilbert curve of (xCell, yCell, zCell); edges by
    their new (smaller, larger) cell pair; vertices by their sorted new cell
    triple."""
    from .mesh import _hilbert_keys

    xyz = np.stack([np.asarray(arr[f"mesh.{c}Cell"], dtype=np.float64) for c in "xyz"], axis=1)
    xyz /= np.linalg.norm(xyz, axis=1, keepdims=True)
    cell = np.argsort(_hilbert_keys(xyz, bits), kind="stable")
    new_c = _inverse(cell)
    coe = new_c[np.asarray(arr["mesh.cellsOnEdge"])]
    edge = np.lexsort((coe.max(axis=1), coe.min(axis=1)))
    cov = np.sort(new_c[np.asarray(arr["mesh.cellsOnVertex"])], axis=1)
    vertex = np.lexsort(cov.T[::-1])
    return Renumbering(cell, edge, vertex)


def neighbour_spread(arr: dict[str, Any]) -> dict[str, float]:
    """Mean |index difference| between an edge and its edgesOnEdge
    neighbours and between a cell and its cellsOnCell neighbours (a
    locality measure of a numbering)."""
    eoe = np.asarray(arr["mesh.edgesOnEdge"])
    e = np.broadcast_to(np.arange(eoe.shape[0])[:, None], eoe.shape)
    coc = np.asarray(arr["mesh.cellsOnCell"])
    c = np.broadcast_to(np.arange(coc.shape[0])[:, None], coc.shape)
    return {"edge": float(np.abs(eoe - e)[eoe >= 0].mean()), "cell": float(np.abs(coc - c)[coc >= 0].mean())}


# state and saved-diagnostic fields: (entity, axis)
FIELD_AXES = {
    "rho": ("cell", 0), "rho_theta": ("cell", 0), "rho_u": ("edge", 0), "rho_w": ("cell", 0),
    "scalars": ("cell", 1), "theta_m": ("cell", 0), "exner": ("cell", 0), "density_perturbation": ("cell", 0),
    "rho_theta_perturbation": ("cell", 0), "pressure_perturbation": ("cell", 0), "normal_velocity": ("edge", 0),
    "vertical_velocity": ("cell", 0),
}


def field(values: np.ndarray, name: str, ren: Renumbering) -> np.ndarray:
    """A logical state or sidecar field ([level][entity], scalars
    [tracer][level][cell]) renumbered by ``ren``."""
    entity, lead = FIELD_AXES[name]
    return np.take(np.asarray(values), ren.of(entity), axis=lead + 1)


def renumber_case(case, ren: Renumbering):
    """A ``hexdyn.case.DycoreCase`` renumbered by ``ren``."""
    from .case import DycoreCase, VerticalGridData, case_arrays
    from .mesh import VoronoiMesh

    arr = apply(case_arrays(case), ren)
    mesh = VoronoiMesh(arrays={k[5:]: v for k, v in arr.items() if k.startswith("mesh.")},
                       level=case.mesh.level, lloyd=case.mesh.lloyd, seed=case.mesh.seed)
    vertical = VerticalGridData(**{k: arr["vertical." + k] for k in VerticalGridData.__dataclass_fields__})
    rest = {k: arr[k] for k in DycoreCase.__dataclass_fields__ if k not in ("mesh", "vertical", "scalar_names",
                                                                              "coef_3rd_order")}
    return DycoreCase(mesh=mesh, vertical=vertical, scalar_names=case.scalar_names,
                      coef_3rd_order=case.coef_3rd_order, **rest)
