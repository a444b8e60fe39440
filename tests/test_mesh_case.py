"""Synthetic mesh and case builders: MPAS conventions and determinism."""

import numpy as np
import pytest

from fixtures import inputs, load_golden
from hexdyn.case import build_case, case_arrays
from hexdyn.mesh import build_mesh


@pytest.fixture(scope="module")
def mesh3():
    return build_mesh(3, lloyd=5, seed=0)


def test_counts():
    for level, (c, e, v) in {2: (162, 480, 320), 3: (642, 1920, 1280), 4: (2562, 7680, 5120)}.items():
        m = build_mesh(level, lloyd=2, seed=0)
        assert (m.n_cells, m.n_edges, m.n_vertices) == (c, e, v)
        assert np.sum(m.nEdgesOnCell == 5) == 12


def test_areas_and_kites(mesh3):
    a = mesh3.arrays
    r = a["sphere_radius"]
    assert np.isclose(a["areaCell"].sum(), 4 * np.pi * r * r, rtol=1e-12)
    assert np.allclose(a["kiteAreasOnVertex"].sum(axis=1), a["areaTriangle"])
    assert np.all(a["kiteAreasOnVertex"] > 0)


def test_edge_orientation(mesh3):
    a = mesh3.arrays
    c1, c2 = a["cellsOnEdge"].T
    assert np.all(c1 < c2)
    # v2 lies to the left of the normal c1 -> c2 (tangent = k x n points to v2)
    xe = np.stack([a["xEdge"], a["yEdge"], a["zEdge"]], 1)
    xv = np.stack([a["xVertex"], a["yVertex"], a["zVertex"]], 1)
    t = a["_edge_tangent"]
    d = xv[a["verticesOnEdge"][:, 1]] - xv[a["verticesOnEdge"][:, 0]]
    assert np.all(np.einsum("ij,ij->i", d, t) > 0)
    del xe


def test_trisk_properties(mesh3):
    """TRiSK weights: antisymmetry and tangential reconstruction (Thuburn 2009)."""
    a = mesh3.arrays
    eoe, w, ne = a["edgesOnEdge"], a["weightsOnEdge"], a["nEdgesOnEdge"]
    dc, dv = a["dcEdge"], a["dvEdge"]
    pairs = {}
    for e in range(eoe.shape[0]):
        for s in range(ne[e]):
            pairs[(e, eoe[e, s])] = w[e, s] * dc[e] / dv[eoe[e, s]]
    assert max(abs(pairs[(e, f)] + pairs[(f, e)]) for (e, f) in pairs) < 1e-12
    xe = np.stack([a["xEdge"], a["yEdge"], a["zEdge"]], 1)
    U = np.cross(np.array([0, 0, 1.0]), xe) / a["sphere_radius"] * 20.0
    u = np.einsum("ij,ij->i", U, a["_edge_normal"])
    vt = np.einsum("ij,ij->i", U, a["_edge_tangent"])
    v = np.zeros_like(u)
    for s in range(eoe.shape[1]):
        act = ne > s
        v[act] += w[act, s] * u[eoe[act, s]]
    assert np.abs(v - vt).max() < 0.1 * 20.0


def test_case_builder_is_deterministic():
    fx = load_golden("l2_L12")
    arr = inputs(fx)
    mesh = build_mesh(2, lloyd=20, seed=0)
    again = case_arrays(build_case(mesh, n_levels=12, seed=0, n_condensates=1))
    for k in ("rho", "rho_theta", "rho_u", "scalars", "zb_cell", "vertical.zz", "adv_coefs"):
        assert np.array_equal(np.asarray(again[k]), np.asarray(arr[k])), k


def test_balanced_state_is_physical():
    mesh = build_mesh(3, lloyd=5, seed=0)
    case = build_case(mesh, n_levels=20, seed=1, n_condensates=2)
    assert np.all(case.rho > 0) and np.all(case.rho_theta > 0)
    u = 2 * case.rho_u / (case.rho[:, mesh.cellsOnEdge[:, 0]] + case.rho[:, mesh.cellsOnEdge[:, 1]])
    assert 25.0 < np.abs(u).max() < 45.0
    assert np.all(np.diff(case.vertical.zgrid, axis=0) > 0)
    assert case.scalars.shape == (3, 20, mesh.n_cells)
    assert np.all(case.scalars >= 0)
