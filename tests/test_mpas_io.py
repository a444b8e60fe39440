"""MPAS mesh files (hexdyn.mpas_io): a mesh written with the MPAS variable
names and 1-based connectivity reads back identical, and a case built on the
read mesh steps exactly like one built on the original (oracle)."""

import numpy as np
import pytest

from hexdyn import mpas_io
from hexdyn.case import build_case, case_arrays
from hexdyn.mesh import build_mesh


def test_mesh_round_trip(tmp_path):
    mesh = build_mesh(2, lloyd=2, seed=0)
    path = tmp_path / "x1.162.grid.nc"
    mpas_io.write_mesh(mesh, path)
    back = mpas_io.read_mesh(path)
    for k, v in mesh.arrays.items():
        if k.startswith("_"):
            continue
        got = np.asarray(back.arrays[k])
        want = np.asarray(v)
        assert got.shape == want.shape, k
        assert np.array_equal(got.astype(want.dtype) if want.dtype.kind in "iub" else got, want), k
    # the derived edge normals agree with the builder's to rounding
    assert np.allclose(back.arrays["_edge_normal"], mesh.arrays["_edge_normal"], atol=1e-12)


def test_read_mesh_steps_like_the_original(tmp_path):
    from oracle.dycore import OracleConfig, OracleDycore, State

    mesh = build_mesh(2, lloyd=2, seed=0)
    path = tmp_path / "mesh.nc"
    mpas_io.write_mesh(mesh, path)
    back = mpas_io.read_mesh(path)
    a = case_arrays(build_case(mesh, n_levels=8, seed=0, n_condensates=1))
    b = case_arrays(build_case(back, n_levels=8, seed=0, n_condensates=1, like=None))
    cfg = OracleConfig(dt=1800.0, n_sub_steps=2, moist="dry")
    names = ("rho", "rho_theta", "rho_u", "rho_w", "scalars")
    # the same case arrays (the state from the read mesh uses its own
    # derived normals; step the original state on both meshes)
    b.update({k: a[k] for k in names})
    sa, _ = OracleDycore(a, cfg).step(State(*(a[k].copy() for k in names)), None)
    sb, _ = OracleDycore(b, cfg).step(State(*(a[k].copy() for k in names)), None)
    for k in names:
        assert np.array_equal(getattr(sa, k), getattr(sb, k)), k


def test_not_netcdf3_is_refused(tmp_path):
    bad = tmp_path / "x.nc"
    bad.write_bytes(b"\x89HDF\r\n\x1a\n" + b"\0" * 64)
    with pytest.raises(ValueError):
        mpas_io.read_mesh(bad)
