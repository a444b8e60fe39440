"""MPAS init / restart files (CPU): ``hexdyn.mpas_io.write_restart`` /
``read_restart`` / ``read_vertical_grid`` / ``read_initial_state``.

* a case written and read back holds the same words in every array;
* the reference's state after one step, written with its saved diagnostics
  and read back, steps (oracle) to the reference's second step word for
  word (tests/golden fixture ``l2_L12``);
* the reader returns, word for word, what the reference's own loaders
  (``load_mpas_vertical_grid``, hexcore/driver.py:1419, and
  ``load_mpas_initial_state``, :1582) return for the same file, for a
  restart-form file (``rho_zz``, ``theta_m``, ``ru``, ``rw`` and the saved
  diagnostics) and a public init-form file (``rho``, ``theta``, ``qv``,
  ``u``, ``w``: the coupled-state conversions and the terrain correction of
  ``rw``).  Those comparisons run where the reference checkout is present
  (its loaders read through a SciPy-backed netCDF4 stand-in).
"""

import numpy as np
import pytest

from fixtures import SIDE, STATE, case_from_arrays, differing_words, import_reference, inputs, load_golden
from hexdyn import mpas_io
from hexdyn.driver import HostSidecar
from oracle.dycore import OracleConfig, OracleDycore, Sidecar, State

CASE_FIELDS = ("rho_base", "rho_theta_base", "pressure_base", "exner_base", "rho", "rho_theta", "rho_u", "rho_w",
               "scalars", "zb_cell", "zb3_cell", "adv_coefs", "adv_coefs_3rd", "n_adv_cells_for_edge",
               "adv_cells_for_edge", "u_init", "v_init")
VERTICAL = ("zw", "dzw", "rdzw", "zu", "dzu", "rdzu", "rdzwp", "rdzwm", "fzp", "fzm", "zgrid", "zz", "zxu", "dss")
# the level arrays an MPAS file stores (zw, dzw, zu, rdzwp, rdzwm are derived
# from rdzw on reading, as the reference's loader derives them)
STORED = ("rdzw", "dzu", "rdzu", "fzp", "fzm", "zgrid", "zz", "zxu", "dss")


def _same(a, b) -> bool:
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.dtype.kind == b.dtype.kind and np.array_equal(
        np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b.astype(a.dtype)).view(np.uint8))


def _golden_case():
    fx = load_golden("l2_L12")
    case = case_from_arrays(inputs(fx))
    case.scalar_names = ("qv", "qc")[: case.scalars.shape[0]]
    case.coef_3rd_order = 0.25
    return fx, case


def _sidecar(fx, step):
    return HostSidecar(*(fx[f"dry.step{step}.side.{k}"] for k in SIDE))


def test_restart_round_trip_is_bitwise(tmp_path):
    """A state with its saved diagnostics (the reference's after one step:
    the file holds rtheta_p, not rho_theta, and the step leaves rho_theta =
    rtheta_p + rtheta_base exactly)."""
    fx, case = _golden_case()
    for k in STATE:
        setattr(case, k, fx[f"dry.step1.{k}"])
    side = _sidecar(fx, 1)
    path = tmp_path / "restart.nc"
    mpas_io.write_restart(path, case, side, time_seconds=1800.0)
    back, bside = mpas_io.read_restart(path)
    for k in CASE_FIELDS:
        assert _same(getattr(case, k), getattr(back, k)), k
    for k in STORED:
        assert _same(getattr(case.vertical, k), getattr(back.vertical, k)), k
    for k in ("cf1", "cf2", "cf3"):
        assert np.float32(getattr(case.vertical, k)) == np.float32(getattr(back.vertical, k)), k
    for k in SIDE:
        assert _same(getattr(side, k), getattr(bside, k)), k
    assert back.scalar_names == case.scalar_names and back.time_seconds == 1800.0
    for k in ("cellsOnEdge", "edgesOnCell", "weightsOnEdge", "dcEdge", "areaCell"):
        assert _same(case.mesh.arrays[k], back.mesh.arrays[k]), k


def test_restart_continues_as_the_reference(tmp_path):
    """The reference's state and saved diagnostics after step 1, through the
    file, then one oracle step: the reference's step 2, every word."""
    fx, case = _golden_case()
    for k in STATE:
        setattr(case, k, fx[f"dry.step1.{k}"])
    path = tmp_path / "restart_step1.nc"
    mpas_io.write_restart(path, case, _sidecar(fx, 1), time_seconds=1800.0)
    back, bside = mpas_io.read_restart(path)
    from hexdyn.case import case_arrays

    arr = case_arrays(back) if hasattr(back, "__dataclass_fields__") else _arrays_of(back)
    orc = OracleDycore(arr, OracleConfig(dt=float(fx["config.dt"]), n_sub_steps=int(fx["config.n_sub_steps"]),
                                         moist="dry"))
    st, sd = orc.step(State(*(np.asarray(getattr(back, k)).copy() for k in STATE)),
                      Sidecar(*(np.asarray(getattr(bside, k)).copy() for k in SIDE)))
    for k in STATE:
        assert differing_words(getattr(st, k), fx[f"dry.step2.{k}"]) == 0, k
    for k in SIDE:
        assert differing_words(getattr(sd, k), fx[f"dry.step2.side.{k}"]) == 0, k


def _arrays_of(case) -> dict:
    out = {"mesh." + k: v for k, v in case.mesh.arrays.items()}
    for k in case.vertical.__dataclass_fields__:
        out["vertical." + k] = getattr(case.vertical, k)
    for k in CASE_FIELDS:
        out[k] = getattr(case, k)
    out["coef_3rd_order"] = case.coef_3rd_order
    return out


# ------------------------------------------------ the reference's own loader

REF = import_reference()
needs_reference = pytest.mark.skipif(REF is None, reason="the reference checkout is not present")


def _reference_mesh(case):
    from hexcore.mesh import Mesh

    a = case.mesh.arrays
    dims = {"nCells": int(a["areaCell"].size), "nEdges": int(a["dcEdge"].size),
            "nVertices": int(a["areaTriangle"].size), "maxEdges": int(a["edgesOnCell"].shape[1]),
            "maxEdges2": int(a["edgesOnEdge"].shape[1]), "vertexDegree": 3}
    return Mesh(arrays=dict(a), dimensions=dims, attrs={"on_a_sphere": "YES"})


def _write_public(path, case, side):
    """An init-form file: physical rho and dry theta, qv, u, w, the base
    state and the vertical grid, and no rho_zz / theta_m / ru / rw / saved
    diagnostics."""
    tmp = str(path) + ".restart"
    mpas_io.write_restart(tmp, case, side)
    from scipy.io import netcdf_file

    src = netcdf_file(tmp, "r", mmap=False)
    dst = netcdf_file(str(path), "w", version=2)
    try:
        for name, size in src.dimensions.items():
            dst.createDimension(name, size)
        for k, val in src._attributes.items():
            setattr(dst, k, val)
        skip = {"rho_zz", "theta_m", "ru", "rw", "exner", "rtheta_p", "rho_p", "pressure_p"}
        for name, var in src.variables.items():
            if name in skip:
                continue
            out = dst.createVariable(name, var.data.dtype.char, var.dimensions)
            if var.dimensions:
                out[:] = var.data
            else:
                out.data[()] = var.data[()]
        zz = np.asarray(case.vertical.zz, np.float32)
        rho = np.asarray(case.rho, np.float32) * zz
        qv = np.asarray(case.scalars[0], np.float32)
        theta = (np.asarray(side.theta_m, np.float32) / (np.float32(1.0) + np.float32(1.6) * qv)).astype(np.float32)
        for name, value, ent, lev in (("rho", rho, "nCells", "nVertLevels"), ("theta", theta, "nCells", "nVertLevels")):
            out = dst.createVariable(name, "f", ("Time", ent, lev))
            out[:] = value.T[None]
    finally:
        src.close()
        dst.close()


@needs_reference
@pytest.mark.parametrize("form", ["restart", "public"])
def test_reader_matches_the_reference_loader(tmp_path, form):
    from hexcore.driver import load_mpas_initial_state, load_mpas_vertical_grid

    fx, case = _golden_case()
    for k in STATE:
        setattr(case, k, fx[f"dry.step1.{k}"])
    side = _sidecar(fx, 1)
    path = tmp_path / f"{form}.nc"
    if form == "restart":
        mpas_io.write_restart(path, case, side)
    else:
        _write_public(path, case, side)
    names = tuple(case.scalar_names)
    mesh = mpas_io.read_mesh(path)
    vg, zb_cell, zb3_cell = mpas_io.read_vertical_grid(path, mesh)
    st, ref, sd = mpas_io.read_initial_state(path, mesh, vg, scalar_names=names, terrain=(zb_cell, zb3_cell))
    rmesh = _reference_mesh(case)
    native = load_mpas_vertical_grid(path, rmesh, config_coef_3rd_order=0.25)
    rvg, rterr = native.vertical_grid, native.terrain_metrics
    for k in VERTICAL:
        assert _same(getattr(rvg, k), getattr(vg, k)), k
    assert _same(rterr.zb_cell, zb_cell) and _same(rterr.zb3_cell, zb3_cell)
    rst, rref, rsd = load_mpas_initial_state(path, rmesh, rvg, scalar_names=names, terrain_metrics=rterr,
                                             return_saved_diagnostics=True)
    for k in STATE:
        assert _same(getattr(rst, k), getattr(st, k)), (form, k)
    for k in ("rho_base", "rho_theta_base", "pressure_base", "exner_base"):
        assert _same(getattr(rref, k), getattr(ref, k)), (form, k)
    if form == "restart":
        for k in SIDE:
            assert _same(getattr(rsd, k), getattr(sd, k)), k
        # and it is the state that was written
        for k in STATE:
            assert _same(getattr(st, k), fx[f"dry.step1.{k}"]), k
    else:
        assert sd is None  # rebuilt on the device from the state


@pytest.mark.gpu
def test_cuda_step_from_a_restart_file_is_the_reference_step(tmp_path):
    """The reference's state after one step through a restart file into the
    CUDA library (saved diagnostics from the file), one step: the
    reference's step 2, word for word."""
    import torch

    from hexdyn.config import DycoreConfig
    from hexdyn.driver import HexDycoreDriver

    assert torch.cuda.is_available()
    torch.cuda.set_device(0)
    fx, case = _golden_case()
    for k in STATE:
        setattr(case, k, fx[f"dry.step1.{k}"])
    path = tmp_path / "restart_step1.nc"
    mpas_io.write_restart(path, case, _sidecar(fx, 1), time_seconds=1800.0)
    back, bside = mpas_io.read_restart(path)
    cfg = DycoreConfig(config_dt=float(fx["config.dt"]), config_number_of_sub_steps=int(fx["config.n_sub_steps"]),
                       moist_coefficients="dry")
    drv = HexDycoreDriver.from_host(back.mesh, back, back.vertical, back, cfg, saved_diagnostics=bside,
                                    terrain_metrics=back, advection_coefficients=back, reference_wind_profiles=back)
    assert drv.time_seconds == 1800.0
    res = drv.step()
    for k in STATE:
        assert differing_words(getattr(res.state, k), fx[f"dry.step2.{k}"]) == 0, k
    for k in SIDE:
        assert differing_words(getattr(res.saved_diagnostics, k), fx[f"dry.step2.side.{k}"]) == 0, k
    drv.close()
