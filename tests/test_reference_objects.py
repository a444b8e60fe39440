"""The drop-in boundary with the reference's own classes (CPU).

Builds the reference's ``V841DryDycoreConfig`` (``hexcore/config_v841.py:114``),
``Mesh`` (``hexcore/mesh.py:1290``), ``PrognosticState``
(``hexcore/state.py:15``), ``VerticalGrid`` (``hexcore/vertical.py:83``),
``DryReferenceState`` / ``TerrainMetrics`` / ``DrySavedDiagnostics``
(``hexcore/driver.py:609,636,661``), ``AdvectionCoefficients``
(``hexcore/transport.py:38``) and ``V841ReferenceWindProfiles``
(``hexcore/dynamics_v841.py``) from a golden fixture, and checks that

* ``DycoreConfig.from_reference`` accepts a configuration this path runs and
  refuses, by name and before any device work, every reference knob it does
  not implement when set away from the reference's default;
* ``HexDycoreDriver.from_host``'s host preparation (the descriptor handed to
  ``hexdyn_create`` and every array behind it) is the same, word for word,
  whether given the reference's objects or the duck-typed stand-ins the GPU
  tests use, so the GPU parity of the stand-ins carries over.

Skipped where the reference checkout is absent.
"""

import dataclasses

import numpy as np
import pytest

from fixtures import STATE, case_from_arrays, import_reference, inputs, load_golden

ROOT = import_reference()
pytestmark = pytest.mark.skipif(ROOT is None, reason="the reference checkout is not present")


def _reference_config(**kw):
    from hexcore.config_v841 import V841DryDycoreConfig

    base = dict(config_dt=1800.0, config_number_of_sub_steps=2, config_dynamics_split_steps=3,
                config_split_dynamics_transport=True, config_monotonic=True, config_positive_definite=False,
                config_coef_3rd_order=0.25, config_apvm_upwinding=0.5)
    base.update(kw)
    return V841DryDycoreConfig(**base)


def test_reference_config_is_accepted():
    from hexdyn.config import DycoreConfig

    cfg = DycoreConfig.from_reference(_reference_config())
    assert cfg.config_dt == 1800.0 and cfg.config_number_of_sub_steps == 2 and cfg.fct


@pytest.mark.parametrize("knob,value", [
    ("config_les_model", "3d_smagorinsky"), ("config_les_surface", "specified"), ("config_mix_scalars", True),
    ("config_mix_full", False), ("config_surface_heat_flux", 0.24), ("config_surface_moisture_flux", 1e-4),
    ("config_surface_drag_coefficient", 1e-3), ("config_physics_suite", "mesoscale_reference"),
    ("config_iau_option", "on"), ("config_h_mom_eddy_visc2", 1000.0), ("config_h_theta_eddy_visc4", 1e12),
    ("config_vertical_mixing", True), ("config_curvature_terms", True), ("config_gpu_aware_mpi", True),
    ("config_terrain_following", False), ("source_release", "v8.2.3"),
])
def test_unmodelled_reference_knob_is_refused_by_name(knob, value):
    from hexdyn.config import ConfigurationRefusal, DycoreConfig

    ref = dataclasses.replace(_reference_config(), **{knob: value})
    with pytest.raises(ConfigurationRefusal) as err:
        DycoreConfig.from_reference(ref)
    assert err.value.knob == knob
    assert err.value.value == value


def test_every_unmodelled_knob_of_the_reference_is_listed():
    """Knobs of the reference's configuration that this path neither models
    nor lists would still be refused (their dataclass default is used), but
    each should carry its own reason."""
    from hexcore.config_v841 import V841DryDycoreConfig

    from hexdyn.config import UNMODELLED_REFERENCE_KNOBS, DycoreConfig

    modelled = {f.name for f in dataclasses.fields(DycoreConfig)}
    ref = {f.name for f in dataclasses.fields(V841DryDycoreConfig)}
    missing = sorted(ref - modelled - set(UNMODELLED_REFERENCE_KNOBS) - {"config_terrain_following"})
    assert missing == []


def _reference_objects(fx):
    from hexcore.driver import DryReferenceState, TerrainMetrics
    from hexcore.dynamics_v841 import V841ReferenceWindProfiles
    from hexcore.mesh import Mesh
    from hexcore.state import PrognosticState
    from hexcore.transport import AdvectionCoefficients
    from hexcore.vertical import VerticalGrid

    arr = inputs(fx)
    stand_in = case_from_arrays(arr)
    marrays = {k[5:]: v for k, v in arr.items() if k.startswith("mesh.")}
    dims = {"nCells": int(marrays["areaCell"].size), "nEdges": int(marrays["dcEdge"].size),
            "nVertices": int(marrays["areaTriangle"].size), "maxEdges": int(marrays["edgesOnCell"].shape[1]),
            "maxEdges2": int(marrays["edgesOnEdge"].shape[1]), "vertexDegree": 3}
    mesh = Mesh(arrays=marrays, dimensions=dims, attrs={"on_a_sphere": "YES"})
    vg = VerticalGrid(**{k: getattr(stand_in.vertical, k) for k in stand_in.vertical.__dataclass_fields__})
    ref = DryReferenceState(stand_in.rho_base, stand_in.rho_theta_base, stand_in.pressure_base,
                            stand_in.exner_base)
    tm = TerrainMetrics(stand_in.zb_cell, stand_in.zb3_cell)
    ac = AdvectionCoefficients(stand_in.adv_coefs, stand_in.adv_coefs_3rd, stand_in.n_adv_cells_for_edge,
                               stand_in.adv_cells_for_edge, 3, None)
    wp = V841ReferenceWindProfiles(stand_in.u_init, stand_in.v_init)
    state = PrognosticState(*(np.asarray(arr[k]).copy() for k in STATE), 0.0)
    return stand_in, (mesh, state, vg, ref, ac, tm, wp)


def test_reference_objects_give_the_stand_in_descriptor():
    from hexdyn.config import DycoreConfig
    from hexdyn.driver import _build_descriptor

    fx = load_golden("l2_L12")
    s, (mesh, state, vg, ref, ac, tm, wp) = _reference_objects(fx)
    cfg = DycoreConfig.from_reference(_reference_config(config_dt=float(fx["config.dt"])))
    d_ref, keep_ref, sizes_ref = _build_descriptor(mesh, state, vg, ref, cfg, tm, ac, wp)
    d_std, keep_std, sizes_std = _build_descriptor(s.mesh, s, s.vertical, s, cfg, s, s, s)
    assert sizes_ref == sizes_std
    assert sorted(keep_ref) == sorted(keep_std)
    for k in keep_ref:
        a, b = keep_ref[k], keep_std[k]
        assert a.dtype == b.dtype and a.shape == b.shape, k
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k
    import ctypes

    for name, _ in d_ref._fields_:
        va, vb = getattr(d_ref, name), getattr(d_std, name)
        if isinstance(va, ctypes._Pointer):  # arrays compared above; NULL where one is NULL
            assert bool(va) == bool(vb), name
        elif isinstance(va, ctypes.Array):
            assert list(va) == list(vb), name
        else:
            assert va == vb, name


def test_reference_state_and_sidecar_attributes_are_read():
    """The state and sidecar uploads read the reference's attribute names:
    every field ``set_state`` reads exists on ``PrognosticState`` and
    ``DrySavedDiagnostics`` with the shape the library expects."""
    from hexcore.driver import DrySavedDiagnostics

    from hexdyn import _lib

    fx = load_golden("l2_L12")
    _, (mesh, state, *_rest) = _reference_objects(fx)
    L, C = fx["in.rho"].shape
    E = fx["in.rho_u"].shape[1]
    side = DrySavedDiagnostics(*(fx[f"dry.step1.side.{k}"] for k in (
        "theta_m", "exner", "density_perturbation", "rho_theta_perturbation", "pressure_perturbation",
        "normal_velocity", "vertical_velocity")))
    for name in _lib.STATE_FIELDS:
        assert np.asarray(getattr(state, name)).shape[-2:] in ((L, C), (L, E), (L + 1, C)), name
    for name in _lib.SIDECAR_FIELDS:
        assert np.asarray(getattr(side, name)).shape in ((L, C), (L, E), (L + 1, C)), name
