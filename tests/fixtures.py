"""Shared test helpers: golden fixtures and synthetic cases as driver inputs."""

from __future__ import annotations

from pathlib import Path
from types import SimpleNamespace

import numpy as np

from hexdyn.case import VerticalGridData
from hexdyn.mesh import VoronoiMesh

GOLDEN = Path(__file__).resolve().parent / "golden"
STATE = ("rho", "rho_theta", "rho_u", "rho_w", "scalars")
SIDE = ("theta_m", "exner", "density_perturbation", "rho_theta_perturbation",
        "pressure_perturbation", "normal_velocity", "vertical_velocity")


def load_golden(name: str) -> dict:
    """A fixture; configuration variants carry only outputs and take their
    inputs from the base case they name."""
    with np.load(GOLDEN / f"step_{name}.npz", allow_pickle=False) as z:
        fx = {k: z[k] for k in z.files}
    if "base" in fx:
        base = load_golden(str(fx["base"]))
        fx.update({k: v for k, v in base.items() if k.startswith("in.")})
        if "config.n_scalars" in fx:
            fx["in.scalars"] = fx["in.scalars"][: int(fx["config.n_scalars"])].copy()
    return fx


def golden_config(fx: dict) -> dict:
    """The configuration a fixture was made with (defaults of the base cases)."""
    return {"dt": float(fx["config.dt"]), "n_sub_steps": int(fx["config.n_sub_steps"]),
            "monotonic": bool(int(fx.get("config.monotonic", 1))),
            "apvm_upwinding": float(fx.get("config.apvm_upwinding", 0.5)),
            "xnutr": float(fx.get("config.xnutr", 0.0)), "zd": float(fx.get("config.zd", 22000.0)),
            "order": int(fx.get("config.order", 3)),
            "smagorinsky": (None if "config.smagorinsky_coef" not in fx else
                            (float(fx["config.smagorinsky_coef"]), float(fx["config.visc4_2dsmag"]),
                             float(fx["config.del4u_div_factor"])))}


VARIANTS = [("l2_L12_sub1", 2), ("l2_L12_sub4", 2), ("l2_L12_nomono", 2), ("l2_L12_noapvm", 1),
            ("l2_L12_notracers", 2), ("l2_L12_xnutr", 2), ("l2_L12_rk2", 2), ("l2_L12_rk2_sub4", 1),
            ("l2_L12_smag", 2)]


def inputs(fx: dict) -> dict:
    """The case arrays (``hexdyn.case.case_arrays`` layout) of a fixture."""
    return {k[3:]: v for k, v in fx.items() if k.startswith("in.")}


def case_from_arrays(arr: dict) -> SimpleNamespace:
    """A duck-typed case (reference attribute names) from case arrays."""
    mesh = VoronoiMesh(arrays={k[5:]: v for k, v in arr.items() if k.startswith("mesh.")})
    vfields = {k[9:]: v for k, v in arr.items() if k.startswith("vertical.")}
    for k in ("cf1", "cf2", "cf3"):
        vfields[k] = float(vfields[k])
    vfields["first_height_level"] = int(vfields["first_height_level"])
    vertical = VerticalGridData(**vfields)
    ns = SimpleNamespace(mesh=mesh, vertical=vertical)
    for k in ("zb_cell", "zb3_cell", "rho_base", "rho_theta_base", "pressure_base", "exner_base",
              "rho", "rho_theta", "rho_u", "rho_w", "scalars", "adv_coefs", "adv_coefs_3rd",
              "n_adv_cells_for_edge", "adv_cells_for_edge", "u_init", "v_init"):
        setattr(ns, k, arr[k])
    ns.time_seconds = 0.0
    return ns


def differing_words(a, b) -> int:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    assert a.shape == b.shape, (a.shape, b.shape)
    return int(np.count_nonzero(a.view(np.uint32) != b.view(np.uint32)))
