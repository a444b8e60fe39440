"""Dycore configuration with refusal-based validation.

Mirrors the knobs of the reference's ``V841DryDycoreConfig``
(``hexcore/config_v841.py:114``, defaults ``:117-140``, base validation
``hexcore/driver.py:232-501``) that the GPU step path reads.  A value outside
what this path implements is refused by name, before any launch, with the
same ``ConfigurationRefusal(knob, value, reason, declaration)`` shape as
``hexcore/errors.py:17``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, fields
from typing import Any, Mapping


class ConfigurationRefusal(RuntimeError):
    """A requested configuration knob has no implementation on this path."""

    def __init__(self, knob: str, value: object, reason: str, declaration: str) -> None:
        self.knob = knob
        self.value = value
        self.reason = reason
        self.declaration = declaration
        super().__init__(f"{knob}={value!r} is refused: {reason}. To run, declare {declaration}.")


def _refuse(knob: str, value: object, reason: str, declaration: str) -> None:
    raise ConfigurationRefusal(knob, value, reason, declaration)


# Knobs of the reference's configuration classes that this path does not
# implement, with the reference's defaults and why each is refused when set
# to anything else: ``V841DryDycoreConfig`` (hexcore/config_v841.py:114-140)
# and its base ``DryDycoreConfig`` (hexcore/driver.py:172-260).
UNMODELLED_REFERENCE_KNOBS: dict[str, tuple[object, str]] = {
    "config_physics_suite": ("none", "physics suites run outside the dycore step"),
    "config_iau_option": ("off", "incremental analysis update forcing is not part of this step"),
    "config_h_theta_eddy_visc2": (0.0, "fixed eddy viscosities (2d_fixed mixing) are not implemented"),
    "config_v_theta_eddy_visc2": (0.0, "fixed eddy viscosities (2d_fixed mixing) are not implemented"),
    "config_h_mom_eddy_visc2": (0.0, "fixed eddy viscosities (2d_fixed mixing) are not implemented"),
    "config_v_mom_eddy_visc2": (0.0, "fixed eddy viscosities (2d_fixed mixing) are not implemented"),
    "config_h_theta_eddy_visc4": (0.0, "fixed eddy viscosities (2d_fixed mixing) are not implemented"),
    "config_h_mom_eddy_visc4": (0.0, "fixed eddy viscosities (2d_fixed mixing) are not implemented"),
    "config_vertical_mixing": (False, "the saved vertical Euler filters are not implemented"),
    "config_curvature_terms": (False, "the optional curvature branch is not implemented"),
    "config_gpu_aware_mpi": (False, "this path has no MPI transport"),
    "config_les_model": ("none", "LES / 3-D Smagorinsky mixing is not implemented"),
    "config_les_surface": ("none", "LES surface forcing is not implemented"),
    "config_mix_scalars": (False, "3-D mixing of scalars is not implemented"),
    "config_mix_full": (True, "the 3-D mixing variants are not implemented"),
    "config_surface_heat_flux": (0.0, "prescribed surface fluxes belong to the LES branch, not implemented"),
    "config_surface_moisture_flux": (0.0, "prescribed surface fluxes belong to the LES branch, not implemented"),
    "config_surface_drag_coefficient": (0.0, "prescribed surface drag belongs to the LES branch, not implemented"),
    "source_release": ("v8.4.1", "this path implements the v8.4.1/8.4.2 numerics"),
}


def _refuse_unmodelled(config: Any, modelled: set[str]) -> None:
    """Refuse, by name, every knob of a reference configuration that this
    path does not model and whose value is not the reference's default.
    Dataclass configurations are checked field by field against their own
    defaults (so knobs added to the reference later are caught too); other
    objects against ``UNMODELLED_REFERENCE_KNOBS``."""
    defaults: dict[str, object] = {}
    try:
        import dataclasses

        for f in dataclasses.fields(config):
            if f.default is not dataclasses.MISSING:
                defaults[f.name] = f.default
            elif f.default_factory is not dataclasses.MISSING:  # type: ignore[misc]
                defaults[f.name] = f.default_factory()  # type: ignore[misc]
    except TypeError:
        pass
    for knob, (default, _) in UNMODELLED_REFERENCE_KNOBS.items():
        defaults.setdefault(knob, default)
    for knob, default in defaults.items():
        if knob in modelled or not hasattr(config, knob):
            continue
        value = getattr(config, knob)
        if knob == "config_terrain_following":
            # hexcore/driver.py:2286-2305: True or None run with the terrain
            # metrics this path always takes; False would drop them
            if value is False:
                _refuse(knob, value, "this path always applies the native terrain metrics",
                        "config_terrain_following=True or None")
            continue
        if knob == "source_release":
            default = UNMODELLED_REFERENCE_KNOBS[knob][0]
        if isinstance(default, bool) or isinstance(value, bool):
            same = type(value) is type(default) and value == default
        else:
            try:
                same = bool(value == default)
            except Exception:  # noqa: BLE001
                same = False
        if not same:
            reason = UNMODELLED_REFERENCE_KNOBS.get(knob, (None, "this knob is not implemented on the GPU step "
                                                                 "path"))[1]
            _refuse(knob, value, reason, f"{knob}={default!r}")


@dataclass(frozen=True)
class DycoreConfig:
    """The v8.4.1/8.4.2 dry-plus-tracer lane on one GPU."""

    config_dt: float = 30.0
    config_time_integration_order: int = 3
    config_number_of_sub_steps: int = 2
    config_dynamics_split_steps: int = 3
    config_split_dynamics_transport: bool = True
    config_scalar_advection: bool = True
    config_monotonic: bool = True
    config_positive_definite: bool = False
    config_scalar_adv_order: int = 3
    config_scalar_vadv_order: int = 3
    config_coef_3rd_order: float = 0.25
    config_apvm_upwinding: float = 0.5
    config_epssm: float = 0.0
    config_epssm_minimum: float = 0.1
    config_epssm_maximum: float = 0.5
    config_epssm_transition_bottom_z: float = 30_000.0
    config_epssm_transition_top_z: float = 50_000.0
    config_divergence_damping: bool = True
    config_smdiv: float = 0.1
    config_len_disp: float = 0.0
    config_xnutr: float = 0.0
    config_zd: float = 22_000.0
    config_horiz_mixing: str = "off"
    # 2-D Smagorinsky knobs (hexcore/driver.py:193-201; port-safe defaults:
    # zero active-only coefficients while mixing is off)
    config_smagorinsky_coef: float = 0.0
    config_visc4_2dsmag: float = 0.0
    config_del4u_div_factor: float = 10.0
    config_h_ScaleWithMesh: bool = True
    config_mpas_cam_coef: float = 0.0
    config_number_cam_damping_levels: int = 4
    config_number_rayleigh_damp_u_levels: int = 6
    config_rayleigh_damp_u_timescale_days: float = 5.0
    config_moist_physics: bool = False
    # End-of-step clamp of negative mixing ratios (where q < 0: q = 0) that
    # the reference's CUDA driver applies on the global path without physics
    # (hexcore/cuda_driver.py:5306-5311); its NumPy authority, which the
    # strict parity follows, applies it only with config_moist_physics
    # (hexcore/driver.py:3531-3534).  The monotonic limiter's output is never
    # negative, so the clamp changes words only with standard transport.
    clamp_negative_scalars: bool = False
    config_rayleigh_damp_u: bool = False
    config_apply_lbcs: bool = False
    # Coefficient semantics of the carried scalars: "native" applies
    # atm_compute_moist_coefficients from every scalar each step (native MPAS
    # and the reference CUDA driver with physics off); "dry" keeps qtot=0,
    # cqu=cqw=1 (the reference CPU driver on a global mesh).
    moist_coefficients: str = "native"
    # "strict": bit-identical to the reference authority; "fast": FMA.
    numerics: str = "strict"

    @classmethod
    def from_mapping(cls, raw: Mapping[str, Any]) -> "DycoreConfig":
        known = {f.name for f in fields(cls)}
        unknown = sorted(set(raw) - known)
        if unknown:
            _refuse(unknown[0], raw[unknown[0]], "this option is not implemented on the GPU step path",
                    f"a supported value after porting {unknown[0]!r}")
        out = cls(**raw)
        out.validate()
        return out

    @classmethod
    def from_reference(cls, config: Any, **overrides: Any) -> "DycoreConfig":
        """Project a reference ``V841DryDycoreConfig`` (or any object with the
        same attribute names) onto this configuration.  Every reference knob
        this path does not model must hold the reference's default; any other
        value is refused by name (``ConfigurationRefusal``) before any device
        work, as ``hexcore/cuda_driver.py:3096-3215`` refuses before launching."""
        modelled = {f.name for f in fields(cls)}
        _refuse_unmodelled(config, modelled)
        values = {f.name: getattr(config, f.name) for f in fields(cls) if hasattr(config, f.name)}
        values.update(overrides)
        out = cls(**values)
        out.validate()
        return out

    def validate(self) -> None:
        if not math.isfinite(self.config_dt) or self.config_dt <= 0.0:
            _refuse("config_dt", self.config_dt, "the timestep must be finite and positive", "config_dt>0")
        if (isinstance(self.config_time_integration_order, bool)
                or self.config_time_integration_order not in (2, 3)):
            _refuse("config_time_integration_order", self.config_time_integration_order,
                    "the MPAS split-explicit loop has only order-2 and order-3 schedules",
                    "config_time_integration_order=2 or 3")
        if not isinstance(self.config_number_of_sub_steps, int) or self.config_number_of_sub_steps < 1:
            _refuse("config_number_of_sub_steps", self.config_number_of_sub_steps,
                    "the split-explicit acoustic loop requires a positive count", "config_number_of_sub_steps>=1")
        if self.config_dynamics_split_steps not in (1, 3):
            _refuse("config_dynamics_split_steps", self.config_dynamics_split_steps,
                    "the drivers implement one and three dynamics subcycles only",
                    "config_dynamics_split_steps=1 or 3")
        if not self.config_split_dynamics_transport:
            _refuse("config_split_dynamics_transport", False,
                    "the GPU path transports scalars after the dynamics subcycles (split transport)",
                    "config_split_dynamics_transport=True")
        if not self.config_scalar_advection:
            _refuse("config_scalar_advection", False, "scalar advection is always active on this path",
                    "config_scalar_advection=True")
        if self.config_scalar_adv_order != 3 or self.config_scalar_vadv_order != 3:
            _refuse("config_scalar_adv_order", (self.config_scalar_adv_order, self.config_scalar_vadv_order),
                    "the path uses the third-order horizontal and vertical fluxes",
                    "config_scalar_adv_order=3 and config_scalar_vadv_order=3")
        if not math.isfinite(self.config_coef_3rd_order) or self.config_coef_3rd_order < 0.0:
            _refuse("config_coef_3rd_order", self.config_coef_3rd_order,
                    "the upwind coefficient must be finite and non-negative", "config_coef_3rd_order=0.25")
        if not math.isfinite(self.config_apvm_upwinding) or self.config_apvm_upwinding < 0.0:
            _refuse("config_apvm_upwinding", self.config_apvm_upwinding,
                    "the APVM branch requires a finite non-negative coefficient", "config_apvm_upwinding>=0")
        if not math.isfinite(self.config_smdiv) or self.config_smdiv < 0.0:
            _refuse("config_smdiv", self.config_smdiv, "the divergence damping coefficient is non-negative",
                    "config_smdiv>=0")
        if self.config_divergence_damping and self.config_smdiv == 0.0:
            _refuse("config_smdiv", 0.0, "the enabled divergence-damping branch would be an accidental no-op",
                    "config_smdiv>0 when config_divergence_damping=True")
        if not self.config_divergence_damping and self.config_smdiv != 0.0:
            _refuse("config_divergence_damping", False, "a nonzero config_smdiv must not be silently ignored",
                    "config_divergence_damping=True when config_smdiv>0")
        if self.config_len_disp < 0.0 or not math.isfinite(self.config_len_disp):
            _refuse("config_len_disp", self.config_len_disp, "a negative filter length is not admitted",
                    "config_len_disp>=0 (zero selects nominalMinDc)")
        mn, mx = self.config_epssm_minimum, self.config_epssm_maximum
        lo, hi = self.config_epssm_transition_bottom_z, self.config_epssm_transition_top_z
        if not (0.0 <= mn <= 1.0) or not (mn <= mx <= 1.0):
            _refuse("config_epssm_minimum", (mn, mx), "the off-centering profile must be ordered in [0,1]",
                    "0<=config_epssm_minimum<=config_epssm_maximum<=1")
        if not (lo >= 0.0 and hi > lo):
            _refuse("config_epssm_transition_top_z", (lo, hi), "the transition must have positive width",
                    "0<=bottom<top")
        # hexcore/driver.py:436-447 (V841DryDycoreConfig validation)
        if not math.isfinite(self.config_xnutr) or not 0.0 <= self.config_xnutr <= 1.0:
            _refuse("config_xnutr", self.config_xnutr, "v8.4.1 requires a finite bounded damping coefficient",
                    "0.0<=config_xnutr<=1.0")
        if not math.isfinite(self.config_zd) or self.config_zd <= 0.0:
            _refuse("config_zd", self.config_zd, "v8.4.1 requires a finite positive damping start height",
                    "config_zd>0")
        if self.config_horiz_mixing not in ("off", "2d_fixed", "2d_smagorinsky"):
            _refuse("config_horiz_mixing", self.config_horiz_mixing,
                    "the v8.4.1 dycore admits off, zero 2d_fixed and 2d_smagorinsky",
                    "config_horiz_mixing='off' or '2d_smagorinsky'")
        # hexcore/mixing_v841.py:71-145 (V841MixingConfig) and driver.py:357-395
        for knob, low, strict in (("config_smagorinsky_coef", 0.0, False), ("config_visc4_2dsmag", 0.0, False),
                                  ("config_del4u_div_factor", 0.0, True), ("config_mpas_cam_coef", 0.0, False)):
            value = float(getattr(self, knob))
            if not math.isfinite(value) or value < low or (strict and value <= low):
                _refuse(knob, value, "the value is outside the Registry domain", f"an admitted finite {knob}")
        if not isinstance(self.config_h_ScaleWithMesh, bool):
            _refuse("config_h_ScaleWithMesh", self.config_h_ScaleWithMesh, "the Registry option is logical",
                    "config_h_ScaleWithMesh=True or False")
        # hexcore/config_v841.py:694-704 upper-damping knobs
        for knob in ("config_number_cam_damping_levels", "config_number_rayleigh_damp_u_levels"):
            value = getattr(self, knob)
            if type(value) is not int or value < 1:
                _refuse(knob, value, "the native damping loop requires a positive integer level count",
                        "a positive integer")
        days = self.config_rayleigh_damp_u_timescale_days
        if not math.isfinite(days) or days <= 0:
            _refuse("config_rayleigh_damp_u_timescale_days", days,
                    "the Rayleigh coefficient divides by a positive timescale", "a finite positive timescale")
        if self.config_horiz_mixing != "2d_smagorinsky":
            for knob in ("config_smagorinsky_coef", "config_visc4_2dsmag"):
                if float(getattr(self, knob)) != 0.0:
                    _refuse(knob, getattr(self, knob), "this Smagorinsky-only knob is inactive when mixing is "
                            "off and must not be silently ignored",
                            f"{knob}=0.0 or config_horiz_mixing='2d_smagorinsky'")
        if self.config_horiz_mixing != "2d_smagorinsky" and self.config_mpas_cam_coef != 0.0:
            _refuse("config_mpas_cam_coef", self.config_mpas_cam_coef,
                    "the CAM floor bounds the Smagorinsky diffusivity and is inactive when mixing is off",
                    "config_mpas_cam_coef=0.0 or config_horiz_mixing='2d_smagorinsky'")
        if not isinstance(self.config_rayleigh_damp_u, bool):
            _refuse("config_rayleigh_damp_u", self.config_rayleigh_damp_u, "the Registry option is logical",
                    "config_rayleigh_damp_u=True or False")
        for knob in ("config_moist_physics", "config_apply_lbcs"):
            if getattr(self, knob):
                _refuse(knob, True, "physics and limited-area branches are outside this path",
                        f"{knob}=False")
        if self.moist_coefficients not in ("native", "dry"):
            _refuse("moist_coefficients", self.moist_coefficients, "unknown coefficient semantics",
                    "moist_coefficients='native' or 'dry'")
        if self.numerics not in ("strict", "fast"):
            _refuse("numerics", self.numerics, "unknown numerics mode", "numerics='strict' or 'fast'")

    @property
    def fct(self) -> bool:
        """RK3 stage uses the monotonic/positive-definite limiter (transport.py:2210)."""
        return bool(self.config_monotonic or self.config_positive_definite)
