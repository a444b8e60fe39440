"""Generate the golden step fixtures by running the reference itself.

Runs the reference's CPU dycore authority (``hexcore.driver.DryDycoreDriver``
with ``V841DryDycoreConfig``, gpuwm-hex 0.5.0) on small synthetic cases built
by ``hexdyn.case`` and stores inputs and outputs as ``.npz`` fixtures.  It
needs the reference checkout, given as the first argument or in the
``HEXDYN_REFERENCE_ROOT`` environment variable, and therefore runs only where
that exists; the fixtures it writes are what the tests read.

At the two large sizes (2562 cells x 55 levels with qv; 40962 cells x 55
levels with qv and 5 condensates, the throughput workload) it stores SHA-256
digests of every input array and every output field instead of the arrays
(``digests_<name>.json``): the inputs are rebuilt by ``hexdyn.case`` where the
tests run, and a test compares digests only where the rebuilt inputs have the
recorded digest (NumPy's transcendental functions take SIMD paths that depend
on the host CPU, so another host may build other input bits).

Harness: a two-class ``netCDF4`` stub and a ``gpuwm``
stub are put on ``sys.path`` (the reference imports them only for file I/O
and LES route checks); the advection coefficients, vertical grid and terrain
metrics the reference would take from its Rust engines are supplied by the
case builder.  The ``native`` fixture wraps the driver so that
``_advance_dynamics_subcycle`` receives the moist coefficients of every
carried scalar (``hexcore/regional_v841.py:1180``), which is what native MPAS
and the reference's CUDA driver apply with physics off.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT [fixture names ...]
       HEXDYN_REFERENCE_ROOT=... python tests/golden/make_golden.py [fixture names ...]
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "gpuwm-hex_b200"))
sys.path.insert(0, str(HERE.parent))

from fixtures import array_digest, inputs_digest, reference_stub_dir  # noqa: E402
from hexdyn.case import build_case, case_arrays  # noqa: E402
from hexdyn.mesh import build_mesh  # noqa: E402

CASES = {
    # name: (mesh level, levels, condensates, dt, sub steps, steps, native moist steps)
    "l2_L12": (2, 12, 1, 1800.0, 2, 2, 1),
    "l3_L20": (3, 20, 0, 1800.0, 2, 1, 0),
    # qv + 5 condensates, the tracer count of the throughput workload
    "l2_L12_t6": (2, 12, 5, 1800.0, 2, 2, 2),
}

# The same inputs with the first 4 and 5 scalars only (every scalar count
# from 4 to 6 then has reference outputs): name -> (base, scalars kept,
# steps); both moist-coefficient semantics.
SCALAR_VARIANTS = {
    "l2_L12_t4": ("l2_L12_t6", 4, 2),
    "l2_L12_t5": ("l2_L12_t6", 5, 2),
}

# Digest-only runs at full size, native moist coefficients:
# name -> (mesh level, levels, condensates, dt, sub steps, steps)
DIGESTS = {
    "c1": (4, 55, 0, 1800.0, 2, 2),
    "c2": (6, 55, 5, 720.0, 2, 1),
}

# Configuration variants on the inputs of a base case (outputs only; the
# fixture names its base): name -> (base, sub steps, monotonic, apvm, steps,
# scalars kept, xnutr, time integration order)
VARIANTS = {
    "l2_L12_sub1": ("l2_L12", 1, True, 0.5, 2, None, 0.0, 3),     # one acoustic substep per stage
    "l2_L12_sub4": ("l2_L12", 4, True, 0.5, 2, None, 0.0, 3),     # (1, 2, 4) substeps
    "l2_L12_nomono": ("l2_L12", 2, False, 0.5, 2, None, 0.0, 3),  # standard RK3 transport
    "l2_L12_noapvm": ("l2_L12", 2, True, 0.0, 1, None, 0.0, 3),   # no APVM upwinding
    "l2_L12_notracers": ("l2_L12", 2, True, 0.5, 2, 0, 0.0, 3),   # no scalars at all
    "l2_L12_xnutr": ("l2_L12", 2, True, 0.5, 2, None, 0.2, 3),    # implicit w damping above 22 km
    "l2_L12_rk2": ("l2_L12", 2, True, 0.5, 2, None, 0.0, 2),      # order-2 schedule, (1, 1, 2) substeps
    "l2_L12_rk2_sub4": ("l2_L12", 4, True, 0.5, 1, None, 0.0, 2), # order 2, (2, 2, 4) substeps
}

# 2-D Smagorinsky horizontal mixing (v8.4.1 deformation form,
# hexcore/mixing_v841.py): name -> (base, steps, coefficient, visc4,
# del4u_div_factor).  The fixture also stores the reference's deformation
# weights of the mesh.
SMAG_VARIANTS = {
    "l2_L12_smag": ("l2_L12", 2, 0.125, 0.05, 10.0),
}


def main(reference_root: str, *only: str) -> None:
    if not (Path(reference_root) / "tree" / "src" / "hexcore").is_dir():
        raise SystemExit(f"{reference_root!r} holds no tree/src/hexcore: give the reference checkout")
    sys.path.insert(0, reference_stub_dir())
    sys.path.insert(0, str(Path(reference_root) / "tree" / "src"))
    from hexcore.config_v841 import V841DryDycoreConfig
    from hexcore.driver import DryDycoreDriver, DryReferenceState, TerrainMetrics
    from hexcore.dynamics_v841 import V841ReferenceWindProfiles
    from hexcore.regional_v841 import compute_moist_coefficients
    from hexcore.state import PrognosticState
    from hexcore.transport import AdvectionCoefficients
    from hexcore.vertical import VerticalGrid

    class NativeMoistDriver(DryDycoreDriver):
        """Moist coefficients of every carried scalar in each subcycle.  With
        split transport the subcycle's scalars are the step's, so this equals
        forming them once per step as native MPAS does."""

        def _advance_dynamics_subcycle(self, state, **kw):
            qtot, cqw, cqu = compute_moist_coefficients(
                state.scalars, moist_indices=range(state.scalars.shape[0]),
                cells_on_edge_remapped=np.asarray(self.mesh.cellsOnEdge), nlev=self.nlev)
            kw.update(moist_cqu=cqu, moist_cqw=cqw, moist_qtot=qtot)
            return super()._advance_dynamics_subcycle(state, **kw)

    def run(cls, mesh, vg, ref, cfg, ac, tm, wp, case, nsteps, label, out):
        drv = cls(mesh, vg, ref, cfg, advection_coefficients=ac, terrain_metrics=tm, reference_wind_profiles=wp)
        state = PrognosticState(case.rho.copy(), case.rho_theta.copy(), case.rho_u.copy(), case.rho_w.copy(),
                                case.scalars.copy(), 0.0)
        side = None
        for step in range(1, nsteps + 1):
            res = drv.step(state, saved_diagnostics=side)
            state, side = res.state, res.saved_diagnostics
            for k in ("rho", "rho_theta", "rho_u", "rho_w", "scalars"):
                out[f"{label}.step{step}.{k}"] = np.asarray(getattr(state, k))
            for k in ("theta_m", "exner", "density_perturbation", "rho_theta_perturbation",
                      "pressure_perturbation", "normal_velocity", "vertical_velocity"):
                out[f"{label}.step{step}.side.{k}"] = np.asarray(getattr(side, k))

    def reference_inputs(case):
        vg = VerticalGrid(**{k: getattr(case.vertical, k) for k in case.vertical.__dataclass_fields__})
        ref = DryReferenceState(case.rho_base, case.rho_theta_base, case.pressure_base, case.exner_base)
        tm = TerrainMetrics(case.zb_cell, case.zb3_cell)
        ac = AdvectionCoefficients(case.adv_coefs, case.adv_coefs_3rd, case.n_adv_cells_for_edge,
                                   case.adv_cells_for_edge, 3, None)
        wp = V841ReferenceWindProfiles(case.u_init, case.v_init)
        return vg, ref, ac, tm, wp

    def base_config(dt, nsub):
        return V841DryDycoreConfig(config_dt=dt, config_number_of_sub_steps=nsub, config_dynamics_split_steps=3,
                                   config_split_dynamics_transport=True, config_monotonic=True,
                                   config_positive_definite=False, config_coef_3rd_order=0.25,
                                   config_apvm_upwinding=0.5)

    for name, (level, nlev, ncond, dt, nsub, nsteps) in DIGESTS.items():
        if name not in only:  # minutes to hours of CPU: only on request
            continue
        t0 = time.time()
        mesh = build_mesh(level, lloyd=20, seed=0)
        case = build_case(mesh, n_levels=nlev, seed=0, n_condensates=ncond)
        arrays = case_arrays(case)
        vg, ref, ac, tm, wp = reference_inputs(case)
        out = {}
        run(NativeMoistDriver, mesh, vg, ref, base_config(dt, nsub), ac, tm, wp, case, nsteps, "native", out)
        record = {"case": {"mesh_level": level, "lloyd": 20, "seed": 0, "levels": nlev, "condensates": ncond,
                           "dt": dt, "sub_steps": nsub, "steps": nsteps, "moist_coefficients": "native"},
                  "made_by": "hexcore.driver.DryDycoreDriver (V841DryDycoreConfig), native moist coefficients",
                  "inputs_sha256": inputs_digest(arrays),
                  "inputs": {k: array_digest(v) for k, v in sorted(arrays.items())},
                  "outputs": {k: array_digest(v) for k, v in sorted(out.items())},
                  "reference_seconds": round(time.time() - t0, 1)}
        path = HERE / f"digests_{name}.json"
        path.write_text(json.dumps(record, indent=1) + "\n")
        print(f"{path.name}: {len(out)} output digests in {time.time() - t0:.1f}s")

    variants = {**VARIANTS, **SMAG_VARIANTS, **SCALAR_VARIANTS}
    for name, (level, nlev, ncond, dt, nsub, nsteps, native_steps) in CASES.items():
        if only and name not in only and not any(v[0] == name for k, v in variants.items() if k in only):
            continue
        t0 = time.time()
        mesh = build_mesh(level, lloyd=20, seed=0)
        case = build_case(mesh, n_levels=nlev, seed=0, n_condensates=ncond)
        vg, ref, ac, tm, wp = reference_inputs(case)
        cfg = base_config(dt, nsub)
        out = {f"in.{k}": v for k, v in case_arrays(case).items()}
        out["config.dt"] = dt
        out["config.n_sub_steps"] = nsub
        if not only or name in only:
            runs = [("dry", DryDycoreDriver, nsteps)] + ([("native", NativeMoistDriver, native_steps)]
                                                         if native_steps else [])
            for label, cls, n in runs:
                run(cls, mesh, vg, ref, cfg, ac, tm, wp, case, n, label, out)
            path = HERE / f"step_{name}.npz"
            np.savez_compressed(path, **out)
            print(f"{path.name}: {path.stat().st_size / 1e6:.2f} MB in {time.time() - t0:.1f}s")
        for vname, (base, vsub, mono, apvm, vsteps, keep, xnutr, order) in VARIANTS.items():
            if base != name or (only and vname not in only):
                continue
            t0 = time.time()
            vcfg = V841DryDycoreConfig(config_dt=dt, config_number_of_sub_steps=vsub, config_dynamics_split_steps=3,
                                       config_split_dynamics_transport=True, config_monotonic=mono,
                                       config_positive_definite=False, config_coef_3rd_order=0.25,
                                       config_apvm_upwinding=apvm, config_xnutr=xnutr, config_zd=22000.0,
                                       config_time_integration_order=order)
            vout = {"base": np.array(base), "config.dt": dt, "config.n_sub_steps": vsub,
                    "config.monotonic": int(mono), "config.apvm_upwinding": apvm}
            if order != 3:
                vout["config.order"] = order
            if xnutr:
                vout["config.xnutr"] = xnutr
                vout["config.zd"] = 22000.0
            vcase = case
            if keep is not None:
                import dataclasses

                vcase = dataclasses.replace(case, scalars=case.scalars[:keep].copy())
                vout["config.n_scalars"] = keep
            run(DryDycoreDriver, mesh, vg, ref, vcfg, ac, tm, wp, vcase, vsteps, "dry", vout)
            path = HERE / f"step_{vname}.npz"
            np.savez_compressed(path, **vout)
            print(f"{path.name}: {path.stat().st_size / 1e6:.2f} MB in {time.time() - t0:.1f}s")
        for vname, (base, vsteps, smag, visc4, divf) in SMAG_VARIANTS.items():
            if base != name or (only and vname not in only):
                continue
            import os

            from hexcore import numerics
            from hexcore.mixing_v841 import initialize_deformation_weights_v841

            # the reference's strict geometry (glibc sinf/cosf, correctly
            # rounded asinf/atan2f), built from its shipped sources into a
            # temporary cache
            os.environ.setdefault("HEXCORE_NATIVE_CPU_CACHE", tempfile.mkdtemp(prefix="hexdyn_ref_native_"))
            numerics.set_mode("strict", source="make_golden")
            t0 = time.time()
            # the v8.4.1 deformation weights need the spherical-mesh attributes
            mesh.attrs = {"on_a_sphere": "YES", "sphere_radius": float(mesh.arrays["sphere_radius"])}
            vcfg = V841DryDycoreConfig(config_dt=dt, config_number_of_sub_steps=nsub, config_dynamics_split_steps=3,
                                       config_split_dynamics_transport=True, config_monotonic=True,
                                       config_positive_definite=False, config_coef_3rd_order=0.25,
                                       config_apvm_upwinding=0.5, config_horiz_mixing="2d_smagorinsky",
                                       config_smagorinsky_coef=smag, config_visc4_2dsmag=visc4,
                                       config_del4u_div_factor=divf, config_len_disp=0.0, config_mpas_cam_coef=0.0)
            vout = {"base": np.array(base), "config.dt": dt, "config.n_sub_steps": nsub,
                    "config.smagorinsky_coef": smag, "config.visc4_2dsmag": visc4, "config.del4u_div_factor": divf}
            w = initialize_deformation_weights_v841(mesh, dtype=np.float32)
            vout["mix.coef_c2"], vout["mix.coef_s2"], vout["mix.coef_cs"] = w.coef_c2, w.coef_s2, w.coef_cs
            run(DryDycoreDriver, mesh, vg, ref, vcfg, ac, tm, wp, case, vsteps, "dry", vout)
            path = HERE / f"step_{vname}.npz"
            np.savez_compressed(path, **vout)
            print(f"{path.name}: {path.stat().st_size / 1e6:.2f} MB in {time.time() - t0:.1f}s")
        for vname, (base, keep, vsteps) in SCALAR_VARIANTS.items():
            if base != name or (only and vname not in only):
                continue
            import dataclasses

            t0 = time.time()
            vcase = dataclasses.replace(case, scalars=case.scalars[:keep].copy())
            vout = {"base": np.array(base), "config.dt": dt, "config.n_sub_steps": nsub, "config.n_scalars": keep}
            run(DryDycoreDriver, mesh, vg, ref, cfg, ac, tm, wp, vcase, vsteps, "dry", vout)
            run(NativeMoistDriver, mesh, vg, ref, cfg, ac, tm, wp, vcase, vsteps, "native", vout)
            path = HERE / f"step_{vname}.npz"
            np.savez_compressed(path, **vout)
            print(f"{path.name}: {path.stat().st_size / 1e6:.2f} MB in {time.time() - t0:.1f}s")


if __name__ == "__main__":
    args = sys.argv[1:]
    env_root = os.environ.get("HEXDYN_REFERENCE_ROOT")
    if args and (Path(args[0]) / "tree").is_dir():
        root, names = args[0], args[1:]
    elif env_root:
        root, names = env_root, args
    else:
        raise SystemExit("usage: make_golden.py REFERENCE_ROOT [names...] (or set HEXDYN_REFERENCE_ROOT)")
    main(root, *names)
