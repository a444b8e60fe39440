"""Train and evaluate the learned corrector (``python -m hexdyn.learned_eval``).

Workload: the 40962-cell mesh (bisection level 6), 55 levels, dt = 720 s
with 2 acoustic substeps (120 s), qv plus 2 condensates.  The reduced step
takes a time step ``ratio`` times longer with ``red_substeps`` acoustic
substeps and stands for ``ratio`` full steps (default: dt 1440 s with 3
substeps of 160 s; 2 x ratio substeps keep the 120 s acoustic step); ratio 1
with 1 substep is the reduced-substep design at the same time step.
Training pairs come from ensemble members (the balanced jet with a seeded
0.1 K theta perturbation smoothed over 3 rings) at ``times`` states spread
over the evaluation window; the evaluation starts from a held-out member.  Reported: the networks' training and validation
losses, and over ``days`` simulated days the speed of the plain path, of
the learned path and of the reduced path without correction, the number of
fallbacks, and the day-N errors of the learned and uncorrected paths
against the plain run (RMS of the lowest-level pressure in hPa, normalised
L2 of theta_m).
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

CP_OVER_R = 1004.5 / 287.0
P0 = 100000.0


def _z_mid_padded(case, S: int):
    import torch

    zg = np.asarray(case.vertical.zgrid, dtype=np.float64)
    zm = (0.5 * (zg[:-1] + zg[1:])).astype(np.float32)  # [L][C]
    out = np.zeros((zm.shape[1], S), dtype=np.float32)
    out[:, : zm.shape[0]] = zm.T
    return torch.from_numpy(out).cuda()


def _surface_pressure(drv) -> np.ndarray:
    from .driver import DeviceAtmosphere

    ex = DeviceAtmosphere(drv).logical("exner")[0].cpu().numpy().astype(np.float64)
    return P0 * ex ** CP_OVER_R


def _theta(drv) -> np.ndarray:
    from .driver import DeviceAtmosphere

    return DeviceAtmosphere(drv).logical("theta_m").cpu().numpy().astype(np.float64)


def _state_errors(drv, ref_theta, ref_ps, ref_u):
    from .driver import DeviceAtmosphere

    th = _theta(drv)
    u = DeviceAtmosphere(drv).logical("normal_velocity").cpu().numpy().astype(np.float64)
    return {"theta_rel_l2": float(np.linalg.norm(th - ref_theta) / np.linalg.norm(ref_theta)),
            "ps_rms_pa": float(np.sqrt(np.mean((_surface_pressure(drv) - ref_ps) ** 2))),
            "u_rms": float(np.sqrt(np.mean((u - ref_u) ** 2)))}


def one_step_errors(full, reduced, col, edge, z, case, *, probes: int = 3, spacing: int = 4, ratio: int = 1) -> dict:
    """Errors of one reduced step, with and without correction, against
    ``ratio`` full steps from the same state, at ``probes`` states along a
    full run."""
    from .corrector import LearnedStepper, copy_state, restore, snapshot
    from .driver import DeviceAtmosphere

    stepper = LearnedStepper(full, reduced, col, edge, z, energy_tol=float("inf"), w_growth_tol=float("inf"),
                             ratio=ratio)
    full.set_state(case)
    out = {"uncorrected": [], "corrected": []}
    for _ in range(probes):
        full.step_async(spacing)
        snap = snapshot(full)
        copy_state(reduced, full)
        full.step_async(ratio)
        ref = (_theta(full), _surface_pressure(full),
               DeviceAtmosphere(full).logical("normal_velocity").cpu().numpy().astype(np.float64))
        reduced.step_async(1)
        out["uncorrected"].append(_state_errors(reduced, *ref))
        restore(reduced, snap)
        stepper.reset()
        stepper.step()
        out["corrected"].append(_state_errors(reduced, *ref))
        restore(full, snap)
        full.step_async(ratio)
    full.read_flag()
    mean = lambda rows, k: float(np.mean([r[k] for r in rows]))  # noqa: E731
    return {kind: {k: mean(rows, k) for k in rows[0]} for kind, rows in out.items()}


def run(*, level: int = 6, levels: int = 55, dt: float = 720.0, members: int = 8, times: int = 8,
        samples: int = 60000, epochs: int = 60, days: float = 5.0, seed: int = 0, lr: float = 1e-3,
        mesh=None, ratio: int = 2, red_substeps: int | None = 3) -> dict:
    import torch

    import hexdyn
    from .case import build_case
    from .config import DycoreConfig
    from .corrector import LearnedStepper, TrainedNet, make_pairs
    from .mesh import build_mesh

    t_setup = time.perf_counter()
    mesh = mesh if mesh is not None else build_mesh(level, lloyd=20, seed=0)
    base = build_case(mesh, n_levels=levels, seed=0, n_condensates=2)
    train_cases = [build_case(mesh, n_levels=levels, seed=2000 + i, n_condensates=2, theta_noise=0.1,
                              theta_noise_rings=3, like=base) for i in range(members)]
    eval_case = build_case(mesh, n_levels=levels, seed=9999, n_condensates=2, theta_noise=0.1, theta_noise_rings=3,
                           like=base)
    full_cfg = DycoreConfig(config_dt=dt, config_number_of_sub_steps=2, moist_coefficients="native")
    if red_substeps is None:
        red_substeps = 2 * ratio if ratio > 1 else 1
    red_cfg = DycoreConfig(config_dt=dt * ratio, config_number_of_sub_steps=red_substeps, moist_coefficients="native")
    full = hexdyn.from_case(base, full_cfg, capture_graph=True)
    reduced = hexdyn.from_case(base, red_cfg, capture_graph=True)
    setup_s = time.perf_counter() - t_setup

    n_steps = int(round(days * 86400.0 / dt / ratio)) * ratio  # full steps
    n_red = n_steps // ratio  # reduced steps over the same span
    # training pairs spread over the evaluation window of every member
    between = max(2, n_steps // times - ratio)
    pairs = make_pairs(full, reduced, [(c, None) for c in train_cases], samples=samples, times=times, seed=seed,
                       ratio=ratio, steps_between=between)
    L = levels
    col = TrainedNet(6 * L, 512, 3, 3 * L, seed=seed + 1)
    edge = TrainedNet(4 * L, 256, 3, L, seed=seed + 2)
    col_rec = col.fit(pairs.col_x, pairs.col_y, epochs=epochs, batch=2048, lr=lr, seed=seed)
    edge_rec = edge.fit(pairs.edge_x, pairs.edge_y, epochs=epochs, batch=2048, lr=lr, seed=seed)

    z = _z_mid_padded(base, full.level_stride)
    stream = torch.cuda.current_stream()
    one_step = one_step_errors(full, reduced, col, edge, z, eval_case, probes=3, ratio=ratio)

    # plain full-substep run (whole step as one CUDA graph)
    full.set_state(eval_case)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    full.step_async(n_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    full.read_flag()
    ps_plain, th_plain = _surface_pressure(full), _theta(full)

    # reduced run without correction
    reduced.set_state(eval_case)
    e0.record(stream)
    reduced.step_async(n_red)
    e1.record(stream)
    torch.cuda.synchronize()
    red_ms = e0.elapsed_time(e1)
    red_flag, red_first_bad = 0, None
    try:
        red_flag = reduced.read_flag()
        ps_red, th_red = _surface_pressure(reduced), _theta(reduced)
    except FloatingPointError:
        red_flag = -1
        ps_red, th_red = None, None
        # the first step whose validation flag is set
        reduced.set_state(eval_case)
        for i in range(n_red):
            reduced.step_async(1)
            try:
                reduced.read_flag()
            except FloatingPointError:
                red_first_bad = i
                break

    # learned run: reduced step + networks, full step as fallback
    reduced.set_state(eval_case)
    stepper = LearnedStepper(full, reduced, col, edge, z, ratio=ratio)
    for _ in range(2):  # warm-up of the network workspaces (not counted in the run)
        stepper.correct()
    reduced.set_state(eval_case)
    stepper.reset()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    failure = None
    try:
        for _ in range(n_red):
            stepper.step()
    except FloatingPointError as exc:
        failure = str(exc)
    torch.cuda.synchronize()
    learned_s = time.perf_counter() - t0
    done = stepper.steps
    if failure is None:
        reduced.read_flag()
        ps_l, th_l = _surface_pressure(reduced), _theta(reduced)
    else:
        ps_l, th_l = None, None

    # ablation: the same reduced step, checks and fallback without the networks
    reduced.set_state(eval_case)
    bare = LearnedStepper(full, reduced, col, edge, z, use_network=False, ratio=ratio)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bare_failure = None
    try:
        for _ in range(n_red):
            bare.step()
    except FloatingPointError as exc:
        bare_failure = str(exc)
    torch.cuda.synchronize()
    bare_s = time.perf_counter() - t0
    ps_b, th_b = (_surface_pressure(reduced), _theta(reduced)) if bare_failure is None else (None, None)

    def rms_hpa(a):
        return None if a is None else float(np.sqrt(np.mean((a - ps_plain) ** 2)) / 100.0)

    def theta_l2(a):
        return None if a is None else float(np.linalg.norm(a - th_plain) / np.linalg.norm(th_plain))

    sim_days = n_steps * dt / 86400.0
    per_hour = lambda seconds: sim_days / (seconds / 3600.0)  # noqa: E731
    red_dt = dt * ratio if ratio > 1 else dt
    red_desc = f"dt {red_dt:g} s, {red_substeps} substeps, standing for {ratio} full step(s)"
    return {
        "workload": f"x1.{mesh.n_cells} (bisection level {level}), {levels} levels, dt {dt:g} s, qv + 2 "
                    f"condensates; training members {members} (theta noise 0.1 K), evaluation member held out; "
                    f"reduced step: {red_desc}",
        "ratio": ratio, "reduced_substeps": red_substeps,
        "setup_s": setup_s,
        "pairs": {"state_pairs": pairs.pairs, "full_steps_between_pairs": between, "column_samples": int(len(pairs.col_x)),
                  "edge_samples": int(len(pairs.edge_x)), "seconds": pairs.seconds, "split": "80/20 seeded"},
        "column_net": {"shape": f"{6 * L} -> 512 x3 (GELU) -> {3 * L}", "train_loss_first": col_rec.train_loss[0],
                       "train_loss_last": col_rec.train_loss[-1], "val_loss_initial": col_rec.val_loss_initial,
                       "val_loss_no_correction": col_rec.val_loss_zero,
                       "val_loss": col_rec.val_loss, "optimizer_steps": col_rec.steps, "seconds": col_rec.seconds},
        "edge_net": {"shape": f"{4 * L} -> 256 x3 (GELU) -> {L}", "train_loss_first": edge_rec.train_loss[0],
                     "train_loss_last": edge_rec.train_loss[-1], "val_loss_initial": edge_rec.val_loss_initial,
                       "val_loss_no_correction": edge_rec.val_loss_zero,
                     "val_loss": edge_rec.val_loss, "optimizer_steps": edge_rec.steps, "seconds": edge_rec.seconds},
        "one_step_vs_full_step": one_step,
        "eval_steps": n_steps, "eval_days": sim_days,
        "plain": {"days_per_hour": per_hour(plain_ms / 1000.0), "ms_per_step": plain_ms / n_steps},
        "reduced_uncorrected": {"days_per_hour": per_hour(red_ms / 1000.0), "ms_per_step": red_ms / n_red,
                                "validation_flag": red_flag, "first_flagged_step": red_first_bad,
                                "ps_rms_hpa": rms_hpa(ps_red),
                                "theta_rel_l2": theta_l2(th_red)},
        "reduced_with_checks_no_network": {
            "days_per_hour": (bare.steps * red_dt / 86400.0) / (bare_s / 3600.0), "steps_done": bare.steps,
            "failure": bare_failure, "fallbacks": bare.fallbacks, "first_fallback_step": bare.first_fallback,
            "ps_rms_hpa": rms_hpa(ps_b), "theta_rel_l2": theta_l2(th_b)},
        "learned": {"days_per_hour": (done * red_dt / 86400.0) / (learned_s / 3600.0),
                    "ms_per_step": 1000.0 * learned_s / max(done, 1),
                    "speedup_vs_plain": (plain_ms / n_steps * (red_dt / dt)) / (1000.0 * learned_s / max(done, 1)),
                    "steps_done": done, "failure": failure, "fallbacks": stepper.fallbacks,
                    "first_fallback_step": stepper.first_fallback, "reduced_steps_flagged": stepper.flagged,
                    "energy_rel_change_median": float(np.nanmedian(stepper.last_rel)),
                    "energy_rel_change_p90": float(np.nanpercentile(stepper.last_rel, 90)),
                    "w_rms_growth_p90": float(np.nanpercentile(stepper.last_growth, 90)),
                    "checks": "fallback when the reduced step's flag is set, the energy changes by > 1e-4 relative, "
                              "or the RMS of w grows by > 5 % in the step",
                    "ps_rms_hpa": rms_hpa(ps_l), "theta_rel_l2": theta_l2(th_l)},
    }


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--members", type=int, default=8)
    ap.add_argument("--samples", type=int, default=60000)
    ap.add_argument("--times", type=int, default=8, help="pair sample times per member over the window")
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--days", type=float, default=5.0)
    ap.add_argument("--ratio", type=int, default=2, help="reduced time step / full time step")
    ap.add_argument("--red-substeps", type=int, default=3,
                    help="acoustic substeps of the reduced step (0: 2 x ratio, or 1 at ratio 1)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    res = run(level=a.level, members=a.members, samples=a.samples, epochs=a.epochs, days=a.days, ratio=a.ratio,
              times=a.times, red_substeps=a.red_substeps or None)
    text = json.dumps(res, indent=1)
    print(text)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
