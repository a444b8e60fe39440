"""Benchmark: simulated days per wall-hour of the MPAS-A v8.4.2 dry-plus-tracer
dycore step on the x1.40962 mesh, 55 levels, FP32.

Workload (default): the bisected icosahedron at level 6 (40962 cells, 122880
edges, 81920 vertices), 55 levels to 30 km, the balanced jet with terrain,
qv plus 5 condensate tracers, dt = 720 s, 2 acoustic sub-steps, split-3 RK3,
monotonic FCT, native moist coefficients, strict numerics (bit-identical to
the reference authority), the whole large step replayed as one CUDA graph.
Synthetic inputs stand in for the reference's x1.40962 grid/init files.

One JSON line is printed by rank 0.  ``--impl reference`` times the
reference's CPU step path restated in NumPy (the oracle) on the host cores
on the same workload instead.

Launch: python bench.py [--gpus N --steps K --warmup W]; for N > 1 under
torch.distributed.run, one process per GPU, each advancing its own replica
(the single-instance step does not shard: replicas only).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "gpuwm-hex_b200"))
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

LEVEL_DT = {4: 1800.0, 5: 1440.0, 6: 720.0, 7: 360.0}
METRIC = "simulated days/wall-hour, x1.40962 55L FP32: plain vs batched vs learned-corrected"
PEAK_FALLBACK_GBS = 6650.0


def parse() -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--levels", type=int, default=55)
    ap.add_argument("--condensates", type=int, default=5)
    ap.add_argument("--numerics", default="strict", choices=["strict", "fast"])
    ap.add_argument("--smagorinsky", action="store_true",
                    help="2-D Smagorinsky horizontal mixing on (coefficient 0.125, visc4 0.05); off in the "
                         "workload's configuration")
    ap.add_argument("--renumber", default="none", choices=["none", "random", "hilbert"],
                    help="renumber the mesh entities before the run (the builder already numbers them along a "
                         "Hilbert curve; random scrambles them, hilbert re-orders a scrambled copy)")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--autotune", default="on", choices=["on", "off"],
                    help="choose the block size of every kernel by timing before capturing the graph")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget-s", type=float, default=60.0)
    ap.add_argument("--batched", default="on", choices=["on", "off"],
                    help="also time the uneven ensemble (24 x 10242-cell members at 1440 s + 16 x 40962-cell "
                         "members at 720 s) batched and looped")
    ap.add_argument("--batch-periods", type=int, default=4, help="timed 1440 s periods of the ensemble leg")
    ap.add_argument("--partition-ranks", type=int, default=2,
                    help="ranks of the partitioned-instance leg, emulated on one GPU (0 or 1: off)")
    ap.add_argument("--learned", default="on", choices=["on", "off"],
                    help="also train the learned corrector (shortened) and time the corrected path for half a day")
    return ap.parse_args()


# ------------------------------------------------------------- byte model
def kernel_bytes(name: str, C: int, E: int, V: int, L: int, T: int, maxE: int = 6, advW: int = 10,
                 damping: bool = False) -> int:
    """Algorithmic bytes of one launch: each distinct array read or written,
    times the extent it touches (L levels or L+1 interfaces per entity), 4 B,
    counted once; connectivity/coefficient tables counted once.  ``damping``:
    the implicit w damping profile is not zero (config_xnutr > 0), so the
    acoustic cell pass also reads dss, rho_zz and w."""
    cl, ci, el, vl = C * L, C * (L + 1), E * L, V * L
    tcl, tel = T * C * L, T * E * L
    conn_c = C * maxE * 3 + C * 2          # eoc, csign (+ coc/voc) and deg, inv_area
    conn_e = E * 2 + E * 4                 # coe and per-edge metrics
    adv = E * advW * 3                     # adv, adv3, adv_cells
    zb = 2 * C * maxE * (L + 1)
    words = {
        "k_diag_vertex": el + 2 * vl + V * 8,
        "k_diag_cell": el + 2 * vl + 2 * cl + conn_c,
        "k_diag_edge": 3 * el + vl + cl + conn_e,                  # u, cached v, pv_edge out
        "k_diag_edge_v": 3 * el + vl + cl + conn_e + E * 24,       # u (+ neighbours), v out, pv_edge out
        "k_moist_cell": tcl + 2 * cl,
        "k_clamp_scalars": 2 * tcl,
        "k_moist_edge": tcl + el + conn_e,
        "k_euler_edge": 3 * el + 4 * cl + conn_e,
        "k_euler_cell": el + 2 * ci + 5 * cl + conn_c,
        "k_hdiv": el + cl + conn_c,
        "k_edge_adv": 3 * el + cl + ci + adv,
        "k_tend_u": 6 * el + ci + 3 * cl + conn_e + E * 24,          # + the first substep's ru_p, ru_avg out
        "k_tend_cell": 5 * el + 5 * ci + 4 * cl + zb + conn_c,
        "k_vcoef": 9 * cl + 6 * cl + ci,
        # the two launches below run only in builds without the acoustic fusions
        "k_ac_edge_first": 3 * el,                                 # tend_ru in; ru_p, ru_avg out
        "k_ac_edge": 7 * el + 6 * cl + conn_e,                     # damping of n-1 + update n
        "k_ac_edge_damp": 2 * el + 3 * cl + conn_e,                # damping only
        # (+ dss, rho_zz, w when the damping profile is not zero)
        "k_ac_cell_first": el + 10 * cl + 6 * ci + conn_c + (2 * cl + ci if damping else 0),  # old perts zero
        "k_ac_cell": el + 14 * cl + 8 * ci + conn_c + (2 * cl + ci if damping else 0),
        # + the last substep's damping: ru_p out, rtpp_new and theta_m at both
        # cells (rtpp_old only after a stage of several substeps: not counted)
        "k_recover_edge": 8 * el + 5 * cl + conn_e,
        "k_recover_cell": el + 16 * cl + 7 * ci + zb + conn_c,       # + the next stage's hdiv
        "k_tr_edge": (tcl + tel) + el + adv,
        "k_tr_edge_mono": (tcl + tel) + el + adv,
        "k_tr_std": 3 * tcl + tel + 2 * cl + el + ci + conn_c,
        "k_fct_target": 2 * cl + el + ci + conn_c,
        "k_fct_cell1": 5 * tcl + T * ci + tel + 2 * cl + el + ci + conn_c,   # + vertical fluxes out
        "k_fct_edge": 3 * tcl + 2 * tel + el + conn_e,
        "k_fct_cell2": 4 * tcl + T * ci + tel + cl + conn_c,             # vertical fluxes in
        # 2-D Smagorinsky mixing (bench --smagorinsky), once per subcycle
        "k_smag_kdiff": 2 * el + cl + 3 * C * maxE + conn_c,
        "k_mix_edge2": 3 * cl + vl + 3 * el + conn_e + E * 2,
        "k_mix_cell2": 3 * cl + 3 * ci + 2 * cl + conn_c,
        "k_mix_lap_vertex": el + vl + V * 6,
        "k_mix_lap_cell": el + cl + conn_c,
        "k_mix_edge4": 2 * cl + vl + 2 * el + conn_e,
        "k_mix_cell4": 4 * ci + 3 * cl + conn_c,
    }
    if name not in words:
        return 0
    return 4 * int(words[name])


def measured_peak() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return PEAK_FALLBACK_GBS, "fallback"


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples (every 200 ms) of the SM clock and throttle reasons."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[4]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [r for r in rows if r[2] > 0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in loaded for i, v in enumerate(r[3]) if v.lower().startswith("active")})
        return {"sm_mhz": float(np.median([r[0] for r in loaded])), "sm_max_mhz": max(r[1] for r in loaded),
                "reasons": reasons, "samples": len(loaded)}


# ---------------------------------------------------------------- helpers
def build_workload(args):
    from hexdyn.case import build_case
    from hexdyn.mesh import build_mesh

    mesh = build_mesh(args.level, lloyd=20, seed=0)
    case = build_case(mesh, n_levels=args.levels, seed=0, n_condensates=args.condensates)
    if getattr(args, "renumber", "none") != "none":
        from hexdyn import reorder
        from hexdyn.case import case_arrays

        ren = reorder.random_order(case_arrays(case), seed=0)
        case = reorder.renumber_case(case, ren)
        if args.renumber == "hilbert":
            case = reorder.renumber_case(case, reorder.hilbert_order(case_arrays(case)))
    return case


def workload_config(args, case) -> dict:
    m = case.mesh
    return {
        "workload": f"x1.{m.n_cells} synthetic icosahedral Voronoi mesh (bisection level {args.level}, 20 Lloyd "
                    f"iterations), {args.levels} levels to 30 km, balanced jet + terrain, "
                    f"{case.scalars.shape[0]} tracers, dt={LEVEL_DT[args.level]:g} s, 2 acoustic sub-steps, "
                    "split-3 RK3, monotonic FCT",
        "cells": m.n_cells, "edges": m.n_edges, "vertices": m.n_vertices, "levels": args.levels,
        "tracers": int(case.scalars.shape[0]), "dt_s": LEVEL_DT[args.level], "path": "plain",
        "numerics": args.numerics, "moist_coefficients": "native",
        "l2": "inputs larger than L2 (per-step working set > 126 MB)",
        "graph": not args.no_graph,
        "horizontal_mixing": "2d_smagorinsky (0.125, visc4 0.05)" if getattr(args, "smagorinsky", False) else "off",
        "numbering": {"none": "Hilbert curve of the generators (mesh builder)", "random": "random permutation",
                      "hilbert": "random permutation re-ordered by hexdyn.reorder.hilbert_order"}[
                          getattr(args, "renumber", "none")],
    }


def oracle_time_per_step(case, dt: float, budget_s: float, max_steps: int) -> tuple[float, int]:
    from hexdyn.case import case_arrays
    from oracle.dycore import OracleConfig, OracleDycore, State

    arr = case_arrays(case)
    orc = OracleDycore(arr, OracleConfig(dt=dt, n_sub_steps=2, moist="native"))
    st = State(*(np.asarray(arr[k]).copy() for k in ("rho", "rho_theta", "rho_u", "rho_w", "scalars")))
    sd = None
    times = []
    t_all = time.perf_counter()
    while len(times) < max_steps:
        t0 = time.perf_counter()
        st, sd = orc.step(st, sd)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > budget_s:
            break
    return float(np.mean(times)), len(times)


def cores_used() -> int:
    """Threads the CPU baseline computes on: the oracle is NumPy, whose
    elementwise FP32 kernels run on the calling thread (the step uses no
    BLAS), so one."""
    return 1


def host_box() -> dict:
    """The host the CPU baseline ran on: logical CPUs, the affinity mask the
    process may use, and the thread-count variables that NumPy, BLAS and the
    reference's host copy helpers read."""
    try:
        affinity = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        affinity = None
    env = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS",
                                          "GPUWM_HEX_HOST_COPY_THREADS")}
    cpu = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                cpu = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "affinity_cpus": affinity, "cpu": cpu, "env": env}


CPU_PATH = ("the oracle: a vectorised NumPy FP32 restatement of the reference's DryDycoreDriver.step "
            "(hexcore/driver.py:3314), bit-identical to it, single-threaded; the reference's own NumPy path "
            "is also single-threaded and was 18x slower at 2562 cells")


# Launch labels that run the same kernel function with other arguments.
KERNEL_OF_LABEL = {"k_ac_edge_first": "kv_ac_edge", "k_ac_edge_damp": "kv_ac_edge", "k_ac_cell_first": "kv_ac_cell",
                   "k_diag_edge_v": "kv_diag_edge", "k_tr_edge_mono": "kv_tr_edge"}


def kernel_of(label: str) -> str:
    """The kernel function a launch label runs (``k_x`` -> ``kv_x``)."""
    return KERNEL_OF_LABEL.get(label, "kv_" + label[2:] if label.startswith("k_") else label)


def by_kernel(kernels: dict, prof_steps: int) -> dict:
    """Per-label profile entries merged per kernel function: launches, share,
    average launch time and algorithmic bytes per launch (launch-weighted)."""
    out: dict[str, dict] = {}
    for label, k in kernels.items():
        name = kernel_of(label)
        n = k["launches_per_step"]
        m = out.setdefault(name, {"labels": [], "launches_per_step": 0.0, "share": 0.0, "_us": 0.0, "_bytes": 0.0})
        m["labels"].append(label)
        m["launches_per_step"] += n
        m["share"] += k["share"]
        m["_us"] += k["avg_us"] * n
        m["_bytes"] += (k["bytes"] or 0) * n
    for m in out.values():
        n = m["launches_per_step"]
        m["avg_us"] = m.pop("_us") / n
        m["bytes"] = m.pop("_bytes") / n
        m["gbs"] = m["bytes"] / (m["avg_us"] * 1e-6) / 1e9 if m["bytes"] else None
    return out


# ------------------------------------------------------------- ensembles
ENSEMBLE = ((5, 24, 1440.0, 1), (6, 16, 720.0, 2))  # (level, members, dt, steps per 1440 s period)


def build_ensemble(args, plain_case):
    """The uneven ensemble: per mesh, members that share its geometry and
    differ in a seeded theta perturbation (0.1 K, smoothed over 3 rings) and
    tracer blobs; qv plus 2 condensates."""
    from hexdyn.case import build_case
    from hexdyn.mesh import build_mesh

    groups = []
    for gi, (level, n, dt, per) in enumerate(ENSEMBLE):
        mesh = plain_case.mesh if level == args.level else build_mesh(level, lloyd=20, seed=0)
        base = plain_case if level == args.level else build_case(mesh, n_levels=args.levels, seed=0,
                                                                   n_condensates=2)
        members = [build_case(mesh, n_levels=args.levels, seed=1000 * (gi + 1) + i, n_condensates=2,
                              theta_noise=0.1, theta_noise_rings=3, like=base) for i in range(n)]
        groups.append((members, dt, per))
    return groups


def run_ensemble(args, stream, dist, world: int, rank: int, plain_case) -> dict:
    """Member-days per hour of the uneven ensemble, batched (one ensemble
    handle per time step, both advanced by hexdyn_step_batched: every kernel
    launch covers all members of a group, the groups run concurrently) and
    looped (each member its own single-instance graph, one after another).
    Members are spread over ranks by cell count (no per-step collective)."""
    import torch

    import hexdyn
    from hexdyn.config import DycoreConfig
    from hexdyn.ensemble import HexEnsemble, assign_members, step_batched

    groups = build_ensemble(args, plain_case)
    flat = [(gi, m) for gi, (members, _, _) in enumerate(groups) for m in range(len(members))]
    cells = [groups[gi][0][m].mesh.n_cells for gi, m in flat]
    mine = set(assign_members(cells, world)[rank])
    cfgs = [DycoreConfig(config_dt=dt, config_number_of_sub_steps=2, moist_coefficients="native",
                         numerics=args.numerics) for _, dt, _ in groups]
    my_groups = []
    for gi, (members, dt, per) in enumerate(groups):
        sel = [members[m] for i, (g, m) in enumerate(flat) if g == gi and i in mine]
        my_groups.append((sel, per))
    n_members = sum(len(sel) for sel, _ in my_groups)
    periods, warm = max(1, args.batch_periods), 2

    def timed(run):
        for _ in range(warm):
            run()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(periods):
            run()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # looped: every member its own single-instance driver (whole step as a graph)
    singles = [(hexdyn.from_case(c, cfgs[gi]), per) for gi, (sel, per) in enumerate(my_groups) for c in sel]
    for drv, _ in singles:
        if args.autotune == "on":
            drv.autotune(1)
        drv.capture_graph()

    def looped():
        for drv, per in singles:
            drv.step_async(per)

    loop_ms = timed(looped)
    loop_flags = [drv.read_flag() for drv, _ in singles]
    launches_single = sum(drv.receipt().launches_per_step * per for drv, per in singles)
    for drv, _ in singles:
        drv.close()
    del singles
    # batched: one ensemble per time step, both groups per call
    ens = [(HexEnsemble.from_cases(sel, cfgs[gi]), per) for gi, (sel, per) in enumerate(my_groups) if sel]
    for e, _ in ens:
        if args.autotune == "on":
            e.autotune(1)
        e.capture_graph()

    def batched():
        step_batched([e for e, _ in ens], [per for _, per in ens], read_flags=False, stream=stream)

    batch_ms = timed(batched)
    batch_flags = [e.read_flag() for e, _ in ens]
    launches_batched = sum(e.receipt().launches_per_step * per for e, per in ens)
    for e, _ in ens:
        e.close()
    total_members = len(flat)
    period_days = 1440.0 / 86400.0
    batched_value = total_members * periods * period_days / (batch_ms / 1000.0 / 3600.0)
    looped_value = total_members * periods * period_days / (loop_ms / 1000.0 / 3600.0)
    return {
        "metric": "member-days/hour", "value": batched_value, "looped_value": looped_value,
        "speedup_vs_looped": batched_value / looped_value,
        "ms_per_period": batch_ms / periods, "looped_ms_per_period": loop_ms / periods,
        "periods": periods, "warmup": warm, "members": total_members, "members_this_rank": n_members,
        "workload": "uneven ensemble: 24 members on the 10242-cell mesh (dt 1440 s, 1 step per period) + 16 "
                    "members on the 40962-cell mesh (dt 720 s, 2 steps per period), 55 levels, qv + 2 "
                    "condensates, theta noise 0.1 K over 3 rings; a period is 1440 simulated seconds",
        "gpu_launches_per_period": int(launches_batched), "looped_gpu_launches_per_period": int(launches_single),
        "validation_flags": [*loop_flags, *batch_flags],
    }


# ------------------------------------------------------ learned corrector
def run_learned(args, plain_case) -> dict:
    """The learned-corrector path on this mesh (qv + 2 condensates, plain dt
    720 s; reduced step dt 1440 s with 3 substeps standing for two plain
    steps): pairs from 4 members, 30 epochs per network, then half a
    simulated day of the plain, reduced-with-checks and learned paths from a
    held-out member.  The 5-day evaluation is ``python -m hexdyn.learned_eval``."""
    from hexdyn.learned_eval import run

    res = run(level=args.level, levels=args.levels, members=4, epochs=30, days=0.5, mesh=plain_case.mesh)
    lp = res["learned"]
    return {
        "metric": "simulated days/hour", "value": lp["days_per_hour"], "plain_value": res["plain"]["days_per_hour"],
        "speedup_vs_plain": lp["speedup_vs_plain"], "fallbacks": lp["fallbacks"], "steps": lp["steps_done"],
        "ps_rms_hpa_vs_plain": lp["ps_rms_hpa"], "theta_rel_l2_vs_plain": lp["theta_rel_l2"],
        "no_network_value": res["reduced_with_checks_no_network"]["days_per_hour"],
        "no_network_fallbacks": res["reduced_with_checks_no_network"]["fallbacks"],
        "no_network_ps_rms_hpa_vs_plain": res["reduced_with_checks_no_network"]["ps_rms_hpa"],
        "no_network_theta_rel_l2_vs_plain": res["reduced_with_checks_no_network"]["theta_rel_l2"],
        "network_net_effect": ("the networks cost speed (value < no_network_value) and buy accuracy only where "
                               "ps_rms_hpa_vs_plain < no_network_ps_rms_hpa_vs_plain; the doubled time step alone "
                               "meets the speed target"),
        "reduced_uncorrected_first_flagged_step": res["reduced_uncorrected"]["first_flagged_step"],
        "column_net_val_loss": res["column_net"]["val_loss"],
        "column_net_val_loss_no_correction": res["column_net"]["val_loss_no_correction"],
        "workload": res["workload"] + f"; {res['eval_steps']} steps ({res['eval_days']:g} days)",
    }


# ------------------------------------------------ partitioned single instance
def run_partitioned(args, case, cfg) -> dict:
    """One instance split over ``args.partition_ranks`` ranks emulated on this
    GPU (``hexdyn.partition.PartitionedDycore``: a thread and a stream per
    rank, halo exchanges as device copies at the step's exchange points).
    The owned regions after one step are compared word for word with a
    single instance's step from the same state, then steps are timed with
    CUDA events on every rank's stream (max over ranks)."""
    import numpy as np
    import torch

    import hexdyn
    from hexdyn import _lib, partition
    from hexdyn.case import case_arrays

    arr = case_arrays(case)
    ranks = args.partition_ranks
    single = hexdyn.from_case(case, cfg)
    single.step_device(1)
    ref_state, ref_side = single.get_state()
    single.close()
    part = partition.PartitionedDycore(arr, cfg, ranks)
    part.step(1)
    got_state, got_side = part.get_state()
    differing = 0
    for name in _lib.STATE_FIELDS:
        differing += int(np.count_nonzero(np.asarray(getattr(ref_state, name), np.float32).view(np.uint32)
                                          != got_state[name].view(np.uint32)))
    for name in _lib.SIDECAR_FIELDS:
        differing += int(np.count_nonzero(np.asarray(getattr(ref_side, name), np.float32).view(np.uint32)
                                          != got_side[name].view(np.uint32)))
    n_before = len(part.exchanges[0])
    part.step(1)   # warm-up
    steps = 3
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ranks)]
    for (e0, _), st in zip(ev, part.streams):
        e0.record(st)
    part.step(steps)
    for (_, e1), st in zip(ev, part.streams):
        e1.record(st)
    torch.cuda.synchronize()
    ms = max(e0.elapsed_time(e1) for e0, e1 in ev) / steps
    exchanges = (len(part.exchanges[0]) - n_before) // (steps + 1)
    lays = part.layouts
    part.close()
    dt = cfg.config_dt
    return {
        "metric": "simulated days/hour", "value": (dt / 86400.0) / (ms / 1000.0 / 3600.0), "ms_per_step": ms,
        "steps": steps, "warmup": 1, "ranks": ranks, "emulated_on_one_gpu": True,
        "halo_rings": partition.halo_rings_for(cfg), "exchanges_per_step": exchanges,
        "owned_cells": [lay.n_owned["cell"] for lay in lays],
        "halo_cells": [int(lay.l2g["cell"].size - lay.n_owned["cell"]) for lay in lays],
        "halo_edges": [int(lay.l2g["edge"].size - lay.n_owned["edge"]) for lay in lays],
        "owned_region_differing_words_vs_single_instance": differing,
        "note": "ranks share one GPU here (eager steps, host hooks between launches): the number shows the path "
                "running and its overhead, not multi-GPU scaling",
    }


# ------------------------------------------------------------------- arms
def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    case = build_workload(args)
    dt = LEVEL_DT[args.level]
    budget = max(30.0, min(170.0, args.cpu_budget_s * 2.5))
    sec, n = oracle_time_per_step(case, dt, budget, max(1, args.steps))
    value = (dt / 86400.0) / (sec / 3600.0)
    sample = (f"{n} full large step(s) of the {case.mesh.n_cells}-cell workload (of --steps {args.steps} "
              f"requested; bounded to ~{budget:.0f} s), no warm-up needed for NumPy")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "simulated days/hour",
        "n_gpus": 0, "steps": n, "warmup": 0, "ms_per_step": sec * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, case),
        "cpu_baseline": {"value": value, "unit": "simulated days/hour", "cores": cores_used(), "kind": "port",
                         "path": CPU_PATH, "host": host_box(), "sample": sample},
        "e2e": {"value": value, "unit": "simulated days/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local_rank: int) -> None:
    import torch

    import hexdyn
    from hexdyn.config import DycoreConfig

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        dist = dist_mod
    dt = LEVEL_DT[args.level]
    case = build_workload(args)
    mixing = (dict(config_horiz_mixing="2d_smagorinsky", config_smagorinsky_coef=0.125, config_visc4_2dsmag=0.05)
              if args.smagorinsky else {})
    cfg = DycoreConfig(config_dt=dt, config_number_of_sub_steps=2, moist_coefficients="native",
                       numerics=args.numerics, **mixing)
    drv = hexdyn.from_case(case, cfg)
    tuning = drv.autotune(2) if args.autotune == "on" else {}
    if not args.no_graph:
        drv.capture_graph()
    stream = torch.cuda.current_stream()
    sampler = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)).split(",")[0])
                           if world == 1 else local_rank).start()
    drv.step_async(max(3, args.warmup))
    drv.read_flag()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    drv.step_async(args.steps)
    stop.record(stream)
    torch.cuda.synchronize()
    barrier()
    elapsed = start.elapsed_time(stop)
    flag = drv.read_flag()
    if dist is not None:
        t = torch.tensor([elapsed], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    clocks = sampler.stop()
    ms_per_step = elapsed / args.steps
    days = args.steps * dt / 86400.0
    value = world * days / (elapsed / 1000.0 / 3600.0)
    launches = drv.receipt().launches_per_step

    # per-kernel CUDA-event profile over the same number of eager steps
    prof = drv.profile(max(1, min(args.steps, 20)))
    prof_steps = max(1, min(args.steps, 20))
    C, E, V = case.mesh.n_cells, case.mesh.n_edges, case.mesh.n_vertices
    L, T = args.levels, int(case.scalars.shape[0])
    peak, peak_kind = measured_peak()
    total_ms = sum(ms for _, ms in prof.values())
    kernels = {}
    for name, (n, ms) in prof.items():
        avg_ms = ms / n
        b = kernel_bytes(name, C, E, V, L, T, advW=int(case.adv_cells_for_edge.shape[1]))
        kernels[name] = {"launches_per_step": n / prof_steps, "avg_us": avg_ms * 1000.0,
                         "share": ms / total_ms, "bytes": b,
                         "gbs": (b / (avg_ms / 1000.0) / 1e9) if b else None}
    merged = by_kernel(kernels, prof_steps)
    dominant = max(merged, key=lambda k: merged[k]["share"])
    dk = merged[dominant]
    achieved = dk["gbs"]
    traffic = None
    traffic_file = ROOT / "profiles" / "traffic.json"
    if traffic_file.exists():
        try:
            # ncu DRAM bytes per launch of each kernel function (the mean
            # over its launches of one step)
            known = json.loads(traffic_file.read_text())
            traffic = known.get(dominant)
        except Exception:  # noqa: BLE001
            traffic = None
    step_bytes = sum(kernel_bytes(k, C, E, V, L, T) * kernels[k]["launches_per_step"] for k in kernels)

    # end to end through host buffers: upload state+sidecar, step, download
    from hexdyn import _lib

    def pinned(shape):
        t = torch.empty(int(np.prod(shape)), dtype=torch.float32, pin_memory=True)
        return t.numpy().reshape(shape), t

    state_now, side_now = drv.get_state()
    hold = []
    sin, sdin, sout, sdout = {}, {}, {}, {}
    for name in _lib.STATE_FIELDS:
        a, t = pinned(drv.field_shape(name))
        a[...] = getattr(state_now, name)
        sin[name] = a
        b, t2 = pinned(drv.field_shape(name))
        sout[name] = b
        hold += [t, t2]
    for name in _lib.SIDECAR_FIELDS:
        a, t = pinned(drv.field_shape(name))
        a[...] = getattr(side_now, name)
        sdin[name] = a
        b, t2 = pinned(drv.field_shape(name))
        sdout[name] = b
        hold += [t, t2]
    h2d = sum(a.nbytes for a in (*sin.values(), *sdin.values()))
    d2h = sum(a.nbytes for a in (*sout.values(), *sdout.values()))
    e2e_steps = max(3, min(args.steps, 20))
    drv.step_host_buffers(sin, sdin, sout, sdout)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        drv.step_host_buffers(sin, sdin, sout, sdout)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * (e2e_steps * dt / 86400.0) / (e2e_ms / 1000.0 / 3600.0)
    drv.read_flag()

    batched = run_ensemble(args, stream, dist, world, rank, case) if args.batched == "on" else None
    learned = run_learned(args, case) if args.learned == "on" and args.level == 6 else None
    partitioned = (run_partitioned(args, case, cfg)
                   if args.partition_ranks > 1 and world == 1 and rank == 0 else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sec, n = oracle_time_per_step(case, dt, args.cpu_budget_s, 2)
        cpu = {"value": (dt / 86400.0) / (sec / 3600.0), "unit": "simulated days/hour", "cores": cores_used(),
               "kind": "port", "path": CPU_PATH, "host": host_box(),
               "sample": f"{n} full large step(s) of this workload by the NumPy oracle (single thread), "
                         f"{sec:.1f} s/step"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "simulated days/hour", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(args, case),
            "parallelism": "replicas" if world > 1 else "single instance",
            "clocks": clocks, "validation_flag": flag,
            "e2e": {"value": e2e_value, "unit": "simulated days/hour", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "gpu_launches": int(launches) * args.steps if not args.no_graph else int(launches) * args.steps,
            "gpu_launches_per_step": int(launches),
            "roofline": {"bound": "hbm", "kernel": dominant, "labels": dk["labels"], "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None,
                         "traffic": traffic, "bytes_per_launch": dk["bytes"], "avg_launch_us": dk["avg_us"],
                         "share": dk["share"]},
            "autotune": {k: v["threads"] for k, v in tuning.items()},
            "step_bytes_algorithmic": step_bytes,
            "step_gbs": step_bytes / (ms_per_step / 1000.0) / 1e9,
            "kernels": kernels,
            "kernel_functions": merged,
            "batched": batched,
            "learned": learned,
            "partitioned": partitioned,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    drv.close()
    del hold


def main() -> None:
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        try:
            run_ours(args, rank, world, local_rank)
        finally:
            dist.destroy_process_group()
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
