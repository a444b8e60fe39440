"""Configuration refusals (hexcore/config_v841.py and hexcore/driver.py:232)."""

import pytest

from hexdyn.config import ConfigurationRefusal, DycoreConfig
from oracle.dycore import schedule


def test_defaults_validate():
    DycoreConfig().validate()


@pytest.mark.parametrize("kw,knob", [
    (dict(config_dt=-1.0), "config_dt"),
    (dict(config_time_integration_order=1), "config_time_integration_order"),
    (dict(config_time_integration_order=4), "config_time_integration_order"),
    (dict(config_dynamics_split_steps=2), "config_dynamics_split_steps"),
    (dict(config_split_dynamics_transport=False), "config_split_dynamics_transport"),
    (dict(config_smdiv=0.0), "config_smdiv"),
    (dict(config_divergence_damping=False), "config_divergence_damping"),
    (dict(config_xnutr=1.5), "config_xnutr"),
    (dict(config_xnutr=0.2, config_zd=0.0), "config_zd"),
    (dict(config_horiz_mixing="3d_smagorinsky"), "config_horiz_mixing"),
    (dict(config_mpas_cam_coef=0.1), "config_mpas_cam_coef"),
    (dict(config_number_rayleigh_damp_u_levels=0), "config_number_rayleigh_damp_u_levels"),
    (dict(config_rayleigh_damp_u_timescale_days=0.0), "config_rayleigh_damp_u_timescale_days"),
    (dict(config_smagorinsky_coef=0.125), "config_smagorinsky_coef"),
    (dict(config_horiz_mixing="2d_smagorinsky", config_del4u_div_factor=0.0), "config_del4u_div_factor"),
    (dict(config_moist_physics=True), "config_moist_physics"),
    (dict(moist_coefficients="wet"), "moist_coefficients"),
])
def test_refusals_name_the_knob(kw, knob):
    with pytest.raises(ConfigurationRefusal) as err:
        DycoreConfig(**kw).validate()
    assert err.value.knob == knob


def test_unknown_option_refused():
    with pytest.raises(ConfigurationRefusal):
        DycoreConfig.from_mapping({"config_les_model": "3d_smagorinsky"})


def test_rk3_schedule_matches_mpas():
    """hexcore/integration.py:104: split 3, 2 sub-steps at dt=1800."""
    st = schedule(1800.0, 2, 3)
    assert [s[0] for s in st] == [1, 2, 3]
    assert [s[1] for s in st] == [200.0, 300.0, 600.0]
    assert [s[2] for s in st] == [200.0, 300.0, 300.0]
    assert [s[3] for s in st] == [1, 1, 2]
    st6 = schedule(720.0, 6, 3)
    assert [s[3] for s in st6] == [1, 3, 6]


@pytest.mark.parametrize("dt,substeps", [(15.0, 2), (20.0, 4), (60.0, 2)])
def test_rk2_schedule_matches_mpas(dt, substeps):
    """tests/test_rk2_v841.py:30-45 of the reference: counts (n/2, n/2, n),
    and the FP32 large steps equal the FP32 rk_timestep of atm_srk3
    (order 2 takes the half-step branch at both first stages)."""
    import numpy as np

    st = schedule(dt, substeps, 3, order=2)
    assert [s[3] for s in st] == [substeps // 2, substeps // 2, substeps]
    dyn = np.float32(np.float32(dt) / np.float32(3.0))
    want = [np.float32(dyn / np.float32(2.0)), np.float32(dyn / np.float32(2.0)), dyn]
    assert [np.float32(s[1]).tobytes() for s in st] == [w.tobytes() for w in want]
    assert np.float32(schedule(dt, substeps, 1, order=2)[0][1]) == np.float32(dt * 0.5)
    DycoreConfig(config_dt=dt, config_time_integration_order=2, config_number_of_sub_steps=substeps).validate()


def test_bench_byte_model_covers_every_step_kernel():
    """bench.py's roofline needs the algorithmic bytes of every launch label
    the step can issue (the labels of csrc/dycore_step.cuh)."""
    import re
    from pathlib import Path

    import bench

    root = Path(__file__).resolve().parent.parent
    step = (root / "gpuwm-hex_b200" / "csrc" / "dycore_step.cuh").read_text()
    labels = set(re.findall(r'\.lpvt?\("(k_[a-z0-9_]+)"', step))
    labels |= set(re.findall(r'LPSN\(L, "(k_[a-z0-9_]+)"', step))
    labels |= {x for pair in re.findall(r'"(k_[a-z0-9_]+)" : "(k_[a-z0-9_]+)"', step) for x in pair}
    labels |= set(re.findall(r'LPG\(L, "(k_[a-z0-9_]+)"', step))
    labels |= {"k_" + m for m in re.findall(r"LPST?\(L, [^,]+, [^,]+, ([a-z0-9_]+),", step)}
    labels |= set(re.findall(r"LP\(L, [^,]+, [^,]+, [^,]+, (k_[a-z0-9_]+),", step))
    labels -= {"k_name", "k_rebuild_cell", "k_recover_u"}  # macro text; the sidecar rebuild, not a step kernel
    assert {"k_tend_u", "k_fct_cell2", "k_clamp_scalars", "k_mix_cell2", "k_diag_vertex"} <= labels
    for name in sorted(labels):
        assert bench.kernel_bytes(name, 10, 30, 20, 12, 3) > 0, name


def test_bench_roofline_merges_labels_of_one_kernel():
    """The roofline names a kernel function: launch labels that run the same
    function (the first acoustic substep's k_ac_cell_first and the later
    k_ac_cell) are merged, shares added, time and bytes launch-weighted."""
    import bench

    kernels = {"k_ac_cell_first": {"launches_per_step": 9, "avg_us": 80.0, "share": 0.09, "bytes": 200e6},
               "k_ac_cell": {"launches_per_step": 3, "avg_us": 90.0, "share": 0.035, "bytes": 260e6},
               "k_tend_u": {"launches_per_step": 9, "avg_us": 92.0, "share": 0.105, "bytes": 159e6}}
    merged = bench.by_kernel(kernels, 1)
    assert set(merged) == {"kv_ac_cell", "kv_tend_u"}
    ac = merged["kv_ac_cell"]
    assert ac["launches_per_step"] == 12 and abs(ac["share"] - 0.125) < 1e-12
    assert abs(ac["avg_us"] - (9 * 80.0 + 3 * 90.0) / 12) < 1e-9
    assert abs(ac["bytes"] - (9 * 200e6 + 3 * 260e6) / 12) < 1e-3
    assert max(merged, key=lambda k: merged[k]["share"]) == "kv_ac_cell"
    assert bench.kernel_of("k_diag_edge_v") == "kv_diag_edge" and bench.kernel_of("k_fct_cell1") == "kv_fct_cell1"
    box = bench.host_box()
    assert box["nproc"] >= 1 and set(box["env"]) == {"OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS",
                                                      "GPUWM_HEX_HOST_COPY_THREADS"}
