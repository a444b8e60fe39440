"""CUDA step parity through the C ABI.

Strict numerics must reproduce the reference's own outputs word for word
(golden fixtures made by running the reference, tests/golden/make_golden.py)
and the oracle at the C1 size (2562 cells x 55 levels).  Fast numerics must
stay within relative L2 1e-5 per field after one step.
"""

import numpy as np
import pytest

import hexdyn
from fixtures import SIDE, STATE, VARIANTS, case_from_arrays, differing_words, golden_config, inputs, load_golden
from hexdyn.case import build_case, case_arrays
from hexdyn.config import DycoreConfig
from hexdyn.mesh import build_mesh
from oracle.dycore import OracleConfig, OracleDycore, State

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("these tests need a CUDA GPU")
    torch.cuda.set_device(0)


def smag_knobs(c: dict) -> dict:
    if not c["smagorinsky"]:
        return {}
    coef, visc4, divf = c["smagorinsky"]
    return dict(config_horiz_mixing="2d_smagorinsky", config_smagorinsky_coef=coef, config_visc4_2dsmag=visc4,
                config_del4u_div_factor=divf)


def make_driver(arr, dt, nsub, moist, numerics="strict", graph=False):
    case = case_from_arrays(arr)
    cfg = DycoreConfig(config_dt=dt, config_number_of_sub_steps=nsub, moist_coefficients=moist, numerics=numerics)
    return hexdyn.from_case(case, cfg, capture_graph=graph)


@pytest.mark.parametrize("name,label,steps", [("l2_L12", "dry", 2), ("l2_L12", "native", 1), ("l3_L20", "dry", 1)])
def test_strict_step_matches_reference_outputs(name, label, steps):
    fx = load_golden(name)
    drv = make_driver(inputs(fx), float(fx["config.dt"]), int(fx["config.n_sub_steps"]), label)
    for step in range(1, steps + 1):
        res = drv.step()
        for k in STATE:
            assert differing_words(getattr(res.state, k), fx[f"{label}.step{step}.{k}"]) == 0, (step, k)
        for k in SIDE:
            assert differing_words(getattr(res.saved_diagnostics, k), fx[f"{label}.step{step}.side.{k}"]) == 0, (step, k)
    drv.close()


@pytest.mark.parametrize("name,steps", VARIANTS)
def test_strict_step_matches_reference_variants(name, steps):
    """One and four acoustic substeps, standard RK3 transport, no APVM, no
    tracers, implicit w damping, the order-2 schedule, 2-D Smagorinsky
    mixing: the CUDA step against the reference run with that
    configuration."""
    fx = load_golden(name)
    c = golden_config(fx)
    cfg = DycoreConfig(config_dt=c["dt"], config_number_of_sub_steps=c["n_sub_steps"],
                       config_monotonic=c["monotonic"], config_apvm_upwinding=c["apvm_upwinding"],
                       config_xnutr=c["xnutr"], config_zd=c["zd"], config_time_integration_order=c["order"],
                       moist_coefficients="dry", **smag_knobs(c))
    drv = hexdyn.from_case(case_from_arrays(inputs(fx)), cfg, capture_graph=True)
    for step in range(1, steps + 1):
        res = drv.step()
        for k in STATE:
            assert differing_words(getattr(res.state, k), fx[f"dry.step{step}.{k}"]) == 0, (name, step, k)
        for k in SIDE:
            assert differing_words(getattr(res.saved_diagnostics, k), fx[f"dry.step{step}.side.{k}"]) == 0, \
                (name, step, k)
    drv.close()


@pytest.mark.parametrize("seed", [7])
def test_renumbered_case_matches_reference(seed):
    """The CUDA step of the 162-cell reference inputs under a random
    renumbering of cells, edges and vertices, mapped back, equals the
    reference's step word for word (hexdyn.reorder)."""
    from hexdyn import reorder

    fx = load_golden("l2_L12")
    arr = inputs(fx)
    ren = reorder.random_order(arr, seed=seed)
    drv = make_driver(reorder.apply(arr, ren), float(fx["config.dt"]), int(fx["config.n_sub_steps"]), "dry")
    back = ren.inverse()
    for step in (1, 2):
        res = drv.step()
        for k in STATE:
            got = reorder.field(getattr(res.state, k), k, back)
            assert differing_words(got, fx[f"dry.step{step}.{k}"]) == 0, (step, k)
        for k in SIDE:
            got = reorder.field(getattr(res.saved_diagnostics, k), k, back)
            assert differing_words(got, fx[f"dry.step{step}.side.{k}"]) == 0, (step, k)
    drv.close()


def test_cells_on_cell_slot_order_does_not_change_the_step():
    """The limiter's bounds are a min/max over cellsOnCell.  When its slots
    follow edgesOnCell (the MPAS convention) the library takes the upwind
    fluxes' cell values from the columns the bounds load; here the slots are
    rotated by one, so it gathers them per edge instead, and the words are
    still the reference's."""
    fx = load_golden("l2_L12")
    arr = dict(inputs(fx))
    coc = arr["mesh.cellsOnCell"].copy()
    counts = arr["mesh.nEdgesOnCell"]
    for c in range(coc.shape[0]):
        m = int(counts[c])
        coc[c, :m] = np.roll(coc[c, :m], 1)
    arr["mesh.cellsOnCell"] = coc
    drv = make_driver(arr, float(fx["config.dt"]), int(fx["config.n_sub_steps"]), "dry")
    for step in (1, 2):
        res = drv.step()
        for k in STATE:
            assert differing_words(getattr(res.state, k), fx[f"dry.step{step}.{k}"]) == 0, (step, k)
    drv.close()


def test_negative_scalar_clamp_matches_oracle():
    """clamp_negative_scalars (the reference CUDA driver's end-of-step
    `putmask(scalars, scalars < 0, 0)`) with standard transport, whose
    undershoots leave negative mixing ratios: the CUDA step equals the
    oracle with the clamp, and the oracle without it holds negatives (so the
    clamp is exercised)."""
    arr = case_arrays(build_case(build_mesh(2, lloyd=2, seed=0), n_levels=12, seed=0, n_condensates=2))
    knobs = dict(dt=1800.0, n_sub_steps=2, moist="native", monotonic=False)
    raw, _ = OracleDycore(arr, OracleConfig(**knobs)).step(State(*(np.asarray(arr[k]).copy() for k in STATE)))
    assert (raw.scalars < 0).sum() > 0
    orc = OracleDycore(arr, OracleConfig(**knobs, clamp_negative_scalars=True))
    cfg = DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2, moist_coefficients="native",
                       config_monotonic=False, clamp_negative_scalars=True)
    drv = hexdyn.from_case(case_from_arrays(arr), cfg, capture_graph=True)
    st, sd = State(*(np.asarray(arr[k]).copy() for k in STATE)), None
    for step in (1, 2):
        st, sd = orc.step(st, sd)
        assert (st.scalars < 0).sum() == 0
        res = drv.step()
        for k in STATE:
            assert differing_words(getattr(res.state, k), getattr(st, k)) == 0, (step, k)
        for k in SIDE:
            assert differing_words(getattr(res.saved_diagnostics, k), getattr(sd, k)) == 0, (step, k)
    drv.close()


@pytest.mark.parametrize("levels", [4, 5, 8])
def test_short_columns_match_oracle(levels):
    """The fewest levels the third-order vertical fluxes allow (4), and 5 and
    8: one or two four-level chunks per column, every chunk holding a
    boundary interface."""
    arr = case_arrays(build_case(build_mesh(2, lloyd=2, seed=0), n_levels=levels, seed=0, n_condensates=1))
    drv = make_driver(arr, 900.0, 2, "native", graph=True)
    orc = OracleDycore(arr, OracleConfig(dt=900.0, n_sub_steps=2, moist="native"))
    state, side = State(*(np.asarray(arr[k]).copy() for k in STATE)), None
    for step in (1, 2):
        res = drv.step()
        state, side = orc.step(state, side)
        for k in STATE:
            assert differing_words(getattr(res.state, k), getattr(state, k)) == 0, (levels, step, k)
        for k in SIDE:
            assert differing_words(getattr(res.saved_diagnostics, k), getattr(side, k)) == 0, (levels, step, k)
    drv.close()


def test_tall_columns_match_oracle():
    """130 levels (stride 136, 34 four-level chunks per column, more than a
    warp): the column sweeps run in their one-level form (k_vcoef,
    k_ac_cell) while every other kernel keeps four levels per thread."""
    arr = case_arrays(build_case(build_mesh(2, lloyd=2, seed=0), n_levels=130, seed=0, n_condensates=1))
    drv = make_driver(arr, 900.0, 2, "native")
    orc = OracleDycore(arr, OracleConfig(dt=900.0, n_sub_steps=2, moist="native"))
    state, side = State(*(np.asarray(arr[k]).copy() for k in STATE)), None
    for step in (1, 2):
        res = drv.step()
        state, side = orc.step(state, side)
        for k in STATE:
            assert differing_words(getattr(res.state, k), getattr(state, k)) == 0, (step, k)
        for k in SIDE:
            assert differing_words(getattr(res.saved_diagnostics, k), getattr(side, k)) == 0, (step, k)
    drv.close()


@pytest.fixture(scope="module")
def c1_case():
    mesh = build_mesh(4, lloyd=20, seed=0)
    return case_arrays(build_case(mesh, n_levels=55, seed=0, n_condensates=0))


@pytest.mark.parametrize("moist", ["dry", "native"])
def test_strict_c1_matches_oracle_two_steps(c1_case, moist):
    arr = c1_case
    orc = OracleDycore(arr, OracleConfig(dt=1800.0, n_sub_steps=2, moist=moist))
    drv = make_driver(arr, 1800.0, 2, moist)
    st = State(*(np.asarray(arr[k]).copy() for k in STATE))
    sd = None
    for step in (1, 2):
        st, sd = orc.step(st, sd)
        res = drv.step()
        for k in STATE:
            assert differing_words(getattr(res.state, k), getattr(st, k)) == 0, (moist, step, k)
        for k in SIDE:
            assert differing_words(getattr(res.saved_diagnostics, k), getattr(sd, k)) == 0, (moist, step, k)
    drv.close()


def test_graph_replay_is_bitwise_eager():
    fx = load_golden("l2_L12")
    arr = inputs(fx)
    eager = make_driver(arr, 1800.0, 2, "native")
    graph = make_driver(arr, 1800.0, 2, "native", graph=True)
    for _ in range(3):
        a, b = eager.step(), graph.step()
    for k in STATE:
        assert differing_words(getattr(a.state, k), getattr(b.state, k)) == 0, k
    assert b.receipt.graph
    eager.close()
    graph.close()


def _pinned(shape):
    import torch

    t = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    return t.numpy(), t


@pytest.mark.parametrize("graph", [False, True])
def test_host_buffer_step_equals_device_step(graph):
    """hexdyn_step_host (uploads, the step, and downloads of every field but
    the scalars on a second stream beside the scalar transport) returns the
    words of a device step followed by downloads, step after step, with the
    outputs fed back as the next inputs."""
    arr = case_arrays(build_case(build_mesh(4, lloyd=2, seed=0), n_levels=55, seed=0, n_condensates=2))
    a = make_driver(arr, 1800.0, 2, "native", graph=graph)
    b = make_driver(arr, 1800.0, 2, "native", graph=graph)
    state, side = a.get_state()
    hold, bufs = [], {}
    for name in (*STATE, *SIDE):
        src = getattr(state, name) if name in STATE else getattr(side, name)
        x, t = _pinned(a.field_shape(name))
        y, u = _pinned(a.field_shape(name))
        x[...] = src
        bufs[name] = (x, y)
        hold += [t, u]
    for step in (1, 2, 3):
        a.step_host_buffers({k: bufs[k][0] for k in STATE}, {k: bufs[k][0] for k in SIDE},
                            {k: bufs[k][1] for k in STATE}, {k: bufs[k][1] for k in SIDE})
        a.synchronize()
        res = b.step()
        for k in STATE:
            assert differing_words(bufs[k][1], getattr(res.state, k)) == 0, (step, k)
        for k in SIDE:
            assert differing_words(bufs[k][1], getattr(res.saved_diagnostics, k)) == 0, (step, k)
        for k in (*STATE, *SIDE):
            bufs[k][0][...] = bufs[k][1]
            bufs[k][1][...] = np.nan
    a.close()
    b.close()


def test_fast_numerics_within_tolerance(c1_case):
    strict = make_driver(c1_case, 1800.0, 2, "native")
    fast = make_driver(c1_case, 1800.0, 2, "native", numerics="fast")
    a, b = strict.step(), fast.step()
    for k in STATE:
        x = getattr(a.state, k).astype(np.float64)
        y = getattr(b.state, k).astype(np.float64)
        if k == "rho_w":
            # rw starts at zero: compare against the field's own scale
            rel = np.linalg.norm(x - y) / max(np.linalg.norm(x), 1e-30)
            assert rel < 1e-3, (k, rel)
            continue
        rel = np.linalg.norm(x - y) / np.linalg.norm(x)
        assert rel <= 1e-5, (k, rel)
    strict.close()
    fast.close()


def test_runs_are_deterministic(c1_case):
    outs = []
    for _ in range(2):
        drv = make_driver(c1_case, 1800.0, 2, "native")
        outs.append(drv.step())
        drv.close()
    for k in STATE:
        assert differing_words(getattr(outs[0].state, k), getattr(outs[1].state, k)) == 0


def test_post_transport_callback_sees_the_step_and_writes_through():
    """physics_post_transport_callback receives logical device views of the
    step's result and of the state the step started from (the reference's
    hand-off after transport); writes into the result land in the library's
    buffers."""
    from hexdyn.config import ConfigurationRefusal

    fx = load_golden("l2_L12")
    drv = make_driver(inputs(fx), float(fx["config.dt"]), int(fx["config.n_sub_steps"]), "dry", graph=True)
    before, _ = drv.get_state()
    seen = {}

    def hand_off(state, saved, outer_state, modified_theta_dynamics_rate):
        seen["rho"] = state.rho.cpu().numpy()
        seen["outer_rho"] = outer_state.rho.cpu().numpy()
        seen["outer_scalars"] = outer_state.scalars.cpu().numpy()
        seen["u"] = saved.normal_velocity.cpu().numpy()
        seen["rate"] = modified_theta_dynamics_rate
        state.scalars.zero_()

    drv._step_device_v841(physics_post_transport_callback=hand_off)
    after, _ = drv.get_state()
    assert differing_words(seen["outer_rho"], before.rho) == 0
    assert differing_words(seen["outer_scalars"], before.scalars) == 0
    assert differing_words(seen["rho"], fx["dry.step1.rho"]) == 0
    assert differing_words(seen["u"], fx["dry.step1.side.normal_velocity"]) == 0
    assert seen["rate"] is None
    assert after.scalars.size > 0 and not after.scalars.any()
    drv.close()
    clamp = hexdyn.from_case(case_from_arrays(inputs(fx)), DycoreConfig(config_dt=1800.0, clamp_negative_scalars=True))
    with pytest.raises(ConfigurationRefusal):
        clamp._step_device_v841(physics_post_transport_callback=hand_off)
    clamp.close()


def test_validation_flag_raises_on_bad_state():
    """A host-side corruption (negative rho_theta in one column) must come back
    as the device validation flag, not as a silent result or a fault."""
    fx = load_golden("l2_L12")
    arr = dict(inputs(fx))
    arr["rho_theta"] = arr["rho_theta"].copy()
    arr["rho_theta"][:, 5] = -arr["rho_theta"][:, 5]
    with pytest.raises(FloatingPointError):
        drv = make_driver(arr, 1800.0, 2, "dry")
        drv.step()


def test_acoustic_words_and_reference_step_signature():
    """_step_device_v841 (the reference's production entry) refuses held
    physics tendencies and a mass-loading count other than the carried
    scalars by name, and hands acoustic_output_callback the final acoustic
    words, equal to the oracle's ru_p and rw_p after the last substep of RK
    stage 3 of the last subcycle (the per-stage physics callback:
    tests/test_physics_hook.py)."""
    from hexdyn.config import ConfigurationRefusal
    from oracle.dycore import OracleConfig, OracleDycore, State

    fx = load_golden("l2_L12")
    arr = inputs(fx)
    drv = make_driver(arr, float(fx["config.dt"]), int(fx["config.n_sub_steps"]), "dry", graph=True)
    with pytest.raises(ConfigurationRefusal) as err:
        drv._step_device_v841(physics_mass_loading_count=arr["scalars"].shape[0] + 1)
    assert err.value.knob == "physics_mass_loading_count"
    with pytest.raises(ConfigurationRefusal) as err:
        drv._step_device_v841(object())
    assert err.value.knob == "held_physics_tendencies"
    got = {}

    def keep(ru_p, rw_p):
        got["ru_p"], got["rw_p"] = ru_p.cpu().numpy(), rw_p.cpu().numpy()

    drv._step_device_v841(acoustic_output_callback=keep)
    record = []
    orc = OracleDycore(arr, OracleConfig(dt=float(fx["config.dt"]), n_sub_steps=int(fx["config.n_sub_steps"]),
                                         moist="dry"))
    orc.step(State(*(arr[k].copy() for k in STATE)), None, record=record)
    words = [r for r in record if "ru_p" in r]
    assert len(words) == 3  # one per dynamics subcycle; the last is the step's
    assert differing_words(got["ru_p"], words[-1]["ru_p"]) == 0
    assert differing_words(got["rw_p"], words[-1]["rw_p"]) == 0
    # the step itself is the reference's
    state = drv.get_state()[0]
    for k in STATE:
        assert differing_words(getattr(state, k), fx[f"dry.step1.{k}"]) == 0, k
    drv.close()


def test_upper_damping_matches_oracle():
    """Rayleigh damping of u over the top 6 levels (5-day timescale) and the
    CAM floor of the Smagorinsky diffusivity over the top 4 levels: the CUDA
    step equals the oracle's restatement of the reference's native operators
    (hexcore/native/upper_damping.rs) word for word over two steps.  (The
    reference's own CPU path for them needs a Rust toolchain, so this
    parity is against the restatement only.)"""
    from oracle.dycore import OracleConfig, OracleDycore, State
    from oracle.mixing import SmagorinskyConfig

    fx = load_golden("l2_L12")
    arr = inputs(fx)
    dt, nsub = float(fx["config.dt"]), int(fx["config.n_sub_steps"])
    cfg = DycoreConfig(config_dt=dt, config_number_of_sub_steps=nsub, moist_coefficients="dry",
                       config_horiz_mixing="2d_smagorinsky", config_smagorinsky_coef=0.125,
                       config_visc4_2dsmag=0.05, config_mpas_cam_coef=2.0, config_rayleigh_damp_u=True)
    drv = hexdyn.from_case(case_from_arrays(arr), cfg, capture_graph=True)
    orc = OracleDycore(arr, OracleConfig(dt=dt, n_sub_steps=nsub, moist="dry", rayleigh=(6, 5.0),
                                         smagorinsky=SmagorinskyConfig(0.125, 0.05, 10.0, cam_coef=2.0)))
    state, side = State(*(arr[k].copy() for k in STATE)), None
    plain = fx["dry.step1.rho_u"]
    for step in (1, 2):
        res = drv.step()
        state, side = orc.step(state, side)
        for k in STATE:
            assert differing_words(getattr(res.state, k), getattr(state, k)) == 0, (step, k)
        for k in SIDE:
            assert differing_words(getattr(res.saved_diagnostics, k), getattr(side, k)) == 0, (step, k)
        if step == 1:
            # the damping acts: the top levels differ from the undamped step
            assert differing_words(res.state.rho_u[-6:], plain[-6:]) > 0
    drv.close()
