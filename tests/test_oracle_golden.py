"""The oracle against the reference's own step outputs (golden fixtures).

The fixtures were produced by running the reference CPU authority
(``hexcore/driver.py:3314`` ``DryDycoreDriver.step`` with
``V841DryDycoreConfig``) on these exact inputs; see tests/golden/make_golden.py.
The oracle must reproduce every output word.
"""

import numpy as np
import pytest

from fixtures import (SCALAR_VARIANTS, SIDE, STATE, VARIANTS, differing_words, digest_case, golden_config, inputs,
                      load_digests, load_golden, mismatched_digests)
from oracle.dycore import OracleConfig, OracleDycore, State


@pytest.mark.parametrize("name,label,steps", [("l2_L12", "dry", 2), ("l2_L12", "native", 1), ("l3_L20", "dry", 1)])
def test_oracle_matches_reference_bitwise(name, label, steps):
    fx = load_golden(name)
    arr = inputs(fx)
    cfg = OracleConfig(dt=float(fx["config.dt"]), n_sub_steps=int(fx["config.n_sub_steps"]), moist=label)
    orc = OracleDycore(arr, cfg)
    state = State(*(arr[k].copy() for k in STATE))
    side = None
    for step in range(1, steps + 1):
        state, side = orc.step(state, side)
        for k in STATE:
            assert differing_words(getattr(state, k), fx[f"{label}.step{step}.{k}"]) == 0, (label, step, k)
        for k in SIDE:
            assert differing_words(getattr(side, k), fx[f"{label}.step{step}.side.{k}"]) == 0, (label, step, k)


@pytest.mark.parametrize("name,steps", VARIANTS)
def test_oracle_matches_reference_variants(name, steps):
    """Configuration variants (one and four acoustic substeps, standard RK3
    transport, no APVM, no tracers, implicit w damping) against the reference
    run with that configuration."""
    fx = load_golden(name)
    c = golden_config(fx)
    arr = inputs(fx)
    if c["xnutr"]:
        from hexdyn.case import vertical_velocity_damping

        arr["vertical.dss"] = vertical_velocity_damping(arr["vertical.zgrid"], c["xnutr"], c["zd"])
        assert np.count_nonzero(arr["vertical.dss"]) > 0
    from oracle.mixing import SmagorinskyConfig

    smag = SmagorinskyConfig(*c["smagorinsky"]) if c["smagorinsky"] else None
    orc = OracleDycore(arr, OracleConfig(dt=c["dt"], n_sub_steps=c["n_sub_steps"], monotonic=c["monotonic"],
                                         apvm_upwinding=c["apvm_upwinding"], moist="dry", order=c["order"],
                                         smagorinsky=smag))
    state = State(*(arr[k].copy() for k in STATE))
    side = None
    for step in range(1, steps + 1):
        state, side = orc.step(state, side)
        for k in STATE:
            assert differing_words(getattr(state, k), fx[f"dry.step{step}.{k}"]) == 0, (name, step, k)
        for k in SIDE:
            assert differing_words(getattr(side, k), fx[f"dry.step{step}.side.{k}"]) == 0, (name, step, k)


def test_native_moist_coefficients_change_the_step():
    fx = load_golden("l2_L12")
    assert differing_words(fx["dry.step1.rho_u"], fx["native.step1.rho_u"]) > 0


def test_dry_state_moist_modes_agree():
    """With no scalars loading the air (qtot=0, cqu=cqw=1) both coefficient
    semantics give the same bits (hexcore/cuda_driver.py:5062-5065)."""
    fx = load_golden("l2_L12")
    arr = inputs(fx)
    arr["scalars"] = np.zeros_like(arr["scalars"])
    outs = []
    for moist in ("dry", "native"):
        orc = OracleDycore(arr, OracleConfig(dt=1800.0, n_sub_steps=2, moist=moist))
        st, sd = orc.step(State(*(arr[k].copy() for k in STATE)))
        outs.append((st, sd))
    for k in STATE:
        assert differing_words(getattr(outs[0][0], k), getattr(outs[1][0], k)) == 0


def test_deformation_weights_match_reference():
    """hexcore/mixing_v841.py:495 deformation weights of the 162-cell mesh,
    computed by the reference with its strict geometry."""
    from oracle.mixing import deformation_weights

    fx = load_golden("l2_L12_smag")
    c2, s2, cs = deformation_weights(inputs(fx))
    for got, key in ((c2, "mix.coef_c2"), (s2, "mix.coef_s2"), (cs, "mix.coef_cs")):
        assert differing_words(got, fx[key]) == 0, key


def test_smagorinsky_steps_match_reference():
    """Two steps with 2-D Smagorinsky mixing (coefficient 0.125, visc4 0.05,
    del4u_div_factor 10, len_disp from nominalMinDc) equal the reference's."""
    from oracle.mixing import SmagorinskyConfig

    fx = load_golden("l2_L12_smag")
    c = golden_config(fx)
    arr = inputs(fx)
    orc = OracleDycore(arr, OracleConfig(dt=c["dt"], n_sub_steps=c["n_sub_steps"], moist="dry",
                                         smagorinsky=SmagorinskyConfig(*c["smagorinsky"])))
    state = State(*(arr[k].copy() for k in STATE))
    side = None
    for step in (1, 2):
        state, side = orc.step(state, side)
        for k in STATE:
            assert differing_words(getattr(state, k), fx[f"dry.step{step}.{k}"]) == 0, (step, k)
        for k in SIDE:
            assert differing_words(getattr(side, k), fx[f"dry.step{step}.side.{k}"]) == 0, (step, k)


def test_oracle_scalar_clamp_zeroes_only_negatives():
    """The end-of-step clamp (`putmask(scalars, scalars < 0, 0)`,
    hexcore/cuda_driver.py:5311) is the step's last operation: the clamped
    step equals the unclamped one with exactly its negative words zeroed."""
    from hexdyn.case import build_case, case_arrays
    from hexdyn.mesh import build_mesh

    arr = case_arrays(build_case(build_mesh(2, lloyd=2, seed=0), n_levels=12, seed=0, n_condensates=2))
    knobs = dict(dt=1800.0, n_sub_steps=2, moist="native", monotonic=False)
    start = State(*(np.asarray(arr[k]).copy() for k in STATE))
    raw, raw_side = OracleDycore(arr, OracleConfig(**knobs)).step(start.copy())
    clamped, side = OracleDycore(arr, OracleConfig(**knobs, clamp_negative_scalars=True)).step(start.copy())
    neg = raw.scalars < 0
    assert neg.sum() > 0
    expect = np.where(neg, np.float32(0.0), raw.scalars)
    assert differing_words(clamped.scalars, expect) == 0
    for k in STATE:
        if k != "scalars":
            assert differing_words(getattr(clamped, k), getattr(raw, k)) == 0, k


@pytest.mark.parametrize("name,steps", SCALAR_VARIANTS)
@pytest.mark.parametrize("label", ["dry", "native"])
def test_oracle_matches_reference_scalar_counts(name, steps, label):
    """qv + 5 condensates (the throughput workload's six scalars) and the
    same inputs cut to 4 and 5 scalars, run by the reference with both
    moist-coefficient semantics."""
    fx = load_golden(name)
    arr = inputs(fx)
    orc = OracleDycore(arr, OracleConfig(dt=float(fx["config.dt"]), n_sub_steps=int(fx["config.n_sub_steps"]),
                                         moist=label))
    state, side = State(*(arr[k].copy() for k in STATE)), None
    for step in range(1, steps + 1):
        state, side = orc.step(state, side)
        for k in STATE:
            assert differing_words(getattr(state, k), fx[f"{label}.step{step}.{k}"]) == 0, (name, label, step, k)
        for k in SIDE:
            assert differing_words(getattr(side, k), fx[f"{label}.step{step}.side.{k}"]) == 0, (name, label, step, k)


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_oracle_matches_reference_digests_at_full_size(name):
    """2562 cells x 55 levels (two steps) and the throughput workload,
    40962 cells x 55 levels with 6 scalars at dt 720 s (one step, about a
    minute here): every output field of the oracle has the digest of the
    reference's own output on the same inputs."""
    record = load_digests(name)
    arr, same_inputs = digest_case(record)
    if not same_inputs:
        pytest.skip(f"the {name} inputs built on this host differ from the recorded ones (host SIMD paths)")
    c = record["case"]
    orc = OracleDycore(arr, OracleConfig(dt=c["dt"], n_sub_steps=c["sub_steps"], moist=c["moist_coefficients"]))
    state, side = State(*(np.asarray(arr[k]).copy() for k in STATE)), None
    for step in range(1, c["steps"] + 1):
        state, side = orc.step(state, side)
        assert mismatched_digests(record, "native", step, state, side) == [], (name, step)
