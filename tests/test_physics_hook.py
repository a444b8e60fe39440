"""The per-stage physics hand-off of ``_step_device_v841``
(``physics_stage_callback``, hexcore/cuda_driver.py:4393-4400).

The same callback -- tendencies formed from the stage's state and saved
diagnostics by single FP32 products, identical on the host and the device --
drives the oracle (``OracleConfig.physics_stage``) and the CUDA step (a host
hook called before every RK stage); the two steps, and the modified theta
dynamics rate handed to the post-transport callback, must agree word for
word.  The oracle places each tendency where the reference's CUDA driver
adds it: ``(tend_ru + saved Euler) + rho_u``; ``tend_rt`` + ``rho x
diabatic_theta``, + the saved mixing, + ``rho_theta``; the density
tendency of a subcycle's last stage into the next subcycle's saved density
tendency; the rate ``(tend_rt - tend_rho theta_m) / rho`` at RK stage 3.
"""

import numpy as np
import pytest

from fixtures import SIDE, STATE, case_from_arrays, differing_words, inputs, load_golden
from oracle.dycore import OracleConfig, OracleDycore, State

F32 = np.float32
C_U, C_RT, C_RHO, C_DTH = F32(-1.0e-5), F32(1.0e-6), F32(1.0e-7), F32(2.0e-6)


class Tendencies:
    def __init__(self, rho_u, rho_theta, rho, diabatic_theta):
        self.rho_u, self.rho_theta, self.rho, self.diabatic_theta = rho_u, rho_theta, rho, diabatic_theta


def numpy_callback(calls):
    def cb(*, rk_step, dynamics_substep, state, saved):
        calls.append((dynamics_substep, rk_step))
        return Tendencies(state.rho_u * C_U, state.rho * C_RT, saved.density_perturbation * C_RHO,
                          saved.theta_m * C_DTH)
    return cb


def test_oracle_hook_runs_before_every_stage_and_changes_the_step():
    fx = load_golden("l2_L12")
    arr = inputs(fx)
    calls = []
    orc = OracleDycore(arr, OracleConfig(dt=1800.0, n_sub_steps=2, moist="native",
                                         physics_stage=numpy_callback(calls)))
    st, sd = orc.step(State(*(arr[k].copy() for k in STATE)))
    assert calls == [(s, r) for s in (1, 2, 3) for r in (1, 2, 3)]
    assert orc.modified_rate is not None and orc.modified_rate.shape == arr["rho"].shape
    plain, _ = OracleDycore(arr, OracleConfig(dt=1800.0, n_sub_steps=2, moist="native")).step(
        State(*(arr[k].copy() for k in STATE)))
    assert differing_words(st.rho_u, plain.rho_u) > 0 and differing_words(st.rho_theta, plain.rho_theta) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("smag", [False, True])
def test_cuda_stage_callback_matches_oracle(smag):
    import torch

    import hexdyn
    from hexdyn.config import DycoreConfig

    assert torch.cuda.is_available()
    torch.cuda.set_device(0)
    fx = load_golden("l2_L12")
    arr = inputs(fx)
    mix = dict(config_horiz_mixing="2d_smagorinsky", config_smagorinsky_coef=0.125,
               config_visc4_2dsmag=0.05) if smag else {}
    cfg = DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2, moist_coefficients="native", **mix)
    drv = hexdyn.from_case(case_from_arrays(arr), cfg)
    calls, rates = [], []
    c = {k: torch.tensor(v, dtype=torch.float32, device="cuda") for k, v in
         (("u", C_U), ("rt", C_RT), ("rho", C_RHO), ("dth", C_DTH))}

    def gpu_cb(*, rk_step, dynamics_substep, state, saved, diagnostics):
        calls.append((dynamics_substep, rk_step))
        return Tendencies(state.rho_u * c["u"], state.rho * c["rt"], saved.density_perturbation * c["rho"],
                          saved.theta_m * c["dth"])

    def post(*, state, saved, outer_state, modified_theta_dynamics_rate):
        rates.append(modified_theta_dynamics_rate.cpu().numpy().copy())

    okw = {}
    if smag:
        from oracle.mixing import SmagorinskyConfig

        okw["smagorinsky"] = SmagorinskyConfig(0.125, 0.05, 10.0)
    ocalls = []
    orc = OracleDycore(arr, OracleConfig(dt=1800.0, n_sub_steps=2, moist="native",
                                         physics_stage=numpy_callback(ocalls), **okw))
    st, sd = State(*(arr[k].copy() for k in STATE)), None
    for step in (1, 2):
        drv._step_device_v841(physics_stage_callback=gpu_cb, physics_post_transport_callback=post,
                              physics_mass_loading_count=arr["scalars"].shape[0])
        got, gside = drv.get_state()
        st, sd = orc.step(st, sd)
        for k in STATE:
            assert differing_words(getattr(got, k), getattr(st, k)) == 0, (step, k)
        for k in SIDE:
            assert differing_words(getattr(gside, k), getattr(sd, k)) == 0, (step, k)
        assert differing_words(rates[-1], orc.modified_rate) == 0, step
    assert calls == ocalls == [(s, r) for _ in (1, 2) for s in (1, 2, 3) for r in (1, 2, 3)]
    drv.close()


@pytest.mark.gpu
def test_stage_callback_errors_and_refusals():
    import torch

    import hexdyn
    from hexdyn.config import ConfigurationRefusal, DycoreConfig

    assert torch.cuda.is_available()
    fx = load_golden("l2_L12")
    arr = inputs(fx)
    drv = hexdyn.from_case(case_from_arrays(arr), DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2))
    before, _ = drv.get_state()
    with pytest.raises(RuntimeError, match="returned no sources"):
        drv._step_device_v841(physics_stage_callback=lambda **kw: None)
    after, _ = drv.get_state()
    for k in STATE:  # nothing was published
        assert differing_words(getattr(before, k), getattr(after, k)) == 0, k
    with pytest.raises(ConfigurationRefusal) as err:
        drv._step_device_v841(physics_tendencies=object())
    assert err.value.knob == "held_physics_tendencies"
    with pytest.raises(ConfigurationRefusal) as err:
        drv._step_device_v841(physics_mass_loading_count=arr["scalars"].shape[0] + 1)
    assert err.value.knob == "physics_mass_loading_count"
    # the plain step still runs, and as a graph, once the callback is gone
    drv.capture_graph()
    drv.step_device(1)
    drv.close()
