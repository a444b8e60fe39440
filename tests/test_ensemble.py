"""Batched ensembles against single instances, bit for bit.

Members on meshes of different size (a 162-cell and a 642-cell mesh) are
concatenated into one handle; after two large steps every member's state and
saved diagnostics must equal those of a driver created from that member
alone.  An uneven batch (members with dt and members with dt/2 stepping
twice) must equal the single instances stepped the same way.
"""

import numpy as np
import pytest

import hexdyn
from fixtures import SIDE, STATE, differing_words
from hexdyn.case import build_case
from hexdyn.config import DycoreConfig
from hexdyn.ensemble import HexEnsemble, step_batched
from hexdyn.mesh import build_mesh

pytestmark = pytest.mark.gpu

LEVELS = 12


@pytest.fixture(scope="module")
def cases():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA GPU")
    torch.cuda.set_device(0)
    m2 = build_mesh(2, lloyd=2, seed=0)
    m3 = build_mesh(3, lloyd=2, seed=0)
    return [build_case(m2, n_levels=LEVELS, seed=1, n_condensates=2, theta_noise=0.1),
            build_case(m3, n_levels=LEVELS, seed=2, n_condensates=2, theta_noise=0.1),
            build_case(m2, n_levels=LEVELS, seed=3, n_condensates=2, theta_noise=0.1)]


def _cfg(dt):
    return DycoreConfig(config_dt=dt, config_number_of_sub_steps=2, moist_coefficients="native")


def _assert_same(ens, m, single):
    st, sd = ens.get_member_state(m)
    ref_st, ref_sd = single.get_state()
    for k in STATE:
        assert differing_words(getattr(st, k), getattr(ref_st, k)) == 0, (m, k)
    for k in SIDE:
        assert differing_words(getattr(sd, k), getattr(ref_sd, k)) == 0, (m, k)


def test_ensemble_members_equal_single_instances(cases):
    cfg = _cfg(900.0)
    singles = [hexdyn.from_case(c, cfg) for c in cases]
    ens = HexEnsemble.from_cases(cases, cfg, capture_graph=True)
    assert ens.member_count == 3
    for m in range(3):
        _assert_same(ens, m, singles[m])  # the rebuilt sidecars agree before stepping
    ens.step_device(2)
    for s in singles:
        s.step_device(2)
    for m in range(3):
        _assert_same(ens, m, singles[m])
    for s in singles:
        s.close()
    ens.close()


def test_mixing_ensemble_members_equal_single_instances(cases):
    """2-D Smagorinsky mixing in an ensemble: the deformation weights and
    mesh scalings of each member are concatenated like its geometry, and
    each member's words equal its own single-instance run."""
    cfg = DycoreConfig(config_dt=900.0, config_number_of_sub_steps=2, moist_coefficients="native",
                       config_horiz_mixing="2d_smagorinsky", config_smagorinsky_coef=0.125,
                       config_visc4_2dsmag=0.05)
    members = [cases[0], cases[2]]  # one mesh: one Smagorinsky length
    singles = [hexdyn.from_case(c, cfg) for c in members]
    ens = HexEnsemble.from_cases(members, cfg, capture_graph=True)
    ens.step_device(2)
    for s in singles:
        s.step_device(2)
    for m in range(2):
        _assert_same(ens, m, singles[m])
    for s in singles:
        s.close()
    ens.close()


def test_uneven_batch_equals_single_instances(cases):
    coarse, fine = _cfg(900.0), _cfg(450.0)
    g1 = HexEnsemble.from_cases([cases[0], cases[2]], coarse, capture_graph=True)
    g2 = HexEnsemble.from_cases([cases[1]], fine, capture_graph=True)
    flags = step_batched([g1, g2], [1, 2])
    assert flags == [0, 0]
    s0, s2 = hexdyn.from_case(cases[0], coarse), hexdyn.from_case(cases[2], coarse)
    s1 = hexdyn.from_case(cases[1], fine)
    s0.step_device(1)
    s2.step_device(1)
    s1.step_device(2)
    _assert_same(g1, 0, s0)
    _assert_same(g1, 1, s2)
    _assert_same(g2, 0, s1)
    assert g1.time_seconds == 900.0 and g2.time_seconds == 900.0
    for d in (g1, g2, s0, s1, s2):
        d.close()


def test_member_upload_round_trip(cases):
    ens = HexEnsemble.from_cases(cases[:2], _cfg(900.0))
    st, _ = ens.get_member_state(1)
    np.testing.assert_array_equal(st.rho, np.asarray(cases[1].rho, dtype=np.float32))
    np.testing.assert_array_equal(st.scalars, np.asarray(cases[1].scalars, dtype=np.float32))
    ens.close()
