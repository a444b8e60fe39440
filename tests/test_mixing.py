"""Host set-up of the 2-D Smagorinsky mixing (hexdyn.mixing): the
deformation weights of the 162-cell mesh equal the reference's
(hexcore/mixing_v841.py:495, strict geometry) word for word, and the
smagorinsky_2d constants follow its FP32 formulas."""

import numpy as np

from fixtures import differing_words, inputs, load_golden
from hexdyn import mixing
from hexdyn.config import DycoreConfig


def test_host_deformation_weights_match_reference():
    fx = load_golden("l2_L12_smag")
    mesh = {k[5:]: v for k, v in inputs(fx).items() if k.startswith("mesh.")}
    c2, s2, cs = mixing.deformation_weights(mesh)
    for got, key in ((c2, "mix.coef_c2"), (s2, "mix.coef_s2"), (cs, "mix.coef_cs")):
        assert differing_words(got, fx[key]) == 0, key


def test_smagorinsky_constants():
    fx = load_golden("l2_L12_smag")
    mesh = {k[5:]: v for k, v in inputs(fx).items() if k.startswith("mesh.")}
    cfg = DycoreConfig(config_dt=1800.0, config_horiz_mixing="2d_smagorinsky", config_smagorinsky_coef=0.125,
                       config_visc4_2dsmag=0.05)
    length = np.float32(float(np.asarray(mesh["nominalMinDc"])))
    m = mixing.setup(mesh, cfg, length)
    f = np.float32
    assert m.strain_scale == (f(0.125) * length) * (f(0.125) * length)
    assert m.ceiling == (f(0.01) * (length * length)) * (f(1.0) / f(1800.0))
    assert m.h4 == f(0.05) * ((length * length) * length)
    assert np.all(m.del2 == f(1.0)) and np.all(m.del4 == f(1.0))  # uniform meshDensity
