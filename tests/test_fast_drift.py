"""Fast numerics (multiply-adds contracted) against strict numerics over 24
simulated hours on the 2562-cell mesh, 55 levels, dt 1800 s (48 large
steps), both replayed as CUDA graphs.  Stated drift bounds (relative L2 per
field; about ten times the drift measured on a B200: rho 4.9e-8, rho_theta
1.5e-8, theta_m 6.0e-8, rho_u 1.9e-6, u 1.9e-6, qv 7.4e-7, rho_w 1.3e-4,
w 4.7e-4):"""

import numpy as np
import pytest

BOUNDS = {"rho": 1e-6, "rho_theta": 1e-6, "theta_m": 1e-6, "rho_u": 2e-5, "normal_velocity": 2e-5,
          "scalars": 1e-5, "rho_w": 2e-3, "vertical_velocity": 5e-3}

pytestmark = pytest.mark.gpu


def test_fast_numerics_drift_over_24_hours():
    import torch

    import hexdyn
    from hexdyn.case import build_case
    from hexdyn.config import DycoreConfig
    from hexdyn.mesh import build_mesh

    assert torch.cuda.is_available()
    case = build_case(build_mesh(4, lloyd=20, seed=0), n_levels=55, seed=0, n_condensates=1)
    strict = hexdyn.from_case(case, DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2), capture_graph=True)
    fast = hexdyn.from_case(case, DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2, numerics="fast"),
                            capture_graph=True)
    strict.step_device(48)
    fast.step_device(48)
    a, sa = strict.get_state()
    b, sb = fast.get_state()
    for k, bound in BOUNDS.items():
        x = getattr(a, k, None)
        y = getattr(b, k, None)
        if x is None:
            x, y = getattr(sa, k), getattr(sb, k)
        x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
        rel = np.linalg.norm(x - y) / np.linalg.norm(x)
        assert rel <= bound, (k, rel, bound)
    strict.close()
    fast.close()
