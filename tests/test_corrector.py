"""The learned-corrector pipeline on a small mesh: pairs of full and reduced
steps, training of both networks with the tensor-core kernels, and corrected
steps with their checks and fallback, for both reduced steps (one substep
at the same time step; a doubled time step with three substeps standing for
two full steps).

What the networks gain is measured on held-out pairs: their error on the
increments (full steps minus reduced step) must be below the error of
applying no correction.  The forecast errors over days are reported by
``python -m hexdyn.learned_eval``.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ratio,red_substeps", [(1, 1), (2, 3)])
def test_corrector_trains_and_steps(ratio, red_substeps):
    import torch

    import hexdyn
    from hexdyn.case import build_case
    from hexdyn.config import DycoreConfig
    from hexdyn.corrector import LearnedStepper, TrainedNet, make_pairs
    from hexdyn.learned_eval import _z_mid_padded
    from hexdyn.mesh import build_mesh

    assert torch.cuda.is_available()
    L = 12
    mesh = build_mesh(3, lloyd=2, seed=0)
    base = build_case(mesh, n_levels=L, seed=0, n_condensates=2)
    members = [build_case(mesh, n_levels=L, seed=10 + i, n_condensates=2, theta_noise=0.1, like=base) for i in range(3)]
    full = hexdyn.from_case(base, DycoreConfig(config_dt=1200.0, config_number_of_sub_steps=2), capture_graph=True)
    red = hexdyn.from_case(base, DycoreConfig(config_dt=1200.0 * ratio, config_number_of_sub_steps=red_substeps),
                           capture_graph=True)
    pairs = make_pairs(full, red, [(m, None) for m in members], samples=1536, times=2, ratio=ratio)
    assert pairs.col_x.shape == (1536, 6 * L) and pairs.col_y.shape == (1536, 3 * L)
    assert np.all(np.isfinite(pairs.col_x)) and np.all(np.isfinite(pairs.edge_y))
    col = TrainedNet(6 * L, 128, 3, 3 * L, seed=1)
    edge = TrainedNet(4 * L, 128, 3, L, seed=2)
    rc = col.fit(pairs.col_x, pairs.col_y, epochs=40, batch=256, lr=1e-3)
    re = edge.fit(pairs.edge_x, pairs.edge_y, epochs=40, batch=256, lr=1e-3)
    assert rc.train_loss[-1] < rc.train_loss[0]
    assert rc.val_loss < rc.val_loss_zero, (rc.val_loss, rc.val_loss_zero)
    assert re.val_loss < re.val_loss_zero, (re.val_loss, re.val_loss_zero)
    # corrected steps with the checks; every step ends finite
    red.set_state(members[0])
    stepper = LearnedStepper(full, red, col, edge, _z_mid_padded(base, red.level_stride), ratio=ratio)
    for _ in range(4):
        stepper.step()
    st, _ = red.get_state()
    assert np.all(np.isfinite(st.rho)) and np.all(np.isfinite(st.rho_u))
    assert stepper.steps == 4
    full.close()
    red.close()
