"""The launch-shape autotuner: it picks a block size per kernel label, leaves
the state and sidecar exactly as they were, and the tuned step (replayed
from graphs captured again after tuning) is bit-identical to the untuned
one."""

import pytest

import hexdyn
from fixtures import SIDE, STATE, case_from_arrays, differing_words, inputs, load_golden
from hexdyn.config import DycoreConfig

pytestmark = pytest.mark.gpu


def test_autotune_keeps_state_and_results():
    import torch

    assert torch.cuda.is_available()
    arr = inputs(load_golden("l2_L12"))
    cfg = DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2, moist_coefficients="native")
    ref = hexdyn.from_case(case_from_arrays(arr), cfg, capture_graph=True)
    tuned = hexdyn.from_case(case_from_arrays(arr), cfg, capture_graph=True)
    before, side_before = tuned.get_state()
    report = tuned.autotune(steps_per_candidate=1)
    sizes = (64, 96, 128, 160, 192, 224, 256)
    assert report and all(v["threads"] in sizes and tuple(v["us"]) == sizes for v in report.values())
    assert "k_tend_u" in report and "k_ac_cell_first" in report
    after, side_after = tuned.get_state()
    for k in STATE:
        assert differing_words(getattr(after, k), getattr(before, k)) == 0, k
    for k in SIDE:
        assert differing_words(getattr(side_after, k), getattr(side_before, k)) == 0, k
    a, b = ref.step(2), tuned.step(2)
    for k in STATE:
        assert differing_words(getattr(a.state, k), getattr(b.state, k)) == 0, k
    for k in SIDE:
        assert differing_words(getattr(a.saved_diagnostics, k), getattr(b.saved_diagnostics, k)) == 0, k
    ref.close()
    tuned.close()
