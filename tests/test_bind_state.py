"""Caller-owned state buffers (hexdyn_bind_state): the handle steps from them
without a copy, the result alternates between them and the library's own
buffers, and it equals an ordinary driver's step bit for bit."""

import ctypes as C

import pytest

import hexdyn
import hexdyn._lib as L
from fixtures import SIDE, STATE, case_from_arrays, differing_words, inputs, load_golden
from hexdyn.config import DycoreConfig
from hexdyn.driver import DeviceAtmosphere

pytestmark = pytest.mark.gpu


def _logical(drv, name, padded):
    rows = drv._rows(name)
    n, blocks = drv._entities(name)
    if blocks > 1:
        return padded.reshape(blocks, n, -1)[:, :, :rows].transpose(1, 2).cpu().numpy()
    return padded[:, :rows].t().cpu().numpy()


def test_bound_buffers_step_like_the_driver():
    import torch

    assert torch.cuda.is_available()
    arr = inputs(load_golden("l2_L12"))
    cfg = DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2, moist_coefficients="native")
    ref = hexdyn.from_case(case_from_arrays(arr), cfg)
    drv = hexdyn.from_case(case_from_arrays(arr), cfg, capture_graph=True)
    atm = DeviceAtmosphere(drv)
    bufs = {k: atm.padded(k).clone() for k in L.FIELDS}
    # a misaligned field is refused before anything changes
    bad = dict(bufs)
    bad["rho"] = bufs["rho"].view(-1)[1:]
    with pytest.raises(L.HexDynError):
        drv.bind_state(bad)
    drv.bind_state(bufs)
    expect = ref.step(2)
    drv.step_device(2)  # even: the new state is back in the bound buffers
    torch.cuda.synchronize()
    for k in STATE:
        assert differing_words(_logical(drv, k, bufs[k]), getattr(expect.state, k)) == 0, k
    for k in SIDE:
        assert differing_words(_logical(drv, k, bufs[k]), getattr(expect.saved_diagnostics, k)) == 0, k
    # unbinding needs the state in the library's buffers (odd step count)
    rc = L.load().hexdyn_bind_state(drv._handle, None, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == L.HEXDYN_E_STATE
    expect = ref.step(1)
    drv.step_device(1)
    drv.bind_state(None)
    got, side = drv.get_state()
    for k in STATE:
        assert differing_words(getattr(got, k), getattr(expect.state, k)) == 0, k
    ref.close()
    drv.close()
