"""The no-allocation step entry point against the ordinary step.

``hexdyn_step_noalloc`` exists for callers that cannot call cudaMalloc when
they step (a framework whose device memory pool must not be bypassed,
ensemble members that own their state buffers but have no workspace): it
takes caller-owned input and output buffers and keeps every intermediate in
the library's fixed 64 MiB device array.  Its results must equal
``hexdyn_step`` word for word (the strict tests' tolerance) on two calls in a
row, also right after a call on another mesh has left its words in the
array.  The buffers below are allocated by the test itself; the entry point
allocates nothing.
"""

import ctypes as C

import numpy as np
import pytest

import hexdyn
import hexdyn._lib as L
from fixtures import SIDE, STATE, case_from_arrays, differing_words, inputs, load_golden
from hexdyn.config import DycoreConfig
from hexdyn.driver import DeviceAtmosphere

pytestmark = pytest.mark.gpu


MIXING = dict(config_horiz_mixing="2d_smagorinsky", config_smagorinsky_coef=0.125, config_visc4_2dsmag=0.05)


def _driver(arr, mixing=False):
    cfg = DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2, moist_coefficients="native",
                       **(MIXING if mixing else {}))
    return hexdyn.from_case(case_from_arrays(arr), cfg)


def _logical(drv, name, padded):
    rows = drv._rows(name)
    n, blocks = drv._entities(name)
    if blocks > 1:
        return padded.reshape(blocks, n, -1)[:, :, :rows].transpose(1, 2).cpu().numpy()
    return padded[:, :rows].t().cpu().numpy()


def _noalloc_once(drv) -> None:
    """One no-alloc step of ``drv``'s uploaded state into fresh buffers."""
    import torch

    atm = DeviceAtmosphere(drv)
    f_in, f_out, keep = L.HexDynFields(), L.HexDynFields(), []
    for k, i in L.FIELDS.items():
        a = atm.padded(k).clone()
        b = torch.empty_like(a)
        keep += [a, b]
        f_in.field[i], f_out.field[i] = a.data_ptr(), b.data_ptr()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.load().hexdyn_step_noalloc(drv._handle, C.byref(f_in), C.byref(f_out), stream, None)
    assert rc == L.HEXDYN_OK, L.last_error()
    torch.cuda.synchronize()


@pytest.mark.parametrize("mixing,other_mesh_first", [(False, False), (True, False), (False, True)])
def test_noalloc_step_equals_step_on_two_calls(mixing, other_mesh_first):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA GPU")
    torch.cuda.set_device(0)
    if other_mesh_first:
        # a 642-cell, 20-level step leaves words of another layout in the array
        other = _driver(inputs(load_golden("l3_L20")), mixing=True)
        _noalloc_once(other)
        other.close()
    arr = inputs(load_golden("l2_L12"))
    ref = _driver(arr, mixing)
    noa = _driver(arr, mixing)
    atm = DeviceAtmosphere(noa)
    names = list(L.FIELDS)
    # caller-owned buffers in the padded layout, the input filled from the
    # driver's uploaded state
    bufs_in = {k: atm.padded(k).clone() for k in names}
    bufs_out = {k: torch.full_like(v, float("nan")) for k, v in bufs_in.items()}
    lib = L.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for step in (1, 2):
        expect = ref.step()
        f_in, f_out = L.HexDynFields(), L.HexDynFields()
        for k in names:
            f_in.field[L.FIELDS[k]] = bufs_in[k].data_ptr()
            f_out.field[L.FIELDS[k]] = bufs_out[k].data_ptr()
        flag = C.c_int(-1)
        rc = lib.hexdyn_step_noalloc(noa._handle, C.byref(f_in), C.byref(f_out), stream, C.byref(flag))
        assert rc == L.HEXDYN_OK, L.last_error()
        assert flag.value == 0
        torch.cuda.synchronize()
        for k in STATE:
            got = _logical(noa, k, bufs_out[k])
            assert differing_words(got, getattr(expect.state, k)) == 0, (step, k)
        for k in SIDE:
            got = _logical(noa, k, bufs_out[k])
            assert differing_words(got, getattr(expect.saved_diagnostics, k)) == 0, (step, k)
        bufs_in, bufs_out = bufs_out, bufs_in
    ref.close()
    noa.close()


def test_noalloc_step_refuses_aliasing_and_oversize():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA GPU")
    arr = inputs(load_golden("l2_L12"))
    drv = _driver(arr)
    atm = DeviceAtmosphere(drv)
    lib = L.load()
    f = L.HexDynFields()
    for k, i in L.FIELDS.items():
        f.field[i] = atm.padded(k).data_ptr()
    rc = lib.hexdyn_step_noalloc(drv._handle, C.byref(f), C.byref(f), None, None)
    assert rc == L.HEXDYN_E_ARG and "same buffer" in L.last_error()
    drv.close()
    # 2562 cells x 55 levels with 6 tracers needs more than the 64 MiB array
    from hexdyn.case import build_case
    from hexdyn.mesh import build_mesh

    big = build_case(build_mesh(4, lloyd=2, seed=0), n_levels=55, seed=0, n_condensates=5)
    cfg = DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2)
    drv = hexdyn.from_case(big, cfg)
    atm = DeviceAtmosphere(drv)
    fin, fout = L.HexDynFields(), L.HexDynFields()
    keep = []
    for k, i in L.FIELDS.items():
        a = atm.padded(k)
        b = torch.empty_like(a)
        keep.append(b)
        fin.field[i] = a.data_ptr()
        fout.field[i] = b.data_ptr()
    rc = lib.hexdyn_step_noalloc(drv._handle, C.byref(fin), C.byref(fout), None, None)
    assert rc == L.HEXDYN_E_CAPACITY and "bytes of step scratch" in L.last_error()
    drv.close()
