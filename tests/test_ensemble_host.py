"""Host-side ensemble logic: refusal of incompatible members (before any
device work) and the assignment of members to GPUs, including two gloo
ranks that compute it independently."""

import ctypes as C
import os
import socket

import numpy as np
import pytest

import hexdyn._lib as L
from fixtures import case_from_arrays, inputs, load_golden
from hexdyn.config import DycoreConfig
from hexdyn.driver import _build_descriptor
from hexdyn.ensemble import assign_members


def _desc(name, dt):
    case = case_from_arrays(inputs(load_golden(name)))
    cfg = DycoreConfig(config_dt=dt, config_number_of_sub_steps=2)
    return _build_descriptor(case.mesh, case, case.vertical, case, cfg, case, case, case)


def test_ensemble_refuses_members_that_differ():
    lib = L.load()
    d0, k0, _ = _desc("l2_L12", 1800.0)
    d1, k1, _ = _desc("l2_L12", 900.0)
    h = C.c_void_p()
    arr = (L.HexDynDesc * 2)(d0, d1)
    assert lib.hexdyn_create_ensemble(arr, 2, C.byref(h)) == L.HEXDYN_E_ARG
    assert "member 1 differs from member 0 in dt" in L.last_error()
    d2, k2, _ = _desc("l3_L20", 1800.0)
    arr = (L.HexDynDesc * 2)(d0, d2)
    assert lib.hexdyn_create_ensemble(arr, 2, C.byref(h)) == L.HEXDYN_E_ARG
    assert "n_levels" in L.last_error()
    assert lib.hexdyn_create_ensemble(arr, 0, C.byref(h)) == L.HEXDYN_E_ARG
    assert not h.value


def _mixing_desc(name, coef):
    case = case_from_arrays(inputs(load_golden(name)))
    cfg = DycoreConfig(config_dt=1800.0, config_number_of_sub_steps=2, config_horiz_mixing="2d_smagorinsky",
                       config_smagorinsky_coef=coef, config_visc4_2dsmag=0.05)
    return _build_descriptor(case.mesh, case, case.vertical, case, cfg, case, case, case)


def test_mixing_ensemble_refuses_members_with_other_mixing():
    """Members of a mixing ensemble share the option and its constants (the
    Smagorinsky length scales with the mesh)."""
    lib = L.load()
    d0, k0, _ = _mixing_desc("l2_L12", 0.125)
    d1, k1, _ = _desc("l2_L12", 1800.0)
    h = C.c_void_p()
    arr = (L.HexDynDesc * 2)(d0, d1)
    assert lib.hexdyn_create_ensemble(arr, 2, C.byref(h)) == L.HEXDYN_E_ARG
    assert "mixing or upper-damping options" in L.last_error()
    d2, k2, _ = _mixing_desc("l2_L12", 0.1)
    arr = (L.HexDynDesc * 2)(d0, d2)
    assert lib.hexdyn_create_ensemble(arr, 2, C.byref(h)) == L.HEXDYN_E_ARG
    assert "mixing or upper-damping constants" in L.last_error()
    assert not h.value


def test_batched_step_refuses_bad_batches():
    lib = L.load()
    assert lib.hexdyn_step_batched(None, None) == L.HEXDYN_E_ARG
    b = L.HexDynBatch(0, None, None, None)
    assert lib.hexdyn_step_batched(C.byref(b), None) == L.HEXDYN_E_ARG
    groups = (C.c_void_p * 1)(None)
    steps = (C.c_int32 * 1)(1)
    b = L.HexDynBatch(1, groups, steps, None)
    assert lib.hexdyn_step_batched(C.byref(b), None) == L.HEXDYN_E_ARG
    assert "NULL" in L.last_error()


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_assign_members_covers_all_and_balances(world):
    cells = [10242] * 24 + [40962] * 16
    shares = assign_members(cells, world)
    flat = sorted(m for s in shares for m in s)
    assert flat == list(range(len(cells)))
    loads = [sum(cells[m] for m in s) for s in shares]
    assert max(loads) - min(loads) <= max(cells)
    assert shares == assign_members(cells, world)  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, cells, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = assign_members(cells, world)[rank]
    everyone = [None] * world
    dist.all_gather_object(everyone, mine)
    # the end-of-run reduction of member-steps (no per-step collective)
    import torch

    t = torch.tensor([len(mine)], dtype=torch.int64)
    dist.all_reduce(t)
    dist.destroy_process_group()
    q.put((rank, mine, everyone, int(t.item())))


def test_two_gloo_ranks_agree_on_the_assignment():
    import multiprocessing as mp

    cells = [10242] * 24 + [40962] * 16
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, cells, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, mine, everyone, total in out:
        assert everyone[rank] == mine
        assert total == len(cells)
    a, b = out[0][1], out[1][1]
    assert not set(a) & set(b) and sorted(a + b) == list(range(len(cells)))
    assert np.isclose(sum(cells[m] for m in a), sum(cells[m] for m in b), rtol=0.1)
