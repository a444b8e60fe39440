"""Partitioned single instance on the device: every rank's owned region
equals the single instance, word for word (the reference's partition
invariance, ``hexcore/partition_executor_v841.py``: owned-region union
byte-compared with the single-GPU run at every step boundary).

The ranks run in one process on one GPU (``hexdyn.partition.PartitionedDycore``:
a thread and a stream per rank, halo exchanges as device copies ordered by
events); the layouts, plans and exchange points are those a rank per GPU
uses (``RankDycore``).  The workload is 2562 cells x 55 levels renumbered
along a Hilbert curve, qv + 5 condensates (the limiter's exchange runs),
dt 720 s, two steps.
"""

import ctypes as C

import numpy as np
import pytest

import hexdyn
from fixtures import differing_words
from hexdyn import _lib, partition, reorder
from hexdyn.case import arrays_case, build_case, case_arrays
from hexdyn.config import DycoreConfig
from hexdyn.mesh import build_mesh

pytestmark = pytest.mark.gpu

SMAG = dict(config_horiz_mixing="2d_smagorinsky", config_smagorinsky_coef=0.125, config_visc4_2dsmag=0.05)


@pytest.fixture(scope="module")
def arrays():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("these tests need a CUDA GPU")
    torch.cuda.set_device(0)
    arr = case_arrays(build_case(build_mesh(4, lloyd=20, seed=0), n_levels=55, seed=0, n_condensates=5))
    return reorder.apply(arr, reorder.hilbert_order(arr))


def _config(mixing):
    return DycoreConfig(config_dt=720.0, config_number_of_sub_steps=2, moist_coefficients="native",
                        **(SMAG if mixing else {}))


def _single(arr, cfg, steps):
    drv = hexdyn.from_case(arrays_case(arr), cfg)
    out = []
    for _ in range(steps):
        drv.step_device(1)
        st, sd = drv.get_state()
        out.append(({k: getattr(st, k) for k in _lib.STATE_FIELDS}, {k: getattr(sd, k) for k in _lib.SIDECAR_FIELDS}))
    drv.close()
    return out


def _differing(got, want) -> dict:
    bad = {}
    for part in (0, 1):
        for k, v in want[part].items():
            n = differing_words(got[part][k], v)
            if n:
                bad[k] = n
    return bad


# per step: the start and the end of each of 3 subcycles x 3 RK stages; the
# initial diagnostics; one acoustic cell pass per substep (1, 1, 2 substeps
# at 2 substeps per stage); 3 transport stages; the limiter once
EXCHANGES_PER_STEP = {_lib.XCH_STATE: 10, _lib.XCH_DIAG: 1, _lib.XCH_ACOUSTIC: 12, _lib.XCH_SCALARS: 3,
                      _lib.XCH_FCT: 1}


@pytest.mark.parametrize("n_parts,mixing", [(2, False), (4, False), (3, True)])
def test_partitioned_steps_are_the_single_instance(arrays, n_parts, mixing):
    cfg = _config(mixing)
    want = _single(arrays, cfg, 2)
    part = partition.PartitionedDycore(arrays, cfg, n_parts)
    assert all(lay.l2g["cell"].size > lay.n_owned["cell"] for lay in part.layouts)
    for step in range(2):
        part.step(1)
        assert _differing(part.get_state(), want[step]) == {}, (n_parts, mixing, step)
    for r in range(n_parts):
        counts = {p: part.exchanges[r].count(p) for p in set(part.exchanges[r])}
        assert counts == {p: 2 * n for p, n in EXCHANGES_PER_STEP.items()}, r
    part.close()


def test_one_ring_of_halo_is_not_enough(arrays):
    """The comparison sees a halo that is too shallow."""
    cfg = _config(False)
    want = _single(arrays, cfg, 1)
    part = partition.PartitionedDycore(arrays, cfg, 2, halo_rings=1)
    part.step(1)
    bad = _differing(part.get_state(), want[0])
    assert bad.get("rho_u", 0) > 0 and bad.get("scalars", 0) > 0
    part.close()


def test_exchange_hook_failure_and_refusals(arrays):
    """A hook that fails aborts the step with nothing published; a hooked
    handle refuses graph capture and steps eagerly."""
    lib = _lib.load()
    cfg = _config(False)
    drv = hexdyn.from_case(arrays_case(arrays), cfg)
    before, _ = drv.get_state()
    seen = []

    def failing(user, point, nbufs, bufs, kinds):
        seen.append(point)
        return -1 if point == _lib.XCH_ACOUSTIC else 0

    hook = _lib.EXCHANGE_HOOK(failing)
    _lib.check(lib.hexdyn_set_exchange_hook(drv._handle, hook, None))
    with pytest.raises(_lib.HexDynError, match="hook aborted step 1"):
        drv.step_device(1)
    assert seen == [_lib.XCH_STATE, _lib.XCH_DIAG, _lib.XCH_ACOUSTIC]
    after, _ = drv.get_state()
    for k in _lib.STATE_FIELDS:
        assert differing_words(getattr(before, k), getattr(after, k)) == 0, k
    assert lib.hexdyn_capture_graph(drv._handle, C.c_void_p(0)) == _lib.HEXDYN_E_STATE
    # a hook that moves nothing leaves the step as it is (the callback object
    # must outlive its registration)
    noop = _lib.EXCHANGE_HOOK(lambda *a: 0)
    _lib.check(lib.hexdyn_set_exchange_hook(drv._handle, noop, None))
    drv.step_device(1)
    _lib.check(lib.hexdyn_set_exchange_hook(drv._handle, _lib.EXCHANGE_HOOK(), None))
    got, gside = drv.get_state()
    want = _single(arrays, cfg, 1)[0]
    assert _differing(({k: getattr(got, k) for k in _lib.STATE_FIELDS},
                       {k: getattr(gside, k) for k in _lib.SIDECAR_FIELDS}), want) == {}
    drv.capture_graph()   # no hook: the graph is allowed again
    drv.close()
    # ensembles take no exchange hook (a partitioned instance is one member)
    ens = hexdyn.HexEnsemble.from_cases([arrays_case(arrays), arrays_case(arrays)], cfg)
    assert lib.hexdyn_set_exchange_hook(ens._handle, noop, None) == _lib.HEXDYN_E_ARG
    ens.close()


def test_halo_pack_and_unpack_move_exactly_the_listed_rows(arrays):
    """The one-launch halo kernels against torch indexing: cell, edge and
    tracer buffers, random row lists; unpack writes those rows only."""
    import torch

    lib = _lib.load()
    drv = hexdyn.from_case(arrays_case(arrays), _config(False))
    s = drv.sizes
    S, nC, nE, T = drv.level_stride, s["n_cells"], s["n_edges"], s["n_scalars"]
    g = torch.Generator(device="cuda").manual_seed(0)
    shapes = [(1, nC), (1, nE), (T, nC), (1, nC)]
    kinds = [_lib.KIND_CELL, _lib.KIND_EDGE, _lib.KIND_TRACER, _lib.KIND_CELL]
    bufs = [torch.randn(b, n, S, device="cuda", generator=g) for b, n in shapes]
    crow = torch.randperm(nC, device="cuda", generator=g)[:777].to(torch.int32)
    erow = torch.randperm(nE, device="cuda", generator=g)[:1234].to(torch.int32)
    ptrs = (C.c_void_p * 4)(*[b.data_ptr() for b in bufs])
    kind_arr = (C.c_int * 4)(*kinds)
    words = lib.hexdyn_halo_words(drv._handle, 4, kind_arr, 777, 1234)
    assert words == (777 + 1234 + T * 777 + 777) * S
    packed = torch.empty(words, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(lib.hexdyn_halo_pack(drv._handle, 4, ptrs, kind_arr, C.c_void_p(crow.data_ptr()), 777,
                                    C.c_void_p(erow.data_ptr()), 1234, C.c_void_p(packed.data_ptr()), st))
    want = torch.cat([b[:, (erow if k == _lib.KIND_EDGE else crow).long()].reshape(-1) for b, k in zip(bufs, kinds)])
    assert torch.equal(packed, want)
    dst = [torch.zeros_like(b) for b in bufs]
    dptrs = (C.c_void_p * 4)(*[b.data_ptr() for b in dst])
    _lib.check(lib.hexdyn_halo_unpack(drv._handle, 4, dptrs, kind_arr, C.c_void_p(crow.data_ptr()), 777,
                                      C.c_void_p(erow.data_ptr()), 1234, C.c_void_p(packed.data_ptr()), st))
    for b, d, k in zip(bufs, dst, kinds):
        rows = (erow if k == _lib.KIND_EDGE else crow).long()
        mask = torch.zeros(b.shape[1], dtype=torch.bool, device="cuda")
        mask[rows] = True
        assert torch.equal(d[:, mask], b[:, mask]) and not d[:, ~mask].any()
    # refusals, before any launch
    many = (C.c_void_p * 25)(*([bufs[0].data_ptr()] * 25))
    many_kinds = (C.c_int * 25)(*([_lib.KIND_CELL] * 25))
    assert lib.hexdyn_halo_pack(drv._handle, 25, many, many_kinds, C.c_void_p(crow.data_ptr()), 777, None, 0,
                                C.c_void_p(packed.data_ptr()), st) == _lib.HEXDYN_E_ARG
    odd = (C.c_void_p * 1)(bufs[0].data_ptr() + 4)
    assert lib.hexdyn_halo_pack(drv._handle, 1, odd, kind_arr, C.c_void_p(crow.data_ptr()), 777, None, 0,
                                C.c_void_p(packed.data_ptr()), st) == _lib.HEXDYN_E_ARG
    torch.cuda.synchronize()
    drv.close()


def test_rank_dycore_runs_over_nccl(arrays):
    """The one-rank-per-GPU runner through its NCCL process group: here one
    rank (every GPU call of this suite has one GPU), so it owns the whole
    mesh, posts no transfers, and steps as the single instance does."""
    import os

    import torch
    import torch.distributed as dist

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", str(29400 + os.getpid() % 500))
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        cfg = _config(False)
        want = _single(arrays, cfg, 2)
        rank = partition.RankDycore(arrays, cfg)
        assert rank.plan.peers() == [] and rank.layout.n_owned["cell"] == arrays["mesh.areaCell"].size
        for step in range(2):
            rank.step(1)
            assert _differing(rank.get_state(), want[step]) == {}, step
        rank.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("label", ["dry", "native"])
def test_partitioned_steps_are_the_reference_outputs(label):
    """Two ranks of the 162-cell, 12-level case with qv + 5 condensates
    (tests/golden fixture made by the reference itself): the assembled owned
    regions are the reference's own two steps, word for word."""
    import torch

    from fixtures import SCALAR_VARIANTS, inputs, load_golden

    assert torch.cuda.is_available()
    torch.cuda.set_device(0)
    name, steps = SCALAR_VARIANTS[0]
    fx = load_golden(name)
    arr = inputs(fx)
    cfg = DycoreConfig(config_dt=float(fx["config.dt"]), config_number_of_sub_steps=int(fx["config.n_sub_steps"]),
                       moist_coefficients=label)
    part = partition.PartitionedDycore(arr, cfg, 2)
    for step in range(1, steps + 1):
        part.step(1)
        st, sd = part.get_state()
        want = ({k: fx[f"{label}.step{step}.{k}"] for k in _lib.STATE_FIELDS},
                {k: fx[f"{label}.step{step}.side.{k}"] for k in _lib.SIDECAR_FIELDS})
        assert _differing((st, sd), want) == {}, (label, step)
    part.close()


def test_a_failing_rank_stops_every_rank_and_publishes_nothing(arrays):
    """A rank whose exchange fails (an exception on the host, at the first
    acoustic exchange) breaks the ranks' barrier: every rank's step returns
    with an error, no state changes, and the instance steps normally after."""
    cfg = _config(False)
    part = partition.PartitionedDycore(arrays, cfg, 2, barrier_timeout=60.0)
    before = part.get_state()
    good = part._hooks[1]
    calls = []

    def failing(user, point, nbufs, bufs, kinds):
        calls.append(point)
        if point == _lib.XCH_ACOUSTIC:
            part._errors.append(RuntimeError("rank 1 lost its peer"))
            part._barrier.abort()
            return -1
        return good(user, point, nbufs, bufs, kinds)

    part._hooks[1] = _lib.EXCHANGE_HOOK(failing)
    with pytest.raises(RuntimeError, match="lost its peer"):
        part.step(1)
    assert _lib.XCH_ACOUSTIC in calls
    after = part.get_state()
    assert _differing(after, before) == {}
    part._hooks[1] = good
    want = _single(arrays, cfg, 1)
    part.step(1)
    assert _differing(part.get_state(), want[0]) == {}
    part.close()
