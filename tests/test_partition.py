"""Partitioned single instance, host side (CPU): ``hexdyn.partition``.

The reference's owned-first / halo-last local meshes
(``hexcore/partition_local_mesh_v841.py``) and its halo rounds as
send/receive pairs (``hexcore/partition_nccl_transport_v841.py``):

* every cell, edge and vertex is owned by exactly one rank; a rank's local
  mesh holds its owned entities first and its halo last, and every halo row
  is owned by exactly one other rank, which sends it;
* the local case arrays are a valid case (connectivity in range, slots kept
  in order) and, at one rank, the global case itself;
* over ``torch.distributed`` (gloo, two and three ranks) one exchange
  (``exchange_packed``: one packed array per peer and direction) fills
  every halo row of cell, edge and tracer buffers with its owner's value and
  leaves every owned row alone.

The device step over these meshes is compared with the single instance in
tests/test_partition_gpu.py.
"""

import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from hexdyn import partition
from hexdyn.case import arrays_case, build_case, case_arrays
from hexdyn.mesh import build_mesh

S = 8


def _arrays(level=3, levels=6, condensates=2):
    return case_arrays(build_case(build_mesh(level, lloyd=2, seed=0), n_levels=levels, seed=0,
                                  n_condensates=condensates))


ARR = _arrays()


@pytest.mark.parametrize("n_parts", [1, 2, 3, 4])
@pytest.mark.parametrize("rings", [1, 2, 3])
def test_layouts_cover_every_entity_once(n_parts, rings):
    lays = partition.layouts(ARR, n_parts, rings)
    for kind, n in (("cell", ARR["mesh.areaCell"].size), ("edge", ARR["mesh.dcEdge"].size),
                    ("vertex", ARR["mesh.areaTriangle"].size)):
        owned = np.concatenate([lay.owned(kind) for lay in lays])
        assert np.array_equal(np.sort(owned), np.arange(n)), kind
        for lay in lays:
            l2g = lay.l2g[kind]
            assert np.unique(l2g).size == l2g.size
            assert np.all(lay.owner[kind][l2g[: lay.n_owned[kind]]] == lay.rank)
            assert np.all(lay.owner[kind][l2g[lay.n_owned[kind]:]] != lay.rank)
    plans = partition.plans(lays)
    for p in plans:
        for (q, kind), (mine, theirs) in p.recv.items():
            # the owner sends exactly these rows, in this order
            assert np.array_equal(plans[q].send[(p.rank, kind)], theirs)
            assert np.array_equal(lays[q].l2g[kind][theirs], lays[p.rank].l2g[kind][mine])


def test_halo_rings_reach_the_stencil():
    """``rings`` rings of cells around the owned set, every edge and vertex
    of a local cell."""
    coc, deg = ARR["mesh.cellsOnCell"], ARR["mesh.nEdgesOnCell"]
    lay1 = partition.layouts(ARR, 3, 1)[1]
    cells = set(lay1.l2g["cell"].tolist())
    for c in lay1.owned("cell"):
        assert set(coc[c, : deg[c]].tolist()) <= cells
    lay2 = partition.layouts(ARR, 3, 2)[1]
    assert set(lay1.l2g["cell"].tolist()) < set(lay2.l2g["cell"].tolist())
    eoc = ARR["mesh.edgesOnCell"]
    edges = set(lay2.l2g["edge"].tolist())
    for c in lay2.l2g["cell"]:
        assert set(eoc[c, : deg[c]].tolist()) <= edges


def test_local_case_is_valid_and_one_rank_is_the_global_case():
    lay = partition.layouts(ARR, 1, 2)[0]
    loc = partition.local_arrays(ARR, lay)
    for k, v in ARR.items():
        a, b = np.asarray(v), np.asarray(loc[k])
        assert a.shape == b.shape and np.array_equal(a, b), k
    for n_parts in (2, 4):
        for lay in partition.layouts(ARR, n_parts, 2):
            loc = partition.local_arrays(ARR, lay)
            nc, ne, nv = (lay.l2g[k].size for k in ("cell", "edge", "vertex"))
            deg = loc["mesh.nEdgesOnCell"]
            slot = np.arange(loc["mesh.cellsOnCell"].shape[1])[None, :] < deg[:, None]
            for key, n in (("mesh.cellsOnCell", nc), ("mesh.edgesOnCell", ne), ("mesh.verticesOnCell", nv)):
                vals = loc[key][slot]
                assert vals.min() >= 0 and vals.max() < n, key
            for key, n in (("mesh.cellsOnEdge", nc), ("mesh.verticesOnEdge", nv), ("mesh.cellsOnVertex", nc),
                           ("mesh.edgesOnVertex", ne)):
                assert loc[key].min() >= 0 and loc[key].max() < n, key
            # an owned cell keeps its neighbours, in slot order
            g2l = lay.g2l("cell")
            for c in lay.owned("cell")[:50]:
                lc = g2l[c]
                assert np.array_equal(lay.l2g["cell"][loc["mesh.cellsOnCell"][lc, : deg[lc]]],
                                      ARR["mesh.cellsOnCell"][c, : deg[lc]])
            case = arrays_case(loc)
            assert case.rho.shape == (ARR["rho"].shape[0], nc) and case.rho_u.shape[1] == ne
            assert case.scalars.shape[2] == nc and case.zb_cell.shape[1] == nc


def _encode(kind_ids: np.ndarray, blocks: int) -> np.ndarray:
    """A (blocks, rows, S) buffer whose row of global id g holds g + 0.5 b
    at every level of block b."""
    b = np.arange(blocks, dtype=np.float32)[:, None, None]
    return (kind_ids.astype(np.float32)[None, :, None] + np.float32(0.5) * b) * np.ones((1, 1, S), np.float32)


def _exchange_worker(rank, world, port, result_dir):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lays = partition.layouts(ARR, world, 2)
        plan = partition.ExchangePlan.build(lays, rank)
        lay = lays[rank]
        bufs, want = [], []
        for kind, blocks in (("cell", 1), ("edge", 1), ("cell", 3)):
            full = _encode(lay.l2g[kind], blocks)
            start = full.copy()
            start[:, lay.n_owned[kind]:] = -7.0   # halo rows not yet received
            bufs.append((torch.from_numpy(start), kind))
            want.append(full)
        packer = partition.TorchRows(bufs)
        partition.exchange_packed(plan, packer)
        partition.exchange_packed(plan, packer)   # idempotent on owner truth
        ok = all(np.array_equal(b.numpy(), w) for (b, _), w in zip(bufs, want))
        open(os.path.join(result_dir, f"rank{rank}"), "w").write("ok" if ok else "bad")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_exchange_fills_every_halo_row(tmp_path, world):
    port = 29500 + (os.getpid() % 1000) + world
    mp.start_processes(_exchange_worker, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn")
    for r in range(world):
        assert (tmp_path / f"rank{r}").read_text() == "ok", r
