"""One dycore instance partitioned over ranks.

The reference partitions a single instance the same way
(``hexcore/partition_local_mesh_v841.py``, ``partition_executor_v841.py``,
``partition_nccl_transport_v841.py``):

* cells are split among the ranks in contiguous ranges of the cell numbering
  (``cell_owners``; the parts are compact when the numbering follows a
  space-filling curve, ``hexdyn.reorder.hilbert_order``); an edge belongs to
  the owner of its first cell, a vertex to the owner of its first cell;
* each rank steps a local mesh (``local_arrays``): its owned cells, edges and
  vertices first, then a halo of ``halo_rings`` rings of neighbouring cells
  and every edge and vertex of a local cell.  Connectivity is mapped to local
  indices; a reference to an entity outside the local set becomes local index
  0 (such rows only feed halo values that the next exchange overwrites);
* owner values reach the halo at the exchange points of the step
  (``hexdyn_set_exchange_hook``): the step's start, after the initial solve
  diagnostics, after every acoustic cell pass, at the end of every RK stage,
  at every transport stage entry and after the limiter's scale factors.
  Every halo entity is owned by exactly one other rank, so an exchange is a
  gather of owned rows on the owner and a scatter into the receiver's halo
  rows (``ExchangePlan``).  An exchange does no arithmetic: with a halo deep
  enough for the stencils between two exchanges (``halo_rings_for``: two
  rings, three with 2-D Smagorinsky mixing, whose fourth-order filter of the
  subcycle's start state reaches one ring further), each rank's owned region
  is the single instance's, word for word.

Two runners share the layouts and plans:

* ``PartitionedDycore`` -- P ranks in one process on one device: one thread
  and one stream per rank, exchanges as device copies between the ranks'
  buffers, ordered by CUDA events and a host barrier (no kernel waits on
  another kernel);
* ``RankDycore`` -- one rank per process and GPU over ``torch.distributed``
  (NCCL): at each point one packed array of owned rows per peer is sent
  and one received (``exchange_packed``), posted in the same order on every
  rank.

Rows move with the library's one-launch kernels (``hexdyn_halo_pack`` /
``hexdyn_halo_unpack``): every buffer of an exchange point in one launch per
peer and direction.
"""

from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import _lib
from .reorder import _CASE, _MESH_ROWS, _PASS, _sizes

ENTITIES = ("cell", "edge", "vertex")


def cell_owners(n_cells: int, n_parts: int) -> np.ndarray:
    """Owner rank of every cell: contiguous, near-equal ranges of the cell
    numbering."""
    if not 1 <= n_parts <= n_cells:
        raise ValueError(f"cannot split {n_cells} cells into {n_parts} parts")
    return (np.arange(n_cells, dtype=np.int64) * n_parts) // n_cells


@dataclass
class Layout:
    """One rank's local numbering: ``l2g[kind][local] = global``, owned
    entities first (ascending global index), halo last (ascending)."""

    rank: int
    l2g: dict[str, np.ndarray]
    n_owned: dict[str, int]
    owner: dict[str, np.ndarray] = field(repr=False)   # global index -> owner rank

    @staticmethod
    def build(arr: dict, owner_cells: np.ndarray, rank: int, halo_rings: int) -> "Layout":
        coc = np.asarray(arr["mesh.cellsOnCell"], dtype=np.int64)
        deg = np.asarray(arr["mesh.nEdgesOnCell"], dtype=np.int64)
        eoc = np.asarray(arr["mesh.edgesOnCell"], dtype=np.int64)
        voc = np.asarray(arr["mesh.verticesOnCell"], dtype=np.int64)
        owner = {"cell": np.asarray(owner_cells, dtype=np.int64)}
        owner["edge"] = owner["cell"][np.asarray(arr["mesh.cellsOnEdge"], dtype=np.int64)[:, 0]]
        owner["vertex"] = owner["cell"][np.asarray(arr["mesh.cellsOnVertex"], dtype=np.int64)[:, 0]]
        slot = np.arange(coc.shape[1])[None, :] < deg[:, None]
        local = owner["cell"] == rank
        if not local.any():
            raise ValueError(f"rank {rank} owns no cell")
        for _ in range(halo_rings):
            local[coc[local[:, None] & slot]] = True
        cells = np.flatnonzero(local)
        members = {"cell": cells, "edge": np.unique(eoc[cells][slot[cells]]),
                   "vertex": np.unique(voc[cells][slot[cells]])}
        l2g, n_owned = {}, {}
        for kind, ids in members.items():
            mine = owner[kind][ids] == rank
            l2g[kind] = np.concatenate([ids[mine], ids[~mine]]).astype(np.int64)
            n_owned[kind] = int(mine.sum())
        return Layout(rank, l2g, n_owned, owner)

    def g2l(self, kind: str) -> np.ndarray:
        """Global index -> local index, -1 where the entity is not local."""
        out = np.full(self.owner[kind].size, -1, dtype=np.int64)
        out[self.l2g[kind]] = np.arange(self.l2g[kind].size)
        return out

    def owned(self, kind: str) -> np.ndarray:
        return self.l2g[kind][: self.n_owned[kind]]


def halo_rings_for(config) -> int:
    """Cell rings the stencils between two exchanges reach: edge values of
    the tracer and theta advection read the second ring; the Smagorinsky
    filter of the subcycle's start state (del2 of del2 on edges) one more."""
    return 3 if getattr(config, "config_horiz_mixing", "") == "2d_smagorinsky" else 2


def layouts(arr: dict, n_parts: int, halo_rings: int = 2) -> list[Layout]:
    owner = cell_owners(_sizes(arr)["cell"], n_parts)
    return [Layout.build(arr, owner, r, halo_rings) for r in range(n_parts)]


def _local_index(values: np.ndarray, g2l: np.ndarray) -> np.ndarray:
    """Connectivity values mapped to local indices: unused slots (negative)
    kept, entities outside the local set mapped to 0."""
    v = np.asarray(values)
    out = v.copy()
    used = v >= 0
    out[used] = np.maximum(g2l[v[used]], 0)
    return out


def local_arrays(arr: dict, lay: Layout) -> dict[str, Any]:
    """The case arrays (``hexdyn.case.case_arrays`` layout) of one rank's
    local mesh: entity-indexed arrays gathered by ``lay.l2g``, connectivity
    mapped to local indices, everything else shared."""
    g2l = {k: lay.g2l(k) for k in ENTITIES}
    out: dict[str, Any] = {}
    for key, value in arr.items():
        if key.startswith("mesh."):
            name = key[5:]
            for entity, table in _MESH_ROWS.items():
                if name in table:
                    a = np.asarray(value)[lay.l2g[entity]]
                    target = table[name]
                    out[key] = _local_index(a, g2l[target]) if target else a
                    break
            else:
                if np.asarray(value).ndim > 0:
                    raise ValueError(f"no partition rule for mesh array {name!r}")
                out[key] = value
        elif key in _CASE:
            entity, axis, target = _CASE[key]
            a = np.take(np.asarray(value), lay.l2g[entity], axis=axis)
            out[key] = _local_index(a, g2l[target]) if target else a
        elif key in _PASS:
            out[key] = value
        else:
            raise ValueError(f"no partition rule for case array {key!r}")
    for key, kind in (("mesh.nCells", "cell"), ("mesh.nEdges", "edge"), ("mesh.nVertices", "vertex")):
        if key in out:
            out[key] = np.array(lay.l2g[kind].size)
    return out


@dataclass
class ExchangePlan:
    """What one rank receives and sends at every exchange.

    ``recv[(peer, kind)] = (local halo rows here, local owned rows on peer)``
    and ``send[(peer, kind)] = local owned rows here``, in the receiver's halo
    order, for ``kind`` in ``cell`` / ``edge`` (vertices carry no exchanged
    state: their values derive from cells and edges each stage)."""

    rank: int
    recv: dict[tuple[int, str], tuple[np.ndarray, np.ndarray]]
    send: dict[tuple[int, str], np.ndarray]

    @staticmethod
    def build(lays: list[Layout], rank: int) -> "ExchangePlan":
        recv: dict[tuple[int, str], tuple[np.ndarray, np.ndarray]] = {}
        send: dict[tuple[int, str], np.ndarray] = {}
        for kind in ("cell", "edge"):
            for p, lay in enumerate(lays):
                halo = np.arange(lay.n_owned[kind], lay.l2g[kind].size)
                owners = lay.owner[kind][lay.l2g[kind][halo]]
                for q in range(len(lays)):
                    if q == p or not (p == rank or q == rank):
                        continue
                    rows = halo[owners == q]
                    if rows.size == 0:
                        continue
                    theirs = lays[q].g2l(kind)[lay.l2g[kind][rows]]
                    if np.any(theirs < 0) or np.any(theirs >= lays[q].n_owned[kind]):
                        raise ValueError(f"{kind} halo of rank {p} is not owned by rank {q}")
                    if p == rank:
                        recv[(q, kind)] = (rows, theirs)
                    else:
                        send[(p, kind)] = theirs
            halo = lays[rank].l2g[kind].size - lays[rank].n_owned[kind]
            got = sum(v[0].size for (q, k), v in recv.items() if k == kind)
            if got != halo:
                raise ValueError(f"rank {rank}: {halo - got} {kind} halo rows have no owner")
        return ExchangePlan(rank, recv, send)

    def peers(self) -> list[int]:
        return sorted({q for q, _ in self.recv} | {q for q, _ in self.send})


def plans(lays: list[Layout]) -> list[ExchangePlan]:
    return [ExchangePlan.build(lays, r) for r in range(len(lays))]


KINDS = ("cell", "edge")


class TorchRows:
    """The buffers of one exchange point as ``(blocks, rows, S)`` tensors of
    any device, packed and unpacked with torch indexing: buffer by buffer,
    the rows of its kind (cell rows for cell and tracer buffers) in list
    order.  The device runners move the same rows with the library's
    one-launch kernels (``DeviceRows``)."""

    def __init__(self, buffers: list):
        self.buffers = buffers   # [(tensor, kind)]

    def words(self, rows: dict) -> int:
        return sum(int(b.shape[0]) * len(rows[k]) * int(b.shape[2]) for b, k in self.buffers if k in rows)

    def pack(self, key, rows: dict, out) -> None:
        import torch

        parts = [b[:, torch.as_tensor(rows[k], dtype=torch.long, device=b.device)].reshape(-1)
                 for b, k in self.buffers if k in rows]
        if parts:
            out.copy_(torch.cat(parts))

    def unpack(self, key, rows: dict, packed) -> None:
        import torch

        off = 0
        for b, k in self.buffers:
            if k not in rows:
                continue
            n = int(b.shape[0]) * len(rows[k]) * int(b.shape[2])
            idx = torch.as_tensor(rows[k], dtype=torch.long, device=b.device)
            b[:, idx] = packed[off:off + n].view(int(b.shape[0]), len(rows[k]), int(b.shape[2]))
            off += n


class DeviceRows:
    """The buffers of one exchange point as the library hands them to the
    hook (device pointers and kinds), moved by ``hexdyn_halo_pack`` /
    ``hexdyn_halo_unpack``: one launch per peer and direction."""

    def __init__(self, driver, nbuf: int, bufs, kinds, stream, index_cache: dict):
        self.lib = _lib.load()
        self.handle = driver._handle
        self.nbuf = nbuf
        self.ptrs = (C.c_void_p * max(1, nbuf))(*[bufs[i] for i in range(nbuf)])
        self.kinds = (C.c_int * max(1, nbuf))(*[kinds[i] for i in range(nbuf)])
        self.stream = stream
        self.cache = index_cache

    def _rows(self, key, kind, rows):
        import torch

        if kind not in rows:
            return None, 0
        t = self.cache.get((key, kind))
        if t is None:
            t = self.cache[(key, kind)] = torch.as_tensor(np.asarray(rows[kind], dtype=np.int32), device="cuda")
        return C.c_void_p(t.data_ptr()), int(t.numel())

    def words(self, rows: dict) -> int:
        n = {k: len(rows[k]) if k in rows else 0 for k in KINDS}
        return int(self.lib.hexdyn_halo_words(self.handle, self.nbuf, self.kinds, n["cell"], n["edge"]))

    def _move(self, fn, key, rows, packed) -> None:
        (cp, cn), (ep, en) = self._rows(key, "cell", rows), self._rows(key, "edge", rows)
        stream = C.c_void_p(int(getattr(self.stream, "cuda_stream", self.stream)))
        _lib.check(fn(self.handle, self.nbuf, self.ptrs, self.kinds, cp, cn, ep, en, C.c_void_p(packed.data_ptr()),
                      stream))

    def pack(self, key, rows: dict, out) -> None:
        self._move(self.lib.hexdyn_halo_pack, key, rows, out)

    def unpack(self, key, rows: dict, packed) -> None:
        self._move(self.lib.hexdyn_halo_unpack, key, rows, packed)


def exchange_packed(plan: ExchangePlan, packer, group=None, alloc=None) -> None:
    """One exchange point over ``torch.distributed``: for every peer (in
    ascending order, the same on every rank) the owned rows it needs, of
    every buffer of the point, are packed into one array and sent; the rows
    received from it are unpacked into this rank's halo.  All sends and
    receives of the point are posted together (``batch_isend_irecv``).
    ``packer``: ``TorchRows`` or ``DeviceRows``; ``alloc(key, words)``
    returns a float32 buffer of at least ``words`` (default: a new tensor on
    the packer's device)."""
    import torch
    import torch.distributed as dist

    def new(key, n):
        dev = packer.buffers[0][0].device if isinstance(packer, TorchRows) else "cuda"
        return torch.empty(n, dtype=torch.float32, device=dev)

    alloc = alloc or new
    ops, pending = [], []
    for q in plan.peers():
        send = {k: plan.send[(q, k)] for k in KINDS if (q, k) in plan.send}
        if send:
            n = packer.words(send)
            buf = alloc(("send", q), n)[:n]
            packer.pack(("send", q), send, buf)
            ops.append(dist.P2POp(dist.isend, buf, q, group=group))
        recv = {k: plan.recv[(q, k)][0] for k in KINDS if (q, k) in plan.recv}
        if recv:
            n = packer.words(recv)
            buf = alloc(("recv", q), n)[:n]
            ops.append(dist.P2POp(dist.irecv, buf, q, group=group))
            pending.append((q, recv, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for q, recv, buf in pending:
        packer.unpack(("recv", q), recv, buf)


class _Buffers:
    """Growing float32 device buffers by key (packed halo rows)."""

    def __init__(self):
        self.bufs: dict = {}

    def __call__(self, key, words: int):
        import torch

        b = self.bufs.get(key)
        if b is None or b.numel() < words:
            b = self.bufs[key] = torch.empty(max(1, words), dtype=torch.float32, device="cuda")
        return b


def gather_owned(lays: list[Layout], parts: list[tuple[Any, Any]]) -> tuple[dict, dict]:
    """Global logical state and saved diagnostics from every rank's owned
    region (``parts[r]`` = rank r's (state, saved diagnostics))."""
    state, side = {}, {}
    for name in (*_lib.STATE_FIELDS, *_lib.SIDECAR_FIELDS):
        kind = "edge" if name in ("rho_u", "normal_velocity") else "cell"
        pieces = []
        for lay, (st, sd) in zip(lays, parts):
            v = np.asarray(getattr(st, name) if name in _lib.STATE_FIELDS else getattr(sd, name))
            pieces.append((lay.owned(kind), v[..., : lay.n_owned[kind]]))
        g = np.full(pieces[0][1].shape[:-1] + (lays[0].owner[kind].size,), np.nan, dtype=np.float32)
        for ids, v in pieces:
            g[..., ids] = v
        (state if name in _lib.STATE_FIELDS else side)[name] = g
    return state, side


def _driver(arr: dict, config, stream=None):
    from . import from_case
    from .case import arrays_case

    return from_case(arrays_case(arr), config, stream=stream)


class PartitionedDycore:
    """P ranks of one instance in this process on the current device.

    Rank r steps its local mesh on its own stream in its own host thread.  At
    an exchange point every rank records an event and meets the others at a
    host barrier; each then makes its stream wait for the owners' events,
    copies its halo rows out of the owners' buffers on its stream, records a
    second event and meets the others again; before its next kernel each
    stream waits for the other ranks' copies (the owners must not overwrite
    rows still being read).  No kernel waits on another kernel."""

    def __init__(self, arr: dict, config, n_parts: int, halo_rings: int | None = None,
                 barrier_timeout: float = 300.0):
        import torch

        if halo_rings is None:
            halo_rings = halo_rings_for(config)
        self.n_parts = n_parts
        self.layouts = layouts(arr, n_parts, halo_rings)
        self.plans = plans(self.layouts)
        self.streams = [torch.cuda.Stream() for _ in range(n_parts)]
        self.drivers = [_driver(local_arrays(arr, lay), config, stream=s)
                        for lay, s in zip(self.layouts, self.streams)]
        torch.cuda.synchronize()
        self.device = torch.cuda.current_device()
        self.timeout = barrier_timeout
        self._barrier = threading.Barrier(n_parts)
        self._points: list = [None] * n_parts
        self._ready = [torch.cuda.Event() for _ in range(n_parts)]
        self._copied = [torch.cuda.Event() for _ in range(n_parts)]
        self._index: dict = {}
        self._packed = _Buffers()
        self._errors: list[BaseException] = []
        self.exchanges: list[list[int]] = [[] for _ in range(n_parts)]
        self._hooks = [_lib.EXCHANGE_HOOK(self._hook_for(r)) for r in range(n_parts)]
        # rows rank r receives from q: its halo rows and q's owned rows
        self._recv = [{q: ({k: self.plans[r].recv[(q, k)][0] for k in KINDS if (q, k) in self.plans[r].recv},
                           {k: self.plans[r].recv[(q, k)][1] for k in KINDS if (q, k) in self.plans[r].recv})
                       for q in range(n_parts)} for r in range(n_parts)]

    def _hook_for(self, r: int):
        import torch

        def hook(user, point, nbufs, bufs, kinds):
            try:
                st = self.streams[r]
                self._points[r] = DeviceRows(self.drivers[r], nbufs, bufs, kinds, st, self._index)
                self._ready[r].record(st)
                self._barrier.wait(self.timeout)
                for q in range(self.n_parts):
                    if q != r:
                        st.wait_event(self._ready[q])
                mine = self._points[r]
                for q in range(self.n_parts):
                    halo, owned = self._recv[r][q]
                    if not halo:
                        continue
                    # q's owned rows packed with q's handle, unpacked into r's
                    # halo with r's, both on r's stream
                    theirs = self._points[q]
                    src = DeviceRows(self.drivers[q], theirs.nbuf, theirs.ptrs, theirs.kinds, st, self._index)
                    n = mine.words(halo)
                    packed = self._packed((r, q), n)
                    src.pack(("own", r, q), owned, packed)
                    mine.unpack(("halo", r, q), halo, packed)
                self._copied[r].record(st)
                self._barrier.wait(self.timeout)
                for q in range(self.n_parts):
                    if q != r:
                        st.wait_event(self._copied[q])
                self.exchanges[r].append(int(point))
                return 0
            except BaseException as exc:  # noqa: BLE001 - re-raised by step()
                self._errors.append(exc)
                self._barrier.abort()
                return -1

        return hook

    def step(self, nsteps: int = 1) -> None:
        lib = _lib.load()
        errors: list[BaseException] = []

        def run(r: int) -> None:
            import torch

            drv = self.drivers[r]
            try:
                torch.cuda.set_device(self.device)
                _lib.check(lib.hexdyn_set_exchange_hook(drv._handle, self._hooks[r], None))
                try:
                    drv.step_device(nsteps)
                finally:
                    lib.hexdyn_set_exchange_hook(drv._handle, _lib.EXCHANGE_HOOK(), None)
            except BaseException as exc:  # noqa: BLE001
                errors.append(exc)
                self._barrier.abort()

        threads = [threading.Thread(target=run, args=(r,)) for r in range(self.n_parts)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        self._barrier.reset()
        if self._errors or errors:
            exc = (self._errors or errors)[0]
            self._errors.clear()
            raise exc

    def get_state(self) -> tuple[dict, dict]:
        """The owned regions of every rank as global logical fields (state,
        saved diagnostics)."""
        return gather_owned(self.layouts, [d.get_state() for d in self.drivers])

    def close(self) -> None:
        for d in self.drivers:
            d.close()


class RankDycore:
    """This process's rank of a partitioned instance, one rank per GPU over
    ``torch.distributed`` (every rank builds the same layouts from the same
    global case arrays)."""

    def __init__(self, arr: dict, config, group=None, halo_rings: int | None = None):
        import torch
        import torch.distributed as dist

        if halo_rings is None:
            halo_rings = halo_rings_for(config)
        self.group = group
        self.rank = dist.get_rank(group)
        self.n_parts = dist.get_world_size(group)
        self.layouts = layouts(arr, self.n_parts, halo_rings)
        self.plan = ExchangePlan.build(self.layouts, self.rank)
        self.layout = self.layouts[self.rank]
        self.stream = torch.cuda.Stream()
        self.driver = _driver(local_arrays(arr, self.layout), config, stream=self.stream)
        self._index: dict = {}
        self._packed = _Buffers()
        self._error: BaseException | None = None
        self._hook = _lib.EXCHANGE_HOOK(self._exchange)

    def _exchange(self, user, point, nbufs, bufs, kinds) -> int:
        import torch

        try:
            with torch.cuda.stream(self.stream):
                exchange_packed(self.plan, DeviceRows(self.driver, nbufs, bufs, kinds, self.stream, self._index),
                                self.group, self._packed)
            return 0
        except BaseException as exc:  # noqa: BLE001 - re-raised by step()
            self._error = exc
            return -1

    def step(self, nsteps: int = 1) -> None:
        lib = _lib.load()
        _lib.check(lib.hexdyn_set_exchange_hook(self.driver._handle, self._hook, None))
        try:
            self.driver.step_device(nsteps)
        except BaseException:
            if self._error is not None:
                err, self._error = self._error, None
                raise err from None
            raise
        finally:
            lib.hexdyn_set_exchange_hook(self.driver._handle, _lib.EXCHANGE_HOOK(), None)

    def get_state(self) -> tuple[dict, dict]:
        """Global logical fields assembled from every rank's owned region
        (``all_gather_object`` of each rank's local fields: for checks and
        output, not for the step)."""
        import torch.distributed as dist

        parts: list = [None] * self.n_parts
        dist.all_gather_object(parts, self.driver.get_state(), group=self.group)
        return gather_owned(self.layouts, parts)

    def close(self) -> None:
        self.driver.close()
