"""Batched ensembles.

The reference runs ensemble members side by side, each with its own
atmosphere, workspaces and CUDA stream, one launch sequence per member
(``hexcore/multi_member.py:1-7``).  Here the members of one time step are
concatenated into a single mesh (``hexdyn_create_ensemble``): member ``m``
owns a contiguous range of cells, edges and vertices, its connectivity is
offset into that range, and every kernel of the large step runs once for all
members.  No stencil reaches across members, so each member's result is the
step of its own single-instance driver, bit for bit.  Members of one ensemble
may live on meshes of different size; they share the configuration, levels,
tracer count and vertical coordinate.

An uneven batch (members with different time steps, e.g. 1440 s members on a
coarse mesh and 720 s members taking two steps per 1440 s) is a list of
ensembles advanced together by :func:`step_batched`: each group steps on its
own stream, concurrently, and the caller's stream waits for all of them.

:func:`assign_members` spreads members over GPUs for multi-GPU runs: members
are independent, so a rank only needs its share (balanced by cell count) and
no collective runs per step.
"""

from __future__ import annotations

import ctypes as C
from typing import Any, Sequence

import numpy as np

from . import _lib
from .config import DycoreConfig
from .driver import F32, HexDycoreDriver, HostSidecar, HostState, _build_descriptor, _refuse_missing


class HexEnsemble(HexDycoreDriver):
    """Several dycore members stepped as one handle on the current device."""

    def __init__(self, handle: C.c_void_p, keep: dict, cfg: DycoreConfig, sizes: dict,
                 member_sizes: list[dict], stream: Any):
        super().__init__(handle, keep, cfg, sizes, stream)
        self.member_sizes = member_sizes

    # ------------------------------------------------------------ creation
    @classmethod
    def from_host_members(cls, members: Sequence[dict], config: DycoreConfig, *, stream: Any = None,
                          capture_graph: bool = False) -> "HexEnsemble":
        """``members``: dicts with the ``from_host`` inputs of each member
        (``mesh``, ``state``, ``vertical``, ``reference``, ``terrain_metrics``,
        ``advection_coefficients``, ``reference_wind_profiles`` and optionally
        ``saved_diagnostics``)."""
        if not members:
            raise ValueError("an ensemble needs at least one member")
        cfg = config
        cfg.validate()
        lib = _lib.load()
        descs, keeps, sizes = [], [], []
        for m in members:
            for key, decl in (("terrain_metrics", "TerrainMetrics(zb_cell, zb3_cell)"),
                              ("advection_coefficients", "AdvectionCoefficients(...)"),
                              ("reference_wind_profiles", "V841ReferenceWindProfiles(u_init, v_init)")):
                if m.get(key) is None:
                    _refuse_missing(key, f"{key}={decl}")
            d, k, s = _build_descriptor(m["mesh"], m["state"], m["vertical"], m["reference"], cfg,
                                        m["terrain_metrics"], m["advection_coefficients"],
                                        m["reference_wind_profiles"])
            descs.append(d)
            keeps.append(k)
            sizes.append(s)
        arr = (_lib.HexDynDesc * len(descs))(*descs)
        handle = C.c_void_p()
        _lib.check(lib.hexdyn_create_ensemble(arr, len(descs), C.byref(handle)))
        total = dict(sizes[0])
        for key in ("n_cells", "n_edges", "n_vertices"):
            total[key] = sum(s[key] for s in sizes)
        ens = cls(handle, {"members": keeps}, cfg, total, sizes, stream)
        for i, m in enumerate(members):
            ens.set_member_state(i, m["state"], m.get("saved_diagnostics"), rebuild=False)
        if any(m.get("saved_diagnostics") is None for m in members):
            # the rebuild is per column and per edge, so rebuilding all members
            # leaves members with a supplied sidecar unchanged only if it was
            # the rebuilt one; supplied sidecars are therefore set again after
            stream_h = ens._stream_handle()
            _lib.check(lib.hexdyn_rebuild_sidecar(ens._handle, stream_h))
            for i, m in enumerate(members):
                if m.get("saved_diagnostics") is not None:
                    ens._put_member_sidecar(i, m["saved_diagnostics"], stream_h)
        ens.time_seconds = float(getattr(members[0]["state"], "time_seconds", 0.0))
        ens.synchronize()
        ens._keep.pop("_uploads", None)
        if capture_graph:
            ens.capture_graph()
        return ens

    @classmethod
    def from_cases(cls, cases: Sequence[Any], config: DycoreConfig, **kwargs) -> "HexEnsemble":
        """Ensemble of synthetic ``hexdyn.case.DycoreCase`` members."""
        members = [dict(mesh=c.mesh, state=c, vertical=c.vertical, reference=c, terrain_metrics=c,
                        advection_coefficients=c, reference_wind_profiles=c) for c in cases]
        return cls.from_host_members(members, config, **kwargs)

    # ------------------------------------------------------------- members
    @property
    def member_count(self) -> int:
        return len(self.member_sizes)

    def member_shape(self, m: int, name: str) -> tuple[int, ...]:
        s = self.member_sizes[m]
        L = s["n_levels"]
        rows = L + 1 if name in ("rho_w", "vertical_velocity") else L
        n = s["n_edges"] if name in ("rho_u", "normal_velocity") else s["n_cells"]
        return (s["n_scalars"], rows, n) if name == "scalars" else (rows, n)

    def _put_member(self, m: int, name: str, value: Any, stream) -> None:
        arr = np.ascontiguousarray(value, dtype=F32)
        if arr.shape != self.member_shape(m, name):
            raise ValueError(f"member {m} {name} shape {arr.shape} != {self.member_shape(m, name)}")
        self._keep.setdefault("_uploads", []).append(arr)
        _lib.check(self._lib.hexdyn_set_member_state(self._handle, m, _lib.FIELDS[name],
                                                     arr.ctypes.data_as(C.POINTER(C.c_float)), arr.size, stream))

    def _put_member_sidecar(self, m: int, side: Any, stream) -> None:
        for name in _lib.SIDECAR_FIELDS:
            self._put_member(m, name, getattr(side, name), stream)

    def set_member_state(self, m: int, state: Any, saved_diagnostics: Any = None, *, rebuild: bool = True) -> None:
        """Upload member ``m``'s prognostic state (and sidecar).  Without a
        sidecar and with ``rebuild``, the saved diagnostics of every member
        are rebuilt from their current states (hexcore/driver.py:2655)."""
        stream = self._stream_handle()
        for name in _lib.STATE_FIELDS:
            if name == "scalars" and self.member_sizes[m]["n_scalars"] == 0:
                continue
            self._put_member(m, name, getattr(state, name), stream)
        if saved_diagnostics is not None:
            self._put_member_sidecar(m, saved_diagnostics, stream)
        elif rebuild:
            _lib.check(self._lib.hexdyn_rebuild_sidecar(self._handle, stream))
        if rebuild or saved_diagnostics is not None:
            self.synchronize()
            self._keep.pop("_uploads", None)

    def get_member_state(self, m: int, stream=None) -> tuple[HostState, HostSidecar]:
        st = self._stream_handle() if stream is None else stream
        out = {}
        for name in (*_lib.STATE_FIELDS, *_lib.SIDECAR_FIELDS):
            arr = np.empty(self.member_shape(m, name), dtype=F32)
            if arr.size:
                _lib.check(self._lib.hexdyn_get_member_state(self._handle, m, _lib.FIELDS[name],
                                                             arr.ctypes.data_as(C.POINTER(C.c_float)), arr.size,
                                                             st))
            out[name] = arr
        self.synchronize()
        state = HostState(**{k: out[k] for k in _lib.STATE_FIELDS}, time_seconds=self.time_seconds)
        return state, HostSidecar(**{k: out[k] for k in _lib.SIDECAR_FIELDS})


def step_batched(groups: Sequence[HexDycoreDriver], steps: Sequence[int], *, read_flags: bool = True,
                 stream: Any = None) -> list[int] | None:
    """Advance each group by its own number of large steps, the groups
    concurrently on private streams (``hexdyn_step_batched``).  With
    ``read_flags`` the validation flags are read (synchronising) and a set
    flag raises ``FloatingPointError``."""
    if len(groups) != len(steps) or not groups:
        raise ValueError("one step count per group")
    lib = _lib.load()
    handles = (C.c_void_p * len(groups))(*[g._handle for g in groups])
    counts = (C.c_int32 * len(groups))(*[int(s) for s in steps])
    flags = (C.c_int32 * len(groups))()
    batch = _lib.HexDynBatch(len(groups), handles, counts, flags if read_flags else None)
    st = groups[0]._stream_handle() if stream is None else C.c_void_p(int(getattr(stream, "cuda_stream", stream)))
    rc = lib.hexdyn_step_batched(C.byref(batch), st)
    if rc == _lib.HEXDYN_E_NUMERIC:
        raise FloatingPointError(_lib.last_error())
    _lib.check(rc)
    for g, n in zip(groups, steps):
        g.time_seconds += n * g.config.config_dt
    return list(flags) if read_flags else None


def assign_members(cells: Sequence[int], world_size: int) -> list[list[int]]:
    """Greedy largest-first bin packing of members (by cell count) onto
    ``world_size`` GPUs; returns the member indices of each rank, each list in
    increasing member order.  Deterministic, so every rank computes the same
    assignment without communicating."""
    if world_size < 1:
        raise ValueError("world_size must be positive")
    load = [0] * world_size
    out: list[list[int]] = [[] for _ in range(world_size)]
    for m in sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i)):
        r = min(range(world_size), key=lambda j: (load[j], j))
        out[r].append(m)
        load[r] += int(cells[m])
    return [sorted(x) for x in out]
