"""Host driver with the reference's dycore step interface.

``HexDycoreDriver`` presents the methods of the reference's
``CudaDryDycoreDriver`` (``hexcore/cuda_driver.py:2658``):

* ``from_host(mesh, state, vertical, reference, config, *, saved_diagnostics,
  terrain_metrics, advection_coefficients, reference_wind_profiles)``
  (``:2826``) uploads once and owns the device copies;
* ``step_device()`` (``:5751``) advances one large step on the device and
  returns a ``DeviceStepResult`` whose ``atmosphere`` exposes the new state as
  torch CUDA tensors (zero copy);
* ``step()`` (``:6112``) is ``step_device()`` plus the download of the state
  and the saved diagnostics.

Arguments are duck-typed on the reference's attribute names
(``PrognosticState``, ``VerticalGrid``, ``DryReferenceState``,
``TerrainMetrics``, ``AdvectionCoefficients``, ``V841ReferenceWindProfiles``,
``DrySavedDiagnostics``), so the reference's own objects can be passed.  All
arithmetic runs in the CUDA library behind the C ABI (include/hexdyn.h);
there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any

import numpy as np

from . import _lib
from .case import vertical_velocity_damping
from .config import ConfigurationRefusal, DycoreConfig

F32 = np.float32


def _nullcontext():
    import contextlib

    return contextlib.nullcontext()


def mesh_array(mesh: Any, name: str) -> np.ndarray:
    """``_mesh_array`` of the reference: attribute first, then ``mesh.arrays``."""
    try:
        return np.asarray(getattr(mesh, name))
    except AttributeError:
        arrays = getattr(mesh, "arrays", None)
        if arrays is None or name not in arrays:
            raise AttributeError(f"mesh has no MPAS field {name!r}") from None
        return np.asarray(arrays[name])


def _schedule_dts(cfg: DycoreConfig) -> list[float]:
    """Acoustic time step of the three RK stages (hexcore/integration.py:104-160)."""
    dt_dyn = cfg.config_dt / cfg.config_dynamics_split_steps
    n = cfg.config_number_of_sub_steps
    if cfg.config_time_integration_order == 2:
        return [dt_dyn / n] * 3
    return [dt_dyn / 3.0, dt_dyn / n, dt_dyn / n]


@dataclass
class HostState:
    rho: np.ndarray
    rho_theta: np.ndarray
    rho_u: np.ndarray
    rho_w: np.ndarray
    scalars: np.ndarray
    time_seconds: float = 0.0


@dataclass
class HostSidecar:
    theta_m: np.ndarray
    exner: np.ndarray
    density_perturbation: np.ndarray
    rho_theta_perturbation: np.ndarray
    pressure_perturbation: np.ndarray
    normal_velocity: np.ndarray
    vertical_velocity: np.ndarray


class _CudaArray:
    """``__cuda_array_interface__`` view of library-owned device memory."""

    def __init__(self, ptr: int, shape: tuple[int, ...], owner: Any):
        self._owner = owner
        self.__cuda_array_interface__ = {
            "shape": shape, "typestr": "<f4", "data": (int(ptr), False), "version": 3, "strides": None,
        }


@dataclass
class DeviceAtmosphere:
    """Device views of the current state: each field is a torch tensor in the
    library's padded [entity][level] layout (``padded``) and as a logical
    [level][entity] view (``logical``)."""

    driver: "HexDycoreDriver"

    def padded(self, name: str):
        import torch

        ptr = C.c_void_p()
        _lib.check(self.driver._lib.hexdyn_device_field(self.driver._handle, _lib.FIELDS[name], C.byref(ptr)))
        n, blocks = self.driver._entities(name)
        shape = (blocks * n, self.driver.level_stride) if blocks > 1 else (n, self.driver.level_stride)
        return torch.as_tensor(_CudaArray(ptr.value, shape, self.driver), device="cuda")

    def logical(self, name: str):
        rows = self.driver._rows(name)
        t = self.padded(name)[:, :rows]
        n, blocks = self.driver._entities(name)
        if blocks > 1:
            return t.reshape(blocks, n, rows).transpose(1, 2)
        return t.t()


@dataclass
class StepReceipt:
    steps: int
    flag: int
    launches_per_step: int
    device_bytes: int
    graph: bool


@dataclass
class DeviceStepResult:
    atmosphere: DeviceAtmosphere
    receipt: StepReceipt


@dataclass
class HostStepResult:
    state: HostState
    saved_diagnostics: HostSidecar
    receipt: StepReceipt


class HexDycoreDriver:
    """One dycore instance resident on the current CUDA device."""

    def __init__(self, handle: C.c_void_p, keep: dict, cfg: DycoreConfig, sizes: dict, stream: Any):
        self._lib = _lib.load()
        self._handle = handle
        self._keep = keep
        self.config = cfg
        self.sizes = sizes
        self._stream = stream
        self.level_stride = int(self._lib.hexdyn_level_stride(handle))
        self.time_seconds = 0.0
        self._graph = False

    # ------------------------------------------------------------ creation
    @classmethod
    def from_host(cls, mesh: Any, state: Any, vertical: Any, reference: Any, config: Any, *,
                  saved_diagnostics: Any = None, terrain_metrics: Any = None,
                  advection_coefficients: Any = None, reference_wind_profiles: Any = None,
                  stream: Any = None, capture_graph: bool = False, **config_overrides: Any) -> "HexDycoreDriver":
        cfg = config if isinstance(config, DycoreConfig) else DycoreConfig.from_reference(config, **config_overrides)
        if config_overrides and isinstance(config, DycoreConfig):
            cfg = DycoreConfig(**{**cfg.__dict__, **config_overrides})
            cfg.validate()
        if terrain_metrics is None:
            _refuse_missing("zb", "terrain_metrics=TerrainMetrics(zb_cell, zb3_cell)")
        if advection_coefficients is None:
            _refuse_missing("adv_coefs", "advection_coefficients=AdvectionCoefficients(...)")
        if reference_wind_profiles is None:
            _refuse_missing("u_init", "reference_wind_profiles=V841ReferenceWindProfiles(u_init, v_init)")
        lib = _lib.load()
        desc, keep, sizes = _build_descriptor(mesh, state, vertical, reference, cfg, terrain_metrics,
                                              advection_coefficients, reference_wind_profiles)
        handle = C.c_void_p()
        _lib.check(lib.hexdyn_create(C.byref(desc), C.byref(handle)))
        drv = cls(handle, keep, cfg, sizes, stream)
        drv.set_state(state, saved_diagnostics)
        if capture_graph:
            drv.capture_graph()
        return drv

    # ----------------------------------------------------------- plumbing
    def _stream_handle(self):
        if self._stream is not None:
            return C.c_void_p(int(getattr(self._stream, "cuda_stream", self._stream)))
        try:
            import torch

            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:  # noqa: BLE001 - no torch: the legacy default stream
            return C.c_void_p(0)

    def _entities(self, name: str) -> tuple[int, int]:
        s = self.sizes
        if name in ("rho_u", "normal_velocity"):
            return s["n_edges"], 1
        if name == "scalars":
            return s["n_cells"], s["n_scalars"]
        return s["n_cells"], 1

    def _rows(self, name: str) -> int:
        L = self.sizes["n_levels"]
        return L + 1 if name in ("rho_w", "vertical_velocity") else L

    def _shape(self, name: str) -> tuple[int, ...]:
        n, blocks = self._entities(name)
        rows = self._rows(name)
        return (blocks, rows, n) if name == "scalars" else (rows, n)

    def _put(self, name: str, value: Any, stream) -> None:
        arr = np.ascontiguousarray(value, dtype=F32)
        if arr.shape != self._shape(name):
            raise ValueError(f"{name} shape {arr.shape} != {self._shape(name)}")
        self._keep.setdefault("_uploads", []).append(arr)
        _lib.check(self._lib.hexdyn_set_state(self._handle, _lib.FIELDS[name],
                                              arr.ctypes.data_as(C.POINTER(C.c_float)), arr.size, stream))

    def set_state(self, state: Any, saved_diagnostics: Any = None) -> None:
        """Upload a prognostic state (and sidecar, else rebuild it on the device
        exactly as ``hexcore/driver.py:2655`` does)."""
        stream = self._stream_handle()
        self._keep["_uploads"] = []
        for name in _lib.STATE_FIELDS:
            if name == "scalars" and self.sizes["n_scalars"] == 0:
                continue
            self._put(name, getattr(state, name), stream)
        if saved_diagnostics is None:
            _lib.check(self._lib.hexdyn_rebuild_sidecar(self._handle, stream))
        else:
            for name in _lib.SIDECAR_FIELDS:
                self._put(name, getattr(saved_diagnostics, name), stream)
        self.time_seconds = float(getattr(state, "time_seconds", 0.0))
        self.synchronize()
        self._keep["_uploads"] = []

    def synchronize(self) -> None:
        import torch

        if torch.cuda.is_available():
            torch.cuda.synchronize()

    def capture_graph(self) -> None:
        """Capture the whole RK3 large step as CUDA graphs (one per buffer parity)."""
        _lib.check(self._lib.hexdyn_capture_graph(self._handle, self._stream_handle()))
        self._graph = True

    def autotune(self, steps_per_candidate: int = 2) -> dict[str, dict]:
        """Choose the block size of every kernel launch by timing (see
        ``hexdyn_autotune``); the state is left as it was.  Returns, per
        launch label, the microseconds at each block size tried and the
        choice."""
        buf = C.create_string_buffer(1 << 16)
        _lib.check(self._lib.hexdyn_autotune(self._handle, self._stream_handle(), int(steps_per_candidate), buf,
                                             len(buf)))
        lines = buf.value.decode().splitlines()
        candidates = [int(x) for x in lines[0].split()[1:]]
        out = {}
        for line in lines[1:]:
            parts = line.split()
            out[parts[0]] = {"us": {t: float(x) for t, x in zip(candidates, parts[1:-1])}, "threads": int(parts[-1])}
        return out

    def bind_state(self, tensors: dict | None) -> None:
        """Step from caller-owned CUDA tensors (padded layout, one per field
        name of ``hexdyn._lib.FIELDS``) without copying; ``None`` unbinds.
        The step alternates between these and the library's own buffers."""
        if tensors is None:
            _lib.check(self._lib.hexdyn_bind_state(self._handle, None, self._stream_handle()))
            self._keep.pop("_bound", None)
            return
        f = _lib.HexDynFields()
        for name, i in _lib.FIELDS.items():
            t = tensors.get(name)
            f.field[i] = None if t is None else int(t.data_ptr())
        _lib.check(self._lib.hexdyn_bind_state(self._handle, C.byref(f), self._stream_handle()))
        self._keep["_bound"] = dict(tensors)

    # -------------------------------------------------------------- steps
    def step_async(self, nsteps: int = 1) -> None:
        _lib.check(self._lib.hexdyn_step_async(self._handle, self._stream_handle(), int(nsteps)))
        self.time_seconds += nsteps * self.config.config_dt

    def read_flag(self) -> int:
        flag = C.c_int(0)
        rc = self._lib.hexdyn_read_flag(self._handle, self._stream_handle(), C.byref(flag))
        if rc == _lib.HEXDYN_E_NUMERIC:
            raise FloatingPointError(_lib.last_error())
        _lib.check(rc)
        return flag.value

    def step_device(self, nsteps: int = 1) -> DeviceStepResult:
        flag = C.c_int(0)
        done = C.c_int(0)
        rc = self._lib.hexdyn_step(self._handle, self._stream_handle(), int(nsteps), C.byref(flag), C.byref(done))
        if rc == _lib.HEXDYN_E_NUMERIC:
            raise FloatingPointError(_lib.last_error())
        _lib.check(rc)
        self.time_seconds += nsteps * self.config.config_dt
        return DeviceStepResult(DeviceAtmosphere(self), self.receipt(nsteps, flag.value))

    def acoustic_words(self) -> dict:
        """The final acoustic words of the last step as logical device views:
        ``ru_p`` [L][E] and ``rw_p`` [L+1][C] after the last substep of RK
        stage 3 of the last dynamics subcycle (the reference's restart words,
        hexcore/cuda_driver.py:4707-4711).  Valid until the next step."""
        import torch

        out = {}
        S = self.level_stride
        for name, which, n, rows in (("ru_p", 0, self.sizes["n_edges"], self.sizes["n_levels"]),
                                     ("rw_p", 1, self.sizes["n_cells"], self.sizes["n_levels"] + 1)):
            ptr = C.c_void_p()
            _lib.check(self._lib.hexdyn_acoustic_field(self._handle, which, C.byref(ptr)))
            t = torch.as_tensor(_CudaArray(ptr.value, (n, S), self), device="cuda")
            out[name] = t[:, :rows].t()
        return out

    def _step_device_v841(self, physics_tendencies: Any = None, *, physics_stage_callback: Any = None,
                          physics_post_transport_callback: Any = None, physics_mass_loading_count: Any = None,
                          acoustic_output_callback: Any = None) -> DeviceStepResult:
        """One large step with the reference's production signature
        (hexcore/cuda_driver.py:4854, called by
        hexcore/mpasphys/runtime_v842.py:2310).

        ``physics_stage_callback(rk_step=, dynamics_substep=, state=, saved=,
        diagnostics=None)`` is called before the tendencies of every RK stage
        of every dynamics subcycle (cuda_driver.py:4393-4400) with logical
        [level][entity] device views of the stage's state and saved
        diagnostics; it returns an object whose ``rho_u`` [L][E],
        ``rho_theta`` [L][C], ``rho`` [L][C] and ``diabatic_theta`` [L][C]
        (any may be absent or None) enter the step as the reference adds
        them: ``(tend_ru + saved Euler) + rho_u``; ``tend_rt`` + ``rho x
        diabatic_theta``, + the saved mixing term, + ``rho_theta``; the
        ``rho`` given at a subcycle's last stage is added to the next
        subcycle's saved density tendency.  A callback returning None is an
        error, as in the reference.  With a callback the step runs eagerly.
        Held ``physics_tendencies`` belong to the reference's full-physics
        configuration and are refused, as the reference's dry configuration
        refuses them; ``physics_mass_loading_count`` must be the carried
        scalar count (the moist coefficients load every carried scalar).

        ``physics_post_transport_callback(state=, saved=, outer_state=,
        modified_theta_dynamics_rate=)`` is called after the scalar transport
        (cuda_driver.py:5299-5305): ``state`` and ``saved`` hold logical
        device views of the step's result (writes land in the library's
        buffers and feed the next step), ``outer_state`` views of the state
        the step started from, and ``modified_theta_dynamics_rate`` the
        [L][C] rate (tend_rt - tend_rho theta_m) / rho of RK stage 3 of the
        last subcycle when a stage callback ran, else None (the reference
        forms it only with physics tendencies).  ``acoustic_output_callback(ru_p=...,
        rw_p=...)`` receives the final acoustic words after the step (the
        reference calls it after RK stage 3 of every dynamics subcycle; its
        last call carries these values)."""
        from .config import ConfigurationRefusal

        if physics_tendencies is not None:
            raise ConfigurationRefusal("held_physics_tendencies", "provided",
                                       "a dry v8.4.1 config cannot be relabelled by supplying physics arrays",
                                       "physics_stage_callback=... for per-stage physics, or None")
        if physics_mass_loading_count is not None and int(physics_mass_loading_count) != self.sizes["n_scalars"]:
            raise ConfigurationRefusal("physics_mass_loading_count", physics_mass_loading_count,
                                       "the moist coefficients load every carried scalar on this path",
                                       f"physics_mass_loading_count={self.sizes['n_scalars']} (or None)")
        outer = None
        if physics_post_transport_callback is not None:
            if self.config.clamp_negative_scalars:
                # the reference skips its end-of-step clamp when the callback
                # takes the transported scalars (cuda_driver.py:5306-5311)
                raise ConfigurationRefusal("clamp_negative_scalars", True, "a post-transport callback receives "
                                           "the unclamped scalars", "clamp_negative_scalars=False")
            outer = self._views(_lib.STATE_FIELDS)  # the step reads these buffers and writes the others
        rate = None
        if physics_stage_callback is None:
            res = self.step_device(1)
        else:
            res = self._step_with_stage_callback(physics_stage_callback)
            rate = self._physics_view(_lib.PHYS_MODIFIED_RATE)
        if physics_post_transport_callback is not None:
            physics_post_transport_callback(state=self._views(_lib.STATE_FIELDS),
                                            saved=self._views(_lib.SIDECAR_FIELDS), outer_state=outer,
                                            modified_theta_dynamics_rate=rate)
        if acoustic_output_callback is not None:
            acoustic_output_callback(**self.acoustic_words())
        return res

    def _physics_view(self, which: int):
        """Logical [L][E|C] view of a physics buffer of the library."""
        import torch

        ptr = C.c_void_p()
        _lib.check(self._lib.hexdyn_physics_buffer(self._handle, which, C.byref(ptr)))
        n = self.sizes["n_edges"] if which == _lib.PHYS_RHO_U else self.sizes["n_cells"]
        t = torch.as_tensor(_CudaArray(ptr.value, (n, self.level_stride), self), device="cuda")
        return t[:, : self.sizes["n_levels"]].t()

    def _field_view(self, ptr: int, name: str):
        import torch

        n, blocks = self._entities(name)
        rows = self._rows(name)
        if blocks > 1:
            t = torch.as_tensor(_CudaArray(ptr, (blocks * n, self.level_stride), self), device="cuda")
            return t[:, :rows].reshape(blocks, n, rows).transpose(1, 2)
        t = torch.as_tensor(_CudaArray(ptr, (n, self.level_stride), self), device="cuda")
        return t[:, :rows].t()

    def _step_with_stage_callback(self, callback) -> DeviceStepResult:
        """One eager step with ``callback`` run before every RK stage
        (hexdyn_set_stage_hook): the stage's fields are wrapped as views, the
        returned tendencies copied into the library's physics buffers on the
        step's stream."""
        import torch
        from types import SimpleNamespace

        errors: list[BaseException] = []
        targets = ((_lib.PHYS_RHO_U, "rho_u"), (_lib.PHYS_RHO_THETA, "rho_theta"), (_lib.PHYS_RHO, "rho"),
                   (_lib.PHYS_DIABATIC_THETA, "diabatic_theta"))
        stream = torch.cuda.ExternalStream(self._stream_handle().value or 0) if self._stream is not None else None
        t0 = self.time_seconds

        def hook(user, substep, rk_step, fields):
            try:
                f = fields.contents
                views = {name: self._field_view(f.field[i], name) for name, i in _lib.FIELDS.items()
                         if f.field[i] and not (name == "scalars" and self.sizes["n_scalars"] == 0)}
                state = SimpleNamespace(**{k: views[k] for k in _lib.STATE_FIELDS if k in views}, time_seconds=t0)
                saved = SimpleNamespace(**{k: views[k] for k in _lib.SIDECAR_FIELDS})
                with torch.cuda.stream(stream) if stream is not None else _nullcontext():
                    tend = callback(rk_step=int(rk_step), dynamics_substep=int(substep), state=state, saved=saved,
                                    diagnostics=None)
                    if tend is None:
                        raise RuntimeError("active MPAS RK callback returned no sources")
                    mask = 0
                    for bit, name in targets:
                        value = getattr(tend, name, None)
                        if value is None:
                            continue
                        dst = self._physics_view(bit)
                        src = torch.as_tensor(value, device="cuda", dtype=torch.float32)
                        if tuple(src.shape) != tuple(dst.shape):
                            raise ValueError(f"physics {name} shape {tuple(src.shape)} != {tuple(dst.shape)}")
                        dst.copy_(src)
                        mask |= bit
                return mask
            except BaseException as exc:  # noqa: BLE001 - reported after the step
                errors.append(exc)
                return -1

        cb = _lib.STAGE_HOOK(hook)
        _lib.check(self._lib.hexdyn_set_stage_hook(self._handle, cb, None))
        try:
            flag = C.c_int(0)
            done = C.c_int(0)
            rc = self._lib.hexdyn_step(self._handle, self._stream_handle(), 1, C.byref(flag), C.byref(done))
        finally:
            self._lib.hexdyn_set_stage_hook(self._handle, _lib.STAGE_HOOK(), None)
        if errors:
            raise errors[0]
        if rc == _lib.HEXDYN_E_NUMERIC:
            raise FloatingPointError(_lib.last_error())
        _lib.check(rc)
        self.time_seconds += self.config.config_dt
        return DeviceStepResult(DeviceAtmosphere(self), self.receipt(1, flag.value))

    def _views(self, names) -> Any:
        """Logical device views of the current buffers of ``names`` (with
        ``time_seconds`` for the state)."""
        from types import SimpleNamespace

        atm = DeviceAtmosphere(self)
        fields = {n: atm.logical(n) for n in names if not (n == "scalars" and self.sizes["n_scalars"] == 0)}
        if "rho" in names:
            fields["time_seconds"] = self.time_seconds
        return SimpleNamespace(**fields)

    def profile(self, nsteps: int = 1) -> dict[str, tuple[int, float]]:
        """Per-kernel launches and total milliseconds over ``nsteps`` eager
        steps, each launch bracketed by CUDA events on the driver's stream."""
        buf = C.create_string_buffer(1 << 16)
        _lib.check(self._lib.hexdyn_profile_steps(self._handle, self._stream_handle(), int(nsteps), buf, len(buf)))
        self.time_seconds += nsteps * self.config.config_dt
        out = {}
        for line in buf.value.decode().splitlines():
            name, launches, ms = line.split()
            out[name] = (int(launches), float(ms))
        return out

    def receipt(self, steps: int = 0, flag: int = 0) -> StepReceipt:
        return StepReceipt(steps=steps, flag=flag,
                           launches_per_step=int(self._lib.hexdyn_launches_per_step(self._handle)),
                           device_bytes=int(self._lib.hexdyn_device_bytes(self._handle)), graph=self._graph)

    def get_state(self, stream=None) -> tuple[HostState, HostSidecar]:
        st = self._stream_handle() if stream is None else stream
        out = {}
        for name in (*_lib.STATE_FIELDS, *_lib.SIDECAR_FIELDS):
            shape = self._shape(name)
            arr = np.empty(shape, dtype=F32)
            if arr.size:
                _lib.check(self._lib.hexdyn_get_state(self._handle, _lib.FIELDS[name],
                                                      arr.ctypes.data_as(C.POINTER(C.c_float)), arr.size, st))
            out[name] = arr
        self.synchronize()
        state = HostState(**{k: out[k] for k in _lib.STATE_FIELDS}, time_seconds=self.time_seconds)
        side = HostSidecar(**{k: out[k] for k in _lib.SIDECAR_FIELDS})
        return state, side

    def step_host_buffers(self, state_in: dict, side_in: dict, state_out: dict, side_out: dict) -> None:
        """One large step from host buffers to host buffers, enqueued on the
        driver's stream without synchronising: upload of the state and sidecar,
        the step, download of both (the reference's from_host upload, step_device
        and step() download, hexcore/cuda_driver.py:2826,5751,6112), through
        ``hexdyn_step_host`` (the downloads of every field but the scalars
        overlap the scalar transport).  Every field is given in and out; use
        pinned arrays for asynchronous copies; synchronise before reading the
        outputs."""
        fin = (C.c_void_p * _lib.HEXDYN_NUM_FIELDS)()
        fout = (C.c_void_p * _lib.HEXDYN_NUM_FIELDS)()
        for src, dst in ((state_in, fin), (side_in, fin), (state_out, fout), (side_out, fout)):
            for name, arr in src.items():
                if arr.shape != self._shape(name) or arr.dtype != F32 or not arr.flags.c_contiguous:
                    raise ValueError(f"{name}: expected a C-contiguous float32 array of shape {self._shape(name)}")
                dst[_lib.FIELDS[name]] = arr.ctypes.data
        names = (*_lib.STATE_FIELDS, *_lib.SIDECAR_FIELDS)
        missing = [n for n in names if n not in {**state_in, **side_in} or n not in {**state_out, **side_out}]
        if missing:
            raise ValueError(f"step_host_buffers needs every field in and out; missing {missing}")
        _lib.check(self._lib.hexdyn_step_host(self._handle, fin, fout, self._stream_handle()))
        self.time_seconds += self.config.config_dt

    def field_shape(self, name: str) -> tuple[int, ...]:
        return self._shape(name)

    def step(self, nsteps: int = 1) -> HostStepResult:
        res = self.step_device(nsteps)
        state, side = self.get_state()
        return HostStepResult(state, side, res.receipt)

    def close(self) -> None:
        if self._handle:
            self._lib.hexdyn_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def _refuse_missing(knob: str, declaration: str) -> None:
    raise ConfigurationRefusal(knob, None, "the v8.4.1 step needs this input", declaration)


def _i32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x), dtype=np.int32)


def _f32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x).astype(F32, copy=False))


def _build_descriptor(mesh, state, vertical, reference, cfg: DycoreConfig, terrain, adv, winds):
    ncells = int(mesh_array(mesh, "areaCell").size)
    nedges = int(mesh_array(mesh, "dcEdge").size)
    nvert = int(mesh_array(mesh, "areaTriangle").size)
    nlev = int(np.asarray(vertical.zz).shape[0])
    scalars = np.asarray(state.scalars)
    keep: dict[str, np.ndarray] = {}
    eoc = _i32(mesh_array(mesh, "edgesOnCell"))
    eoe = _i32(mesh_array(mesh, "edgesOnEdge"))
    adv_cells = _i32(adv.adv_cells_for_edge)
    angle = np.asarray(mesh_array(mesh, "angleEdge")).astype(F32)
    # cos/sin of the FP32 angle with NumPy's scalar kernel, as the reference
    # evaluates them (hexcore/dynamics_v841.py:163-165).
    cos_a = np.asarray([np.cos(a) for a in angle], dtype=F32)
    sin_a = np.asarray([np.sin(a) for a in angle], dtype=F32)
    arrays = {
        "cells_on_edge": _i32(mesh_array(mesh, "cellsOnEdge")),
        "edges_on_cell": eoc,
        "cells_on_cell": _i32(mesh_array(mesh, "cellsOnCell"))[:, : eoc.shape[1]].copy(),
        "vertices_on_cell": _i32(mesh_array(mesh, "verticesOnCell"))[:, : eoc.shape[1]].copy(),
        "n_edges_on_cell": _i32(mesh_array(mesh, "nEdgesOnCell")),
        "vertices_on_edge": _i32(mesh_array(mesh, "verticesOnEdge")),
        "edges_on_vertex": _i32(mesh_array(mesh, "edgesOnVertex")),
        "cells_on_vertex": _i32(mesh_array(mesh, "cellsOnVertex")),
        "edges_on_edge": eoe,
        "n_edges_on_edge": _i32(mesh_array(mesh, "nEdgesOnEdge")),
        "adv_cells": adv_cells,
        "n_adv_cells": _i32(adv.n_adv_cells_for_edge),
        "dc_edge": _f32(mesh_array(mesh, "dcEdge")),
        "dv_edge": _f32(mesh_array(mesh, "dvEdge")),
        "area_cell": _f32(mesh_array(mesh, "areaCell")),
        "area_triangle": _f32(mesh_array(mesh, "areaTriangle")),
        "kite_areas": _f32(mesh_array(mesh, "kiteAreasOnVertex")),
        "weights_on_edge": _f32(mesh_array(mesh, "weightsOnEdge")),
        "f_vertex": _f32(mesh_array(mesh, "fVertex")),
        "f_edge": _f32(mesh_array(mesh, "fEdge")),
        "cos_angle_edge": cos_a,
        "sin_angle_edge": sin_a,
        "adv_coefs": _f32(adv.adv_coefs),
        "adv_coefs_3rd": _f32(adv.adv_coefs_3rd),
        "fzm": _f32(vertical.fzm), "fzp": _f32(vertical.fzp),
        "rdzw": _f32(vertical.rdzw), "rdzu": _f32(vertical.rdzu),
        "zz": _f32(vertical.zz), "zxu": _f32(vertical.zxu),
        # implicit w damping from the configuration (hexcore/driver.py:2417)
        "dss": vertical_velocity_damping(np.asarray(vertical.zgrid), cfg.config_xnutr, cfg.config_zd),
        "zb_cell": _f32(terrain.zb_cell), "zb3_cell": _f32(terrain.zb3_cell),
        "rho_base": _f32(reference.rho_base), "rho_theta_base": _f32(reference.rho_theta_base),
        "exner_base": _f32(reference.exner_base),
        "u_init": _f32(winds.u_init), "v_init": _f32(winds.v_init),
    }
    desc = _lib.HexDynDesc()
    for name, arr in arrays.items():
        keep[name] = arr
        ptype = C.POINTER(C.c_int32) if arr.dtype == np.int32 else C.POINTER(C.c_float)
        setattr(desc, name, arr.ctypes.data_as(ptype))
    desc.n_cells, desc.n_edges, desc.n_vertices, desc.n_levels = ncells, nedges, nvert, nlev
    desc.max_edges = eoc.shape[1]
    desc.max_edges2 = eoe.shape[1]
    desc.adv_width = adv_cells.shape[1]
    desc.n_scalars = int(scalars.shape[0])
    desc.cf1, desc.cf2, desc.cf3 = float(vertical.cf1), float(vertical.cf2), float(vertical.cf3)
    nominal = np.asarray(mesh_array(mesh, "nominalMinDc")).reshape(-1)
    desc.nominal_min_dc = float(F32(float(nominal[0])))
    desc.dt = float(cfg.config_dt)
    desc.n_sub_steps = cfg.config_number_of_sub_steps
    desc.split_steps = cfg.config_dynamics_split_steps
    desc.monotonic = 1 if cfg.fct else 0
    desc.moist = 1 if cfg.moist_coefficients == "native" else 0
    desc.numerics = 1 if cfg.numerics == "fast" else 0
    desc.coef_3rd_order = cfg.config_coef_3rd_order
    desc.apvm_upwinding = cfg.config_apvm_upwinding
    desc.smdiv = cfg.config_smdiv
    desc.len_disp = cfg.config_len_disp
    desc.epssm_minimum = cfg.config_epssm_minimum
    desc.epssm_maximum = cfg.config_epssm_maximum
    desc.epssm_bottom_z = cfg.config_epssm_transition_bottom_z
    desc.epssm_top_z = cfg.config_epssm_transition_top_z
    desc.rgas, desc.cp, desc.gravity, desc.p0 = 287.0, 1004.5, 9.80616, 100000.0
    for i, dts in enumerate(_schedule_dts(cfg)):
        desc.acoustic_dts2[i] = float(F32(dts) ** 2)
    desc.time_integration_order = int(cfg.config_time_integration_order)
    if cfg.config_horiz_mixing == "2d_smagorinsky":
        # hexcore/mixing_v841.py: weights, mesh scalings and smagorinsky_2d
        # constants on the host; the filter length is config_len_disp or,
        # when zero, nominalMinDc (hexcore/mixing.py:231)
        from . import mixing

        length = F32(cfg.config_len_disp) if cfg.config_len_disp > 0.0 else F32(float(nominal[0]))
        geo = {k: mesh_array(mesh, k) for k in ("nEdgesOnCell", "edgesOnCell", "verticesOnCell", "cellsOnEdge",
                                                 "xCell", "yCell", "zCell", "xVertex", "yVertex", "zVertex",
                                                 "meshDensity")}
        try:
            geo["sphere_radius"] = mesh_array(mesh, "sphere_radius")
        except AttributeError:
            geo["sphere_radius"] = np.asarray(float(getattr(mesh, "attrs")["sphere_radius"]))
        mix = mixing.setup(geo, cfg, length)
        for name, arr in (("deform_c2", mix.coef_c2), ("deform_s2", mix.coef_s2), ("deform_cs", mix.coef_cs),
                          ("mix_del2", mix.del2), ("mix_del4", mix.del4)):
            arr = np.ascontiguousarray(arr, dtype=F32)
            keep[name] = arr
            setattr(desc, name, arr.ctypes.data_as(C.POINTER(C.c_float)))
        desc.horiz_mixing = 1
        desc.smag_strain_scale, desc.smag_ceiling = float(mix.strain_scale), float(mix.ceiling)
        desc.smag_h4, desc.smag_div_factor = float(mix.h4), float(mix.div_factor)
        if cfg.config_mpas_cam_coef > 0.0:
            # hexcore/native/upper_damping.rs CAM floor: ((4 x 2.0833) len) coef in FP32
            desc.cam_levels = int(cfg.config_number_cam_damping_levels)
            desc.cam_base = float(((F32(4.0) * F32(2.0833)) * length) * F32(cfg.config_mpas_cam_coef))
    if cfg.config_rayleigh_damp_u:
        # hexcore/native/upper_damping.rs Rayleigh coefficient base 1/(levels (days 86400)) in FP32
        levels = int(cfg.config_number_rayleigh_damp_u_levels)
        days = F32(cfg.config_rayleigh_damp_u_timescale_days)
        desc.rayleigh_levels = levels
        desc.rayleigh_inverse = float(F32(1.0) / (F32(levels) * (days * F32(86400.0))))
    desc.clamp_negative_scalars = 1 if cfg.clamp_negative_scalars else 0
    sizes = dict(n_cells=ncells, n_edges=nedges, n_vertices=nvert, n_levels=nlev, n_scalars=int(scalars.shape[0]))
    return desc, keep, sizes
