"""Shared test helpers: golden fixtures and synthetic cases as driver inputs."""

from __future__ import annotations

import hashlib
import json
from pathlib import Path
from types import SimpleNamespace

import numpy as np

from hexdyn.case import VerticalGridData
from hexdyn.mesh import VoronoiMesh

GOLDEN = Path(__file__).resolve().parent / "golden"
REPO = Path(__file__).resolve().parent.parent
STATE = ("rho", "rho_theta", "rho_u", "rho_w", "scalars")
SIDE = ("theta_m", "exner", "density_perturbation", "rho_theta_perturbation",
        "pressure_perturbation", "normal_velocity", "vertical_velocity")


def load_golden(name: str) -> dict:
    """A fixture; configuration variants carry only outputs and take their
    inputs from the base case they name."""
    with np.load(GOLDEN / f"step_{name}.npz", allow_pickle=False) as z:
        fx = {k: z[k] for k in z.files}
    if "base" in fx:
        base = load_golden(str(fx["base"]))
        fx.update({k: v for k, v in base.items() if k.startswith("in.")})
        if "config.n_scalars" in fx:
            fx["in.scalars"] = fx["in.scalars"][: int(fx["config.n_scalars"])].copy()
    return fx


def golden_config(fx: dict) -> dict:
    """The configuration a fixture was made with (defaults of the base cases)."""
    return {"dt": float(fx["config.dt"]), "n_sub_steps": int(fx["config.n_sub_steps"]),
            "monotonic": bool(int(fx.get("config.monotonic", 1))),
            "apvm_upwinding": float(fx.get("config.apvm_upwinding", 0.5)),
            "xnutr": float(fx.get("config.xnutr", 0.0)), "zd": float(fx.get("config.zd", 22000.0)),
            "order": int(fx.get("config.order", 3)),
            "smagorinsky": (None if "config.smagorinsky_coef" not in fx else
                            (float(fx["config.smagorinsky_coef"]), float(fx["config.visc4_2dsmag"]),
                             float(fx["config.del4u_div_factor"])))}


VARIANTS = [("l2_L12_sub1", 2), ("l2_L12_sub4", 2), ("l2_L12_nomono", 2), ("l2_L12_noapvm", 1),
            ("l2_L12_notracers", 2), ("l2_L12_xnutr", 2), ("l2_L12_rk2", 2), ("l2_L12_rk2_sub4", 1),
            ("l2_L12_smag", 2)]


# The 162-cell case with qv + 5 condensates and the same inputs cut to 4 and 5
# scalars: (name, steps); each fixture holds dry and native-moist outputs.
SCALAR_VARIANTS = [("l2_L12_t6", 2), ("l2_L12_t5", 2), ("l2_L12_t4", 2)]


def array_digest(a) -> str:
    """SHA-256 of an array's dtype, shape and C-order bytes."""
    a = np.ascontiguousarray(a)
    h = hashlib.sha256(f"{a.dtype.str}{a.shape}".encode())
    h.update(a.tobytes())
    return h.hexdigest()


def inputs_digest(arrays: dict) -> str:
    """One SHA-256 over every input array (case arrays), in name order."""
    h = hashlib.sha256()
    for k in sorted(arrays):
        h.update(k.encode())
        h.update(array_digest(arrays[k]).encode())
    return h.hexdigest()


def load_digests(name: str) -> dict:
    """A digest record of the reference's outputs at full size
    (tests/golden/digests_<name>.json)."""
    path = GOLDEN / f"digests_{name}.json"
    if not path.exists():
        import pytest

        pytest.skip(f"{path.name} has not been generated (tests/golden/make_golden.py REFERENCE_ROOT {name})")
    return json.loads(path.read_text())


def digest_case(record: dict):
    """The case a digest record was made from, rebuilt here, and whether its
    inputs carry the recorded digest (NumPy's SIMD transcendental paths
    depend on the host CPU, so another host may build other bits)."""
    from hexdyn.case import build_case, case_arrays
    from hexdyn.mesh import build_mesh

    c = record["case"]
    mesh = build_mesh(c["mesh_level"], lloyd=c["lloyd"], seed=c["seed"])
    arr = case_arrays(build_case(mesh, n_levels=c["levels"], seed=c["seed"], n_condensates=c["condensates"]))
    return arr, inputs_digest(arr) == record["inputs_sha256"]


def mismatched_digests(record: dict, label: str, step: int, state, side) -> list:
    """Names of the fields of one step whose words differ from the record."""
    bad = []
    for k in STATE:
        if array_digest(np.asarray(getattr(state, k), dtype=np.float32)) != record["outputs"][f"{label}.step{step}.{k}"]:
            bad.append(k)
    for k in SIDE:
        got = array_digest(np.asarray(getattr(side, k), dtype=np.float32))
        if got != record["outputs"][f"{label}.step{step}.side.{k}"]:
            bad.append(k)
    return bad


def inputs(fx: dict) -> dict:
    """The case arrays (``hexdyn.case.case_arrays`` layout) of a fixture."""
    return {k[3:]: v for k, v in fx.items() if k.startswith("in.")}


def case_from_arrays(arr: dict) -> SimpleNamespace:
    """A duck-typed case (reference attribute names) from case arrays."""
    mesh = VoronoiMesh(arrays={k[5:]: v for k, v in arr.items() if k.startswith("mesh.")})
    vfields = {k[9:]: v for k, v in arr.items() if k.startswith("vertical.")}
    for k in ("cf1", "cf2", "cf3"):
        vfields[k] = float(vfields[k])
    vfields["first_height_level"] = int(vfields["first_height_level"])
    vertical = VerticalGridData(**vfields)
    ns = SimpleNamespace(mesh=mesh, vertical=vertical)
    for k in ("zb_cell", "zb3_cell", "rho_base", "rho_theta_base", "pressure_base", "exner_base",
              "rho", "rho_theta", "rho_u", "rho_w", "scalars", "adv_coefs", "adv_coefs_3rd",
              "n_adv_cells_for_edge", "adv_cells_for_edge", "u_init", "v_init"):
        setattr(ns, k, arr[k])
    ns.time_seconds = 0.0
    return ns


def differing_words(a, b) -> int:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    assert a.shape == b.shape, (a.shape, b.shape)
    return int(np.count_nonzero(a.view(np.uint32) != b.view(np.uint32)))


# A read-only ``netCDF4`` for the reference's loaders, over SciPy's netCDF-3
# reader (classic and 64-bit offset files): ``Dataset`` as a context
# manager, ``variables`` with ``dimensions``, ``shape``, ``dtype``, ``name``
# and indexing that returns native-endian arrays, as netCDF4-python does
# with masking off.
NETCDF4_SHIM = """
import numpy as _np
from scipy.io import netcdf_file as _nc


class Variable:
    def __init__(self, name, var):
        self.name = name
        self._var = var
        self.dimensions = tuple(var.dimensions)
        self.shape = tuple(var.shape)
        self.dtype = _np.dtype(var.data.dtype).newbyteorder('=')
        self.ndim = len(self.shape)

    def __getitem__(self, index):
        return _np.asarray(self._var.data[index]).astype(self.dtype)

    def ncattrs(self):
        return list(self._var._attributes)

    def getncattr(self, name):
        return self._var._attributes[name]

    def set_auto_mask(self, flag):
        pass

    def set_auto_maskandscale(self, flag):
        pass


class Dataset:
    def __init__(self, path, mode='r', **kw):
        if mode != 'r':
            raise RuntimeError('read-only netCDF shim')
        self._f = _nc(str(path), 'r', mmap=False)
        self.variables = {k: Variable(k, v) for k, v in self._f.variables.items()}
        self.dimensions = dict(self._f.dimensions)

    def ncattrs(self):
        return list(self._f._attributes)

    def getncattr(self, name):
        return self._f._attributes[name]

    def set_auto_mask(self, flag):
        pass

    def close(self):
        self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
"""


def reference_stub_dir() -> str:
    """A temporary directory holding a read-only ``netCDF4`` over SciPy and a
    ``gpuwm`` stub: the reference's dycore modules import them at module
    level for file I/O and LES route checks only."""
    import tempfile

    d = Path(tempfile.mkdtemp(prefix="hexdyn_ref_stubs_"))
    (d / "netCDF4").mkdir()
    (d / "netCDF4" / "__init__.py").write_text(NETCDF4_SHIM)
    (d / "gpuwm").mkdir()
    (d / "gpuwm" / "__init__.py").write_text("")
    (d / "gpuwm" / "backend.py").write_text(
        "def compilation_target(*a, **k):\n    raise RuntimeError('no gpuwm')\n")
    return str(d)


def reference_root():
    """The reference checkout: ``HEXDYN_REFERENCE_ROOT``, else a ``reference``
    directory beside this repository; None when neither holds the sources."""
    import os

    for cand in (os.environ.get("HEXDYN_REFERENCE_ROOT"), str(REPO.parent / "reference")):
        if cand and (Path(cand) / "tree" / "src" / "hexcore").is_dir():
            return Path(cand)
    return None


def import_reference():
    """Put the reference's sources (and the stubs) on ``sys.path``; returns
    the root, or None when the checkout is absent."""
    import sys

    root = reference_root()
    if root is None:
        return None
    src = str(root / "tree" / "src")
    if src not in sys.path:
        sys.path.insert(0, reference_stub_dir())
        sys.path.insert(0, src)
    return root
