"""Host-side set-up of the 2-D Smagorinsky horizontal mixing (v8.4.1).

``hexcore/mixing_v841.py`` computes, once per mesh, the deformation weights
``coef_c2/coef_s2/coef_cs`` of every cell slot (``atm_initialize_deformation
_weights``, spherical branch) and the per-edge mesh scalings
``meshScalingDel2/Del4``; per dynamics subcycle the GPU kernels then form the
Smagorinsky diffusivity and the momentum, w and theta filters from them.

The weights are float32 spherical geometry evaluated in the reference's
operation order; ``sin``/``cos`` come from the C library's ``sinf``/``cosf``
(the functions the reference's strict geometry binds) and ``asin``/``atan2``
are correctly rounded (evaluated in float64 and rounded once).  The work is
vectorised over the cells of equal edge count.
"""

from __future__ import annotations

import ctypes
import ctypes.util
from dataclasses import dataclass
from typing import Any

import numpy as np

F32 = np.float32


def _libm(name: str, nargs: int = 1):
    fn = getattr(ctypes.CDLL(ctypes.util.find_library("m")), name)
    fn.argtypes = [ctypes.c_float] * nargs
    fn.restype = ctypes.c_float
    return fn


_SINF = _libm("sinf")
_COSF = _libm("cosf")
_POWF = _libm("powf", 2)
_vsin = np.frompyfunc(lambda x: _SINF(float(x)), 1, 1)
_vcos = np.frompyfunc(lambda x: _COSF(float(x)), 1, 1)


def _sin(x):
    return np.asarray(_vsin(np.asarray(x, dtype=F32)), dtype=F32)


def _cos(x):
    return np.asarray(_vcos(np.asarray(x, dtype=F32)), dtype=F32)


def _asin(x):
    return np.arcsin(np.asarray(x, dtype=F32).astype(np.float64)).astype(F32)


def _atan2(y, x):
    return np.arctan2(np.asarray(y, dtype=F32).astype(np.float64),
                      np.asarray(x, dtype=F32).astype(np.float64)).astype(F32)


def _arc(a, b):
    """mpas_arc_length of unit-sphere points a, b (tuples of float32 arrays)."""
    one = F32(1.0)
    two = one + one
    cx, cy, cz = b[0] - a[0], b[1] - a[1], b[2] - a[2]
    r = np.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
    c = np.sqrt(cx * cx + cy * cy + cz * cz)
    return r * two * _asin(c / (two * r))


def _angle(a, b, c):
    """mpas_sphere_angle at a between b and c (arrays of float32)."""
    one = F32(1.0)
    zero = one - one
    half = one / (one + one)
    two = one + one
    sa, sb, sc = _arc(b, c), _arc(a, c), _arc(a, b)
    abx, aby, abz = b[0] - a[0], b[1] - a[1], b[2] - a[2]
    acx, acy, acz = c[0] - a[0], c[1] - a[1], c[2] - a[2]
    dx = (aby * acz) - (abz * acy)
    dy = -((abx * acz) - (abz * acx))
    dz = (abx * acy) - (aby * acx)
    s = half * (sa + sb + sc)
    ratio = (_sin(s - sb) * _sin(s - sc)) / (_sin(sb) * _sin(sc))
    sin_angle = np.sqrt(np.minimum(one, np.maximum(zero, ratio)))
    magnitude = two * _asin(np.maximum(np.minimum(sin_angle, one), -one))
    return np.where((dx * a[0] + dy * a[1] + dz * a[2]) >= zero, magnitude, -magnitude).astype(F32)


def deformation_weights(mesh: Any) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """``coef_c2, coef_s2, coef_cs`` [cell][slot] of a spherical mesh."""
    arr = mesh.arrays if hasattr(mesh, "arrays") else mesh
    radius = F32(float(np.asarray(arr["sphere_radius"])))
    counts = np.asarray(arr["nEdgesOnCell"], dtype=np.int64)
    eoc = np.asarray(arr["edgesOnCell"], dtype=np.int64)
    voc = np.asarray(arr["verticesOnCell"], dtype=np.int64)
    coe = np.asarray(arr["cellsOnEdge"], dtype=np.int64)
    cell_xyz = [np.asarray(arr[k], dtype=F32) / radius for k in ("xCell", "yCell", "zCell")]
    vert_xyz = [np.asarray(arr[k], dtype=F32) for k in ("xVertex", "yVertex", "zVertex")]
    n, width = eoc.shape
    out = [np.zeros((n, width), dtype=F32) for _ in range(3)]
    one, zero, quarter = F32(1.0), F32(0.0), F32(0.25)
    pii = (one + one) * _asin(one)
    half_pi = pii / (one + one)
    for cnt in np.unique(counts):
        cells = np.flatnonzero(counts == cnt)
        cnt = int(cnt)
        c = tuple(x[cells] for x in cell_xyz)
        v = [tuple(x[voc[cells, j]] / radius for x in vert_xyz) for j in range(cnt)]
        pole = (zero, zero, one)
        first = _angle(c, v[0], tuple(np.full(cells.size, p, dtype=F32) for p in pole))
        theta_abs = np.where(c[2] == one, half_pi, half_pi - first).astype(F32)
        thetav = [_angle(c, v[j], v[(j + 1) % cnt]) for j in range(cnt)]
        dl_sphere = [radius * _arc(c, v[j]) for j in range(cnt)]
        thetat = [theta_abs]
        for j in range(1, cnt):
            thetat.append((thetat[j - 1] + thetav[j - 1]).astype(F32))
        xp = [_cos(thetat[j]) * dl_sphere[j] for j in range(cnt)]
        yp = [_sin(thetat[j]) * dl_sphere[j] for j in range(cnt)]
        area = np.zeros(cells.size, dtype=F32)
        theta_edge = []
        for j in range(cnt):
            jp = (j + 1) % cnt
            dx, dy = xp[jp] - xp[j], yp[jp] - yp[j]
            area = (area + quarter * (xp[j] + xp[jp]) * (yp[jp] - yp[j])
                    - quarter * (yp[j] + yp[jp]) * (xp[jp] - xp[j]))
            theta_edge.append((_atan2(dy, dx) - half_pi).astype(F32))
        for j in range(cnt):
            jp = (j + 1) % cnt
            dx, dy = xp[jp] - xp[j], yp[jp] - yp[j]
            dl = np.sqrt(dx * dx + dy * dy)
            st, ct = _sin(theta_edge[j]), _cos(theta_edge[j])
            sign = np.where(coe[eoc[cells, j], 0] != cells, F32(-1.0), F32(1.0))
            out[0][cells, j] = (dl * (ct * ct) / area) * sign
            out[1][cells, j] = (dl * (st * st) / area) * sign
            out[2][cells, j] = (dl * (st * ct) / area) * sign
    return out[0], out[1], out[2]


@dataclass
class MixingSetup:
    """Everything the library takes for the mixing of one mesh."""

    coef_c2: np.ndarray
    coef_s2: np.ndarray
    coef_cs: np.ndarray
    del2: np.ndarray        # [E] meshScalingDel2
    del4: np.ndarray        # [E] meshScalingDel4
    strain_scale: np.float32
    ceiling: np.float32
    h4: np.float32
    div_factor: np.float32


def setup(mesh: Any, cfg, length: np.float32) -> MixingSetup:
    """Weights, mesh scalings and the FP32 constants of ``smagorinsky_2d``
    (``hexcore/mixing_v841.py:615-707``, ``hexcore/mixing.py:271``) for the
    configuration ``cfg`` and the filter length (config_len_disp, or
    nominalMinDc when it is zero)."""
    arr = mesh.arrays if hasattr(mesh, "arrays") else mesh
    c2, s2, cs = deformation_weights(mesh)
    coe = np.asarray(arr["cellsOnEdge"], dtype=np.int64)
    if cfg.config_h_ScaleWithMesh:
        density = np.asarray(arr["meshDensity"], dtype=F32)
        mean = F32(0.5) * (density[coe[:, 0]] + density[coe[:, 1]])
        del2 = np.array([F32(1.0) / F32(_POWF(float(x), 0.25)) for x in mean], dtype=F32)
        del4 = np.array([F32(1.0) / F32(_POWF(float(x), 0.75)) for x in mean], dtype=F32)
    else:
        del2 = np.ones(coe.shape[0], dtype=F32)
        del4 = np.ones(coe.shape[0], dtype=F32)
    length = F32(length)
    coef = F32(cfg.config_smagorinsky_coef)
    strain_scale = (coef * length) * (coef * length)
    inv_dt = F32(1.0) / F32(cfg.config_dt)
    ceiling = (F32(0.01) * (length * length)) * inv_dt
    h4 = F32(cfg.config_visc4_2dsmag) * ((length * length) * length)
    return MixingSetup(c2, s2, cs, del2, del4, strain_scale, ceiling, h4, F32(cfg.config_del4u_div_factor))
