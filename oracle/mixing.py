"""CPU oracle of the v8.4.1 2-D Smagorinsky horizontal mixing (test
infrastructure only).

A NumPy restatement, in float32 with the reference's operation order, of
``hexcore/mixing_v841.py`` (deformation weights, ``smagorinsky_2d``
diffusivity) and of the filters it applies from ``hexcore/mixing.py``
(``momentum_horizontal_filter_tendency`` :391, ``vertical_momentum_horizontal
_filter_tendency`` :533, ``theta_horizontal_filter_tendency`` :638, with the
stored-inverse arithmetic of v8.4.1), as ``hexcore/driver.py:2826-2880``
computes them once per dynamics subcycle and adds them to the saved Euler
terms.  Pinned by ``tests/golden/step_l2_L12_smag.npz`` (the reference's
deformation weights and step outputs).

The reference's strict geometry (``hexcore/native_geometry_math.py``) takes
float32 ``sin`` and ``cos`` from the GNU C library's ``sinf``/``cosf`` (equal
to this host's glibc 2.39 on every input compared) and ``asin`` and
``atan2`` correctly rounded (CORE-MATH).  This restatement calls the C
library's ``sinf``/``cosf`` and obtains the correctly rounded ``asin`` and
``atan2`` by evaluating in float64 and rounding once to float32 (a correctly
rounded result is unique; the float64 error is far below half a float32 ulp,
so the rounding lands on it except for arguments within 2^-29 relative of a
rounding boundary).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np

F32 = np.float32


def _cr(fn, *args) -> np.float32:
    return F32(fn(*[np.float64(a) for a in args]))


def _asin(x):
    return _cr(np.arcsin, x)


def _libm(name: str):
    import ctypes
    import ctypes.util

    fn = getattr(ctypes.CDLL(ctypes.util.find_library("m")), name)
    fn.argtypes = [ctypes.c_float]
    fn.restype = ctypes.c_float
    return fn


_SINF, _COSF = _libm("sinf"), _libm("cosf")


def _sin(x):
    return F32(_SINF(float(x)))


def _cos(x):
    return F32(_COSF(float(x)))


def _atan2(y, x):
    return _cr(np.arctan2, y, x)


def _arc_length(ax, ay, az, bx, by, bz, one):
    """``mpas_arc_length`` as ``mixing_v841.py:167``."""
    cx, cy, cz = bx - ax, by - ay, bz - az
    r = np.sqrt(ax * ax + ay * ay + az * az)
    c = np.sqrt(cx * cx + cy * cy + cz * cz)
    two = one + one
    return r * two * _asin(c / (two * r))


def _sphere_angle(ax, ay, az, bx, by, bz, cx, cy, cz, one):
    """``mpas_sphere_angle`` as ``mixing_v841.py:181``."""
    zero = one - one
    half = one / (one + one)
    two = one + one
    a = _arc_length(bx, by, bz, cx, cy, cz, one)
    b = _arc_length(ax, ay, az, cx, cy, cz, one)
    c = _arc_length(ax, ay, az, bx, by, bz, one)
    abx, aby, abz = bx - ax, by - ay, bz - az
    acx, acy, acz = cx - ax, cy - ay, cz - az
    dx = (aby * acz) - (abz * acy)
    dy = -((abx * acz) - (abz * acx))
    dz = (abx * acy) - (aby * acx)
    s = half * (a + b + c)
    ratio = (_sin(s - b) * _sin(s - c)) / (_sin(b) * _sin(c))
    sin_angle = np.sqrt(np.minimum(one, np.maximum(zero, ratio)))
    magnitude = two * _asin(np.maximum(np.minimum(sin_angle, one), -one))
    return magnitude if (dx * ax + dy * ay + dz * az) >= zero else -magnitude


def deformation_weights(arr: dict[str, Any]):
    """``initialize_deformation_weights_v841`` (``mixing_v841.py:495``, per
    cell as its row kernel :329): coef_c2, coef_s2, coef_cs [cell][slot]."""
    m = lambda k: np.asarray(arr["mesh." + k])  # noqa: E731
    radius = F32(float(m("sphere_radius")))
    counts = m("nEdgesOnCell").astype(np.int64)
    eoc = m("edgesOnCell").astype(np.int64)
    voc = m("verticesOnCell").astype(np.int64)
    coe = m("cellsOnEdge").astype(np.int64)
    xc, yc, zc = (m(k).astype(F32) for k in ("xCell", "yCell", "zCell"))
    xv, yv, zv = (m(k).astype(F32) for k in ("xVertex", "yVertex", "zVertex"))
    n, w = eoc.shape
    c2o, s2o, cso = (np.zeros((n, w), dtype=F32) for _ in range(3))
    one, zero, quarter = F32(1.0), F32(0.0), F32(0.25)
    pii = (one + one) * _asin(one)
    for cell in range(n):
        cnt = int(counts[cell])
        cx, cy, cz = xc[cell] / radius, yc[cell] / radius, zc[cell] / radius
        verts = voc[cell, :cnt]
        vx, vy, vz = xv[verts] / radius, yv[verts] / radius, zv[verts] / radius
        if cz == one:
            theta_abs = pii / (one + one)
        else:
            theta_abs = pii / (one + one) - _sphere_angle(cx, cy, cz, vx[0], vy[0], vz[0], zero, zero, one, one)
        thetav = np.zeros(cnt, dtype=F32)
        dl_sphere = np.zeros(cnt, dtype=F32)
        for j in range(cnt):
            jp = (j + 1) % cnt
            thetav[j] = _sphere_angle(cx, cy, cz, vx[j], vy[j], vz[j], vx[jp], vy[jp], vz[jp], one)
            dl_sphere[j] = radius * _arc_length(cx, cy, cz, vx[j], vy[j], vz[j], one)
        thetat = np.zeros(cnt, dtype=F32)
        thetat[0] = theta_abs
        for j in range(1, cnt):
            thetat[j] = thetat[j - 1] + thetav[j - 1]
        xp = np.array([_cos(t) for t in thetat], dtype=F32) * dl_sphere
        yp = np.array([_sin(t) for t in thetat], dtype=F32) * dl_sphere
        area = zero
        theta_edge = np.zeros(cnt, dtype=F32)
        for j in range(cnt):
            jp = (j + 1) % cnt
            dx, dy = xp[jp] - xp[j], yp[jp] - yp[j]
            area = (area + quarter * (xp[j] + xp[jp]) * (yp[jp] - yp[j])
                    - quarter * (yp[j] + yp[jp]) * (xp[jp] - xp[j]))
            theta_edge[j] = _atan2(dy, dx) - pii / (one + one)
        for j in range(cnt):
            jp = (j + 1) % cnt
            dx, dy = xp[jp] - xp[j], yp[jp] - yp[j]
            dl = np.sqrt(dx * dx + dy * dy)
            st, ct = _sin(theta_edge[j]), _cos(theta_edge[j])
            c2 = dl * (ct * ct) / area
            s2 = dl * (st * st) / area
            cs = dl * (st * ct) / area
            if int(coe[eoc[cell, j], 0]) != cell:
                c2, s2, cs = -c2, -s2, -cs
            c2o[cell, j], s2o[cell, j], cso[cell, j] = c2, s2, cs
    return c2o, s2o, cso


@dataclass
class SmagorinskyConfig:
    coef: float = 0.125            # config_smagorinsky_coef
    visc4: float = 0.05            # config_visc4_2dsmag
    del4u_div_factor: float = 10.0  # config_del4u_div_factor
    cam_coef: float = 0.0           # config_mpas_cam_coef (CAM floor of kdiff when > 0)
    cam_levels: int = 4             # config_number_cam_damping_levels


class SmagorinskyMixing:
    """The per-subcycle mixing of ``hexcore/driver.py:2826-2880`` on the
    geometry ``g`` of ``oracle.dycore`` (weights from ``deformation_weights``)."""

    def __init__(self, g, arr: dict[str, Any], cfg: SmagorinskyConfig, dt: float):
        self.g = g
        self.c2, self.s2, self.cs = deformation_weights(arr)
        length = g.len_disp
        cs_coef = F32(cfg.coef)
        self.strain_scale = (cs_coef * length) * (cs_coef * length)
        inv_dt = F32(1.0) / F32(dt)
        self.ceiling = (F32(0.01) * (length * length)) * inv_dt
        self.h4 = F32(cfg.visc4) * ((length * length) * length)
        self.factor4 = F32(cfg.del4u_div_factor)
        # CAM floor (hexcore/native/upper_damping.rs upper_cam)
        self.cam_levels = int(cfg.cam_levels) if cfg.cam_coef > 0.0 else 0
        self.cam_base = ((F32(4.0) * F32(2.0833)) * length) * F32(cfg.cam_coef)
        # meshScalingDel2/Del4 (mixing.py:271, config_h_ScaleWithMesh)
        from oracle.powf import powf_gnu

        density = np.asarray(arr["mesh.meshDensity"], dtype=F32)
        mean = F32(0.5) * (density[g.c0] + density[g.c1])
        self.del2 = F32(1.0) / powf_gnu(mean, F32(0.25))
        self.del4 = F32(1.0) / powf_gnu(mean, F32(0.75))
        self.inv_dv_limited = np.minimum(g.inv_dv, F32(4.0) * g.inv_dc)

    def kdiff(self, u, v):
        """``compute_smagorinsky_coefficients_v841`` (``mixing_v841.py:615``)."""
        g = self.g
        L = u.shape[0]
        kd = np.zeros((L, g.ncells), dtype=F32)
        two, quarter = F32(2.0), F32(0.25)
        for cell in range(g.ncells):
            dudx = np.zeros(L, dtype=F32)
            dudy = np.zeros(L, dtype=F32)
            dvdx = np.zeros(L, dtype=F32)
            dvdy = np.zeros(L, dtype=F32)
            for s in range(int(g.deg[cell])):
                e = g.eoc[cell, s]
                c2, s2, ccs = self.c2[cell, s], self.s2[cell, s], self.cs[cell, s]
                dudx = (dudx + c2 * u[:, e]) - ccs * v[:, e]
                dudy = (dudy + ccs * u[:, e]) - s2 * v[:, e]
                dvdx = (dvdx + ccs * u[:, e]) + c2 * v[:, e]
                dvdy = (dvdy + s2 * u[:, e]) + ccs * v[:, e]
            d11, d22, d12 = two * dudx, two * dvdy, dudy + dvdx
            diff = d11 - d22
            strain = np.sqrt(quarter * (diff * diff) + d12 * d12)
            kd[:, cell] = np.minimum(self.strain_scale * strain, self.ceiling)
        lv = self.cam_levels
        for k in range(L - lv, L) if lv else ():
            floor = self.cam_base * (F32(1.0) - F32(L - 1 - k) / F32(lv))
            kd[k] = np.fmax(kd[k], floor)
        return kd

    def tendencies(self, u, v, w, theta, rho, divergence, vorticity, euler_ru, euler_rw):
        """Saved Euler terms with mixing: (u = euler_ru + filter, w = euler_rw
        + filter, theta filter), ``hexcore/driver.py:2868-2872``."""
        g = self.g
        L = u.shape[0]
        kd = self.kdiff(u, v)
        h = F32(0.5) * (rho[:, g.c0] + rho[:, g.c1])     # diagnostics h_edge
        half, quarter, one = F32(0.5), F32(0.25), F32(1.0)
        # momentum (mixing.py:391, stored inverses)
        delsq_u = np.zeros_like(u)
        tu = euler_ru.copy()
        for e in range(g.nedges):
            c0, c1 = g.c0[e], g.c1[e]
            v0, v1 = g.voe[e]
            diffusion = ((divergence[:, c1] - divergence[:, c0]) * g.inv_dc[e]
                         - (vorticity[:, v1] - vorticity[:, v0]) * self.inv_dv_limited[e])
            delsq_u[:, e] += diffusion
            kdu = half * (kd[:, c0] + kd[:, c1])
            tu[:, e] += h[:, e] * kdu * diffusion * self.del2[e]
        inv_area_tri = g.inv_area_tri      # 1/areaTriangle in float32
        if self.h4 > F32(0.0):
            dvort = np.zeros((L, g.nvert), dtype=F32)
            for vtx in range(g.nvert):
                for s in range(g.eov.shape[1]):
                    e = g.eov[vtx, s]
                    factor = (inv_area_tri[vtx] * g.dc[e]) * g.vsign[vtx, s]
                    dvort[:, vtx] += factor * delsq_u[:, e]
            ddiv = np.zeros((L, g.ncells), dtype=F32)
            for cell in range(g.ncells):
                ia = g.inv_area[cell]
                for s in range(int(g.deg[cell])):
                    e = g.eoc[cell, s]
                    factor = (ia * g.dv[e]) * g.csign[cell, s]
                    ddiv[:, cell] += factor * delsq_u[:, e]
            for e in range(g.nedges):
                c0, c1 = g.c0[e], g.c1[e]
                v0, v1 = g.voe[e]
                scale = self.del4[e] * self.h4
                r_dc = scale * self.factor4 * g.inv_dc[e]
                r_dv = scale * self.inv_dv_limited[e]
                tu[:, e] -= h[:, e] * ((ddiv[:, c1] - ddiv[:, c0]) * r_dc - (dvort[:, v1] - dvort[:, v0]) * r_dv)
        # w (mixing.py:533) and theta (mixing.py:638)
        tw = np.zeros_like(w)
        tt = np.zeros_like(theta)
        dw = np.zeros((L, g.ncells), dtype=F32)
        dt_ = np.zeros_like(theta)
        for cell in range(g.ncells):
            ia = one / g.area[cell]
            for s in range(int(g.deg[cell])):
                e = g.eoc[cell, s]
                c0, c1 = g.c0[e], g.c1[e]
                sgn = g.csign[cell, s]
                esw = half * ia * sgn * g.dv[e] * (one / g.dc[e])
                for k in range(1, L):
                    flux = esw * (h[k, e] + h[k - 1, e]) * (w[k, c1] - w[k, c0])
                    dw[k, cell] += flux
                    sum_k = kd[k, c0] + kd[k, c1] + kd[k - 1, c0] + kd[k - 1, c1]
                    tw[k, cell] += flux * self.del2[e] * quarter * sum_k
                est = ia * sgn * g.dv[e] * (one / g.dc[e])
                flux_t = est * (theta[:, c1] - theta[:, c0]) * h[:, e]
                dt_[:, cell] += flux_t
                tt[:, cell] += flux_t * half * (kd[:, c0] + kd[:, c1]) * self.del2[e]
        if self.h4 > F32(0.0):
            for cell in range(g.ncells):
                scale = self.h4 * (one / g.area[cell])
                for s in range(int(g.deg[cell])):
                    e = g.eoc[cell, s]
                    c0, c1 = g.c0[e], g.c1[e]
                    es = self.del4[e] * scale * g.dv[e] * g.csign[cell, s] * (one / g.dc[e])
                    tw[1:L, cell] -= es * (dw[1:L, c1] - dw[1:L, c0])
                    tt[:, cell] -= es * (dt_[:, c1] - dt_[:, c0])
        return tu, euler_rw + tw, tt
