"""Oracle (test infrastructure only): the MPAS-A v8.4.1/8.4.2 dry-plus-tracer
dycore step, restated in vectorised NumPy FP32.

The CUDA path is compared against it in the tests.  Nothing in the
product imports it.  It restates the reference's CPU authority
(``DryDycoreDriver.step`` with ``V841DryDycoreConfig``), operation for
operation and in the same order, so that its FP32 results are bit-identical:
every NumPy ufunc on FP32 arrays rounds each operation once (no contraction),
so the same expression tree gives the same bits.  Every per-entity loop of
the reference accumulates its neighbour slots in slot order; here each slot
is one vectorised pass over all entities, which keeps that order per entity.

Reference anchors (``hexcore/`` = ``tree/src/hexcore/`` of gpuwm-hex 0.5.0):

* step / subcycle orchestration: ``driver.py:3314-3603`` and
  ``driver.py:2710-3312``;
* diagnostics: ``diagnostics.py:95-306`` (v8.4.1 stored-inverse branch);
* saved Euler terms: ``dynamics.py:188`` (pressure gradient), ``dynamics.py:122``
  (density tendency), ``driver.py:2804-2820`` (Euler w);
* tendencies: ``dynamics.py:227`` (vertical u transport),
  ``dynamics_v841.py:121`` (momentum), ``driver.py:933`` (rho-theta),
  ``driver.py:1081`` (w), ``acoustic.py:246`` (omega conversion);
* acoustic: ``acoustic_v841.py:81`` (coefficients), ``acoustic_v841.py:299``
  (substep), ``acoustic_v841.py:236`` (Thomas sweep), ``mixing.py:851``
  (divergence damping);
* recovery: ``driver.py:3166-3292``, ``terrain.py:491`` (w recovery),
  ``driver.py:790-863`` (Exner, pressure perturbation);
* split flux: ``integration.py:27,58``;
* transport: ``transport.py:1649`` (RK1/RK2), ``transport.py:1829`` (RK3
  monotonic FCT), ``transport.py:1461`` (edge values), ``transport.py:1389``
  (vertical flux);
* moist coefficients (native semantics): ``regional_v841.py:1180``.

Two moist-coefficient semantics are supported.  ``moist="dry"`` is the
reference CPU driver on a global mesh (qtot=0, cqu=cqw=1).  ``moist="native"``
applies ``atm_compute_moist_coefficients`` from every carried scalar once per
step, as native MPAS and the reference's CUDA driver do with physics off
(``cuda_driver.py:5050-5075``); on a dry state both give the same bits.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np

from .powf import powf_gnu

F32 = np.float32
ONE = F32(1.0)
ZERO = F32(0.0)
HALF = F32(0.5)


@dataclass
class OracleConfig:
    dt: float = 1800.0
    n_sub_steps: int = 2
    split_steps: int = 3
    coef_3rd_order: float = 0.25
    apvm_upwinding: float = 0.5
    smdiv: float = 0.1
    len_disp: float = 0.0
    epssm_minimum: float = 0.1
    epssm_maximum: float = 0.5
    epssm_bottom_z: float = 30000.0
    epssm_top_z: float = 50000.0
    monotonic: bool = True
    moist: str = "dry"          # "dry" (reference CPU driver) or "native"
    rgas: float = 287.0
    cp: float = 1004.5
    gravity: float = 9.80616
    p0: float = 100000.0
    order: int = 3              # config_time_integration_order (2 or 3)
    smagorinsky: Any = None     # oracle.mixing.SmagorinskyConfig: 2-D Smagorinsky mixing on
    rayleigh: Any = None        # (levels, days): Rayleigh damping of u over the top levels
    clamp_negative_scalars: bool = False  # cuda_driver.py:5311 end-of-step clamp
    # Per-stage physics hand-off (hexcore/cuda_driver.py:4393-4400):
    # callable(rk_step=, dynamics_substep=, state=State, saved=Sidecar) ->
    # object with rho_u / rho_theta / rho / diabatic_theta (or None each)
    physics_stage: Any = None


def schedule(dt: float, n_sub: int, splits: int, order: int = 3):
    """``RKSchedule.from_mpas`` (``integration.py:104-160``), orders 3 and 2."""
    dt_dyn = dt / splits
    if order == 2:
        large = (dt_dyn / 2.0, dt_dyn / 2.0, dt_dyn)
        acoustic = (dt_dyn / n_sub,) * 3
        counts = (max(1, n_sub // 2), max(1, n_sub // 2), n_sub)
    else:
        large = (dt_dyn / 3.0, dt_dyn / 2.0, dt_dyn)
        acoustic = (dt_dyn / 3.0, dt_dyn / n_sub, dt_dyn / n_sub)
        counts = (1, max(1, n_sub // 2), n_sub)
    return [(i + 1, large[i], acoustic[i], counts[i]) for i in range(3)]


def offcentering(rdzw: np.ndarray, cfg: OracleConfig):
    """``offcentering_v841.py:47`` etp/etm/ewp/ewm in source loop order."""
    nlev = rdzw.size
    lower, upper = F32(cfg.epssm_bottom_z), F32(cfg.epssm_top_z)
    mn, mx = F32(cfg.epssm_minimum), F32(cfg.epssm_maximum)
    hw = np.zeros(nlev + 1, dtype=F32)
    hu = np.zeros(nlev, dtype=F32)
    for k in range(nlev):
        hw[k + 1] = hw[k] + ONE / rdzw[k]
        hu[k] = HALF * (hw[k + 1] + hw[k])
    width = upper - lower
    pi = np.arccos(F32(-1.0))

    def coef(h):
        if h <= lower:
            return mn
        if h >= upper:
            return mx
        z = (h - lower) / width
        s = F32(np.sin(np.float64(HALF * pi * z)))
        return mn + s ** 2 * (mx - mn)

    etp = np.array([HALF * (ONE + F32(coef(h))) for h in hu], dtype=F32)
    etm = np.array([HALF * (ONE - F32(coef(h))) for h in hu], dtype=F32)
    ewp = np.array([HALF * (ONE + F32(coef(h))) for h in hw], dtype=F32)
    ewm = np.array([HALF * (ONE - F32(coef(h))) for h in hw], dtype=F32)
    return etp, etm, ewp, ewm


def _pos(x):
    """Python ``max(0, x)`` on FP32: x where x > 0 else +0."""
    return np.where(x > ZERO, x, ZERO).astype(F32)


def _neg(x):
    """Python ``min(0, x)`` on FP32: x where x < 0 else +0."""
    return np.where(x < ZERO, x, ZERO).astype(F32)


def _pymin(a, b):
    """Python ``min(a, b)``: a unless b < a."""
    return np.where(b < a, b, a).astype(F32)


def _pymax(a, b):
    return np.where(b > a, b, a).astype(F32)


class Geometry:
    """FP32 casts and index arrays of one mesh + vertical grid."""

    def __init__(self, arrays: dict[str, Any], cfg: OracleConfig):
        m = lambda k: arrays["mesh." + k]  # noqa: E731
        v = lambda k: arrays["vertical." + k]  # noqa: E731
        self.cfg = cfg
        self.coe = np.asarray(m("cellsOnEdge"), dtype=np.int64)
        self.c0, self.c1 = self.coe[:, 0], self.coe[:, 1]
        self.voe = np.asarray(m("verticesOnEdge"), dtype=np.int64)
        self.eoc = np.asarray(m("edgesOnCell"), dtype=np.int64)
        self.coc = np.asarray(m("cellsOnCell"), dtype=np.int64)
        self.voc = np.asarray(m("verticesOnCell"), dtype=np.int64)
        self.deg = np.asarray(m("nEdgesOnCell"), dtype=np.int64)
        self.eov = np.asarray(m("edgesOnVertex"), dtype=np.int64)
        self.cov = np.asarray(m("cellsOnVertex"), dtype=np.int64)
        self.eoe = np.asarray(m("edgesOnEdge"), dtype=np.int64)
        self.neoe = np.asarray(m("nEdgesOnEdge"), dtype=np.int64)
        self.ncells, self.nedges = self.deg.size, self.coe.shape[0]
        self.nvert = self.eov.shape[0]
        self.maxedges = self.eoc.shape[1]
        # edgesOnCell_sign (acoustic.py:224) and edgesOnVertex sign (diagnostics.py:49)
        cs = np.zeros(self.eoc.shape, dtype=F32)
        for s in range(self.maxedges):
            act = np.flatnonzero(self.deg > s)
            e = self.eoc[act, s]
            cs[act, s] = np.where(self.coe[e, 0] == act, ONE, F32(-1.0))
        self.csign = cs
        self.tsign = -cs                      # transport.py:369 operator signs
        self.vsign = np.where(self.voe[self.eov, 1] == np.arange(self.nvert)[:, None],
                              ONE, F32(-1.0)).astype(F32)
        ks = np.full(self.voc.shape, -1, dtype=np.int64)
        for s in range(self.maxedges):
            act = np.flatnonzero(self.deg > s)
            ks[act, s] = np.argmax(self.cov[self.voc[act, s]] == act[:, None], axis=1)
        self.kite_slot = ks
        self.dc = np.asarray(m("dcEdge")).astype(F32)
        self.dv = np.asarray(m("dvEdge")).astype(F32)
        self.area = np.asarray(m("areaCell")).astype(F32)
        self.inv_area = np.reciprocal(self.area)
        self.inv_area_tri = np.reciprocal(np.asarray(m("areaTriangle")).astype(F32))
        self.inv_dc = np.reciprocal(self.dc)
        self.inv_dv = np.reciprocal(self.dv)
        self.kite = np.asarray(m("kiteAreasOnVertex")).astype(F32)
        self.weights = np.asarray(m("weightsOnEdge")).astype(F32)
        self.f_vertex = np.asarray(m("fVertex")).astype(F32)
        self.f_edge = np.asarray(m("fEdge")).astype(F32)
        ang = np.asarray(m("angleEdge")).astype(F32)
        self.cos_angle = np.asarray([np.cos(a) for a in ang], dtype=F32)
        self.sin_angle = np.asarray([np.sin(a) for a in ang], dtype=F32)
        self.len_disp = F32(cfg.len_disp) if cfg.len_disp > 0 else F32(float(np.asarray(m("nominalMinDc")).reshape(-1)[0]))
        # vertical
        self.zz = np.asarray(v("zz"), dtype=F32)
        self.zxu = np.asarray(v("zxu"), dtype=F32)
        self.dss = np.asarray(v("dss"), dtype=F32)
        self.fzm = np.asarray(v("fzm"), dtype=F32)
        self.fzp = np.asarray(v("fzp"), dtype=F32)
        self.rdzw = np.asarray(v("rdzw"), dtype=F32)
        self.rdzu = np.asarray(v("rdzu"), dtype=F32)
        self.cf = (F32(float(v("cf1"))), F32(float(v("cf2"))), F32(float(v("cf3"))))
        self.nlev = self.zz.shape[0]
        self.zb = np.asarray(arrays["zb_cell"], dtype=F32)
        self.zb3 = np.asarray(arrays["zb3_cell"], dtype=F32)
        self.rho_base = np.asarray(arrays["rho_base"], dtype=F32)
        self.rtheta_base = np.asarray(arrays["rho_theta_base"], dtype=F32)
        self.exner_base = np.asarray(arrays["exner_base"], dtype=F32)
        self.u_init = np.asarray(arrays["u_init"], dtype=F32)
        self.v_init = np.asarray(arrays["v_init"], dtype=F32)
        self.adv = np.asarray(arrays["adv_coefs"]).astype(F32)
        self.adv3 = np.asarray(arrays["adv_coefs_3rd"]).astype(F32)
        self.n_adv = np.asarray(arrays["n_adv_cells_for_edge"], dtype=np.int64)
        self.adv_cells = np.asarray(arrays["adv_cells_for_edge"], dtype=np.int64)
        self.etp, self.etm, self.ewp, self.ewm = offcentering(self.rdzw, cfg)
        self.coef3 = F32(cfg.coef_3rd_order)
        self.g = F32(cfg.gravity)
        self.rgas = F32(cfg.rgas)
        self.rcv = F32(cfg.rgas) / (F32(cfg.cp) - F32(cfg.rgas))
        self.c2 = F32(cfg.cp) * self.rcv


@dataclass
class State:
    rho: np.ndarray
    rho_theta: np.ndarray
    rho_u: np.ndarray
    rho_w: np.ndarray
    scalars: np.ndarray

    def copy(self) -> "State":
        return State(self.rho.copy(), self.rho_theta.copy(), self.rho_u.copy(),
                     self.rho_w.copy(), self.scalars.copy())


@dataclass
class Sidecar:
    """``DrySavedDiagnostics`` (``driver.py:661``)."""

    theta_m: np.ndarray
    exner: np.ndarray
    density_perturbation: np.ndarray
    rho_theta_perturbation: np.ndarray
    pressure_perturbation: np.ndarray
    normal_velocity: np.ndarray
    vertical_velocity: np.ndarray

    def copy(self) -> "Sidecar":
        return Sidecar(*(getattr(self, k).copy() for k in self.__dataclass_fields__))


@dataclass
class Diag:
    ke: np.ndarray
    pv_edge: np.ndarray
    v: np.ndarray
    extra: dict = field(default_factory=dict)


class OracleDycore:
    def __init__(self, arrays: dict[str, Any], cfg: OracleConfig | None = None):
        self.cfg = cfg or OracleConfig()
        self.g = Geometry(arrays, self.cfg)
        self.smag = None
        if self.cfg.smagorinsky is not None:
            from oracle.mixing import SmagorinskyMixing

            self.smag = SmagorinskyMixing(self.g, arrays, self.cfg.smagorinsky, self.cfg.dt)

    # ----------------------------------------------------------- recovery
    def exner(self, rho_theta):
        g = self.g
        arg = (g.zz * F32(self.cfg.rgas / self.cfg.p0)) * rho_theta
        return powf_gnu(arg, F32(self.cfg.rgas / (self.cfg.cp - self.cfg.rgas)))

    def pressure_perturbation(self, exner, rtp):
        g = self.g
        return (g.zz * g.rgas) * (exner * rtp + g.rtheta_base * (exner - g.exner_base))

    def normal_velocity(self, rho, rho_u):
        g = self.g
        return (F32(2.0) * rho_u) / (rho[:, g.c0] + rho[:, g.c1])

    def vertical_velocity(self, rho, rho_u, rho_w):
        """``terrain.py:491`` recover_velocities (w part)."""
        g = self.g
        L = g.nlev
        cf1, cf2, cf3 = g.cf
        w = np.zeros((L + 1, g.ncells), dtype=F32)
        izz = g.fzm[1:L, None] * g.zz[1:L] + g.fzp[1:L, None] * g.zz[:L - 1]
        w[1:L] = rho_w[1:L] / izz
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            edge = g.eoc[cell, s]
            sign = g.csign[cell, s]
            flux = cf1 * rho_u[0, edge] + cf2 * rho_u[1, edge] + cf3 * rho_u[2, edge]
            w[0, cell] = w[0, cell] + sign * (g.zb[0, cell, s] + np.copysign(ONE, flux) * g.zb3[0, cell, s]) * flux
            flux = g.fzm[1:L, None] * rho_u[1:L, edge] + g.fzp[1:L, None] * rho_u[:L - 1, edge]
            w[1:L, cell] = w[1:L, cell] + sign * (g.zb[1:L, cell, s] + np.copysign(ONE, flux) * g.zb3[1:L, cell, s]) * flux
        bottom = cf1 * rho[0] + cf2 * rho[1] + cf3 * rho[2]
        irho = g.fzm[1:L, None] * rho[1:L] + g.fzp[1:L, None] * rho[:L - 1]
        w[0] = w[0] / bottom
        w[1:L] = w[1:L] / irho
        return w

    def rebuild_sidecar(self, s: State) -> Sidecar:
        """``driver.py:2655`` _rebuild_saved_diagnostics."""
        g = self.g
        theta = s.rho_theta / s.rho
        exner = self.exner(s.rho_theta)
        rp = s.rho - g.rho_base
        rtp = s.rho_theta - g.rtheta_base
        pp = self.pressure_perturbation(exner, rtp)
        return Sidecar(theta, exner, rp, rtp, pp, self.normal_velocity(s.rho, s.rho_u),
                       self.vertical_velocity(s.rho, s.rho_u, s.rho_w))

    # -------------------------------------------------------- diagnostics
    def diagnostics(self, rho, u, rk_step, cached_v) -> Diag:
        """``diagnostics.py:95`` compute_solve_diagnostics, stored inverses."""
        g = self.g
        L = g.nlev
        ke_edge = (g.dc * g.dv)[None, :] * (u * u)
        vort = np.zeros((L, g.nvert), dtype=F32)
        for s in range(3):
            e = g.eov[:, s]
            vort = vort + (g.vsign[:, s] * g.dc[e]) * u[:, e]
        vort = vort * g.inv_area_tri
        ke = np.zeros((L, g.ncells), dtype=F32)
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            e = g.eoc[cell, s]
            ke[:, cell] = ke[:, cell] + F32(0.25) * ke_edge[:, e]
        ke = ke * g.inv_area
        r = F32(0.25) * g.inv_area_tri
        ke_v = (ke_edge[:, g.eov[:, 0]] + ke_edge[:, g.eov[:, 1]] + ke_edge[:, g.eov[:, 2]]) * r
        kef = F32(0.625)
        ke = ke * kef
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            vtx = g.voc[cell, s]
            corr = ((ONE - kef) * g.kite[vtx, g.kite_slot[cell, s]]) * ke_v[:, vtx]
            ke[:, cell] = ke[:, cell] + corr * g.inv_area[cell]
        if rk_step == 3:
            v = np.zeros_like(u)
            for s in range(g.eoe.shape[1]):
                e = np.flatnonzero(g.neoe > s)
                nb = g.eoe[e, s]
                v[:, e] = v[:, e] + g.weights[e, s] * u[:, nb]
        else:
            v = cached_v.copy()
        pv_v = g.f_vertex[None, :] + vort
        pv_edge = HALF * (pv_v[:, g.voe[:, 0]] + pv_v[:, g.voe[:, 1]])
        if self.cfg.apvm_upwinding > 0.0:
            pv_c = np.zeros((L, g.ncells), dtype=F32)
            for s in range(g.maxedges):
                cell = np.flatnonzero(g.deg > s)
                vtx = g.voc[cell, s]
                contrib = g.kite[vtx, g.kite_slot[cell, s]] * pv_v[:, vtx]
                pv_c[:, cell] = pv_c[:, cell] + contrib * g.inv_area[cell]
            scale = F32(self.cfg.apvm_upwinding) * F32(self.cfg.dt)
            gpt = (pv_v[:, g.voe[:, 1]] - pv_v[:, g.voe[:, 0]]) * g.inv_dv
            gpn = (pv_c[:, g.c1] - pv_c[:, g.c0]) * g.inv_dc
            pv_edge = pv_edge - scale * (v * gpt + u * gpn)
        div = np.zeros((L, g.ncells), dtype=F32)
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            e = g.eoc[cell, s]
            div[:, cell] = div[:, cell] + (g.csign[cell, s] * g.dv[e]) * u[:, e]
        div = div * g.inv_area
        return Diag(ke=ke, pv_edge=pv_edge, v=v, extra={"vorticity": vort, "pv_vertex": pv_v, "divergence": div})

    # ------------------------------------------------------- coefficients
    def moist_coefficients(self, scalars):
        """``regional_v841.py:1180`` with every carried scalar loading the air."""
        g = self.g
        L = g.nlev
        if self.cfg.moist == "dry":
            return (np.zeros((L, g.ncells), dtype=F32), np.ones((L, g.ncells), dtype=F32),
                    np.ones((L, g.nedges), dtype=F32))
        qtot = np.zeros((L, g.ncells), dtype=F32)
        for q in scalars:
            qtot = qtot + q
        cqw = np.ones_like(qtot)
        for k in range(1, L):
            cqw[k] = ONE / (ONE + HALF * (qtot[k] + qtot[k - 1]))
        qe = np.zeros((L, g.nedges), dtype=F32)
        for q in scalars:
            qe = qe + HALF * (q[:, g.c0] + q[:, g.c1])
        cqu = ONE / (ONE + qe)
        return qtot, cqw, cqu

    def vertical_coefficients(self, dts, exner, theta, rtp, cqw, qtot):
        """``acoustic_v841.py:81`` in released source order."""
        g = self.g
        L = g.nlev
        zz = g.zz
        dts2 = F32(dts) ** 2
        g_r = g.g
        cofrz = g.rdzw.copy()
        cofwr = np.zeros_like(zz)
        cofwz = np.zeros_like(zz)
        coftz = np.zeros((L + 1, g.ncells), dtype=F32)
        for k in range(1, L):
            izz = g.fzm[k] * zz[k] + g.fzp[k] * zz[k - 1]
            cofwr[k] = HALF * g_r * izz
            cofwz[k] = g.c2 * izz * g.rdzu[k] * cqw[k] * (g.fzm[k] * exner[k] + g.fzp[k] * exner[k - 1])
            coftz[k] = g.fzm[k] * theta[k] + g.fzp[k] * theta[k - 1]
        cofwt = (HALF * g.rcv * zz * g_r * g.rho_base / (ONE + qtot) * exner
                 / ((g.rtheta_base + rtp) * g.exner_base))
        a = np.zeros_like(zz)
        b = np.zeros_like(zz)
        c = np.zeros_like(zz)
        alpha = np.zeros_like(zz)
        gamma = np.zeros_like(zz)
        b[0] = ONE
        etp, ewp, rdzw = g.etp, g.ewp, g.rdzw
        for k in range(1, L):
            a[k] = (-cofwz[k] * coftz[k - 1] * rdzw[k - 1] * zz[k - 1]
                    + cofwr[k] * cofrz[k - 1] - cofwt[k - 1] * coftz[k - 1] * rdzw[k - 1])
            a[k] = a[k] * etp[k - 1] * ewp[k - 1]
            b[k] = (cofwz[k] * coftz[k] * (etp[k] * rdzw[k] * zz[k] + etp[k - 1] * rdzw[k - 1] * zz[k - 1])
                    - coftz[k] * (etp[k] * cofwt[k] * rdzw[k] - etp[k - 1] * cofwt[k - 1] * rdzw[k - 1])
                    + cofwr[k] * (etp[k] * cofrz[k] - etp[k - 1] * cofrz[k - 1]))
            b[k] = b[k] * ewp[k]
            c[k] = (-cofwz[k] * coftz[k + 1] * rdzw[k] * zz[k] - cofwr[k] * cofrz[k]
                    + cofwt[k] * coftz[k + 1] * rdzw[k])
            c[k] = c[k] * etp[k] * ewp[k + 1]
        c[L - 1] = ZERO
        for k in range(1, L):
            den = ONE + dts2 * (b[k] - a[k] * gamma[k - 1])
            alpha[k] = ONE / den
            gamma[k] = dts2 * c[k] * alpha[k]
        return dict(cofrz=cofrz, cofwr=cofwr, cofwz=cofwz, coftz=coftz, cofwt=cofwt,
                    a=a, b=b, c=c, alpha=alpha, gamma=gamma)

    # --------------------------------------------------------- tendencies
    @staticmethod
    def _flux4(qm2, qm1, q0, qp1, vel):
        return vel * (F32(7.0) * (q0 + qm1) - (qp1 + qm2)) / F32(12.0)

    def _flux3(self, qm2, qm1, q0, qp1, vel, coef):
        return self._flux4(qm2, qm1, q0, qp1, vel) + F32(coef) * np.abs(vel) * (
            (qp1 - qm2) - F32(3.0) * (q0 - qm1)) / F32(12.0)

    def euler_terms(self, saved: State, T1: Sidecar, qtot, cqw, cqu):
        g = self.g
        L = g.nlev
        if self.cfg.moist == "dry":
            dpdz = -g.g * T1.density_perturbation
        else:
            dpdz = -g.g * (g.rho_base * qtot + T1.density_perturbation * (ONE + qtot))
        pp = T1.pressure_perturbation
        # dynamics.py:188 pressure_gradient_euler_tendency (stored inverse)
        euler_ru = -cqu * ((pp[:, g.c1] - pp[:, g.c0]) * g.inv_dc / (HALF * (g.zz[:, g.c1] + g.zz[:, g.c0]))
                           - HALF * g.zxu * (dpdz[:, g.c0] + dpdz[:, g.c1]))
        # dynamics.py:122 density_tendency
        hdiv = self.mass_flux_divergence(saved.rho_u)
        tend_rho = -hdiv - g.rdzw[:, None] * np.diff(saved.rho_w, axis=0)
        euler_rw = np.zeros_like(saved.rho_w)
        for k in range(1, L):
            inner = (g.rdzu[k] * (pp[k] - pp[k - 1]) - (g.fzm[k] * dpdz[k] + g.fzp[k] * dpdz[k - 1]))
            euler_rw[k] = -inner if self.cfg.moist == "dry" else -(cqw[k] * inner)
        return euler_ru, tend_rho, euler_rw

    def mass_flux_divergence(self, ru):
        """``dynamics.py:86``: per cell, slot order, then x inverse area."""
        g = self.g
        out = np.zeros((g.nlev, g.ncells), dtype=F32)
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            e = g.eoc[cell, s]
            out[:, cell] = out[:, cell] + g.csign[cell, s] * g.dv[e] * ru[:, e]
        return out * g.inv_area

    def vertical_transport_u(self, u, rw):
        """``dynamics.py:227`` vertical transport of normal momentum."""
        g = self.g
        L = g.nlev
        rwe = lambda k: HALF * (rw[k, g.c0] + rw[k, g.c1])  # noqa: E731
        wduz = np.zeros((L + 1, g.nedges), dtype=F32)
        wduz[1] = rwe(1) * (g.fzm[1] * u[1] + g.fzp[1] * u[0])
        for k in range(2, L - 1):
            wduz[k] = self._flux3(u[k - 2], u[k - 1], u[k], u[k + 1], rwe(k), 1.0)
        k = L - 1
        wduz[k] = rwe(k) * (g.fzm[k] * u[k] + g.fzp[k] * u[k - 1])
        return -g.rdzw[:, None] * np.diff(wduz, axis=0)

    def momentum(self, u, rho_edge, pv_edge, ke, hdiv, initial):
        """``dynamics_v841.py:121`` with perturbation-Coriolis subtraction."""
        g = self.g
        q = np.zeros_like(u)
        for s in range(g.eoe.shape[1]):
            act = np.flatnonzero(g.neoe > s)
            nb = g.eoe[act, s]
            work_pv = HALF * (pv_edge[:, act] + pv_edge[:, nb])
            q[:, act] = q[:, act] + g.weights[act, s] * u[:, nb] * work_pv
        for s in range(g.eoe.shape[1]):
            act = np.flatnonzero(g.neoe > s)
            nb = g.eoe[act, s]
            ref_u = g.u_init[:, None] * g.cos_angle[nb] - g.v_init[:, None] * g.sin_angle[nb]
            q[:, act] = q[:, act] - g.weights[act, s] * ref_u * g.f_edge[act]
        horizontal = rho_edge * (q - (ke[:, g.c1] - ke[:, g.c0]) * g.inv_dc)
        horizontal = initial + horizontal
        return horizontal - u * HALF * (hdiv[:, g.c0] + hdiv[:, g.c1])

    def rho_theta_tendency(self, cur: State, saved: State, theta, theta_saved, rk_step):
        """``driver.py:933`` stored-inverse branch."""
        g = self.g
        L = g.nlev
        coef = g.coef3
        # Edge theta once per edge (the reference recomputes it per cell slot
        # with identical arithmetic).
        sgn = np.copysign(ONE, cur.rho_u)
        et = np.zeros((L, g.nedges), dtype=F32)
        for ss in range(g.adv_cells.shape[1]):
            lanes = np.flatnonzero(g.n_adv > ss)
            donor = g.adv_cells[lanes, ss]
            w = g.adv[lanes, ss] + coef * sgn[:, lanes] * g.adv3[lanes, ss]
            et[:, lanes] = et[:, lanes] + w * theta[:, donor]
        res = np.zeros((L, g.ncells), dtype=F32)
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            e = g.eoc[cell, s]
            res[:, cell] = res[:, cell] - g.csign[cell, s] * cur.rho_u[:, e] * et[:, e]
        if rk_step > 1:
            for s in range(g.maxedges):
                cell = np.flatnonzero(g.deg > s)
                e = g.eoc[cell, s]
                corr = (g.csign[cell, s] * g.dv[e] * (saved.rho_u[:, e] - cur.rho_u[:, e]) * HALF
                        * (theta_saved[:, g.c1[e]] + theta_saved[:, g.c0[e]]))
                res[:, cell] = res[:, cell] - corr
        res = res * g.inv_area
        vf = np.zeros((L + 1, g.ncells), dtype=F32)
        rw, rws = cur.rho_w, saved.rho_w
        k = 1
        vf[k] = rw[k] * (g.fzm[k] * theta[k] + g.fzp[k] * theta[k - 1])
        vf[k] = vf[k] + (rws[k] - rw[k]) * (g.fzm[k] * theta_saved[k] + g.fzp[k] * theta_saved[k - 1])
        for k in range(2, L - 1):
            vf[k] = self._flux3(theta[k - 2], theta[k - 1], theta[k], theta[k + 1], rw[k], self.cfg.coef_3rd_order)
            vf[k] = vf[k] + (rws[k] - rw[k]) * (g.fzm[k] * theta_saved[k] + g.fzp[k] * theta_saved[k - 1])
        k = L - 1
        if k > 1:
            vf[k] = rws[k] * (g.fzm[k] * theta[k] + g.fzp[k] * theta[k - 1])
        return res - g.rdzw[:, None] * np.diff(vf, axis=0)

    def w_tendency(self, cur: State, w):
        """``driver.py:1081`` stored-inverse branch."""
        g = self.g
        L = g.nlev
        coef = g.coef3
        ru = cur.rho_u
        rui = g.fzm[1:L, None] * ru[1:L] + g.fzp[1:L, None] * ru[:L - 1]
        sgn = np.copysign(ONE, rui)
        ew = np.zeros((L - 1, g.nedges), dtype=F32)
        for ss in range(g.adv_cells.shape[1]):
            lanes = np.flatnonzero(g.n_adv > ss)
            donor = g.adv_cells[lanes, ss]
            wt = g.adv[lanes, ss] + coef * sgn[:, lanes] * g.adv3[lanes, ss]
            ew[:, lanes] = ew[:, lanes] + wt * w[1:L, donor]
        res = np.zeros((L + 1, g.ncells), dtype=F32)
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            e = g.eoc[cell, s]
            res[1:L, cell] = res[1:L, cell] - g.csign[cell, s] * rui[:, e] * ew[:, e]
        res = res * g.inv_area
        rw = cur.rho_w
        vf = np.zeros((L + 1, g.ncells), dtype=F32)
        k = 1
        vf[k] = F32(0.25) * (rw[k] + rw[k - 1]) * (w[k] + w[k - 1])
        for k in range(2, L - 1):
            vf[k] = self._flux3(w[k - 2], w[k - 1], w[k], w[k + 1], HALF * (rw[k] + rw[k - 1]), 1.0)
        k = L - 1
        if k > 1:
            vf[k] = F32(0.25) * (rw[k] + rw[k - 1]) * (w[k] + w[k - 1])
        for k in range(1, L):
            res[k] = res[k] - g.rdzu[k] * (vf[k + 1] - vf[k])
        res[0] = ZERO
        res[-1] = ZERO
        return res

    def omega(self, tend_rw, tend_ru):
        """``acoustic.py:246`` convert_w_tendency_to_omega."""
        g = self.g
        L = g.nlev
        out = tend_rw.copy()
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            e = g.eoc[cell, s]
            flux = g.csign[cell, s] * (g.fzm[1:L, None] * tend_ru[1:L, e] + g.fzp[1:L, None] * tend_ru[:L - 1, e])
            up = np.copysign(ONE, tend_ru[1:L, e])
            out[1:L, cell] = out[1:L, cell] - (g.zb[1:L, cell, s] + up * g.zb3[1:L, cell, s]) * flux
        out[1:L] = out[1:L] * (g.fzm[1:L, None] * g.zz[1:L] + g.fzp[1:L, None] * g.zz[:L - 1])
        return out

    # ----------------------------------------------------------- acoustic
    def acoustic_substep(self, st: dict, fo: dict, co: dict, dts: float, small_step: int):
        """``acoustic_v841.py:299`` one closed-mesh substep (in place on ``st``)."""
        g = self.g
        L = g.nlev
        dts_r = F32(dts)
        etp, etm, ewp, ewm = g.etp, g.etm, g.ewp, g.ewm
        if small_step != 1:
            pg = (st["rtheta_pp"][:, g.c1] - st["rtheta_pp"][:, g.c0]) * g.inv_dc / (HALF * (g.zz[:, g.c1] + g.zz[:, g.c0]))
            pg = fo["cqu"] * HALF * g.c2 * (fo["exner"][:, g.c0] + fo["exner"][:, g.c1]) * pg
            pg = pg + HALF * g.zxu * g.g * (st["rho_pp"][:, g.c0] + st["rho_pp"][:, g.c1])
            st["ru_p"] = st["ru_p"] + dts_r * (fo["tend_ru"] - pg)
            st["ru_avg"] = st["ru_avg"] + st["ru_p"]
        else:
            st["ru_p"] = dts_r * fo["tend_ru"]
            st["ru_avg"] = st["ru_p"].copy()
        st["rtheta_pp_old"] = np.zeros_like(st["rtheta_pp"]) if small_step == 1 else st["rtheta_pp"].copy()
        ru_p = st["ru_p"]
        rs = np.zeros((L, g.ncells), dtype=F32)
        ts = np.zeros_like(rs)
        th = fo["theta_m"]
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            e = g.eoc[cell, s]
            flux = g.csign[cell, s] * dts_r * g.dv[e] * ru_p[:, e] * g.inv_area[cell]
            rs[:, cell] = rs[:, cell] - flux
            ts[:, cell] = ts[:, cell] - flux * HALF * (th[:, g.c1[e]] + th[:, g.c0[e]])
        rw_p, rho_pp, rtpp = st["rw_p"], st["rho_pp"], st["rtheta_pp"]
        coftz = co["coftz"]
        rs = rho_pp + dts_r * fo["tend_rho"] + rs - dts_r * co["cofrz"][:, None] * (
            ewm[1:, None] * rw_p[1:] - ewm[:-1, None] * rw_p[:-1])
        ts = rtpp + dts_r * fo["tend_rt"] + ts - dts_r * g.rdzw[:, None] * (
            ewm[1:, None] * coftz[1:] * rw_p[1:] - ewm[:-1, None] * coftz[:-1] * rw_p[:-1])
        st["ww_avg"][1:L] = st["ww_avg"][1:L] + ewm[1:L, None] * rw_p[1:L]
        zz = g.zz
        cofwz, cofwr, cofwt = co["cofwz"], co["cofwr"], co["cofwt"]
        for k in range(1, L):
            rw_p[k] = rw_p[k] + dts_r * (
                fo["tend_rw"][k]
                - cofwz[k] * ((etp[k] * zz[k] * ts[k] - etp[k - 1] * zz[k - 1] * ts[k - 1])
                              + (etm[k] * zz[k] * rtpp[k] - etm[k - 1] * zz[k - 1] * rtpp[k - 1]))
                - cofwr[k] * ((etp[k] * rs[k] + etp[k - 1] * rs[k - 1])
                              + (etm[k] * rho_pp[k] + etm[k - 1] * rho_pp[k - 1]))
                + cofwt[k] * (etp[k] * ts[k] + etm[k] * rtpp[k])
                + cofwt[k - 1] * (etp[k - 1] * ts[k - 1] + etm[k - 1] * rtpp[k - 1]))
        dts2 = F32(dts) ** 2
        a, alpha, gamma = co["a"], co["alpha"], co["gamma"]
        for k in range(1, L):
            rw_p[k] = (rw_p[k] - dts2 * a[k] * rw_p[k - 1]) * alpha[k]
        for k in range(L - 1, -1, -1):
            rw_p[k] = rw_p[k] - gamma[k] * rw_p[k + 1]
        for k in range(1, L):
            delta = fo["rw_save"][k] - fo["rw"][k]
            damp = g.dss[k]
            zzi = g.fzm[k] * zz[k] + g.fzp[k] * zz[k - 1]
            rhoi = g.fzm[k] * fo["rho_zz"][k] + g.fzp[k] * fo["rho_zz"][k - 1]
            rw_p[k] = (rw_p[k] + delta - dts_r * damp * zzi * rhoi * fo["w"][k]) / (ONE + dts_r * damp) - delta
        st["ww_avg"][1:L] = st["ww_avg"][1:L] + ewp[1:L, None] * rw_p[1:L]
        st["rho_pp"] = rs - dts_r * co["cofrz"][:, None] * (ewp[1:, None] * rw_p[1:] - ewp[:-1, None] * rw_p[:-1])
        st["rtheta_pp"] = ts - dts_r * g.rdzw[:, None] * (
            ewp[1:, None] * coftz[1:] * rw_p[1:] - ewp[:-1, None] * coftz[:-1] * rw_p[:-1])

    def divergence_damping(self, st, theta, dts):
        """``mixing.py:851`` with the v8.4.1 stored inverse of dts."""
        g = self.g
        base = F32(2.0) * F32(self.cfg.smdiv) * g.len_disp
        coef = base * (ONE / F32(float(dts)))
        delta = st["rtheta_pp"] - st["rtheta_pp_old"]
        mask = np.zeros(g.nedges, dtype=F32)
        st["ru_p"] = st["ru_p"] + coef * (delta[:, g.c0] - delta[:, g.c1]) * (ONE - mask) / (
            theta[:, g.c0] + theta[:, g.c1])

    # ----------------------------------------------------------- subcycle
    def subcycle(self, state: State, T1: Sidecar, diag: Diag, moist, record=None, substep: int = 1):
        g = self.g
        cfg = self.cfg
        L = g.nlev
        qtot, cqw, cqu = moist
        stages = schedule(cfg.dt, cfg.n_sub_steps, cfg.split_steps, cfg.order)
        saved = state.copy()
        exner_s, theta_s = T1.exner, T1.theta_m
        rp_s, rtp_s = T1.density_perturbation, T1.rho_theta_perturbation
        co = self.vertical_coefficients(stages[0][2], exner_s, theta_s, rtp_s, cqw, qtot)
        cur = saved.copy()
        cur_theta, cur_rp, cur_rtp = theta_s.copy(), rp_s.copy(), rtp_s.copy()
        cur_exner, cur_pp = exner_s.copy(), T1.pressure_perturbation.copy()
        cur_u, cur_w = T1.normal_velocity.copy(), T1.vertical_velocity.copy()
        cached_v = diag.v
        euler_ru, tend_rho, euler_rw = self.euler_terms(saved, T1, qtot, cqw, cqu)
        # the density physics of the previous subcycle's last stage joins the
        # saved density tendency (hexcore/cuda_driver.py:4275-4305,
        # density_tendency(physics_tendency=) adds it last)
        tend_rho_dyn = tend_rho
        if cfg.physics_stage is not None and getattr(self, "_held_rho", None) is not None:
            tend_rho = tend_rho + self._held_rho
        mix_theta = None
        if self.smag is not None:
            # driver.py:2826-2880: the mixing of the subcycle's start state,
            # saved with the Euler terms for all three RK stages
            euler_ru, euler_rw, mix_theta = self.smag.tendencies(
                T1.normal_velocity, diag.v, T1.vertical_velocity, theta_s, saved.rho,
                diag.extra["divergence"], diag.extra["vorticity"], euler_ru, euler_rw)
        flux_u = flux_w = None
        for stage, large_dt, dts, n_ac in stages:
            phys = None
            if cfg.physics_stage is not None:
                phys = cfg.physics_stage(
                    rk_step=stage, dynamics_substep=substep, state=cur,
                    saved=Sidecar(cur_theta, cur_exner, cur_rp, cur_rtp, cur_pp, cur_u, cur_w))
                if phys is None:
                    raise RuntimeError("active MPAS RK callback returned no sources")
            if stage == 2 and cfg.order == 3:  # driver.py:2894
                co = self.vertical_coefficients(dts, exner_s, cur_theta, cur_rtp, cqw, qtot)
            rho_edge = HALF * (cur.rho[:, g.c0] + cur.rho[:, g.c1])
            hdiv = self.mass_flux_divergence(cur.rho_u)
            tend_ru = self.vertical_transport_u(cur_u, cur.rho_w)
            tend_ru = self.momentum(cur_u, rho_edge, diag.pv_edge, diag.ke, hdiv, tend_ru)
            if self.cfg.rayleigh is not None:
                # Rayleigh damping of u before the saved Euler term
                # (hexcore/native/upper_damping.rs upper_rayleigh, driver.py:2941)
                levels, days = self.cfg.rayleigh
                inv = F32(1.0) / (F32(levels) * (F32(days) * F32(86400.0)))
                for k in range(L - levels, L):
                    tend_ru[k] = tend_ru[k] - (rho_edge[k] * cur_u[k]) * (F32(k - (L - levels) + 1) * inv)
            tend_ru = tend_ru + euler_ru
            if phys is not None and getattr(phys, "rho_u", None) is not None:
                tend_ru = tend_ru + phys.rho_u  # cuda_driver.py:4445 add_pair
            tend_rt = self.rho_theta_tendency(cur, saved, cur_theta, theta_s, stage)
            if phys is not None:
                if stage == 3:
                    # cuda_driver.py:4459-4475 modified_theta_dynamics_rate
                    self.modified_rate = (tend_rt - tend_rho_dyn * cur_theta) / cur.rho
                dth = getattr(phys, "diabatic_theta", None)
                if dth is not None:
                    tend_rt = tend_rt + cur.rho * dth  # add_lagged_diabatic_theta
            if mix_theta is not None:
                tend_rt = tend_rt + mix_theta  # driver.py:2967
            if phys is not None and getattr(phys, "rho_theta", None) is not None:
                tend_rt = tend_rt + phys.rho_theta  # cuda_driver.py:4489-4494
            tend_rw = self.w_tendency(cur, cur_w)
            tend_rw = tend_rw + euler_rw
            tend_om = self.omega(tend_rw, tend_ru)
            if record is not None:
                record.append(dict(stage=stage, tend_ru=tend_ru, tend_rt=tend_rt, tend_rw=tend_om))
            st = dict(ru_p=np.zeros_like(cur.rho_u), rw_p=np.zeros_like(cur.rho_w),
                      rtheta_pp=np.zeros_like(cur.rho), rtheta_pp_old=np.zeros_like(cur.rho),
                      rho_pp=np.zeros_like(cur.rho), ru_avg=np.zeros_like(cur.rho_u),
                      ww_avg=np.zeros_like(cur.rho_w))
            fo = dict(rho_zz=cur.rho, theta_m=theta_s, exner=exner_s, cqu=cqu, tend_ru=tend_ru,
                      tend_rho=tend_rho, tend_rt=tend_rt, tend_rw=tend_om, w=cur_w, rw=cur.rho_w,
                      rw_save=saved.rho_w)
            for small in range(1, n_ac + 1):
                self.acoustic_substep(st, fo, co, dts, small)
                self.divergence_damping(st, theta_s, dts)
            if record is not None and stage == 3:
                # the acoustic words the reference hands to its
                # acoustic_output_callback (cuda_driver.py:4707-4711)
                record.append(dict(ru_p=st["ru_p"].copy(), rw_p=st["rw_p"].copy()))
            cand_rp = rp_s + st["rho_pp"]
            cand_rtp = rtp_s + st["rtheta_pp"]
            cand = State(cand_rp + g.rho_base, cand_rtp + g.rtheta_base,
                         saved.rho_u + st["ru_p"], saved.rho_w + st["rw_p"], cur.scalars.copy())
            cand.rho_w[0] = ZERO
            cand.rho_w[-1] = ZERO
            if np.any(cand.rho <= 0.0) or np.any(cand.rho_theta <= 0.0):
                raise FloatingPointError(f"non-positive density in RK stage {stage}")
            inv_steps = ONE / F32(n_ac)
            fu = saved.rho_u + st["ru_avg"] * inv_steps
            fw = saved.rho_w + st["ww_avg"] * inv_steps
            if stage == 3:
                flux_u, flux_w = fu.copy(), fw.copy()
            cand.scalars = saved.scalars.copy()
            cur = cand
            cur_rp, cur_rtp = cand_rp, cand_rtp
            cur_theta = cur.rho_theta / cur.rho
            if stage == 3:
                cur_exner = self.exner(cur.rho_theta)
                cur_pp = self.pressure_perturbation(cur_exner, cur_rtp)
                cur_theta = cur.rho_theta / cur.rho
            cur_u = self.normal_velocity(cur.rho, cur.rho_u)
            cur_w = self.vertical_velocity(cur.rho, cur.rho_u, cur.rho_w)
            diag = self.diagnostics(cur.rho, cur_u, stage, cached_v)
            cached_v = diag.v
            if phys is not None and stage == stages[-1][0]:
                self._held_rho = getattr(phys, "rho", None)
        side = Sidecar(cur_theta.copy(), cur_exner.copy(), cur_rp.copy(), cur_rtp.copy(),
                       cur_pp.copy(), cur_u.copy(), cur_w.copy())
        return cur, side, diag, flux_u, flux_w

    # ---------------------------------------------------------- transport
    def _vflux(self, q, ww):
        """``transport.py:1389`` with the atmosphere flux3 (+ correction)."""
        g = self.g
        L = g.nlev
        coef = F32(self.cfg.coef_3rd_order)
        out = np.zeros((L + 1, q.shape[1]), dtype=F32)
        for k in range(1, L):
            if k == 1 or k == L - 1:
                out[k] = ww[k] * (g.fzm[k] * q[k] + g.fzp[k] * q[k - 1])
            else:
                base = ww[k] * (F32(7.0) * (q[k] + q[k - 1]) - (q[k + 1] + q[k - 2])) / F32(12.0)
                corr = coef * np.abs(ww[k]) * ((q[k + 1] - q[k - 2]) - F32(3.0) * (q[k] - q[k - 1])) / F32(12.0)
                out[k] = base + corr
        return out

    def _edge_values(self, q, hv, monotonic):
        """``transport.py:1461`` third order, for one scalar (L, C) -> (L, E)."""
        g = self.g
        coef = g.coef3
        sgn = np.copysign(ONE, hv)
        out = np.zeros((g.nlev, g.nedges), dtype=F32)
        active = np.ones(g.nedges, dtype=bool)
        if monotonic:
            ten = np.flatnonzero(g.n_adv == 10)
            if ten.size:
                s = sgn[:, ten]
                val = (g.adv[ten, 0] + coef * s * g.adv3[ten, 0]) * q[:, g.adv_cells[ten, 0]]
                for ss in range(1, 10):
                    val = val + (g.adv[ten, ss] + coef * s * g.adv3[ten, ss]) * q[:, g.adv_cells[ten, ss]]
                out[:, ten] = hv[:, ten] * val
            active &= g.n_adv != 10
        for ss in range(g.adv_cells.shape[1]):
            e = np.flatnonzero(active & (g.n_adv > ss))
            cell = g.adv_cells[e, ss]
            w = g.adv[e, ss] + coef * sgn[:, e] * g.adv3[e, ss]
            if monotonic:
                w = hv[:, e] * w
            out[:, e] = out[:, e] + w * q[:, cell]
        return out

    def advance_scalars(self, old, stage_q, rho_old, rho_new, hv, ww, dt, rk_step):
        """``transport.py:1649`` (split transport, stored inverse area)."""
        g = self.g
        L = g.nlev
        step = F32(dt)
        # transport.py:1749-1755
        wn = (F32(1.0 / (3.0 if self.cfg.order == 3 else 2.0)) if rk_step == 1
              else (HALF if rk_step == 2 else ONE))
        target = (ONE - wn) * rho_old + wn * rho_new
        out = stage_q.copy()
        for i in range(old.shape[0]):
            ev = self._edge_values(stage_q[i], hv, False)
            vf = self._vflux(stage_q[i], ww)
            t = np.zeros((L, g.ncells), dtype=F32)
            for s in range(g.maxedges):
                cell = np.flatnonzero(g.deg > s)
                e = g.eoc[cell, s]
                t[:, cell] = t[:, cell] + g.tsign[cell, s] * hv[:, e] * ev[:, e]
            t = t * g.inv_area + ZERO
            num = old[i] * rho_old + step * (t - g.rdzw[:, None] * (vf[1:] - vf[:-1]))
            out[i] = num * (ONE / target)
        return out

    def advance_scalars_mono(self, old_in, stage_q, rho_old, rho_new, hv, ww, dt):
        """``transport.py:1829`` monotonic FCT, v8.4.1 source order."""
        g = self.g
        L = g.nlev
        step = F32(dt)
        eps = F32(1.0e-20)
        old = old_in + step * np.zeros_like(old_in) / rho_old[None]
        hd = np.zeros((L, g.ncells), dtype=F32)
        for s in range(g.maxedges):
            cell = np.flatnonzero(g.deg > s)
            e = g.eoc[cell, s]
            hd[:, cell] = hd[:, cell] + g.tsign[cell, s] * hv[:, e] * g.dv[e] * g.inv_area[cell]
        target = rho_old + step * (hd - g.rdzw[:, None] * (ww[1:] - ww[:-1]))
        if np.any(target <= 0):
            raise ValueError("limited transport target density must stay positive")
        out = stage_q.copy()
        for i in range(old.shape[0]):
            o = old[i]
            high_e = self._edge_values(stage_q[i], hv, True)
            high_v = self._vflux(stage_q[i], ww)
            mn = o.copy()
            mx = o.copy()
            lo = np.concatenate([o[:1], o[:-1]])
            hi = np.concatenate([o[1:], o[-1:]])
            mn = np.minimum(np.minimum(lo, o), hi)
            mx = np.maximum(np.maximum(lo, o), hi)
            for s in range(g.maxedges):
                cell = np.flatnonzero(g.deg > s)
                nb = g.coc[cell, s]
                mn[:, cell] = _pymin(mn[:, cell], o[:, nb])
                mx[:, cell] = _pymax(mx[:, cell], o[:, nb])
            mass = o * rho_old
            vres = step * high_v
            fcol = np.zeros((L + 1, g.ncells), dtype=F32)
            for k in range(1, L):
                fcol[k] = step * (_pos(ww[k]) * o[k - 1] + _neg(ww[k]) * o[k])
            for k in range(L - 1):
                mass[k] = mass[k] - fcol[k + 1] * g.rdzw[k]
            for k in range(1, L):
                mass[k] = mass[k] + fcol[k] * g.rdzw[k]
                vres[k] = vres[k] - fcol[k]
            s_in = -g.rdzw[:, None] * (_neg(vres[1:]) - _pos(vres[:-1]))
            s_out = -g.rdzw[:, None] * (_pos(vres[1:]) - _neg(vres[:-1]))
            upw = (g.dv * step) * (_pos(hv) * o[:, g.c0] + _neg(hv) * o[:, g.c1])
            hres = step * high_e - upw
            for s in range(g.maxedges):
                cell = np.flatnonzero(g.deg > s)
                e = g.eoc[cell, s]
                ia = g.inv_area[cell]
                mass[:, cell] = mass[:, cell] + g.tsign[cell, s] * upw[:, e] * ia
                sr = (-g.tsign[cell, s]) * hres[:, e]
                s_out[:, cell] = s_out[:, cell] - _pos(sr) * ia
                s_in[:, cell] = s_in[:, cell] - _neg(sr) * ia
            sf = (mx * target - mass) / (s_in + eps)
            s_in = _pymin(np.full_like(sf, ONE), _pos(sf))
            sf = (mn * target - mass) / (s_out - eps)
            s_out = _pymin(np.full_like(sf, ONE), _pos(sf))
            hres = (_pos(hres) * _pymin(s_out[:, g.c0], s_in[:, g.c1])
                    + _neg(hres) * _pymin(s_in[:, g.c0], s_out[:, g.c1]))
            for k in range(1, L):
                f = vres[k]
                vres[k] = (_pos(f) * _pymin(s_out[k - 1], s_in[k])
                           + _neg(f) * _pymin(s_out[k], s_in[k - 1]))
            for s in range(g.maxedges):
                cell = np.flatnonzero(g.deg > s)
                e = g.eoc[cell, s]
                mass[:, cell] = mass[:, cell] + g.tsign[cell, s] * hres[:, e] * g.inv_area[cell]
            mass = mass - g.rdzw[:, None] * (vres[1:] - vres[:-1])
            out[i] = _pos(mass / target)
        return out

    # --------------------------------------------------------------- step
    def step(self, state: State, sidecar: Sidecar | None = None, record=None):
        """One outer step: 3 dynamics subcycles then 3 scalar RK stages."""
        cfg = self.cfg
        g = self.g
        outer = state.copy()
        T0 = self.rebuild_sidecar(outer) if sidecar is None else sidecar.copy()
        moist = self.moist_coefficients(outer.scalars)
        diag = self.diagnostics(outer.rho, T0.normal_velocity, 3, None)
        cur, carried = outer, T0
        fu_sum = fw_sum = None
        self._held_rho = None
        self.modified_rate = None
        for sub in range(cfg.split_steps):
            cur, carried, diag, fu, fw = self.subcycle(cur, carried, diag, moist, record, substep=sub + 1)
            fu_sum = fu.copy() if fu_sum is None else fu + fu_sum
            fw_sum = fw.copy() if fw_sum is None else fw + fw_sum
        inv = ONE / F32(cfg.split_steps)
        flux_u, flux_w = fu_sum * inv, fw_sum * inv
        if outer.scalars.shape[0] > 0:
            q = outer.scalars.copy()
            for stage, large_dt, _, _ in schedule(cfg.dt, cfg.n_sub_steps, 1, cfg.order):
                if stage == 3 and cfg.monotonic:
                    q = self.advance_scalars_mono(outer.scalars, q, outer.rho, cur.rho, flux_u, flux_w, large_dt)
                else:
                    q = self.advance_scalars(outer.scalars, q, outer.rho, cur.rho, flux_u, flux_w, large_dt, stage)
            if cfg.clamp_negative_scalars:
                # hexcore/cuda_driver.py:5311 putmask(scalars, scalars < 0, 0):
                # -0 and NaN compare false and keep their words
                q = q.copy()
                q[q < 0] = ZERO
            cur.scalars = q
        if record is not None:
            record.append(dict(flux_u=flux_u, flux_w=flux_w))
        del g
        return cur, carried
