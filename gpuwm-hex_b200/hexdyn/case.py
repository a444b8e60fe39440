"""Synthetic dycore cases: vertical grid, terrain metrics, balanced jet, tracers.

Everything the reference reads from MPAS grid/static/init files or computes
with its (absent) Rust engines is built here from published formulas:

* a stretched height coordinate to ``ztop`` with a smoothly decaying
  terrain-following hybrid (``zgrid``), its metrics ``zz``/``zxu``, the
  interface weights ``fzm``/``fzp`` and the bottom extrapolation ``cf1..3``
  (the fields of ``hexcore/vertical.py:83`` ``VerticalGrid``);
* the cell-oriented omega-conversion metrics ``zb``/``zb3`` of the MPAS init
  core (``hexcore/driver.py:636`` ``TerrainMetrics``; ``zb3`` already carries
  ``config_coef_3rd_order`` as ``hexcore/terrain.py:39`` states);
* quadratic-fit second derivatives ``deriv_two`` and the compressed
  third-order advection stencil (``hexcore/transport.py:38``
  ``AdvectionCoefficients``), in the native v8.4.1 insertion order;
* a zonally balanced mid-latitude jet in hydrostatic and gradient-wind
  balance (thermal-wind integration in latitude), a Gaussian zonal-wind
  perturbation, water vapour ``qv = 0.8 qsat exp(-z/3 km)`` and optional
  log-normal condensate blobs.

Fields are FP32 where the dycore consumes them (MPAS single precision) and
float64 where they are static geometry, exactly like MPAS files.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np

from .mesh import OMEGA, VoronoiMesh

RGAS = 287.0
CP = 1004.5
GRAVITY = 9.80616
P0 = 100000.0
RV = 461.6
F32 = np.float32


@dataclass
class VerticalGridData:
    """Field-for-field the reference's ``VerticalGrid`` (FP32 arrays)."""

    zw: np.ndarray
    dzw: np.ndarray
    rdzw: np.ndarray
    zu: np.ndarray
    dzu: np.ndarray
    rdzu: np.ndarray
    rdzwp: np.ndarray
    rdzwm: np.ndarray
    fzp: np.ndarray
    fzm: np.ndarray
    ah: np.ndarray
    hx: np.ndarray
    zgrid: np.ndarray
    zz: np.ndarray
    zxu: np.ndarray
    dss: np.ndarray
    cf1: float
    cf2: float
    cf3: float
    first_height_level: int

    @property
    def n_vert_levels(self) -> int:
        return int(self.dzw.size)


@dataclass
class DycoreCase:
    """One synthetic instance: mesh, vertical grid, base state, state, metrics."""

    mesh: VoronoiMesh
    vertical: VerticalGridData
    zb_cell: np.ndarray          # (L+1, C, maxEdges) FP32
    zb3_cell: np.ndarray         # (L+1, C, maxEdges) FP32, x config_coef_3rd_order
    rho_base: np.ndarray         # (L, C)
    rho_theta_base: np.ndarray
    pressure_base: np.ndarray
    exner_base: np.ndarray
    rho: np.ndarray              # rho_zz (L, C)
    rho_theta: np.ndarray        # (L, C)
    rho_u: np.ndarray            # (L, E)
    rho_w: np.ndarray            # (L+1, C)
    scalars: np.ndarray          # (T, L, C)
    scalar_names: tuple[str, ...]
    adv_coefs: np.ndarray        # (E, W) float64
    adv_coefs_3rd: np.ndarray    # (E, W) float64
    n_adv_cells_for_edge: np.ndarray
    adv_cells_for_edge: np.ndarray
    u_init: np.ndarray           # (L,) FP32 reference wind profiles
    v_init: np.ndarray
    coef_3rd_order: float = 0.25


# ---------------------------------------------------------------- vertical


def stretched_levels(n_levels: int, ztop: float) -> np.ndarray:
    """Interface heights of the flat coordinate: quadratic stretching."""
    s = np.arange(n_levels + 1, dtype=np.float64) / n_levels
    return ztop * (0.35 * s + 0.65 * s * s)


def hybrid_decay(zw: np.ndarray, ztop: float, scale: float = 8000.0) -> np.ndarray:
    """Terrain influence B(z): 1 at the ground, 0 at the top (SLEVE-like)."""
    return np.sinh((ztop - zw) / scale) / np.sinh(ztop / scale)


def smooth_cells(mesh: VoronoiMesh, values: np.ndarray, passes: int) -> np.ndarray:
    out = np.asarray(values, dtype=np.float64).copy()
    coc, deg = mesh.cellsOnCell, mesh.nEdgesOnCell
    for _ in range(passes):
        acc = np.zeros_like(out)
        for s in range(coc.shape[1]):
            act = deg > s
            acc[act] += out[coc[act, s]] - out[act]
        out = out + 0.125 * acc
    return out


def gaussian_terrain(mesh: VoronoiMesh, *, seed: int, n_mountains: int = 3,
                     height: float = 2000.0, half_width: float = 1.5e6,
                     smoothing_passes: int = 2) -> np.ndarray:
    """Sum of seeded Gaussian mountains (height at centre, half height at
    ``half_width`` great-circle distance), smoothed on the mesh."""
    rng = np.random.default_rng(seed)
    lat, lon = mesh.latCell, mesh.lonCell
    radius = mesh.sphere_radius
    h = np.zeros_like(lat)
    for _ in range(n_mountains):
        lat0 = np.arcsin(rng.uniform(-0.8, 0.8))
        lon0 = rng.uniform(0.0, 2.0 * np.pi)
        cosd = np.sin(lat) * np.sin(lat0) + np.cos(lat) * np.cos(lat0) * np.cos(lon - lon0)
        d = radius * np.arccos(np.clip(cosd, -1.0, 1.0))
        h += height * np.exp(-np.log(2.0) * (d / half_width) ** 2)
    return smooth_cells(mesh, h, smoothing_passes)


def build_vertical_grid(mesh: VoronoiMesh, terrain: np.ndarray, *, n_levels: int,
                        ztop: float = 30000.0) -> VerticalGridData:
    zw = stretched_levels(n_levels, ztop)
    dzw = np.diff(zw)
    zu = 0.5 * (zw[:-1] + zw[1:])
    dzu = np.zeros(n_levels)
    dzu[1:] = 0.5 * (dzw[1:] + dzw[:-1])
    rdzu = np.zeros(n_levels)
    rdzu[1:] = 1.0 / dzu[1:]
    fzm = np.zeros(n_levels)
    fzp = np.zeros(n_levels)
    # Interface k sits dzw[k-1]/2 above the centre of layer k-1 and dzw[k]/2
    # below the centre of layer k: fzm weighs layer k, fzp layer k-1.
    fzm[1:] = 0.5 * dzw[:-1] / dzu[1:]
    fzp[1:] = 0.5 * dzw[1:] / dzu[1:]
    rdzwp = np.zeros(n_levels)
    rdzwm = np.zeros(n_levels)
    rdzwp[1:] = dzw[:-1] / (dzw[1:] * (dzw[1:] + dzw[:-1]))
    rdzwm[1:] = dzw[1:] / (dzw[:-1] * (dzw[1:] + dzw[:-1]))
    # Quadratic extrapolation of layer-centre values to the ground (z = 0).
    z1, z2, z3 = zu[0], zu[1], zu[2]
    cf1 = (z2 * z3) / ((z1 - z2) * (z1 - z3))
    cf2 = (z1 * z3) / ((z2 - z1) * (z2 - z3))
    cf3 = (z1 * z2) / ((z3 - z1) * (z3 - z2))
    ah = hybrid_decay(zw, ztop)
    hx = np.broadcast_to(np.asarray(terrain, dtype=np.float64)[None, :], (n_levels + 1, terrain.size)).copy()
    zgrid = zw[:, None] + ah[:, None] * hx
    zz = dzw[:, None] / np.diff(zgrid, axis=0)
    c1, c2 = mesh.cellsOnEdge[:, 0], mesh.cellsOnEdge[:, 1]
    dz_edge = zgrid[:, c2] - zgrid[:, c1]
    zxu = 0.5 * (dz_edge[:-1] + dz_edge[1:]) / mesh.dcEdge[None, :]
    f = F32
    return VerticalGridData(
        zw=zw.astype(f), dzw=dzw.astype(f), rdzw=(1.0 / dzw).astype(f), zu=zu.astype(f),
        dzu=dzu.astype(f), rdzu=rdzu.astype(f), rdzwp=rdzwp.astype(f), rdzwm=rdzwm.astype(f),
        fzp=fzp.astype(f), fzm=fzm.astype(f), ah=ah.astype(f), hx=hx.astype(f),
        zgrid=zgrid.astype(f), zz=zz.astype(f), zxu=zxu.astype(f),
        dss=np.zeros((n_levels, terrain.size), dtype=f),
        cf1=float(cf1), cf2=float(cf2), cf3=float(cf3), first_height_level=n_levels + 1)


# ------------------------------------------------------- deriv_two / stencil


def deriv_two(mesh: VoronoiMesh, width: int = 15) -> np.ndarray:
    """Second derivative along each edge normal, fitted per cell.

    MPAS ``mpas_initialize_deriv_two`` (Skamarock and Gassmann 2011): for each
    cell, a quadratic ``a + bx + cy + dx^2 + exy + fy^2`` is least-squares
    fitted to the cell and its neighbours in local tangent-plane coordinates
    (neighbour at arc distance r along its azimuth), and the directional
    second derivative ``2(d cos^2 + e cos sin + f sin^2)`` towards each edge
    is written as weights over [cell, cellsOnCell...].  Shape
    ``(nEdges, 2, width)``; side 0 is the fit of cellsOnEdge[:,0].
    """
    deg = mesh.nEdgesOnCell
    coc, eoc = mesh.cellsOnCell, mesh.edgesOnCell
    coe = mesh.cellsOnEdge
    radius = mesh.sphere_radius
    xyz = np.stack([mesh.xCell, mesh.yCell, mesh.zCell], axis=1) / radius
    exyz = np.stack([mesh.xEdge, mesh.yEdge, mesh.zEdge], axis=1) / radius
    out = np.zeros((coe.shape[0], 2, width))
    zhat = np.array([0.0, 0.0, 1.0])
    for n in np.unique(deg):
        cells = np.flatnonzero(deg == n)
        p0 = xyz[cells]
        east = np.cross(np.broadcast_to(zhat, p0.shape), p0)
        east /= np.linalg.norm(east, axis=1, keepdims=True)
        north = np.cross(p0, east)

        def local(q: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
            dist = 2.0 * np.arcsin(np.clip(0.5 * np.linalg.norm(q - p0, axis=1), 0, 1)) * radius
            az = np.arctan2(np.einsum("ij,ij->i", q, north), np.einsum("ij,ij->i", q, east))
            return dist, az

        design = np.zeros((cells.size, n + 1, 6))
        design[:, :, 0] = 1.0
        for s in range(n):
            dist, az = local(xyz[coc[cells, s]])
            x, y = dist * np.cos(az), dist * np.sin(az)
            design[:, s + 1, 1:] = np.stack([x, y, x * x, x * y, y * y], axis=1)
        fit = np.linalg.pinv(design)            # (cells, 6, n+1)
        for s in range(n):
            edge = eoc[cells, s]
            _, az = local(exyz[edge])
            cs, sn = np.cos(az), np.sin(az)
            w = 2.0 * (cs * cs)[:, None] * fit[:, 3, :] + 2.0 * (cs * sn)[:, None] * fit[:, 4, :] \
                + 2.0 * (sn * sn)[:, None] * fit[:, 5, :]
            side = np.where(coe[edge, 0] == cells, 0, 1)
            out[edge, side, : n + 1] = w
    return out


def advection_stencil(mesh: VoronoiMesh, d2: np.ndarray, *, width: int = 25):
    """Compressed third-order flux stencil (MPAS ``atm_adv_coef_compression``).

    The stencil of edge (c1, c2) is c1, c2, then the neighbours of c1 other
    than c2, then the neighbours of c2 not yet listed (native v8.4.1
    insertion order).  ``adv_coefs`` gathers ``deriv_two`` of both sides and
    ``adv_coefs_3rd`` their difference, each scaled by ``-dc^2/12``; 1/2 is
    added for c1 and c2 and everything is multiplied by ``dvEdge``.
    """
    coe, coc, deg = mesh.cellsOnEdge, mesh.cellsOnCell, mesh.nEdgesOnCell
    n_edges = coe.shape[0]
    cells = np.full((n_edges, width), -1, dtype=np.int64)
    adv = np.zeros((n_edges, width))
    adv3 = np.zeros((n_edges, width))
    count = np.zeros(n_edges, dtype=np.int64)
    for e in range(n_edges):
        c1, c2 = int(coe[e, 0]), int(coe[e, 1])
        lst = [c1, c2]
        for s in range(deg[c1]):
            if coc[c1, s] != c2:
                lst.append(int(coc[c1, s]))
        for s in range(deg[c2]):
            nb = int(coc[c2, s])
            if nb != c1 and nb not in lst:
                lst.append(nb)
        pos = {c: i for i, c in enumerate(lst)}
        a = np.zeros(len(lst))
        a3 = np.zeros(len(lst))
        for side, sgn, cell in ((0, 1.0, c1), (1, -1.0, c2)):
            stencil = [cell] + [int(coc[cell, s]) for s in range(deg[cell])]
            for i, sc in enumerate(stencil):
                a[pos[sc]] += d2[e, side, i]
                a3[pos[sc]] += sgn * d2[e, side, i]
        dc2 = mesh.dcEdge[e] ** 2
        a = -dc2 * a / 12.0
        a3 = -dc2 * a3 / 12.0
        a[0] += 0.5
        a[1] += 0.5
        n = len(lst)
        cells[e, :n] = lst
        adv[e, :n] = mesh.dvEdge[e] * a
        adv3[e, :n] = mesh.dvEdge[e] * a3
        count[e] = n
    w = int(count.max())
    return adv[:, :w], adv3[:, :w], count, cells[:, :w]


def terrain_metrics(mesh: VoronoiMesh, vertical: VerticalGridData, d2: np.ndarray,
                    coef_3rd_order: float) -> tuple[np.ndarray, np.ndarray]:
    """MPAS init ``zb``/``zb3`` flattened to cells (third-order theta advection).

    ``z_edge = (z1+z2)/2 - dc^2 (d2z1 + d2z2)/12`` and
    ``z_edge3 = -dc^2 (d2z1 - d2z2)/12`` from the deriv_two fits of both
    cells; ``zb(k, side) = (z_edge - z_side) dv/A_side`` and
    ``zb3(k, side) = z_edge3 dv/A_side``.  The top interface row stays zero.
    """
    zgrid = np.asarray(vertical.zgrid, dtype=np.float64)
    nlev = vertical.n_vert_levels
    coe, coc, deg, eoc = mesh.cellsOnEdge, mesh.cellsOnCell, mesh.nEdgesOnCell, mesh.edgesOnCell
    n_edges = coe.shape[0]
    d2z = np.zeros((nlev, 2, n_edges))
    for side in (0, 1):
        cell = coe[:, side]
        d2z[:, side] = d2[:, side, 0][None, :] * zgrid[:nlev, cell]
        for s in range(deg.max()):
            act = deg[cell] > s
            nb = coc[cell[act], s]
            d2z[:, side, act] += d2[act, side, s + 1][None, :] * zgrid[:nlev, nb]
    dc2 = mesh.dcEdge ** 2
    z1, z2 = zgrid[:nlev, coe[:, 0]], zgrid[:nlev, coe[:, 1]]
    z_edge = 0.5 * (z1 + z2) - dc2 * (d2z[:, 0] + d2z[:, 1]) / 12.0
    z_edge3 = -dc2 * (d2z[:, 0] - d2z[:, 1]) / 12.0
    zb = np.zeros((nlev + 1, 2, n_edges))
    zb3 = np.zeros((nlev + 1, 2, n_edges))
    for side, zs in ((0, z1), (1, z2)):
        scale = mesh.dvEdge / mesh.areaCell[coe[:, side]]
        zb[:nlev, side] = (z_edge - zs) * scale
        zb3[:nlev, side] = z_edge3 * scale
    n_cells = deg.size
    zb_cell = np.zeros((nlev + 1, n_cells, eoc.shape[1]))
    zb3_cell = np.zeros_like(zb_cell)
    for s in range(eoc.shape[1]):
        act = np.flatnonzero(deg > s)
        edge = eoc[act, s]
        side = np.where(coe[edge, 0] == act, 0, 1)
        zb_cell[:, act, s] = zb[:, side, edge]
        zb3_cell[:, act, s] = coef_3rd_order * zb3[:, side, edge]
    return zb_cell.astype(F32), zb3_cell.astype(F32)


# ------------------------------------------------------------- atmosphere


def jet_profile(z: np.ndarray, z_jet: float = 10000.0, decay: float = 12000.0) -> tuple[np.ndarray, np.ndarray]:
    """Vertical shape of the jet and its derivative, continuous to first
    order: sin(pi z / (2 z_jet)) from 0 at the ground to 1 at ``z_jet``, then
    a Gaussian decay above.  The shear is largest at the ground and decreases
    upward, so the thermal-wind temperature field stays statically stable."""
    z = np.asarray(z, dtype=np.float64)
    below = z <= z_jet
    g = np.exp(-((z - z_jet) / decay) ** 2)
    arg = 0.5 * np.pi * np.minimum(z, z_jet) / z_jet
    vz = np.where(below, np.sin(arg), g)
    dvz = np.where(below, 0.5 * np.pi / z_jet * np.cos(arg), -2.0 * (z - z_jet) / decay ** 2 * g)
    return vz, dvz


def reference_stability(z: np.ndarray, n2_trop: float = 1.0e-4, n2_strat: float = 4.0e-4,
                        z_trop: float = 12000.0, width: float = 1500.0) -> np.ndarray:
    """Brunt-Vaisala frequency squared of the equatorial column: tropospheric
    below ``z_trop``, stratospheric above, joined by a tanh."""
    return n2_trop + (n2_strat - n2_trop) * 0.5 * (1.0 + np.tanh((np.asarray(z) - z_trop) / width))


def equatorial_theta(z: np.ndarray, theta0: float = 300.0) -> np.ndarray:
    """theta(z) of the equatorial (and base-state) column from its N^2(z)."""
    z = np.asarray(z, dtype=np.float64)
    fine = np.arange(0.0, float(np.max(z)) + 100.0, 10.0)
    n2 = reference_stability(fine)
    ln = np.log(theta0) + np.concatenate([[0.0], np.cumsum(0.5 * (n2[1:] + n2[:-1]) * 10.0)]) / GRAVITY
    return np.exp(np.interp(z, fine, ln))


def hydrostatic_exner(z: np.ndarray, theta: np.ndarray) -> np.ndarray:
    """Exner function of a column theta(z), 1 at z[0] = 0 (trapezoidal rule)."""
    integrand = GRAVITY / (CP * np.asarray(theta))
    steps = 0.5 * (integrand[..., 1:] + integrand[..., :-1]) * np.diff(z)
    zeros = np.zeros(integrand.shape[:-1] + (1,))
    return 1.0 - np.concatenate([zeros, np.cumsum(steps, axis=-1)], axis=-1)


def _balanced_jet(u0: float, z_jet: float, theta0: float, radius: float,
                  n_lat: int = 1441, dz: float = 50.0, ztop: float = 34000.0):
    """theta(lat, z) and exner(lat, z) in hydrostatic + gradient-wind balance.

    u = u0 sin^2(2 lat) V(z) with V(0) = 0, so the surface Exner function is
    uniform (1).  Cross-differentiating the gradient-wind balance
    dπ/dlat = -F/(cp θ), F = a f u + u^2 tan(lat), with the hydrostatic
    dπ/dz = -g/(cp θ) gives the thermal-wind equation
    g dlnθ/dlat = F dlnθ/dz - dF/dz, marched from the equator (where θ is the
    stratified column of ``equatorial_theta``) with RK2.  The result is
    checked to be statically stable everywhere.
    """
    z = np.arange(0.0, ztop + dz, dz)
    lat = np.linspace(-np.pi / 2, np.pi / 2, n_lat)
    vz, dvz = jet_profile(z, z_jet)

    def forcing(phi: float) -> tuple[np.ndarray, np.ndarray]:
        s, c = np.sin(phi), np.cos(phi)
        shape = (2.0 * s * c) ** 2
        f = 2.0 * OMEGA * s
        # F = a f u + u^2 tan: u^2 tan = u0^2 vz^2 16 s^5 c^3 (regular at poles)
        big_f = radius * f * u0 * shape * vz + (u0 * vz) ** 2 * 16.0 * s ** 5 * c ** 3
        big_fz = radius * f * u0 * shape * dvz + u0 ** 2 * 2.0 * vz * dvz * 16.0 * s ** 5 * c ** 3
        return big_f, big_fz

    def rhs(phi: float, ln_theta: np.ndarray) -> np.ndarray:
        big_f, big_fz = forcing(phi)
        lz = np.gradient(ln_theta, dz)
        return (big_f * lz - big_fz) / GRAVITY

    eq = n_lat // 2
    ln_t = np.zeros((n_lat, z.size))
    ln_t[eq] = np.log(equatorial_theta(z, theta0))
    for direction in (1, -1):
        cur = ln_t[eq].copy()
        j = eq
        while 0 <= j + direction < n_lat:
            phi, dphi = lat[j], lat[j + direction] - lat[j]
            k1 = rhs(phi, cur)
            k2 = rhs(phi + dphi, cur + dphi * k1)
            cur = cur + 0.5 * dphi * (k1 + k2)
            j += direction
            ln_t[j] = cur
    theta = np.exp(ln_t)
    exner = hydrostatic_exner(z, theta)
    n2 = GRAVITY * np.gradient(ln_t, z, axis=1)
    if n2.min() <= 0.0:
        raise RuntimeError(f"balanced jet is statically unstable (min N^2 = {n2.min():.3e})")
    return lat, z, theta, exner


def _bilinear(lat_grid, z_grid, field, lat, z):
    fi = np.clip((lat - lat_grid[0]) / (lat_grid[1] - lat_grid[0]), 0, lat_grid.size - 1.000001)
    fj = np.clip((z - z_grid[0]) / (z_grid[1] - z_grid[0]), 0, z_grid.size - 1.000001)
    i, j = np.floor(fi).astype(np.int64), np.floor(fj).astype(np.int64)
    a, b = fi - i, fj - j
    return ((1 - a) * (1 - b) * field[i, j] + a * (1 - b) * field[i + 1, j]
            + (1 - a) * b * field[i, j + 1] + a * b * field[i + 1, j + 1])


def qsat(temperature: np.ndarray, pressure: np.ndarray) -> np.ndarray:
    """Saturation mixing ratio over liquid (Bolton 1980)."""
    es = 611.2 * np.exp(17.67 * (temperature - 273.15) / (temperature - 29.65))
    es = np.minimum(es, 0.5 * pressure)
    return 0.622 * es / (pressure - 0.378 * es)


def _libm_sinf():
    import ctypes
    import ctypes.util

    name = ctypes.util.find_library("m")
    if name is None:
        return None
    fn = ctypes.CDLL(name).sinf
    fn.argtypes = [ctypes.c_float]
    fn.restype = ctypes.c_float
    return fn


def vertical_velocity_damping(zgrid: np.ndarray, xnutr: float, zd: float) -> np.ndarray:
    """Implicit w-damping coefficients dss [L][C] of MPAS-A v8.4.1
    (``hexcore/damping_v841.py:23`` build_v841_vertical_velocity_damping,
    float32 lane): above the layer midpoint height zd, dss = xnutr *
    sin^2(pi/2 (z_mid - zd) / (z_top - zd)) with every operation in float32
    and the sine from the C library's sinf, as the reference evaluates it."""
    h = np.asarray(zgrid, dtype=F32)
    nlev, ncell = h.shape[0] - 1, h.shape[1]
    dss = np.zeros((nlev, ncell), dtype=F32)
    x = F32(xnutr)
    if x == F32(0.0):
        return dss
    half = F32(0.5)
    pi = np.arccos(F32(-1.0))
    start = F32(zd)
    midpoint = half * (h[:-1] + h[1:])
    active = midpoint > start
    denominator = np.broadcast_to(h[-1] - start, midpoint.shape)
    phase = (half * pi) * (midpoint[active] - start) / denominator[active]
    sinf = _libm_sinf()
    if sinf is None:
        raise RuntimeError("the damping profile needs the C library's sinf")
    sine = np.array([sinf(float(p)) for p in phase], dtype=F32)
    dss[active] = x * (sine * sine)
    return dss


def build_case(mesh: VoronoiMesh, *, n_levels: int = 55, ztop: float = 30000.0,
               seed: int = 0, n_condensates: int = 0, jet_speed: float = 35.0,
               perturbation: float = 1.0, coef_3rd_order: float = 0.25,
               theta_noise: float = 0.0, theta_noise_rings: int = 3,
               terrain: bool = True, like: DycoreCase | None = None) -> DycoreCase:
    """The balanced-jet dry state with qv (+ condensates) on ``mesh``.

    ``like``: an earlier case on the same mesh whose terrain, vertical grid,
    terrain metrics and advection stencil are reused (ensemble members that
    differ only in their state); ``seed`` then draws only the state's noise
    and tracer blobs."""
    rng = np.random.default_rng(seed + 1)
    radius = mesh.sphere_radius
    if like is not None:
        if like.mesh is not mesh or like.vertical.zz.shape[0] != n_levels or like.coef_3rd_order != coef_3rd_order:
            raise ValueError("like= must be a case on the same mesh, levels and coef_3rd_order")
        vertical = like.vertical
        zb_cell, zb3_cell = like.zb_cell, like.zb3_cell
        adv, adv3, n_adv, adv_cells = (like.adv_coefs, like.adv_coefs_3rd, like.n_adv_cells_for_edge,
                                       like.adv_cells_for_edge)
    else:
        ter = gaussian_terrain(mesh, seed=seed) if terrain else np.zeros(mesh.n_cells)
        vertical = build_vertical_grid(mesh, ter, n_levels=n_levels, ztop=ztop)
        d2 = deriv_two(mesh)
        zb_cell, zb3_cell = terrain_metrics(mesh, vertical, d2, coef_3rd_order)
        adv, adv3, n_adv, adv_cells = advection_stencil(mesh, d2)

    theta0 = 300.0
    lat_g, z_g, theta_g, exner_g = _balanced_jet(jet_speed, 10000.0, theta0, radius)
    zgrid = np.asarray(vertical.zgrid, dtype=np.float64)
    z_mid = 0.5 * (zgrid[:-1] + zgrid[1:])
    lat_c = np.broadcast_to(mesh.latCell[None, :], z_mid.shape)
    theta = _bilinear(lat_g, z_g, theta_g, lat_c, z_mid)
    exner = _bilinear(lat_g, z_g, exner_g, lat_c, z_mid)
    if theta_noise > 0.0:
        noise = rng.standard_normal(z_mid.shape) * theta_noise
        for k in range(n_levels):
            sm = smooth_cells(mesh, noise[k], theta_noise_rings)
            noise[k] = sm * (theta_noise / max(sm.std(), 1e-30))
        theta = theta + noise
    pressure = P0 * exner ** (CP / RGAS)
    rho_dry = pressure / (RGAS * theta * exner)
    zz = np.asarray(vertical.zz, dtype=np.float64)

    # Hydrostatic base state: the equatorial column, interpolated in height.
    zb_fine = np.arange(0.0, 34000.0 + 10.0, 10.0)
    thb_fine = equatorial_theta(zb_fine, theta0)
    exb_fine = hydrostatic_exner(zb_fine, thb_fine)
    theta_b = np.interp(z_mid, zb_fine, thb_fine)
    exner_b = np.interp(z_mid, zb_fine, exb_fine)
    pressure_b = P0 * exner_b ** (CP / RGAS)
    rho_b = pressure_b / (RGAS * theta_b * exner_b)

    rho_zz = (rho_dry / zz).astype(F32)
    rho_theta = (rho_dry / zz * theta).astype(F32)
    rho_base = (rho_b / zz).astype(F32)
    rho_theta_base = (rho_b / zz * theta_b).astype(F32)

    # Winds at edges: balanced zonal jet + Gaussian perturbation at (20E, 40N).
    c1, c2 = mesh.cellsOnEdge[:, 0], mesh.cellsOnEdge[:, 1]
    z_edge = 0.5 * (z_mid[:, c1] + z_mid[:, c2])
    lat_e, lon_e = mesh.latEdge, mesh.lonEdge
    vz, _ = jet_profile(z_edge)
    u_east = jet_speed * np.sin(2.0 * lat_e)[None, :] ** 2 * vz
    lat0, lon0 = np.deg2rad(40.0), np.deg2rad(20.0)
    cosd = np.sin(lat_e) * np.sin(lat0) + np.cos(lat_e) * np.cos(lat0) * np.cos(lon_e - lon0)
    dist = np.arccos(np.clip(cosd, -1.0, 1.0))
    u_east = u_east + perturbation * np.exp(-(dist / 0.1) ** 2)[None, :]
    u_normal = u_east * np.cos(mesh.angleEdge)[None, :]
    rho_edge = 0.5 * (rho_zz[:, c1].astype(np.float64) + rho_zz[:, c2].astype(np.float64))
    rho_u = (rho_edge * u_normal).astype(F32)
    rho_w = np.zeros((n_levels + 1, mesh.n_cells), dtype=F32)

    temperature = theta * exner
    qv = 0.8 * qsat(temperature, pressure) * np.exp(-z_mid / 3000.0)
    scalars = [qv]
    names = ["qv"]
    for i, name in enumerate(("qc", "qr", "qi", "qs", "qg")[:n_condensates]):
        blob = np.zeros_like(qv)
        cols = rng.choice(mesh.n_cells, size=max(1, int(0.05 * mesh.n_cells)), replace=False)
        amp = np.exp(np.log(1.0e-5) + rng.standard_normal(cols.size))
        zc = z_mid[:, cols]
        shape = np.where((zc >= 2000.0) & (zc <= 8000.0), 1.0, 0.0)
        shape *= np.sin(np.pi * np.clip((zc - 2000.0) / 6000.0, 0, 1)) ** 2
        blob[:, cols] = amp[None, :] * shape
        scalars.append(blob)
        names.append(name)
    scalars_arr = np.stack(scalars).astype(F32)
    return DycoreCase(
        mesh=mesh, vertical=vertical, zb_cell=zb_cell, zb3_cell=zb3_cell,
        rho_base=rho_base, rho_theta_base=rho_theta_base,
        pressure_base=pressure_b.astype(F32), exner_base=exner_b.astype(F32),
        rho=rho_zz, rho_theta=rho_theta, rho_u=rho_u, rho_w=rho_w,
        scalars=scalars_arr, scalar_names=tuple(names),
        adv_coefs=adv, adv_coefs_3rd=adv3, n_adv_cells_for_edge=n_adv,
        adv_cells_for_edge=adv_cells,
        u_init=np.zeros(n_levels, dtype=F32), v_init=np.zeros(n_levels, dtype=F32),
        coef_3rd_order=coef_3rd_order)


def case_arrays(case: DycoreCase) -> dict[str, Any]:
    """Flat dict of every array of a case (mesh fields prefixed ``mesh.``)."""
    out: dict[str, Any] = {}
    for k, v in case.mesh.arrays.items():
        out["mesh." + k] = v
    vg = case.vertical
    for k in vg.__dataclass_fields__:
        out["vertical." + k] = getattr(vg, k)
    for k in ("zb_cell", "zb3_cell", "rho_base", "rho_theta_base", "pressure_base",
              "exner_base", "rho", "rho_theta", "rho_u", "rho_w", "scalars",
              "adv_coefs", "adv_coefs_3rd", "n_adv_cells_for_edge", "adv_cells_for_edge",
              "u_init", "v_init"):
        out[k] = getattr(case, k)
    out["coef_3rd_order"] = case.coef_3rd_order
    out["scalar_names"] = np.array(case.scalar_names)
    return out


def arrays_case(arr: dict[str, Any]) -> DycoreCase:
    """The case of a flat array dict (inverse of ``case_arrays``)."""
    mesh = VoronoiMesh(arrays={k[5:]: v for k, v in arr.items() if k.startswith("mesh.")})
    vfields = {k[9:]: v for k, v in arr.items() if k.startswith("vertical.")}
    for k in ("cf1", "cf2", "cf3"):
        vfields[k] = float(vfields[k])
    vfields["first_height_level"] = int(vfields["first_height_level"])
    names = arr.get("scalar_names")
    names = tuple(str(n) for n in np.asarray(names).reshape(-1)) if names is not None else \
        tuple(f"q{i}" for i in range(np.asarray(arr["scalars"]).shape[0]))
    return DycoreCase(mesh=mesh, vertical=VerticalGridData(**vfields), scalar_names=names,
                      coef_3rd_order=float(arr.get("coef_3rd_order", 0.25)),
                      **{k: arr[k] for k in ("zb_cell", "zb3_cell", "rho_base", "rho_theta_base", "pressure_base",
                                             "exner_base", "rho", "rho_theta", "rho_u", "rho_w", "scalars",
                                             "adv_coefs", "adv_coefs_3rd", "n_adv_cells_for_edge",
                                             "adv_cells_for_edge", "u_init", "v_init")})
