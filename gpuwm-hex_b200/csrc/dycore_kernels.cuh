// Dycore kernels and the step orchestration.  This file is compiled twice,
// inside namespace hexdyn_strict (nvcc -fmad=false: every FP32 operation is
// rounded on its own, in the reference's order, so results are bit-identical
// to the NumPy authority) and inside hexdyn_fast (-fmad=true: the same
// arithmetic with multiply-adds contracted).
//
// Operation order follows the reference CPU authority line by line
// (hexcore/ = tree/src/hexcore/ of gpuwm-hex 0.5.0); each kernel names the
// function it restates.  Expressions are written in the reference's textual
// order: C evaluates a*b*c as (a*b)*c and a-b-c as (a-b)-c exactly as NumPy
// does, every literal is float, and reductions run over neighbour slots in
// slot order inside one thread.
//
// Thread layout of the level-parallel kernels: blockDim = (S, EPB); x is the
// level (0..S-1), y the entity within the block; the S threads of an entity
// are consecutive, so a warp reads 32 consecutive words of one column.

#include "dycore_geo.cuh"
#include "hexdyn_ctx.h"
#include "powf_gnu.cuh"

#define HEX_LEVEL_PARALLEL(n)                         \
  const int k = threadIdx.x;                          \
  const int ent = blockIdx.x * blockDim.y + threadIdx.y; \
  if (ent >= (n)) return;

__device__ __forceinline__ float pos0(float x) { return x > 0.0f ? x : 0.0f; }
__device__ __forceinline__ float neg0(float x) { return x < 0.0f ? x : 0.0f; }
// Python min(a, b) / max(a, b): a unless b is strictly smaller / larger.
__device__ __forceinline__ float pymin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float pymax(float a, float b) { return b > a ? b : a; }

__device__ __forceinline__ float flux4f(float qm2, float qm1, float q0, float qp1, float vel) {
  return vel * (7.0f * (q0 + qm1) - (qp1 + qm2)) / 12.0f;
}
// hexcore/dynamics.py:71 flux3 and hexcore/transport.py:440 (both add the
// coefficient term).
__device__ __forceinline__ float flux3f(float qm2, float qm1, float q0, float qp1, float vel, float coef) {
  return flux4f(qm2, qm1, q0, qp1, vel) + coef * fabsf(vel) * ((qp1 - qm2) - 3.0f * (q0 - qm1)) / 12.0f;
}

// ------------------------------------------------------------ recovery

// hexcore/terrain.py:491 recover_velocities, w at interface k of cell c.
// rho(k) is evaluated through the functor so that callers may recompute the
// candidate density instead of reading a buffer being written.
template <class RhoF>
__device__ __forceinline__ float recover_w_at(const HexGeo& g, int c, int k, RhoF rho,
                                              const float* __restrict__ ru, float rw_k) {
  const int S = g.S, L = g.L;
  if (k == 0) {
    float acc = 0.0f;
    const int n = g.deg[c];
    for (int s = 0; s < n; ++s) {
      const int e = g.eoc[c * g.maxE + s];
      const float sign = g.csign[c * g.maxE + s];
      const float flux = g.cf1 * ru[e * S + 0] + g.cf2 * ru[e * S + 1] + g.cf3 * ru[e * S + 2];
      const int zi = (c * g.maxE + s) * S;
      acc = acc + sign * (g.zb[zi] + copysignf(1.0f, flux) * g.zb3[zi]) * flux;
    }
    const float bottom = g.cf1 * rho(0) + g.cf2 * rho(1) + g.cf3 * rho(2);
    return acc / bottom;
  }
  if (k >= L) return 0.0f;
  const float izz = g.fzm[k] * g.zz[c * S + k] + g.fzp[k] * g.zz[c * S + k - 1];
  float acc = rw_k / izz;
  const int n = g.deg[c];
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float sign = g.csign[c * g.maxE + s];
    const float flux = g.fzm[k] * ru[e * S + k] + g.fzp[k] * ru[e * S + k - 1];
    const int zi = (c * g.maxE + s) * S + k;
    acc = acc + sign * (g.zb[zi] + copysignf(1.0f, flux) * g.zb3[zi]) * flux;
  }
  const float irho = g.fzm[k] * rho(k) + g.fzp[k] * rho(k - 1);
  return acc / irho;
}

// hexcore/driver.py:866 _normal_velocity (u = 2 ru / (rho1 + rho2)).
__global__ void k_recover_u(HexGeo g, const float* __restrict__ rho, const float* __restrict__ ru,
                            float* __restrict__ u) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
  u[e * S + k] = 2.0f * ru[e * S + k] / (rho[c0 * S + k] + rho[c1 * S + k]);
}

// hexcore/driver.py:2655 _rebuild_saved_diagnostics (cell part) with
// hexcore/driver.py:790 _pressure_exner and :819 _pressure_perturbation.
__global__ void k_rebuild_cell(HexGeo g, const float* __restrict__ rho, const float* __restrict__ rt,
                               const float* __restrict__ ru, const float* __restrict__ rw, HexSide side,
                               int* flag) {
  HEX_LEVEL_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  if (k < L) {
    const int i = c * S + k;
    const float theta = rt[i] / rho[i];
    int bad = 0;
    const float arg = g.zz[i] * g.r_over_p0 * rt[i];
    const float exner = hexdyn_powf::powf_gnu(arg, g.kappa, &bad);
    if (bad) atomicOr(flag, HEX_FLAG_POWF);
    const float rp = rho[i] - g.rho_base[i];
    const float rtp = rt[i] - g.rtheta_base[i];
    side.theta_m[i] = theta;
    side.exner[i] = exner;
    side.rho_p[i] = rp;
    side.rtheta_p[i] = rtp;
    side.pressure_p[i] = g.zz[i] * g.rgas * (exner * rtp + g.rtheta_base[i] * (exner - g.exner_base[i]));
  }
  if (k <= L) {
    auto rho_at = [&](int kk) { return rho[c * S + kk]; };
    side.w[c * S + k] = recover_w_at(g, c, k, rho_at, ru, rw[c * S + k]);
  }
}

// ---------------------------------------------------------- diagnostics
// hexcore/diagnostics.py:95 compute_solve_diagnostics, v8.4.1 stored inverses.

__device__ __forceinline__ float ke_edge_at(const HexGeo& g, const float* __restrict__ u, int e, int k) {
  const float ue = u[e * g.S + k];
  return g.dc[e] * g.dv[e] * (ue * ue);
}

__global__ void k_diag_vertex(HexGeo g, const float* __restrict__ u, float* __restrict__ pv_vertex,
                              float* __restrict__ ke_vertex) {
  HEX_LEVEL_PARALLEL(g.nV)
  if (k >= g.L) return;
  const int v = ent, S = g.S;
  float vort = 0.0f;
  for (int s = 0; s < 3; ++s) {
    const int e = g.eov[3 * v + s];
    vort = vort + g.vsign[3 * v + s] * g.dc[e] * u[e * S + k];
  }
  vort = vort * g.inv_area_tri[v];
  pv_vertex[v * S + k] = g.f_vertex[v] + vort;
  const float r = 0.25f * g.inv_area_tri[v];
  const float ke0 = ke_edge_at(g, u, g.eov[3 * v], k);
  const float ke1 = ke_edge_at(g, u, g.eov[3 * v + 1], k);
  const float ke2 = ke_edge_at(g, u, g.eov[3 * v + 2], k);
  ke_vertex[v * S + k] = (ke0 + ke1 + ke2) * r;
}

__global__ void k_diag_cell(HexGeo g, const float* __restrict__ u, const float* __restrict__ pv_vertex,
                            const float* __restrict__ ke_vertex, float* __restrict__ ke_out,
                            float* __restrict__ pv_cell) {
  HEX_LEVEL_PARALLEL(g.nC)
  if (k >= g.L) return;
  const int c = ent, S = g.S;
  const int n = g.deg[c];
  const float ia = g.inv_area[c];
  float ke = 0.0f;
  for (int s = 0; s < n; ++s) ke = ke + 0.25f * ke_edge_at(g, u, g.eoc[c * g.maxE + s], k);
  ke = ke * ia;
  ke = ke * 0.625f;
  for (int s = 0; s < n; ++s) {
    const int vtx = g.voc[c * g.maxE + s];
    const float corr = (1.0f - 0.625f) * g.kite[3 * vtx + g.kite_slot[c * g.maxE + s]] * ke_vertex[vtx * S + k];
    ke = ke + corr * ia;
  }
  ke_out[c * S + k] = ke;
  if (g.apvm_on) {
    float pvc = 0.0f;
    for (int s = 0; s < n; ++s) {
      const int vtx = g.voc[c * g.maxE + s];
      const float contrib = g.kite[3 * vtx + g.kite_slot[c * g.maxE + s]] * pv_vertex[vtx * S + k];
      pvc = pvc + contrib * ia;
    }
    pv_cell[c * S + k] = pvc;
  }
}

__global__ void k_diag_edge(HexGeo g, const float* __restrict__ u, const float* __restrict__ pv_vertex,
                            const float* __restrict__ pv_cell, float* __restrict__ v, float* __restrict__ pv_edge,
                            int recompute_v) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  float vt;
  if (recompute_v) {
    vt = 0.0f;
    const int n = g.neoe[e];
    for (int s = 0; s < n; ++s) vt = vt + g.weights[e * g.maxE2 + s] * u[g.eoe[e * g.maxE2 + s] * S + k];
    v[e * S + k] = vt;
  } else {
    vt = v[e * S + k];
  }
  const int v0 = g.voe[2 * e], v1 = g.voe[2 * e + 1];
  float pve = 0.5f * (pv_vertex[v0 * S + k] + pv_vertex[v1 * S + k]);
  if (g.apvm_on) {
    const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
    const float gpt = (pv_vertex[v1 * S + k] - pv_vertex[v0 * S + k]) * g.inv_dv[e];
    const float gpn = (pv_cell[c1 * S + k] - pv_cell[c0 * S + k]) * g.inv_dc[e];
    pve = pve - g.apvm_scale * (vt * gpt + u[e * S + k] * gpn);
  }
  pv_edge[e * S + k] = pve;
}

// --------------------------------------------------- moist coefficients
// hexcore/regional_v841.py:1180 compute_moist_coefficients, every scalar.

__global__ void k_moist_cell(HexGeo g, const float* __restrict__ q, int nT, float* __restrict__ qtot,
                             float* __restrict__ cqw) {
  HEX_LEVEL_PARALLEL(g.nC)
  if (k >= g.L) return;
  const int c = ent, S = g.S;
  auto qt = [&](int kk) {
    float acc = 0.0f;
    for (int t = 0; t < nT; ++t) acc = acc + q[((size_t)t * g.nC + c) * S + kk];
    return acc;
  };
  const float here = qt(k);
  qtot[c * S + k] = here;
  cqw[c * S + k] = k == 0 ? 1.0f : 1.0f / (1.0f + 0.5f * (here + qt(k - 1)));
}

__global__ void k_moist_edge(HexGeo g, const float* __restrict__ q, int nT, float* __restrict__ cqu) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
  float acc = 0.0f;
  for (int t = 0; t < nT; ++t) {
    const float* qt = q + (size_t)t * g.nC * S;
    acc = acc + 0.5f * (qt[c0 * S + k] + qt[c1 * S + k]);
  }
  cqu[e * S + k] = 1.0f / (1.0f + acc);
}

// --------------------------------------------------------- Euler terms

__device__ __forceinline__ float dpdz_at(const HexGeo& g, const float* __restrict__ rp,
                                         const float* __restrict__ qtot, int i) {
  if (!g.moist) return -g.g * rp[i];
  // atm_compute_dyn_tend_work: dpdz = -gravity*(rb*qtot + rr_save*(1+qtot))
  return -g.g * (g.rho_base[i] * qtot[i] + rp[i] * (1.0f + qtot[i]));
}

// hexcore/dynamics.py:188 pressure_gradient_euler_tendency.
__global__ void k_euler_edge(HexGeo g, const float* __restrict__ pp, const float* __restrict__ rp,
                             const float* __restrict__ qtot, const float* __restrict__ cqu,
                             float* __restrict__ euler_ru) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  const int i0 = g.coe[2 * e] * S + k, i1 = g.coe[2 * e + 1] * S + k;
  const float d0 = dpdz_at(g, rp, qtot, i0), d1 = dpdz_at(g, rp, qtot, i1);
  euler_ru[e * S + k] = -cqu[e * S + k] * ((pp[i1] - pp[i0]) * g.inv_dc[e] / (0.5f * (g.zz[i1] + g.zz[i0]))
                                            - 0.5f * g.zxu[e * S + k] * (d0 + d1));
}

// hexcore/dynamics.py:86 mass_flux_divergence (stored inverse area).
__device__ __forceinline__ float mass_flux_div(const HexGeo& g, const float* __restrict__ ru, int c, int k) {
  float acc = 0.0f;
  const int n = g.deg[c];
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    acc = acc + g.csign[c * g.maxE + s] * g.dv[e] * ru[e * g.S + k];
  }
  return acc * g.inv_area[c];
}

// hexcore/dynamics.py:122 density_tendency and hexcore/driver.py:2804 Euler w.
__global__ void k_euler_cell(HexGeo g, const float* __restrict__ ru, const float* __restrict__ rw,
                             const float* __restrict__ pp, const float* __restrict__ rp,
                             const float* __restrict__ qtot, const float* __restrict__ cqw,
                             float* __restrict__ tend_rho, float* __restrict__ euler_rw) {
  HEX_LEVEL_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  const int i = c * S + k;
  if (k < L) tend_rho[i] = -mass_flux_div(g, ru, c, k) - g.rdzw[k] * (rw[i + 1] - rw[i]);
  if (k <= L) {
    float out = 0.0f;
    if (k >= 1 && k < L) {
      const float inner = g.rdzu[k] * (pp[i] - pp[i - 1])
                          - (g.fzm[k] * dpdz_at(g, rp, qtot, i) + g.fzp[k] * dpdz_at(g, rp, qtot, i - 1));
      out = g.moist ? -(cqw[i] * inner) : -inner;
    }
    euler_rw[i] = out;
  }
}

// ------------------------------------------------- stage tendencies

__global__ void k_hdiv(HexGeo g, const float* __restrict__ ru, float* __restrict__ hdiv) {
  HEX_LEVEL_PARALLEL(g.nC)
  if (k >= g.L) return;
  hdiv[ent * g.S + k] = mass_flux_div(g, ru, ent, k);
}

// Third-order edge values of theta_m (levels) and w (interfaces): the
// per-edge stencil sums of hexcore/driver.py:1023-1034 and :1159-1172.
__global__ void k_edge_adv(HexGeo g, const float* __restrict__ ru, const float* __restrict__ theta,
                           const float* __restrict__ w, float* __restrict__ edge_theta,
                           float* __restrict__ edge_w) {
  HEX_LEVEL_PARALLEL(g.nE)
  const int e = ent, S = g.S, L = g.L;
  const int n = g.n_adv[e];
  const int* cells = g.adv_cells + (size_t)e * g.advW;
  const float* a1 = g.adv + (size_t)e * g.advW;
  const float* a3 = g.adv3 + (size_t)e * g.advW;
  if (k < L) {
    const float sgn = copysignf(1.0f, ru[e * S + k]);
    float acc = 0.0f;
    for (int s = 0; s < n; ++s) acc = acc + (a1[s] + g.coef3 * sgn * a3[s]) * theta[cells[s] * S + k];
    edge_theta[e * S + k] = acc;
  }
  if (k >= 1 && k < L) {
    const float rui = g.fzm[k] * ru[e * S + k] + g.fzp[k] * ru[e * S + k - 1];
    const float sgn = copysignf(1.0f, rui);
    float acc = 0.0f;
    for (int s = 0; s < n; ++s) acc = acc + (a1[s] + g.coef3 * sgn * a3[s]) * w[cells[s] * S + k];
    edge_w[e * S + k] = acc;
  }
}

// hexcore/dynamics.py:227 vertical_transport_u (wduz at interface j).
__device__ __forceinline__ float wduz_at(const HexGeo& g, const float* __restrict__ u,
                                         const float* __restrict__ rw, int e, int c0, int c1, int j) {
  const int S = g.S, L = g.L;
  if (j <= 0 || j >= L) return 0.0f;
  const float rwe = 0.5f * (rw[c0 * S + j] + rw[c1 * S + j]);
  const float* ue = u + e * S;
  if (j == 1 || j == L - 1) return rwe * (g.fzm[j] * ue[j] + g.fzp[j] * ue[j - 1]);
  return flux3f(ue[j - 2], ue[j - 1], ue[j], ue[j + 1], rwe, 1.0f);
}

// tend_ru: vertical transport + hexcore/dynamics_v841.py:121 momentum + saved Euler.
__global__ void k_tend_u(HexGeo g, const float* __restrict__ u, const float* __restrict__ rw,
                         const float* __restrict__ rho, const float* __restrict__ pv_edge,
                         const float* __restrict__ ke, const float* __restrict__ hdiv,
                         const float* __restrict__ euler_ru, float* __restrict__ tend_ru) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
  const float tv = -g.rdzw[k] * (wduz_at(g, u, rw, e, c0, c1, k + 1) - wduz_at(g, u, rw, e, c0, c1, k));
  const int n = g.neoe[e];
  const float pve = pv_edge[e * S + k];
  float q = 0.0f;
  for (int s = 0; s < n; ++s) {
    const int nb = g.eoe[e * g.maxE2 + s];
    const float work_pv = 0.5f * (pve + pv_edge[nb * S + k]);
    q = q + g.weights[e * g.maxE2 + s] * u[nb * S + k] * work_pv;
  }
  for (int s = 0; s < n; ++s) {
    const int nb = g.eoe[e * g.maxE2 + s];
    const float ref_u = g.u_init[k] * g.cos_angle[nb] - g.v_init[k] * g.sin_angle[nb];
    q = q - g.weights[e * g.maxE2 + s] * ref_u * g.f_edge[e];
  }
  const float rho_edge = 0.5f * (rho[c0 * S + k] + rho[c1 * S + k]);
  float horizontal = rho_edge * (q - (ke[c1 * S + k] - ke[c0 * S + k]) * g.inv_dc[e]);
  horizontal = tv + horizontal;
  const float res = horizontal - u[e * S + k] * 0.5f * (hdiv[c0 * S + k] + hdiv[c1 * S + k]);
  tend_ru[e * S + k] = res + euler_ru[e * S + k];
}

// hexcore/driver.py:933 theta vertical flux at interface j.
__device__ __forceinline__ float vflux_theta(const HexGeo& g, const float* __restrict__ th,
                                             const float* __restrict__ ths, const float* __restrict__ rw,
                                             const float* __restrict__ rws, int j) {
  const int L = g.L;
  if (j <= 0 || j >= L) return 0.0f;
  if (j == 1) {
    float vf = rw[j] * (g.fzm[j] * th[j] + g.fzp[j] * th[j - 1]);
    return vf + (rws[j] - rw[j]) * (g.fzm[j] * ths[j] + g.fzp[j] * ths[j - 1]);
  }
  if (j == L - 1) return rws[j] * (g.fzm[j] * th[j] + g.fzp[j] * th[j - 1]);
  const float vf = flux3f(th[j - 2], th[j - 1], th[j], th[j + 1], rw[j], g.coef3);
  return vf + (rws[j] - rw[j]) * (g.fzm[j] * ths[j] + g.fzp[j] * ths[j - 1]);
}

// hexcore/driver.py:1081 w vertical flux at interface j.
__device__ __forceinline__ float vflux_w(const HexGeo& g, const float* __restrict__ w,
                                         const float* __restrict__ rw, int j) {
  const int L = g.L;
  if (j <= 0 || j >= L) return 0.0f;
  if (j == 1 || j == L - 1) return 0.25f * (rw[j] + rw[j - 1]) * (w[j] + w[j - 1]);
  return flux3f(w[j - 2], w[j - 1], w[j], w[j + 1], 0.5f * (rw[j] + rw[j - 1]), 1.0f);
}

// tend_rt (hexcore/driver.py:933), tend_rw (:1081) + Euler w, then
// hexcore/acoustic.py:246 convert_w_tendency_to_omega.
__global__ void k_tend_cell(HexGeo g, const float* __restrict__ ru, const float* __restrict__ ru_s,
                            const float* __restrict__ rw, const float* __restrict__ rws,
                            const float* __restrict__ theta, const float* __restrict__ theta_s,
                            const float* __restrict__ w, const float* __restrict__ edge_theta,
                            const float* __restrict__ edge_w, const float* __restrict__ euler_rw,
                            const float* __restrict__ tend_ru, float* __restrict__ tend_rt,
                            float* __restrict__ tend_rw, int rk_step) {
  HEX_LEVEL_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  const int n = g.deg[c];
  const int i = c * S + k;
  const float ia = g.inv_area[c];
  const int* eoc = g.eoc + c * g.maxE;
  const float* cs = g.csign + c * g.maxE;
  if (k < L) {
    float res = 0.0f;
    for (int s = 0; s < n; ++s) {
      const int e = eoc[s];
      res = res - cs[s] * ru[e * S + k] * edge_theta[e * S + k];
    }
    if (rk_step > 1) {
      for (int s = 0; s < n; ++s) {
        const int e = eoc[s];
        const int e0 = g.coe[2 * e], e1 = g.coe[2 * e + 1];
        const float corr = cs[s] * g.dv[e] * (ru_s[e * S + k] - ru[e * S + k]) * 0.5f
                           * (theta_s[e1 * S + k] + theta_s[e0 * S + k]);
        res = res - corr;
      }
    }
    res = res * ia;
    const float* th = theta + c * S;
    const float* ths = theta_s + c * S;
    const float* rwc = rw + c * S;
    const float* rwsc = rws + c * S;
    tend_rt[i] = res - g.rdzw[k] * (vflux_theta(g, th, ths, rwc, rwsc, k + 1) - vflux_theta(g, th, ths, rwc, rwsc, k));
  }
  if (k <= L) {
    float out = 0.0f;
    if (k >= 1 && k < L) {
      float hres = 0.0f;
      for (int s = 0; s < n; ++s) {
        const int e = eoc[s];
        const float rui = g.fzm[k] * ru[e * S + k] + g.fzp[k] * ru[e * S + k - 1];
        hres = hres - cs[s] * rui * edge_w[e * S + k];
      }
      hres = hres * ia;
      const float* wc = w + c * S;
      const float* rwc = rw + c * S;
      float res = hres - g.rdzu[k] * (vflux_w(g, wc, rwc, k + 1) - vflux_w(g, wc, rwc, k));
      out = res + euler_rw[i];
      for (int s = 0; s < n; ++s) {
        const int e = eoc[s];
        const float flux = cs[s] * (g.fzm[k] * tend_ru[e * S + k] + g.fzp[k] * tend_ru[e * S + k - 1]);
        const float up = copysignf(1.0f, tend_ru[e * S + k]);
        const int zi = (c * g.maxE + s) * S + k;
        out = out - (g.zb[zi] + up * g.zb3[zi]) * flux;
      }
      out = out * (g.fzm[k] * g.zz[i] + g.fzp[k] * g.zz[i - 1]);
    } else {
      out = 0.0f + euler_rw[i];
    }
    tend_rw[i] = out;
  }
}

// -------------------------------------------------- vertical coefficients
// hexcore/acoustic_v841.py:81 compute_vertical_implicit_coefficients_v841.
__global__ void k_vcoef(HexGeo g, float dts2, const float* __restrict__ exner,
                        const float* __restrict__ theta, const float* __restrict__ rtp,
                        const float* __restrict__ cqw, const float* __restrict__ qtot, float* __restrict__ cofwr,
                        float* __restrict__ cofwz, float* __restrict__ coftz, float* __restrict__ cofwt,
                        float* __restrict__ a_tri, float* __restrict__ alpha_tri, float* __restrict__ gamma_tri,
                        int* flag) {
  extern __shared__ float sm[];
  const int k = threadIdx.x;
  const int S = g.S, L = g.L;
  const int c = blockIdx.x * blockDim.y + threadIdx.y;
  const bool live = c < g.nC;
  float* s_wr = sm + threadIdx.y * S * 7;
  float* s_wz = s_wr + S;
  float* s_tz = s_wz + S;
  float* s_wt = s_tz + S;
  float* s_a = s_wt + S;
  float* s_b = s_a + S;
  float* s_c = s_b + S;
  const int i = c * S + k;
  if (live) {
    float wr = 0.0f, wz = 0.0f, tz = 0.0f, wt = 0.0f;
    if (k >= 1 && k < L) {
      const float izz = g.fzm[k] * g.zz[i] + g.fzp[k] * g.zz[i - 1];
      wr = 0.5f * g.g * izz;
      wz = g.c2 * izz * g.rdzu[k] * cqw[i] * (g.fzm[k] * exner[i] + g.fzp[k] * exner[i - 1]);
      tz = g.fzm[k] * theta[i] + g.fzp[k] * theta[i - 1];
    }
    if (k < L) {
      wt = 0.5f * g.rcv * g.zz[i] * g.g * g.rho_base[i] / (1.0f + qtot[i]) * exner[i]
           / ((g.rtheta_base[i] + rtp[i]) * g.exner_base[i]);
    }
    s_wr[k] = wr;
    s_wz[k] = wz;
    s_tz[k] = tz;
    s_wt[k] = wt;
  }
  __syncthreads();
  if (live) {
    float a = 0.0f, b = 0.0f, cc = 0.0f;
    if (k == 0) b = 1.0f;
    if (k >= 1 && k < L) {
      const float* rdzw = g.rdzw;
      const float* etp = g.etp;
      const float* ewp = g.ewp;
      const float zzk = g.zz[i], zzm = g.zz[i - 1];
      a = -s_wz[k] * s_tz[k - 1] * rdzw[k - 1] * zzm + s_wr[k] * rdzw[k - 1] - s_wt[k - 1] * s_tz[k - 1] * rdzw[k - 1];
      a = a * etp[k - 1] * ewp[k - 1];
      b = s_wz[k] * s_tz[k] * (etp[k] * rdzw[k] * zzk + etp[k - 1] * rdzw[k - 1] * zzm)
          - s_tz[k] * (etp[k] * s_wt[k] * rdzw[k] - etp[k - 1] * s_wt[k - 1] * rdzw[k - 1])
          + s_wr[k] * (etp[k] * rdzw[k] - etp[k - 1] * rdzw[k - 1]);
      b = b * ewp[k];
      if (k < L - 1) {
        cc = -s_wz[k] * s_tz[k + 1] * rdzw[k] * zzk - s_wr[k] * rdzw[k] + s_wt[k] * s_tz[k + 1] * rdzw[k];
        cc = cc * etp[k] * ewp[k + 1];
      }
    }
    s_a[k] = a;
    s_b[k] = b;
    s_c[k] = cc;
  }
  __syncthreads();
  if (live && k == 0) {
    float gam = 0.0f;
    s_b[0] = 0.0f;   // reused below as alpha
    s_c[0] = 0.0f;   // reused as gamma
    for (int kk = 1; kk < L; ++kk) {
      const float den = 1.0f + dts2 * (s_b[kk] - s_a[kk] * gam);
      if (den == 0.0f) atomicOr(flag, HEX_FLAG_SINGULAR);
      const float alpha = 1.0f / den;
      gam = dts2 * s_c[kk] * alpha;
      s_b[kk] = alpha;
      s_c[kk] = gam;
    }
  }
  __syncthreads();
  if (live) {
    if (k <= L) coftz[i] = s_tz[k];
    if (k < L) {
      cofwr[i] = s_wr[k];
      cofwz[i] = s_wz[k];
      cofwt[i] = s_wt[k];
      a_tri[i] = s_a[k];
      alpha_tri[i] = s_b[k];
      gamma_tri[i] = s_c[k];
    }
  }
}

// ------------------------------------------------------------- acoustic

// One acoustic edge pass: optionally the 3-D divergence damping of the
// previous substep (hexcore/mixing.py:851, stored inverse of dts), then the
// ru_p update of this substep (hexcore/acoustic_v841.py:416-460).
// mode 0: first substep (ru_p = dts*tend_ru); 1: damping + update; 2: damping only.
__global__ void k_ac_edge(HexGeo g, int mode, int old_is_zero, float dts, float damp_coef,
                          const float* __restrict__ tend_ru, const float* __restrict__ rtpp_new,
                          const float* __restrict__ rtpp_old, const float* __restrict__ rho_pp,
                          const float* __restrict__ theta_s, const float* __restrict__ exner_s,
                          const float* __restrict__ cqu, float* __restrict__ ru_p, float* __restrict__ ru_avg) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  const int j = e * S + k;
  if (mode == 0) {
    const float r = dts * tend_ru[j];
    ru_p[j] = r;
    ru_avg[j] = r;
    return;
  }
  const int i0 = g.coe[2 * e] * S + k, i1 = g.coe[2 * e + 1] * S + k;
  float r = ru_p[j];
  {
    const float d0 = old_is_zero ? rtpp_new[i0] - 0.0f : rtpp_new[i0] - rtpp_old[i0];
    const float d1 = old_is_zero ? rtpp_new[i1] - 0.0f : rtpp_new[i1] - rtpp_old[i1];
    r = r + damp_coef * (d0 - d1) * (1.0f - 0.0f) / (theta_s[i0] + theta_s[i1]);
  }
  if (mode == 1) {
    float pg = (rtpp_new[i1] - rtpp_new[i0]) * g.inv_dc[e] / (0.5f * (g.zz[i1] + g.zz[i0]));
    pg = cqu[j] * 0.5f * g.c2 * (exner_s[i0] + exner_s[i1]) * pg;
    pg = pg + 0.5f * g.zxu[j] * g.g * (rho_pp[i0] + rho_pp[i1]);
    r = r + dts * (tend_ru[j] - pg);
    ru_avg[j] = ru_avg[j] + r;
  }
  ru_p[j] = r;
}

// One acoustic cell pass (hexcore/acoustic_v841.py:461-567): rs/ts from the
// edge fluxes of ru_p, the rw_p right-hand side, the dts^2 Thomas sweep
// (:236-257, one thread per column, levels in order), implicit Rayleigh
// damping, ww_avg, and the rho_pp / rtheta_pp updates.  Everything the
// sequential sweep reads (rhs, dts2*a, alpha, gamma) is staged in shared
// memory by the level-parallel phase first, so the recurrence never waits
// on a global load.
#define HEX_AC_SMEM_ARRAYS 8
__global__ void k_ac_cell(HexGeo g, int first, float dts, float dts2, const float* __restrict__ ru_p,
                          const float* __restrict__ theta_s, const float* __restrict__ tend_rho,
                          const float* __restrict__ tend_rt, const float* __restrict__ tend_rw,
                          const float* __restrict__ cofwr, const float* __restrict__ cofwz,
                          const float* __restrict__ coftz, const float* __restrict__ cofwt,
                          const float* __restrict__ a_tri, const float* __restrict__ alpha_tri,
                          const float* __restrict__ gamma_tri, const float* __restrict__ rho_zz,
                          const float* __restrict__ w, const float* __restrict__ rw,
                          const float* __restrict__ rw_save, const float* __restrict__ rtpp_old,
                          float* __restrict__ rtpp_new, float* __restrict__ rho_pp, float* __restrict__ rw_p,
                          float* __restrict__ ww_avg) {
  extern __shared__ float sm[];
  const int k = threadIdx.x;
  const int S = g.S, L = g.L;
  const int c = blockIdx.x * blockDim.y + threadIdx.y;
  const bool live = c < g.nC;
  float* s_rs = sm + threadIdx.y * S * HEX_AC_SMEM_ARRAYS;
  float* s_ts = s_rs + S;
  float* s_rho = s_ts + S;
  float* s_rt = s_rho + S;
  float* s_r = s_rt + S;
  float* s_da = s_r + S;
  float* s_al = s_da + S;
  float* s_ga = s_al + S;
  const int i = c * S + k;
  const float* ewm = g.ewm;
  const float* ewp = g.ewp;
  const float* etp = g.etp;
  const float* etm = g.etm;
  float wa = 0.0f, rwp_old = 0.0f;
  if (live) {
    if (k <= L) rwp_old = first ? 0.0f : rw_p[i];
    s_r[k] = rwp_old;
    if (k < L) {
      s_da[k] = dts2 * a_tri[i];
      s_al[k] = alpha_tri[i];
      s_ga[k] = gamma_tri[i];
    }
  }
  __syncthreads();
  if (live) {
    if (k < L) {
      const float rho_old = first ? 0.0f : rho_pp[i];
      const float rt_old = first ? 0.0f : rtpp_old[i];
      float rs = 0.0f, ts = 0.0f;
      const int n = g.deg[c];
      const float ia = g.inv_area[c];
      for (int s = 0; s < n; ++s) {
        const int e = g.eoc[c * g.maxE + s];
        const int e0 = g.coe[2 * e], e1 = g.coe[2 * e + 1];
        const float flux = g.csign[c * g.maxE + s] * dts * g.dv[e] * ru_p[e * S + k] * ia;
        rs = rs - flux;
        ts = ts - flux * 0.5f * (theta_s[e1 * S + k] + theta_s[e0 * S + k]);
      }
      const float cofrz = g.rdzw[k];
      rs = rho_old + dts * tend_rho[i] + rs - dts * cofrz * (ewm[k + 1] * s_r[k + 1] - ewm[k] * s_r[k]);
      ts = rt_old + dts * tend_rt[i] + ts
           - dts * g.rdzw[k] * (ewm[k + 1] * coftz[i + 1] * s_r[k + 1] - ewm[k] * coftz[i] * s_r[k]);
      s_rs[k] = rs;
      s_ts[k] = ts;
      s_rho[k] = rho_old;
      s_rt[k] = rt_old;
    }
    if (k >= 1 && k < L) wa = (first ? 0.0f : ww_avg[i]) + ewm[k] * rwp_old;
  }
  __syncthreads();
  float rhs = rwp_old;
  if (live && k >= 1 && k < L) {
    const float zzk = g.zz[i], zzm = g.zz[i - 1];
    rhs = rwp_old + dts * (tend_rw[i]
                           - cofwz[i] * ((etp[k] * zzk * s_ts[k] - etp[k - 1] * zzm * s_ts[k - 1])
                                         + (etm[k] * zzk * s_rt[k] - etm[k - 1] * zzm * s_rt[k - 1]))
                           - cofwr[i] * ((etp[k] * s_rs[k] + etp[k - 1] * s_rs[k - 1])
                                         + (etm[k] * s_rho[k] + etm[k - 1] * s_rho[k - 1]))
                           + cofwt[i] * (etp[k] * s_ts[k] + etm[k] * s_rt[k])
                           + cofwt[i - 1] * (etp[k - 1] * s_ts[k - 1] + etm[k - 1] * s_rt[k - 1]));
  }
  __syncthreads();
  if (live && k <= L) s_r[k] = rhs;
  __syncthreads();
  if (live && k == 0) {
    float prev = s_r[0];
#pragma unroll 4
    for (int kk = 1; kk < L; ++kk) {
      prev = (s_r[kk] - s_da[kk] * prev) * s_al[kk];
      s_r[kk] = prev;
    }
    float next = s_r[L];
#pragma unroll 4
    for (int kk = L - 1; kk >= 0; --kk) {
      next = s_r[kk] - s_ga[kk] * next;
      s_r[kk] = next;
    }
  }
  __syncthreads();
  float rwp = 0.0f;
  if (live && k <= L) {
    rwp = s_r[k];
    if (k >= 1 && k < L) {
      const float delta = rw_save[i] - rw[i];
      const float damp = g.dss[i];
      const float zzi = g.fzm[k] * g.zz[i] + g.fzp[k] * g.zz[i - 1];
      const float rhoi = g.fzm[k] * rho_zz[i] + g.fzp[k] * rho_zz[i - 1];
      rwp = (rwp + delta - dts * damp * zzi * rhoi * w[i]) / (1.0f + dts * damp) - delta;
      ww_avg[i] = wa + ewp[k] * rwp;
    } else {
      ww_avg[i] = 0.0f;
    }
    rw_p[i] = rwp;
  }
  __syncthreads();
  if (live && k <= L) s_r[k] = rwp;
  __syncthreads();
  if (live && k < L) {
    rho_pp[i] = s_rs[k] - dts * g.rdzw[k] * (ewp[k + 1] * s_r[k + 1] - ewp[k] * s_r[k]);
    rtpp_new[i] = s_ts[k] - dts * g.rdzw[k] * (ewp[k + 1] * coftz[i + 1] * s_r[k + 1] - ewp[k] * coftz[i] * s_r[k]);
  }
}

// ---------------------------------------------------------- stage recovery
// hexcore/driver.py:3166-3292: candidate state, rw end conditions, u, w,
// theta_m, Exner and p' at stage 3, and the split mass-flux average
// (hexcore/integration.py:27,58).

__global__ void k_recover_edge(HexGeo g, const float* __restrict__ ru_s, const float* __restrict__ ru_p,
                               const float* __restrict__ ru_avg, const float* __restrict__ rp_s,
                               const float* __restrict__ rho_pp, float* __restrict__ ru_out,
                               float* __restrict__ u_out, float* __restrict__ flux_u, int flux_mode,
                               float inv_steps, float inv_splits) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  const int j = e * S + k;
  const int i0 = g.coe[2 * e] * S + k, i1 = g.coe[2 * e + 1] * S + k;
  const float rho0 = rp_s[i0] + rho_pp[i0] + g.rho_base[i0];
  const float rho1 = rp_s[i1] + rho_pp[i1] + g.rho_base[i1];
  const float ru = ru_s[j] + ru_p[j];
  ru_out[j] = ru;
  u_out[j] = 2.0f * ru / (rho0 + rho1);
  // flux_mode: bit 2 active, bit 0 first subcycle, bit 1 last subcycle
  if (flux_mode & 4) {
    const float f = ru_s[j] + ru_avg[j] * inv_steps;
    float acc = (flux_mode & 1) ? f : f + flux_u[j];
    if (flux_mode & 2) acc = acc * inv_splits;
    flux_u[j] = acc;
  }
}

__global__ void k_recover_cell(HexGeo g, int stage3, const float* __restrict__ rp_s,
                               const float* __restrict__ rtp_s, const float* __restrict__ rw_s,
                               const float* __restrict__ rho_pp, const float* __restrict__ rtpp,
                               const float* __restrict__ rw_p, const float* __restrict__ ww_avg,
                               const float* __restrict__ ru_new, HexState out, HexSide side,
                               float* __restrict__ flux_w, int flux_mode, float inv_steps, float inv_splits,
                               int* flag) {
  HEX_LEVEL_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  const int i = c * S + k;
  if (k < L) {
    const float rp = rp_s[i] + rho_pp[i];
    const float rtp = rtp_s[i] + rtpp[i];
    const float rho = rp + g.rho_base[i];
    const float rt = rtp + g.rtheta_base[i];
    if (!(rho > 0.0f) || !(rt > 0.0f)) atomicOr(flag, HEX_FLAG_DENSITY);
    out.rho[i] = rho;
    out.rho_theta[i] = rt;
    side.rho_p[i] = rp;
    side.rtheta_p[i] = rtp;
    side.theta_m[i] = rt / rho;
    if (stage3) {
      int bad = 0;
      const float exner = hexdyn_powf::powf_gnu(g.zz[i] * g.r_over_p0 * rt, g.kappa, &bad);
      if (bad) atomicOr(flag, HEX_FLAG_POWF);
      side.exner[i] = exner;
      side.pressure_p[i] = g.zz[i] * g.rgas * (exner * rtp + g.rtheta_base[i] * (exner - g.exner_base[i]));
    }
  }
  if (k <= L) {
    const float rw = (k == 0 || k == L) ? 0.0f : rw_s[i] + rw_p[i];
    out.rho_w[i] = rw;
    auto rho_at = [&](int kk) { return rp_s[c * S + kk] + rho_pp[c * S + kk] + g.rho_base[c * S + kk]; };
    side.w[i] = recover_w_at(g, c, k, rho_at, ru_new, rw);
    if (flux_mode & 4) {
      const float f = rw_s[i] + ww_avg[i] * inv_steps;
      float acc = (flux_mode & 1) ? f : f + flux_w[i];
      if (flux_mode & 2) acc = acc * inv_splits;
      flux_w[i] = acc;
    }
  }
}

// ------------------------------------------------------------ transport
// hexcore/transport.py:1461 third-order edge values, one tracer per blockIdx.z.
// mono: the monotonic source flux (velocity folded in; the literal ten-term
// association for ten-cell stencils).
__global__ void k_tr_edge(HexGeo g, int mono, const float* __restrict__ q, const float* __restrict__ hv,
                          float* __restrict__ out) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  const size_t toff = (size_t)blockIdx.z * g.nC * S;
  const float* qt = q + toff;
  const int n = g.n_adv[e];
  const int* cells = g.adv_cells + (size_t)e * g.advW;
  const float* a1 = g.adv + (size_t)e * g.advW;
  const float* a3 = g.adv3 + (size_t)e * g.advW;
  const float vel = hv[e * S + k];
  const float sgn = copysignf(1.0f, vel);
  float res;
  if (mono && n == 10) {
    float val = (a1[0] + g.coef3 * sgn * a3[0]) * qt[cells[0] * S + k];
    for (int s = 1; s < 10; ++s) val = val + (a1[s] + g.coef3 * sgn * a3[s]) * qt[cells[s] * S + k];
    res = vel * val;
  } else {
    res = 0.0f;
    for (int s = 0; s < n; ++s) {
      float wgt = a1[s] + g.coef3 * sgn * a3[s];
      if (mono) wgt = vel * wgt;
      res = res + wgt * qt[cells[s] * S + k];
    }
  }
  out[(size_t)blockIdx.z * g.nE * S + e * S + k] = res;
}

// hexcore/transport.py:1389 with the atmosphere flux3 (+ correction).
__device__ __forceinline__ float tr_vflux(const HexGeo& g, const float* __restrict__ qc,
                                          const float* __restrict__ wwc, int j) {
  const int L = g.L;
  if (j <= 0 || j >= L) return 0.0f;
  if (j == 1 || j == L - 1) return wwc[j] * (g.fzm[j] * qc[j] + g.fzp[j] * qc[j - 1]);
  const float vel = wwc[j];
  const float base = vel * (7.0f * (qc[j] + qc[j - 1]) - (qc[j + 1] + qc[j - 2])) / 12.0f;
  const float corr = g.coef3 * fabsf(vel) * ((qc[j + 1] - qc[j - 2]) - 3.0f * (qc[j] - qc[j - 1])) / 12.0f;
  return base + corr;
}

// hexcore/transport.py:1649 advance_scalars (RK1/RK2, split transport).
__global__ void k_tr_std(HexGeo g, float step, float wn, const float* __restrict__ q_old,
                         const float* __restrict__ q_stage, const float* __restrict__ rho_old,
                         const float* __restrict__ rho_new, const float* __restrict__ hv,
                         const float* __restrict__ ww, const float* __restrict__ edge_q,
                         float* __restrict__ q_out) {
  HEX_LEVEL_PARALLEL(g.nC)
  if (k >= g.L) return;
  const int c = ent, S = g.S;
  const int i = c * S + k;
  const size_t toff = (size_t)blockIdx.z * g.nC * S;
  const float* ev = edge_q + (size_t)blockIdx.z * g.nE * S;
  const int n = g.deg[c];
  float t = 0.0f;
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    t = t + -g.csign[c * g.maxE + s] * hv[e * S + k] * ev[e * S + k];
  }
  t = t * g.inv_area[c] + 0.0f;
  const float* qc = q_stage + toff + c * S;
  const float* wwc = ww + c * S;
  const float target = (1.0f - wn) * rho_old[i] + wn * rho_new[i];
  const float num = q_old[toff + i] * rho_old[i]
                    + step * (t - g.rdzw[k] * (tr_vflux(g, qc, wwc, k + 1) - tr_vflux(g, qc, wwc, k)));
  q_out[toff + i] = num * (1.0f / target);
}

// hexcore/transport.py:1887-1906 split-transport target density.
__global__ void k_fct_target(HexGeo g, float step, const float* __restrict__ rho_old,
                             const float* __restrict__ hv, const float* __restrict__ ww,
                             float* __restrict__ target, int* flag) {
  HEX_LEVEL_PARALLEL(g.nC)
  if (k >= g.L) return;
  const int c = ent, S = g.S;
  const int i = c * S + k;
  const int n = g.deg[c];
  const float ia = g.inv_area[c];
  float hd = 0.0f;
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    hd = hd + -g.csign[c * g.maxE + s] * hv[e * S + k] * g.dv[e] * ia;
  }
  const float td = rho_old[i] + step * (hd - g.rdzw[k] * (ww[i + 1] - ww[i]));
  if (!(td > 0.0f)) atomicOr(flag, HEX_FLAG_TARGET);
  target[i] = td;
}

// source-updated old scalar (scalar_tendency is zero): old + step*0/rho.
__device__ __forceinline__ float fct_old(const float* __restrict__ q_old, size_t i) { return q_old[i] + 0.0f; }

__device__ __forceinline__ float fct_fcol(const HexGeo& g, float step, const float* __restrict__ oc,
                                          const float* __restrict__ wwc, int j) {
  return step * (pos0(wwc[j]) * (oc[j - 1] + 0.0f) + neg0(wwc[j]) * (oc[j] + 0.0f));
}

// Unlimited vertical antidiffusive residual at interface j.
__device__ __forceinline__ float fct_vres(const HexGeo& g, float step, const float* __restrict__ qc,
                                          const float* __restrict__ oc, const float* __restrict__ wwc, int j) {
  const float hv = step * tr_vflux(g, qc, wwc, j);
  if (j <= 0 || j >= g.L) return hv;
  return hv - fct_fcol(g, step, oc, wwc, j);
}

__device__ __forceinline__ float fct_upwind(const HexGeo& g, float step, const float* __restrict__ ot,
                                            const float* __restrict__ hv, int e, int k) {
  const int S = g.S;
  const float vel = hv[e * S + k];
  return g.dv[e] * step * (pos0(vel) * (ot[g.coe[2 * e] * S + k] + 0.0f) + neg0(vel) * (ot[g.coe[2 * e + 1] * S + k] + 0.0f));
}

// hexcore/transport.py:1919-2118 (v8.4.1 order): bounds, low-order mass,
// incoming/outgoing antidiffusive totals and the scale factors.
__global__ void k_fct_cell1(HexGeo g, float step, const float* __restrict__ q_old,
                            const float* __restrict__ q_stage, const float* __restrict__ rho_old,
                            const float* __restrict__ hv, const float* __restrict__ ww,
                            const float* __restrict__ high_e, const float* __restrict__ target,
                            float* __restrict__ scale_in, float* __restrict__ scale_out, float* __restrict__ mass_out) {
  HEX_LEVEL_PARALLEL(g.nC)
  if (k >= g.L) return;
  const int c = ent, S = g.S, L = g.L;
  const int i = c * S + k;
  const size_t toff = (size_t)blockIdx.z * g.nC * S;
  const float* ot = q_old + toff;
  const float* oc = ot + c * S;
  const float* qc = q_stage + toff + c * S;
  const float* wwc = ww + c * S;
  const float* he = high_e + (size_t)blockIdx.z * g.nE * S;
  const float o = oc[k] + 0.0f;
  // bounds: the column triple, then the neighbours at this level
  float mn = o, mx = o;
  {
    const int lo = k > 0 ? k - 1 : 0, hi = k + 1 < L ? k + 1 : L - 1;
    float a = oc[lo] + 0.0f, b = oc[hi] + 0.0f;
    mn = fminf(fminf(a, o), b);
    mx = fmaxf(fmaxf(a, o), b);
  }
  const int n = g.deg[c];
  for (int s = 0; s < n; ++s) {
    const float on = ot[g.coc[c * g.maxE + s] * S + k] + 0.0f;
    mn = pymin(mn, on);
    mx = pymax(mx, on);
  }
  float mass = o * rho_old[i];
  if (k < L - 1) mass = mass - fct_fcol(g, step, oc, wwc, k + 1) * g.rdzw[k];
  if (k >= 1) mass = mass + fct_fcol(g, step, oc, wwc, k) * g.rdzw[k];
  const float vr1 = fct_vres(g, step, qc, oc, wwc, k + 1);
  const float vr0 = fct_vres(g, step, qc, oc, wwc, k);
  float s_in = -g.rdzw[k] * (neg0(vr1) - pos0(vr0));
  float s_out = -g.rdzw[k] * (pos0(vr1) - neg0(vr0));
  const float ia = g.inv_area[c];
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float tsign = -g.csign[c * g.maxE + s];
    const float upw = fct_upwind(g, step, ot, hv, e, k);
    mass = mass + tsign * upw * ia;
    const float hres = step * he[e * S + k] - upw;
    const float sr = -tsign * hres;
    s_out = s_out - pos0(sr) * ia;
    s_in = s_in - neg0(sr) * ia;
  }
  const float td = target[i];
  float sf = (mx * td - mass) / (s_in + 1.0e-20f);
  scale_in[toff + i] = pymin(1.0f, pos0(sf));
  sf = (mn * td - mass) / (s_out - 1.0e-20f);
  scale_out[toff + i] = pymin(1.0f, pos0(sf));
  mass_out[toff + i] = mass;
}

__global__ void k_fct_edge(HexGeo g, float step, const float* __restrict__ q_old, const float* __restrict__ hv,
                           const float* __restrict__ high_e, const float* __restrict__ scale_in,
                           const float* __restrict__ scale_out, float* __restrict__ hres_lim) {
  HEX_LEVEL_PARALLEL(g.nE)
  if (k >= g.L) return;
  const int e = ent, S = g.S;
  const size_t toff = (size_t)blockIdx.z * g.nC * S;
  const size_t eoff = (size_t)blockIdx.z * g.nE * S;
  const int i0 = g.coe[2 * e] * S + k, i1 = g.coe[2 * e + 1] * S + k;
  const float upw = fct_upwind(g, step, q_old + toff, hv, e, k);
  const float flux = step * high_e[eoff + e * S + k] - upw;
  const float* si = scale_in + toff;
  const float* so = scale_out + toff;
  hres_lim[eoff + e * S + k] = pos0(flux) * pymin(so[i0], si[i1]) + neg0(flux) * pymin(si[i0], so[i1]);
}

__global__ void k_fct_cell2(HexGeo g, float step, const float* __restrict__ q_old,
                            const float* __restrict__ q_stage, const float* __restrict__ ww,
                            const float* __restrict__ scale_in, const float* __restrict__ scale_out,
                            const float* __restrict__ mass_in, const float* __restrict__ hres_lim,
                            const float* __restrict__ target, float* __restrict__ q_out) {
  HEX_LEVEL_PARALLEL(g.nC)
  if (k >= g.L) return;
  const int c = ent, S = g.S, L = g.L;
  const int i = c * S + k;
  const size_t toff = (size_t)blockIdx.z * g.nC * S;
  const float* oc = q_old + toff + c * S;
  const float* qc = q_stage + toff + c * S;
  const float* wwc = ww + c * S;
  const float* si = scale_in + toff + c * S;
  const float* so = scale_out + toff + c * S;
  const float* hl = hres_lim + (size_t)blockIdx.z * g.nE * S;
  float mass = mass_in[toff + i];
  const int n = g.deg[c];
  const float ia = g.inv_area[c];
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    mass = mass + -g.csign[c * g.maxE + s] * hl[e * S + k] * ia;
  }
  auto vlim = [&](int j) {
    const float f = fct_vres(g, step, qc, oc, wwc, j);
    if (j <= 0 || j >= L) return f;
    return pos0(f) * pymin(so[j - 1], si[j]) + neg0(f) * pymin(so[j], si[j - 1]);
  };
  mass = mass - g.rdzw[k] * (vlim(k + 1) - vlim(k));
  q_out[toff + i] = pos0(mass / target[i]);
}
