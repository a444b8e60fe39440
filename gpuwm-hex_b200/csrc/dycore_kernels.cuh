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
// This file holds the one-level-per-thread kernels: the sidecar rebuild, the
// moist coefficients, and the column-sweep kernels for columns of more than
// 128 levels (S/4 > 32 lanes, beyond one warp).  The stencil kernels of the
// step take four levels per thread (dycore_kernels_vec.cuh).
//
// Thread layout: blockDim = (S, EPB); x is the level (0..S-1), y the entity
// within the block; the S threads of an entity are consecutive, so a warp
// reads 32 consecutive words of one column.

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
