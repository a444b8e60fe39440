// Level-vector kernels: each thread owns four consecutive levels of one
// entity and moves them with 128-bit loads and stores.  The [entity][level]
// layout with a stride S that is a multiple of 8 makes every 4-level chunk
// 16-byte aligned.  Per-level arithmetic follows the reference's expressions
// and order exactly (one FP32 rounding per operation in the strict build);
// the index loads, coefficient loads and address arithmetic of an entity
// are shared by its four levels and each thread carries four independent
// chains.  Stores keep the levels a field defines (levels < L, or <= L for
// interface fields) and write +0 into the chunk's other words (st4m).
//
// Thread layout: blockDim = (S/4, EPB4); x selects the chunk k0 = 4*x.

// Blocks hold at most 256 threads (S/4 <= 256, checked at create).  The
// resident-block target per SM sets the register cap: 4 blocks allow 64
// registers a thread, 3 allow 80.
#ifndef HEX_VEC_MIN_BLOCKS
#define HEX_VEC_MIN_BLOCKS 4
#endif
#define HEX_VEC_BOUNDS __launch_bounds__(256, HEX_VEC_MIN_BLOCKS)
// Third-order stencil weights A + (coef3 sign v) B selected from A + X and
// A - X per level (1) or formed per level (0): the same words.  Measured:
// the tracer edge values 162.6 -> 155.3 us per launch with the selection,
// the theta/w edge values 58.5 -> 60.5 (kept per level).
#ifndef HEX_PM_SELECT_EDGE_ADV
#define HEX_PM_SELECT_EDGE_ADV 0
#endif
#ifndef HEX_PM_SELECT_TR_EDGE
#define HEX_PM_SELECT_TR_EDGE 1
#endif
// Kernels measured faster at another cap: the momentum tendency (a
// latency-bound ten-point gather) at 6 blocks (40 registers), the tracer
// edge values (three tracers' accumulators per thread) at 2 (128), the
// limited antidiffusive flux at 6 and the standard tracer update at 5.
#ifndef HEX_TEND_U_MIN_BLOCKS
#define HEX_TEND_U_MIN_BLOCKS 6
#endif
#ifndef HEX_EDGE_ADV_MIN_BLOCKS
#define HEX_EDGE_ADV_MIN_BLOCKS HEX_VEC_MIN_BLOCKS
#endif
#ifndef HEX_TR_EDGE_MIN_BLOCKS
#define HEX_TR_EDGE_MIN_BLOCKS 2
#endif
#ifndef HEX_FCT_EDGE_MIN_BLOCKS
#define HEX_FCT_EDGE_MIN_BLOCKS 6
#endif
#ifndef HEX_TR_STD_MIN_BLOCKS
#define HEX_TR_STD_MIN_BLOCKS 5
#endif

#define HEX_VEC_PARALLEL(n)                                \
  const int k0 = threadIdx.x * 4;                          \
  const int ent = blockIdx.x * blockDim.y + threadIdx.y;   \
  if (ent >= (n)) return;

// Transport kernels over nT tracers: block b serves tracer b % nT of entity
// block b / nT, so the nT tracers of an entity block run back to back and
// share the reads of the velocities and stencil tables through L2.
#define HEX_VEC_TRACER(n, nT)                                     \
  const int k0 = threadIdx.x * 4;                                 \
  const int tr = blockIdx.x % (nT);                               \
  const int ent = (blockIdx.x / (nT)) * blockDim.y + threadIdx.y; \
  if (ent >= (n)) return;

// Neighbour gathers: each iteration loads an index and then the neighbour's
// levels, so unrolling lets the loads of several neighbours be in flight
// together.  HEX_GATHER_UNROLL sets the unroll factor (0: the compiler's choice).
#ifndef HEX_GATHER_UNROLL
#define HEX_GATHER_UNROLL 2
#endif
// Per-kernel unroll of the neighbour loop (default HEX_GATHER_UNROLL).
// Swept on the x1.40962 workload: the theta/w edge values run fastest
// unrolled by five (55.5 vs 58.3 us per launch; three 57.7); the momentum
// tendency by four or five (with 64 registers) and the tracer edge values by
// three or five were slower than two.
#ifndef HEX_TEND_U_UNROLL
#define HEX_TEND_U_UNROLL HEX_GATHER_UNROLL
#endif
#ifndef HEX_TR_EDGE_UNROLL
#define HEX_TR_EDGE_UNROLL HEX_GATHER_UNROLL
#endif
#ifndef HEX_EDGE_ADV_UNROLL
#define HEX_EDGE_ADV_UNROLL 5
#endif
#define HEX_PRAGMA(x) _Pragma(#x)
#define HEX_UNROLL_N(n) HEX_PRAGMA(unroll n)
#if HEX_GATHER_UNROLL > 0
#define HEX_GATHER HEX_UNROLL_N(HEX_GATHER_UNROLL)
#else
#define HEX_GATHER
#endif

struct V4 {
  float a[4];
};

__device__ __forceinline__ V4 v4zero() { return V4{{0.0f, 0.0f, 0.0f, 0.0f}}; }

// read-only (non-coherent) 128-bit load: the array is not written by the kernel
__device__ __forceinline__ V4 ld4(const float* __restrict__ p) {
  const float4 t = __ldg(reinterpret_cast<const float4*>(p));
  return V4{{t.x, t.y, t.z, t.w}};
}
// coherent 128-bit load for arrays the kernel also writes
__device__ __forceinline__ V4 ld4rw(const float* p) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  return V4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ void st4(float* p, const V4& v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.a[0], v.a[1], v.a[2], v.a[3]);
}
// Store the levels k0+j in [lo, hi) of a chunk; the other words of the chunk
// (the padding levels past the field's last level, and level 0 of a field
// defined from level 1) are written as +0.  No kernel writes anything else
// there and every buffer starts zeroed, so those words stay +0, as they
// would if left alone, while every lane runs the same single 128-bit store
// (a per-word store for the chunk holding the top level would split the warp).
#ifndef HEX_MASKED_STORE_ZERO
#define HEX_MASKED_STORE_ZERO 1
#endif
__device__ __forceinline__ void st4m(float* p, const V4& v, int k0, int lo, int hi) {
#if HEX_MASKED_STORE_ZERO
  V4 w;
#pragma unroll
  for (int j = 0; j < 4; ++j) w.a[j] = (k0 + j >= lo && k0 + j < hi) ? v.a[j] : 0.0f;
  st4(p, w);
#else
  if (k0 >= lo && k0 + 4 <= hi) {
    st4(p, v);
    return;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (k0 + j >= lo && k0 + j < hi) p[j] = v.a[j];
#endif
}

// Column window col[k0-4 .. k0+7] around a thread's chunk; entries outside
// [0, S) read as zero and are never used by a formula.
struct Win {
  float a[12];
  __device__ __forceinline__ float operator()(int d) const { return a[d + 4]; }
};
__device__ __forceinline__ Win win(const float* __restrict__ col, int k0, int S) {
  Win w;
  const V4 m = ld4(col + k0);
  const V4 lo = k0 >= 4 ? ld4(col + k0 - 4) : v4zero();
  const V4 hi = k0 + 4 < S ? ld4(col + k0 + 4) : v4zero();
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    w.a[j] = lo.a[j];
    w.a[j + 4] = m.a[j];
    w.a[j + 8] = hi.a[j];
  }
  return w;
}

// End-of-step clamp of negative mixing ratios (hexcore/cuda_driver.py:5311,
// `putmask(scalars, scalars < 0, 0)`): -0 and NaN compare false and stay.
// blockIdx.z selects the scalar.
__global__ void HEX_VEC_BOUNDS kv_clamp_scalars(HexGeo g, float* __restrict__ q) {
  HEX_VEC_PARALLEL(g.nC)
  float* p = q + ((size_t)blockIdx.z * g.nC + ent) * g.S + k0;
  V4 v = ld4rw(p);
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (v.a[j] < 0.0f) v.a[j] = 0.0f;
  st4m(p, v, k0, 0, g.L);
}

// --------------------------------------------------- moist coefficients
// hexcore/regional_v841.py:1180 compute_moist_coefficients, every scalar:
// qtot = sum of the scalars in scalar order, cqw = 1/(1 + (qtot(k) +
// qtot(k-1))/2) above the surface, cqu = 1/(1 + sum of the two-cell means).
// Scalars are stored [scalar][cell][S].
__global__ void HEX_VEC_BOUNDS kv_moist_cell(HexGeo g, const float* __restrict__ q, int nT,
                                             float* __restrict__ qtot, float* __restrict__ cqw) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S;
  const size_t tstride = (size_t)g.nC * S;
  const float* qc = q + c * S + k0;
  V4 acc = v4zero();
  float below = 0.0f;  // qtot at level k0 - 1
  HEX_GATHER
  for (int t = 0; t < nT; ++t) {
    const V4 v = ld4(qc + t * tstride);
#pragma unroll
    for (int j = 0; j < 4; ++j) acc.a[j] = acc.a[j] + v.a[j];
    if (k0 > 0) below = below + (qc - 1)[t * tstride];
  }
  V4 cw;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float prev = j == 0 ? below : acc.a[j - 1];
    cw.a[j] = k0 + j == 0 ? 1.0f : 1.0f / (1.0f + 0.5f * (acc.a[j] + prev));
  }
  st4m(qtot + c * S + k0, acc, k0, 0, g.L);
  st4m(cqw + c * S + k0, cw, k0, 0, g.L);
}

__global__ void HEX_VEC_BOUNDS kv_moist_edge(HexGeo g, const float* __restrict__ q, int nT,
                                             float* __restrict__ cqu) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  const size_t tstride = (size_t)g.nC * S;
  const float* q0 = q + g.coe[2 * e] * S + k0;
  const float* q1 = q + g.coe[2 * e + 1] * S + k0;
  V4 acc = v4zero();
  HEX_GATHER
  for (int t = 0; t < nT; ++t) {
    const V4 a = ld4(q0 + t * tstride), b = ld4(q1 + t * tstride);
#pragma unroll
    for (int j = 0; j < 4; ++j) acc.a[j] = acc.a[j] + 0.5f * (a.a[j] + b.a[j]);
  }
  V4 out;
#pragma unroll
  for (int j = 0; j < 4; ++j) out.a[j] = 1.0f / (1.0f + acc.a[j]);
  st4m(cqu + e * S + k0, out, k0, 0, g.L);
}

// ---------------------------------------------------------- diagnostics
// hexcore/diagnostics.py:95 compute_solve_diagnostics, v8.4.1 stored inverses.

__global__ void HEX_VEC_BOUNDS kv_diag_vertex(HexGeo g, const float* __restrict__ u, float* __restrict__ pv_vertex,
                               float* __restrict__ ke_vertex, float* __restrict__ vorticity) {
  HEX_VEC_PARALLEL(g.nV)
  const int v = ent, S = g.S;
  V4 vort = v4zero(), ke[3];
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int e = g.eov[3 * v + s];
    const float vd = g.vsign[3 * v + s] * g.dc[e];
    const float dd = g.dc[e] * g.dv[e];
    const V4 ue = ld4(u + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      vort.a[j] = vort.a[j] + vd * ue.a[j];
      ke[s].a[j] = dd * (ue.a[j] * ue.a[j]);
    }
  }
  const float ia = g.inv_area_tri[v], r = 0.25f * g.inv_area_tri[v], f = g.f_vertex[v];
  V4 pv, kv, vo;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    vo.a[j] = vort.a[j] * ia;
    pv.a[j] = f + vo.a[j];
    kv.a[j] = (ke[0].a[j] + ke[1].a[j] + ke[2].a[j]) * r;
  }
  st4m(pv_vertex + v * S + k0, pv, k0, 0, g.L);
  st4m(ke_vertex + v * S + k0, kv, k0, 0, g.L);
  if (vorticity) st4m(vorticity + v * S + k0, vo, k0, 0, g.L);  // the mixing's input
}

// Cell kinetic energy (v8.4.1 kite blend 0.625) and, with APVM, cell PV;
// DIV: also the divergence of u (the horizontal mixing's input).
template <bool DIV>
__global__ void HEX_VEC_BOUNDS kv_diag_cell(HexGeo g, const float* __restrict__ u, const float* __restrict__ pv_vertex,
                             const float* __restrict__ ke_vertex, float* __restrict__ ke_out,
                             float* __restrict__ pv_cell, float* __restrict__ divergence) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S;
  const int n = g.deg[c];
  const float ia = g.inv_area[c];
  V4 ke = v4zero(), dv = v4zero();
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float dd = g.dc[e] * g.dv[e];
    const V4 ue = ld4(u + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) ke.a[j] = ke.a[j] + 0.25f * (dd * (ue.a[j] * ue.a[j]));
    if (DIV) {
      const float sd = g.csign[c * g.maxE + s] * g.dv[e];
#pragma unroll
      for (int j = 0; j < 4; ++j) dv.a[j] = dv.a[j] + sd * ue.a[j];
    }
  }
  if (DIV) {
#pragma unroll
    for (int j = 0; j < 4; ++j) dv.a[j] = dv.a[j] * ia;
    st4m(divergence + c * S + k0, dv, k0, 0, g.L);  // the mixing's input
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) ke.a[j] = ke.a[j] * ia * 0.625f;
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int vtx = g.voc[c * g.maxE + s];
    const float kt = (1.0f - 0.625f) * g.kite[3 * vtx + g.kite_slot[c * g.maxE + s]];
    const V4 kv = ld4(ke_vertex + vtx * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) ke.a[j] = ke.a[j] + kt * kv.a[j] * ia;
  }
  st4m(ke_out + c * S + k0, ke, k0, 0, g.L);
  if (g.apvm_on) {
    V4 pvc = v4zero();
    HEX_GATHER
    for (int s = 0; s < n; ++s) {
      const int vtx = g.voc[c * g.maxE + s];
      const float kite = g.kite[3 * vtx + g.kite_slot[c * g.maxE + s]];
      const V4 pv = ld4(pv_vertex + vtx * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) pvc.a[j] = pvc.a[j] + kite * pv.a[j] * ia;
    }
    st4m(pv_cell + c * S + k0, pvc, k0, 0, g.L);
  }
}

// Tangential velocity (TRiSK weights) and edge PV with APVM upwinding.
__global__ void HEX_VEC_BOUNDS kv_diag_edge(HexGeo g, const float* __restrict__ u, const float* __restrict__ pv_vertex,
                             const float* __restrict__ pv_cell, float* __restrict__ v, float* __restrict__ pv_edge,
                             int recompute_v) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  V4 vt;
  if (recompute_v) {
    vt = v4zero();
    const int n = g.neoe[e];
    HEX_GATHER
    for (int s = 0; s < n; ++s) {
      const float w = g.weights[e * g.maxE2 + s];
      const V4 un = ld4(u + g.eoe[e * g.maxE2 + s] * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) vt.a[j] = vt.a[j] + w * un.a[j];
    }
    st4m(v + e * S + k0, vt, k0, 0, g.L);
  } else {
    vt = ld4rw(v + e * S + k0);
  }
  const int v0 = g.voe[2 * e], v1 = g.voe[2 * e + 1];
  const V4 p0 = ld4(pv_vertex + v0 * S + k0), p1 = ld4(pv_vertex + v1 * S + k0);
  V4 pve;
#pragma unroll
  for (int j = 0; j < 4; ++j) pve.a[j] = 0.5f * (p0.a[j] + p1.a[j]);
  if (g.apvm_on) {
    const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
    const V4 q0 = ld4(pv_cell + c0 * S + k0), q1 = ld4(pv_cell + c1 * S + k0);
    const V4 ue = ld4(u + e * S + k0);
    const float idv = g.inv_dv[e], idc = g.inv_dc[e];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float gpt = (p1.a[j] - p0.a[j]) * idv;
      const float gpn = (q1.a[j] - q0.a[j]) * idc;
      pve.a[j] = pve.a[j] - g.apvm_scale * (vt.a[j] * gpt + ue.a[j] * gpn);
    }
  }
  st4m(pv_edge + e * S + k0, pve, k0, 0, g.L);
}

// --------------------------------------------------------- Euler terms

__device__ __forceinline__ float dpdz_of(const HexGeo& g, float rp, float qt, float rb) {
  if (!g.moist) return -g.g * rp;
  return -g.g * (rb * qt + rp * (1.0f + qt));
}

// hexcore/dynamics.py:188 pressure_gradient_euler_tendency.
__global__ void HEX_VEC_BOUNDS kv_euler_edge(HexGeo g, const float* __restrict__ pp, const float* __restrict__ rp,
                              const float* __restrict__ qtot, const float* __restrict__ cqu,
                              float* __restrict__ euler_ru) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  const int i0 = g.coe[2 * e] * S + k0, i1 = g.coe[2 * e + 1] * S + k0;
  const V4 p0 = ld4(pp + i0), p1 = ld4(pp + i1), r0 = ld4(rp + i0), r1 = ld4(rp + i1);
  // moisture terms of dpdz are read only with native moist coefficients
  const bool m = g.moist;
  const V4 q0 = m ? ld4(qtot + i0) : v4zero(), q1 = m ? ld4(qtot + i1) : v4zero();
  const V4 b0 = m ? ld4(g.rho_base + i0) : v4zero(), b1 = m ? ld4(g.rho_base + i1) : v4zero();
  const V4 z0 = ld4(g.zz + i0), z1 = ld4(g.zz + i1);
  const V4 cq = ld4(cqu + e * S + k0), zx = ld4(g.zxu + e * S + k0);
  const float idc = g.inv_dc[e];
  V4 out;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float d0 = dpdz_of(g, r0.a[j], q0.a[j], b0.a[j]);
    const float d1 = dpdz_of(g, r1.a[j], q1.a[j], b1.a[j]);
    out.a[j] = -cq.a[j] * ((p1.a[j] - p0.a[j]) * idc / (0.5f * (z1.a[j] + z0.a[j])) - 0.5f * zx.a[j] * (d0 + d1));
  }
  st4m(euler_ru + e * S + k0, out, k0, 0, g.L);
}

// hexcore/dynamics.py:86 mass_flux_divergence (stored inverse area), 4 levels.
__device__ __forceinline__ V4 mass_flux_div4(const HexGeo& g, const float* __restrict__ ru, int c, int k0) {
  V4 acc = v4zero();
  const int n = g.deg[c];
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float sd = g.csign[c * g.maxE + s] * g.dv[e];
    const V4 r = ld4(ru + e * g.S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) acc.a[j] = acc.a[j] + sd * r.a[j];
  }
  const float ia = g.inv_area[c];
#pragma unroll
  for (int j = 0; j < 4; ++j) acc.a[j] = acc.a[j] * ia;
  return acc;
}

// hexcore/dynamics.py:122 density_tendency and hexcore/driver.py:2804 Euler w.
__global__ void HEX_VEC_BOUNDS kv_euler_cell(HexGeo g, const float* __restrict__ ru, const float* __restrict__ rw,
                              const float* __restrict__ pp, const float* __restrict__ rp,
                              const float* __restrict__ qtot, const float* __restrict__ cqw,
                              float* __restrict__ tend_rho, float* __restrict__ euler_rw,
                              const float* __restrict__ phys_rho, float* __restrict__ tend_rho_dyn) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  const V4 hd = mass_flux_div4(g, ru, c, k0);
  const Win rww = win(rw + c * S, k0, S);
  const Win ppw = win(pp + c * S, k0, S), rpw = win(rp + c * S, k0, S);
  const bool m = g.moist;
  const Win qtw = m ? win(qtot + c * S, k0, S) : Win{}, rbw = m ? win(g.rho_base + c * S, k0, S) : Win{};
  const V4 cq = m ? ld4(cqw + c * S + k0) : v4zero();
  V4 tr, er;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    tr.a[j] = -hd.a[j] - g.rdzw[k] * (rww(j + 1) - rww(j));
    float out = 0.0f;
    if (k >= 1 && k < L) {
      const float dk = dpdz_of(g, rpw(j), qtw(j), rbw(j));
      const float dm = dpdz_of(g, rpw(j - 1), qtw(j - 1), rbw(j - 1));
      const float inner = g.rdzu[k] * (ppw(j) - ppw(j - 1)) - (g.fzm[k] * dk + g.fzp[k] * dm);
      out = m ? -(cq.a[j] * inner) : -inner;
    }
    er.a[j] = out;
  }
  if (tend_rho_dyn) {
    // physics hand-off: the dynamics-only tendency for the modified theta
    // rate, and the held density physics added after it
    // (hexcore/cuda_horizontal.py:1060, density_tendency(physics_tendency=))
    st4m(tend_rho_dyn + c * S + k0, tr, k0, 0, g.L);
    if (phys_rho) {
      const V4 pr = ld4(phys_rho + c * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) tr.a[j] = tr.a[j] + pr.a[j];
    }
  }
  st4m(tend_rho + c * S + k0, tr, k0, 0, g.L);
  st4m(euler_rw + c * S + k0, er, k0, 0, g.L + 1);
}

// ------------------------------------------------- stage tendencies
// hexcore/dynamics.py:86 mass_flux_divergence of the stage rho*u.
__global__ void HEX_VEC_BOUNDS kv_hdiv(HexGeo g, const float* __restrict__ ru, float* __restrict__ hdiv) {
  HEX_VEC_PARALLEL(g.nC)
  st4m(hdiv + ent * g.S + k0, mass_flux_div4(g, ru, ent, k0), k0, 0, g.L);
}

// Third-order edge values of theta_m (levels) and w (interfaces):
// hexcore/driver.py:1023-1034 and :1159-1172.
__global__ void __launch_bounds__(256, HEX_EDGE_ADV_MIN_BLOCKS) kv_edge_adv(HexGeo g, const float* __restrict__ ru, const float* __restrict__ theta,
                            const float* __restrict__ w, float* __restrict__ edge_theta,
                            float* __restrict__ edge_w) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  const int n = g.n_adv[e];
  const int* cells = g.adv_cells + (size_t)e * g.advW;
  const float* a1 = g.adv + (size_t)e * g.advW;
  const float* a3 = g.adv3 + (size_t)e * g.advW;
  const V4 r = ld4(ru + e * S + k0);
  const float rm = k0 > 0 ? ru[e * S + k0 - 1] : 0.0f;
#if HEX_PM_SELECT_EDGE_ADV
  // The stencil weight A + (coef3 sign(v)) B is A + X or A - X with
  // X = coef3 B (a product's sign is exact, and a - b == a + (-b)): both are
  // formed once per stencil point and each level selects by the sign bit
  // of its velocity, the words of the per-level form.
  bool nt[4], nw[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    nt[j] = signbit(r.a[j]);
    const float rprev = j == 0 ? rm : r.a[j - 1];
    nw[j] = signbit(g.fzm[k] * r.a[j] + g.fzp[k] * rprev);
  }
  V4 at = v4zero(), aw = v4zero();
  HEX_UNROLL_N(HEX_EDGE_ADV_UNROLL)
  for (int s = 0; s < n; ++s) {
    const int cs = cells[s] * S + k0;
    const float A = a1[s], X = g.coef3 * a3[s];
    const float P = A + X, M = A - X;
    const V4 th = ld4(theta + cs), wv = ld4(w + cs);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      at.a[j] = at.a[j] + (nt[j] ? M : P) * th.a[j];
      aw.a[j] = aw.a[j] + (nw[j] ? M : P) * wv.a[j];
    }
  }
#else
  float ct[4], cw[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    ct[j] = g.coef3 * copysignf(1.0f, r.a[j]);
    const float rprev = j == 0 ? rm : r.a[j - 1];
    const float rui = g.fzm[k] * r.a[j] + g.fzp[k] * rprev;
    cw[j] = g.coef3 * copysignf(1.0f, rui);
  }
  V4 at = v4zero(), aw = v4zero();
  HEX_UNROLL_N(HEX_EDGE_ADV_UNROLL)
  for (int s = 0; s < n; ++s) {
    const int cs = cells[s] * S + k0;
    const float A = a1[s], B = a3[s];
    const V4 th = ld4(theta + cs), wv = ld4(w + cs);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      at.a[j] = at.a[j] + (A + ct[j] * B) * th.a[j];
      aw.a[j] = aw.a[j] + (A + cw[j] * B) * wv.a[j];
    }
  }
#endif
  st4m(edge_theta + e * S + k0, at, k0, 0, g.L);
  st4m(edge_w + e * S + k0, aw, k0, 1, g.L);
}

// wduz at interface j of the edge (hexcore/dynamics.py:227), from windows of
// u (edge) and rw at both cells; d = j - k0 in [0, 4].
__device__ __forceinline__ float wduz_win(const HexGeo& g, const Win& uw, const Win& r0, const Win& r1, int k0,
                                          int d) {
  const int j = k0 + d, L = g.L;
  if (j <= 0 || j >= L) return 0.0f;
  const float rwe = 0.5f * (r0(d) + r1(d));
  if (j == 1 || j == L - 1) return rwe * (g.fzm[j] * uw(d) + g.fzp[j] * uw(d - 1));
  return flux3f(uw(d - 2), uw(d - 1), uw(d), uw(d + 1), rwe, 1.0f);
}

// tend_ru: vertical transport + hexcore/dynamics_v841.py:121 momentum + saved Euler.
// RAYLEIGH: the upper Rayleigh damping of u is compiled in (an instance
// without it keeps the common path's registers).
template <bool RAYLEIGH>
__global__ void __launch_bounds__(256, HEX_TEND_U_MIN_BLOCKS) kv_tend_u(HexGeo g, const float* __restrict__ u, const float* __restrict__ rw,
                          const float* __restrict__ rho, const float* __restrict__ pv_edge,
                          const float* __restrict__ ke, const float* __restrict__ hdiv,
                          const float* __restrict__ euler_ru, float* __restrict__ tend_ru,
                          const float* __restrict__ phys_ru, float first_dts, float* __restrict__ ru_p0,
                          float* __restrict__ ru_avg0) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
  const Win uw = win(u + e * S, k0, S);
  const Win r0 = win(rw + c0 * S, k0, S), r1 = win(rw + c1 * S, k0, S);
  float wd[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) wd[d] = wduz_win(g, uw, r0, r1, k0, d);
  const int n = g.neoe[e];
  const V4 pve = ld4(pv_edge + e * S + k0);
  V4 q = v4zero();
  HEX_UNROLL_N(HEX_TEND_U_UNROLL)
  for (int s = 0; s < n; ++s) {
    const int nb = g.eoe[e * g.maxE2 + s];
    const float w = g.weights[e * g.maxE2 + s];
    const V4 un = ld4(u + nb * S + k0), pn = ld4(pv_edge + nb * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float work_pv = 0.5f * (pve.a[j] + pn.a[j]);
      q.a[j] = q.a[j] + w * un.a[j] * work_pv;
    }
  }
  // Perturbation-Coriolis subtraction.  With all-zero reference winds every
  // subtracted term is a signed zero, and q - (+-0) == q bit for bit unless
  // q is itself zero or NaN, so the loop runs only when it can change a
  // stored bit: the padding levels k >= L (whose u is zero) are not tested,
  // or every warp holding a column's top chunk would run it.
  bool need = !g.winds_zero;
#pragma unroll
  for (int j = 0; j < 4; ++j) need = need || (k0 + j < g.L && !(fabsf(q.a[j]) > 0.0f));
  if (need) {
    const float fe = g.f_edge[e];
    HEX_UNROLL_N(HEX_TEND_U_UNROLL)
    for (int s = 0; s < n; ++s) {
      const int nb = g.eoe[e * g.maxE2 + s];
      const float w = g.weights[e * g.maxE2 + s];
      const float ca = g.cos_angle[nb], sa = g.sin_angle[nb];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + j;
        const float ref_u = g.u_init[k] * ca - g.v_init[k] * sa;
        q.a[j] = q.a[j] - w * ref_u * fe;
      }
    }
  }
  const V4 rh0 = ld4(rho + c0 * S + k0), rh1 = ld4(rho + c1 * S + k0);
  const V4 ke0 = ld4(ke + c0 * S + k0), ke1 = ld4(ke + c1 * S + k0);
  const V4 hd0 = ld4(hdiv + c0 * S + k0), hd1 = ld4(hdiv + c1 * S + k0);
  const V4 eu = ld4(euler_ru + e * S + k0);
  const float idc = g.inv_dc[e];
  V4 out;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    const float tv = -g.rdzw[k] * (wd[j + 1] - wd[j]);
    const float rho_edge = 0.5f * (rh0.a[j] + rh1.a[j]);
    float horizontal = rho_edge * (q.a[j] - (ke1.a[j] - ke0.a[j]) * idc);
    horizontal = tv + horizontal;
    float res = horizontal - uw(j) * 0.5f * (hd0.a[j] + hd1.a[j]);
    if (RAYLEIGH && k >= g.L - g.rayleigh_levels && k < g.L) {
      // Rayleigh damping of u before the saved Euler term
      // (hexcore/native/upper_damping.rs, mpas_atm_time_integration.F:6610-6627)
      const float coefficient = (float)(k - (g.L - g.rayleigh_levels) + 1) * g.rayleigh_inverse;
      res = res - (rho_edge * uw(j)) * coefficient;
    }
    out.a[j] = res + eu.a[j];
  }
  if (phys_ru) {
    // (tend + saved Euler) + physics (hexcore/cuda_driver.py:4445, add_pair)
    const V4 pu = ld4(phys_ru + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) out.a[j] = out.a[j] + pu.a[j];
  }
  st4m(tend_ru + e * S + k0, out, k0, 0, g.L);
  if (ru_p0) {
    // the stage's first acoustic substep starts from ru_p = ru_avg = dts x
    // tend_ru (kv_ac_edge mode 0), formed here from the tendency in registers
    V4 r;
#pragma unroll
    for (int j = 0; j < 4; ++j) r.a[j] = first_dts * out.a[j];
    st4m(ru_p0 + e * S + k0, r, k0, 0, g.L);
    st4m(ru_avg0 + e * S + k0, r, k0, 0, g.L);
  }
}

// theta vertical flux at interface j = k0 + d (hexcore/driver.py:1048-1076).
__device__ __forceinline__ float vflux_theta_win(const HexGeo& g, const Win& th, const Win& ths, const Win& rw,
                                                 const Win& rws, int k0, int d) {
  const int j = k0 + d, L = g.L;
  if (j <= 0 || j >= L) return 0.0f;
  if (j == 1) {
    const float vf = rw(d) * (g.fzm[j] * th(d) + g.fzp[j] * th(d - 1));
    return vf + (rws(d) - rw(d)) * (g.fzm[j] * ths(d) + g.fzp[j] * ths(d - 1));
  }
  if (j == L - 1) return rws(d) * (g.fzm[j] * th(d) + g.fzp[j] * th(d - 1));
  const float vf = flux3f(th(d - 2), th(d - 1), th(d), th(d + 1), rw(d), g.coef3);
  return vf + (rws(d) - rw(d)) * (g.fzm[j] * ths(d) + g.fzp[j] * ths(d - 1));
}

// w vertical flux at interface j = k0 + d (hexcore/driver.py:1176-1200).
__device__ __forceinline__ float vflux_w_win(const HexGeo& g, const Win& w, const Win& rw, int k0, int d) {
  const int j = k0 + d, L = g.L;
  if (j <= 0 || j >= L) return 0.0f;
  if (j == 1 || j == L - 1) return 0.25f * (rw(d) + rw(d - 1)) * (w(d) + w(d - 1));
  return flux3f(w(d - 2), w(d - 1), w(d), w(d + 1), 0.5f * (rw(d) + rw(d - 1)), 1.0f);
}

// tend_rt (hexcore/driver.py:933), tend_rw (:1081) + Euler w, then
// hexcore/acoustic.py:246 convert_w_tendency_to_omega.
__global__ void HEX_VEC_BOUNDS kv_tend_cell(HexGeo g, const float* __restrict__ ru, const float* __restrict__ ru_s,
                             const float* __restrict__ rw, const float* __restrict__ rws,
                             const float* __restrict__ theta, const float* __restrict__ theta_s,
                             const float* __restrict__ w, const float* __restrict__ edge_theta,
                             const float* __restrict__ edge_w, const float* __restrict__ euler_rw,
                             const float* __restrict__ tend_ru, float* __restrict__ tend_rt,
                             float* __restrict__ tend_rw, int rk_step, const float* __restrict__ mix_theta,
                             HexPhysCell phys) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  const int n = g.deg[c];
  const float ia = g.inv_area[c];
  const int* eoc = g.eoc + c * g.maxE;
  const float* cs = g.csign + c * g.maxE;
  // horizontal parts: rho-theta flux divergence, RK>1 correction, w flux
  V4 res = v4zero(), hres = v4zero();
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = eoc[s];
    const float sg = cs[s];
    const V4 r = ld4(ru + e * S + k0), et = ld4(edge_theta + e * S + k0), ew = ld4(edge_w + e * S + k0);
    const float rm = k0 > 0 ? ru[e * S + k0 - 1] : 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      res.a[j] = res.a[j] - sg * r.a[j] * et.a[j];
      const float rprev = j == 0 ? rm : r.a[j - 1];
      const float rui = g.fzm[k] * r.a[j] + g.fzp[k] * rprev;
      hres.a[j] = hres.a[j] - sg * rui * ew.a[j];
    }
  }
  if (rk_step > 1) {
    const V4 tc = ld4(theta_s + c * S + k0);
    HEX_GATHER
    for (int s = 0; s < n; ++s) {
      const int e = eoc[s];
      const int e0 = g.coe[2 * e], e1 = g.coe[2 * e + 1];
      const float dvs = cs[s] * g.dv[e];
      const V4 r = ld4(ru + e * S + k0), rs = ld4(ru_s + e * S + k0);
      const V4 tn = ld4(theta_s + (e0 == c ? e1 : e0) * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        // theta_s[e1] + theta_s[e0] with this cell as one operand (IEEE
        // addition commutes, so the operand order changes no bit)
        const float corr = dvs * (rs.a[j] - r.a[j]) * 0.5f * (tn.a[j] + tc.a[j]);
        res.a[j] = res.a[j] - corr;
      }
    }
  }
  const Win th = win(theta + c * S, k0, S), ths = win(theta_s + c * S, k0, S);
  const Win rww = win(rw + c * S, k0, S), rwsw = win(rws + c * S, k0, S);
  const Win ww = win(w + c * S, k0, S), zzw = win(g.zz + c * S, k0, S);
  const V4 er = ld4(euler_rw + c * S + k0);
  float vt[5], vw[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    vt[d] = vflux_theta_win(g, th, ths, rww, rwsw, k0, d);
    vw[d] = vflux_w_win(g, ww, rww, k0, d);
  }
  V4 trt, trw;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    trt.a[j] = res.a[j] * ia - g.rdzw[k] * (vt[j + 1] - vt[j]);
    if (k >= 1 && k < L) {
      const float rsw = hres.a[j] * ia - g.rdzu[k] * (vw[j + 1] - vw[j]);
      trw.a[j] = rsw + er.a[j];
    } else {
      trw.a[j] = 0.0f + er.a[j];
    }
  }
  // omega conversion (interfaces 1..L-1)
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = eoc[s];
    const float sg = cs[s];
    const V4 t = ld4(tend_ru + e * S + k0);
    const float tm = k0 > 0 ? tend_ru[e * S + k0 - 1] : 0.0f;
    const int zi = (c * g.maxE + s) * S + k0;
    const V4 zb = ld4(g.zb + zi), zb3 = ld4(g.zb3 + zi);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      if (k >= 1 && k < L) {
        const float tprev = j == 0 ? tm : t.a[j - 1];
        const float flux = sg * (g.fzm[k] * t.a[j] + g.fzp[k] * tprev);
        const float up = copysignf(1.0f, t.a[j]);
        trw.a[j] = trw.a[j] - (zb.a[j] + up * zb3.a[j]) * flux;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    if (k >= 1 && k < L) trw.a[j] = trw.a[j] * (g.fzm[k] * zzw(j) + g.fzp[k] * zzw(j - 1));
    if (k > L) trw.a[j] = 0.0f;
  }
  if (phys.on) {
    // physics hand-off (hexcore/cuda_driver.py:4459-4494): at RK stage 3 the
    // modified theta dynamics rate (tend_rt - tend_rho theta_m) / rho of the
    // dynamics-only tendencies, then the lagged diabatic heating rho x dth
    const V4 rh = ld4(phys.rho + c * S + k0);
    if (phys.mod_rate) {
      const V4 td = ld4(phys.tend_rho_dyn + c * S + k0);
      V4 mr;
#pragma unroll
      for (int j = 0; j < 4; ++j) mr.a[j] = (trt.a[j] - td.a[j] * th(j)) / rh.a[j];
      st4m(phys.mod_rate + c * S + k0, mr, k0, 0, g.L);
    }
    if (phys.dth) {
      const V4 dth = ld4(phys.dth + c * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) trt.a[j] = trt.a[j] + rh.a[j] * dth.a[j];
    }
  }
  if (mix_theta) {
    // hexcore/driver.py:2967: the saved horizontal theta mixing
    const V4 mt = ld4(mix_theta + c * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) trt.a[j] = trt.a[j] + mt.a[j];
  }
  if (phys.rt) {
    const V4 pt = ld4(phys.rt + c * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) trt.a[j] = trt.a[j] + pt.a[j];
  }
  st4m(tend_rt + c * S + k0, trt, k0, 0, g.L);
  st4m(tend_rw + c * S + k0, trw, k0, 0, g.L + 1);
}

// ------------------------------------------------- horizontal mixing
// 2-D Smagorinsky mixing of the dynamics subcycle's start state
// (hexcore/driver.py:2826-2880), v8.4.1 stored-inverse arithmetic.

// NumPy minimum: NaN if either operand is NaN, else the smaller.
__device__ __forceinline__ float np_min(float a, float b) { return a != a ? a : (b != b ? b : (b < a ? b : a)); }

// hexcore/mixing_v841.py:615 smagorinsky_2d: kdiff of every cell level from
// the deformation of the edge normal (u) and tangential (v) velocities.
__global__ void HEX_VEC_BOUNDS kv_smag_kdiff(HexGeo g, const float* __restrict__ u, const float* __restrict__ v,
                              float* __restrict__ kdiff) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S;
  const int n = g.deg[c];
  V4 dudx = v4zero(), dudy = v4zero(), dvdx = v4zero(), dvdy = v4zero();
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float c2 = g.deform_c2[c * g.maxE + s], s2 = g.deform_s2[c * g.maxE + s];
    const float ccs = g.deform_cs[c * g.maxE + s];
    const V4 ue = ld4(u + e * S + k0), ve = ld4(v + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      dudx.a[j] = (dudx.a[j] + c2 * ue.a[j]) - ccs * ve.a[j];
      dudy.a[j] = (dudy.a[j] + ccs * ue.a[j]) - s2 * ve.a[j];
      dvdx.a[j] = (dvdx.a[j] + ccs * ue.a[j]) + c2 * ve.a[j];
      dvdy.a[j] = (dvdy.a[j] + s2 * ue.a[j]) + ccs * ve.a[j];
    }
  }
  V4 kd;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float d11 = 2.0f * dudx.a[j], d22 = 2.0f * dvdy.a[j], d12 = dudy.a[j] + dvdx.a[j];
    const float diff = d11 - d22;
    const float strain = sqrtf(0.25f * (diff * diff) + d12 * d12);
    kd.a[j] = np_min(g.smag_strain_scale * strain, g.smag_ceiling);
    const int k = k0 + j;
    if (k >= g.L - g.cam_levels && k < g.L) {
      // CAM floor of the diffusivity (hexcore/native/upper_damping.rs,
      // mpas_atm_time_integration.F:6401-6403)
      const float floor_k = g.cam_base * (1.0f - (float)(g.L - 1 - k) / (float)g.cam_levels);
      kd.a[j] = fmaxf(kd.a[j], floor_k);
    }
  }
  st4m(kdiff + c * S + k0, kd, k0, 0, g.L);
}

// hexcore/mixing.py:391-474 second-order momentum filter: delsq_u and the
// Euler u term plus rho_edge kdiff delsq_u meshScalingDel2 (rho_edge the
// diagnostics' h_edge of the subcycle's start density).
__global__ void HEX_VEC_BOUNDS kv_mix_edge2(HexGeo g, const float* __restrict__ div, const float* __restrict__ vort,
                             const float* __restrict__ kdiff, const float* __restrict__ rho,
                             const float* __restrict__ euler_ru, float* __restrict__ delsq_u,
                             float* __restrict__ mix_u) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  const int i0 = g.coe[2 * e] * S + k0, i1 = g.coe[2 * e + 1] * S + k0;
  const int j0 = g.voe[2 * e] * S + k0, j1 = g.voe[2 * e + 1] * S + k0;
  const V4 d0 = ld4(div + i0), d1 = ld4(div + i1), z0 = ld4(vort + j0), z1 = ld4(vort + j1);
  const V4 k0v = ld4(kdiff + i0), k1v = ld4(kdiff + i1), r0 = ld4(rho + i0), r1 = ld4(rho + i1);
  const V4 eu = ld4(euler_ru + e * S + k0);
  const float idc = g.inv_dc[e], idv = g.inv_dv_lim[e], del2 = g.mix_del2[e];
  V4 dq, mu;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float diffusion = (d1.a[j] - d0.a[j]) * idc - (z1.a[j] - z0.a[j]) * idv;
    dq.a[j] = 0.0f + diffusion;
    const float h = 0.5f * (r0.a[j] + r1.a[j]);
    const float kdu = 0.5f * (k0v.a[j] + k1v.a[j]);
    mu.a[j] = eu.a[j] + h * kdu * diffusion * del2;
  }
  st4m(delsq_u + e * S + k0, dq, k0, 0, g.L);
  st4m(mix_u + e * S + k0, mu, k0, 0, g.L);
}

// hexcore/mixing.py:533 (w, interfaces 1..L-1) and :638 (theta) second-order
// filters of a cell, with their Laplacians delsq_w and delsq_theta.
#ifndef HEX_MIX_CELL2_MIN_BLOCKS
#define HEX_MIX_CELL2_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(256, HEX_MIX_CELL2_MIN_BLOCKS) kv_mix_cell2(HexGeo g, const float* __restrict__ kdiff, const float* __restrict__ rho,
                             const float* __restrict__ w, const float* __restrict__ theta,
                             float* __restrict__ w_mix, float* __restrict__ delsq_w,
                             float* __restrict__ theta_mix, float* __restrict__ delsq_theta) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  const int n = g.deg[c];
  const float ia = g.inv_area[c];
  V4 tw = v4zero(), dw = v4zero(), tt = v4zero(), dt = v4zero();
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
    const float sg = g.csign[c * g.maxE + s];
    const float del2 = g.mix_del2[e];
    const float esw = 0.5f * ia * sg * g.dv[e] * g.inv_dc[e];
    const float est = ia * sg * g.dv[e] * g.inv_dc[e];
    const V4 r0 = ld4(rho + c0 * S + k0), r1 = ld4(rho + c1 * S + k0);
    const V4 kd0 = ld4(kdiff + c0 * S + k0), kd1 = ld4(kdiff + c1 * S + k0);
    const V4 w0 = ld4(w + c0 * S + k0), w1 = ld4(w + c1 * S + k0);
    const V4 t0 = ld4(theta + c0 * S + k0), t1 = ld4(theta + c1 * S + k0);
    // level k0-1 of rho and kdiff (for the interface below the chunk)
    const float rm0 = k0 > 0 ? rho[c0 * S + k0 - 1] : 0.0f, rm1 = k0 > 0 ? rho[c1 * S + k0 - 1] : 0.0f;
    const float km0 = k0 > 0 ? kdiff[c0 * S + k0 - 1] : 0.0f, km1 = k0 > 0 ? kdiff[c1 * S + k0 - 1] : 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      const float h = 0.5f * (r0.a[j] + r1.a[j]);
      if (k >= 1 && k < L) {
        const float hm = j == 0 ? 0.5f * (rm0 + rm1) : 0.5f * (r0.a[j - 1] + r1.a[j - 1]);
        const float kdm0 = j == 0 ? km0 : kd0.a[j - 1], kdm1 = j == 0 ? km1 : kd1.a[j - 1];
        const float flux = esw * (h + hm) * (w1.a[j] - w0.a[j]);
        dw.a[j] = dw.a[j] + flux;
        const float sum_k = kd0.a[j] + kd1.a[j] + kdm0 + kdm1;
        tw.a[j] = tw.a[j] + flux * del2 * 0.25f * sum_k;
      }
      const float ft = est * (t1.a[j] - t0.a[j]) * h;
      dt.a[j] = dt.a[j] + ft;
      tt.a[j] = tt.a[j] + ft * 0.5f * (kd0.a[j] + kd1.a[j]) * del2;
    }
  }
  st4m(w_mix + c * S + k0, tw, k0, 0, L + 1);
  st4m(delsq_w + c * S + k0, dw, k0, 0, L + 1);
  st4m(theta_mix + c * S + k0, tt, k0, 0, L);
  st4m(delsq_theta + c * S + k0, dt, k0, 0, L);
}

// hexcore/mixing.py:464-476: the Laplacians of delsq_u at vertices
// (vorticity form) and cells (divergence form).
__global__ void HEX_VEC_BOUNDS kv_mix_lap_vertex(HexGeo g, const float* __restrict__ delsq_u,
                                  float* __restrict__ delsq_vort) {
  HEX_VEC_PARALLEL(g.nV)
  const int v = ent, S = g.S;
  V4 acc = v4zero();
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int e = g.eov[3 * v + s];
    const float factor = g.inv_area_tri[v] * g.dc[e] * g.vsign[3 * v + s];
    const V4 d = ld4(delsq_u + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) acc.a[j] = acc.a[j] + factor * d.a[j];
  }
  st4m(delsq_vort + v * S + k0, acc, k0, 0, g.L);
}
__global__ void HEX_VEC_BOUNDS kv_mix_lap_cell(HexGeo g, const float* __restrict__ delsq_u,
                                float* __restrict__ delsq_div) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S;
  const int n = g.deg[c];
  V4 acc = v4zero();
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float factor = g.inv_area[c] * g.dv[e] * g.csign[c * g.maxE + s];
    const V4 d = ld4(delsq_u + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) acc.a[j] = acc.a[j] + factor * d.a[j];
  }
  st4m(delsq_div + c * S + k0, acc, k0, 0, g.L);
}

// hexcore/mixing.py:478-490 fourth-order momentum filter (subtracted).
__global__ void HEX_VEC_BOUNDS kv_mix_edge4(HexGeo g, const float* __restrict__ rho,
                             const float* __restrict__ delsq_div, const float* __restrict__ delsq_vort,
                             float* __restrict__ mix_u) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  const int i0 = g.coe[2 * e] * S + k0, i1 = g.coe[2 * e + 1] * S + k0;
  const int j0 = g.voe[2 * e] * S + k0, j1 = g.voe[2 * e + 1] * S + k0;
  const V4 d0 = ld4(delsq_div + i0), d1 = ld4(delsq_div + i1);
  const V4 z0 = ld4(delsq_vort + j0), z1 = ld4(delsq_vort + j1);
  const V4 r0 = ld4(rho + i0), r1 = ld4(rho + i1);
  const float scale = g.mix_del4[e] * g.smag_h4;
  const float r_dc = scale * g.smag_div_factor * g.inv_dc[e];
  const float r_dv = scale * g.inv_dv_lim[e];
  V4 mu = ld4rw(mix_u + e * S + k0);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float h = 0.5f * (r0.a[j] + r1.a[j]);
    const float diffusion = h * ((d1.a[j] - d0.a[j]) * r_dc - (z1.a[j] - z0.a[j]) * r_dv);
    mu.a[j] = mu.a[j] - diffusion;
  }
  st4m(mix_u + e * S + k0, mu, k0, 0, g.L);
}

// hexcore/mixing.py:576-590 and :719-733 fourth-order w and theta filters
// (when visc4 > 0), then the saved w term euler_rw + w filter (driver.py:2870).
__global__ void HEX_VEC_BOUNDS kv_mix_cell4(HexGeo g, const float* __restrict__ delsq_w,
                             const float* __restrict__ delsq_theta, const float* __restrict__ euler_rw,
                             const float* __restrict__ w_mix, float* __restrict__ theta_mix,
                             float* __restrict__ mix_w) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  V4 tw = ld4(w_mix + c * S + k0), tt = ld4rw(theta_mix + c * S + k0);
  if (g.smag_h4 > 0.0f) {
    const int n = g.deg[c];
    const float scale = g.smag_h4 * g.inv_area[c];
    HEX_GATHER
    for (int s = 0; s < n; ++s) {
      const int e = g.eoc[c * g.maxE + s];
      const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
      const float es = g.mix_del4[e] * scale * g.dv[e] * g.csign[c * g.maxE + s] * g.inv_dc[e];
      const V4 w0 = ld4(delsq_w + c0 * S + k0), w1 = ld4(delsq_w + c1 * S + k0);
      const V4 t0 = ld4(delsq_theta + c0 * S + k0), t1 = ld4(delsq_theta + c1 * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + j;
        if (k >= 1 && k < L) tw.a[j] = tw.a[j] - es * (w1.a[j] - w0.a[j]);
        tt.a[j] = tt.a[j] - es * (t1.a[j] - t0.a[j]);
      }
    }
  }
  const V4 er = ld4(euler_rw + c * S + k0);
  V4 mw;
#pragma unroll
  for (int j = 0; j < 4; ++j) mw.a[j] = er.a[j] + tw.a[j];
  st4m(theta_mix + c * S + k0, tt, k0, 0, L);
  st4m(mix_w + c * S + k0, mw, k0, 0, L + 1);
}

// ------------------------------------------------------------- acoustic

// One acoustic edge pass: the 3-D divergence damping of the previous
// substep (hexcore/mixing.py:851, stored inverse of dts), then the ru_p
// update of this substep (hexcore/acoustic_v841.py:416-460).  mode 0: first
// substep (ru_p = dts*tend_ru); 1: damping + update; 2: damping only.
__global__ void HEX_VEC_BOUNDS kv_ac_edge(HexGeo g, int mode, int old_is_zero, float dts, float inv_dts,
                           const float* __restrict__ tend_ru, const float* __restrict__ rtpp_new,
                           const float* __restrict__ rtpp_old, const float* __restrict__ rho_pp,
                           const float* __restrict__ theta_s, const float* __restrict__ exner_s,
                           const float* __restrict__ cqu, float* __restrict__ ru_p, float* __restrict__ ru_avg) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  const int jj = e * S + k0;
  if (mode == 0) {
    const V4 t = ld4(tend_ru + jj);
    V4 r;
#pragma unroll
    for (int j = 0; j < 4; ++j) r.a[j] = dts * t.a[j];
    st4m(ru_p + jj, r, k0, 0, g.L);
    st4m(ru_avg + jj, r, k0, 0, g.L);
    return;
  }
  const int i0 = g.coe[2 * e] * S + k0, i1 = g.coe[2 * e + 1] * S + k0;
  // smdiv_base * (1/dts), the damping coefficient of the edge's mesh
  const float damp_coef = g.smdiv_edge[e] * inv_dts;
  V4 r = ld4rw(ru_p + jj);
  const V4 n0 = ld4(rtpp_new + i0), n1 = ld4(rtpp_new + i1);
  const V4 o0 = old_is_zero ? v4zero() : ld4(rtpp_old + i0);
  const V4 o1 = old_is_zero ? v4zero() : ld4(rtpp_old + i1);
  const V4 t0 = ld4(theta_s + i0), t1 = ld4(theta_s + i1);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float d0 = n0.a[j] - o0.a[j];
    const float d1 = n1.a[j] - o1.a[j];
    r.a[j] = r.a[j] + damp_coef * (d0 - d1) * (1.0f - 0.0f) / (t0.a[j] + t1.a[j]);
  }
  if (mode == 1) {
    const V4 z0 = ld4(g.zz + i0), z1 = ld4(g.zz + i1), x0 = ld4(exner_s + i0), x1 = ld4(exner_s + i1);
    const V4 p0 = ld4(rho_pp + i0), p1 = ld4(rho_pp + i1);
    const V4 cq = ld4(cqu + jj), zx = ld4(g.zxu + jj), t = ld4(tend_ru + jj);
    V4 av = ld4rw(ru_avg + jj);
    const float idc = g.inv_dc[e];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float pg = (n1.a[j] - n0.a[j]) * idc / (0.5f * (z1.a[j] + z0.a[j]));
      pg = cq.a[j] * 0.5f * g.c2 * (x0.a[j] + x1.a[j]) * pg;
      pg = pg + 0.5f * zx.a[j] * g.g * (p0.a[j] + p1.a[j]);
      r.a[j] = r.a[j] + dts * (t.a[j] - pg);
      av.a[j] = av.a[j] + r.a[j];
    }
    st4m(ru_avg + jj, av, k0, 0, g.L);
  }
  st4m(ru_p + jj, r, k0, 0, g.L);
}

// ---------------------------------------------------------- stage recovery
// hexcore/driver.py:3166-3292 stage recovery, edge part: ru = ru_s + ru_p,
// u = 2 ru / (rho1 + rho2) (hexcore/driver.py:866), and the split mass-flux
// average (hexcore/integration.py:27,58).
// damp: the divergence damping of the stage's last acoustic substep
// (kv_ac_edge mode 2: rtpp_new/rtpp_old its output/input, old_is_zero when
// it was the first) is applied to ru_p here, stored, and recovered from.
__global__ void HEX_VEC_BOUNDS kv_recover_edge(HexGeo g, const float* __restrict__ ru_s, float* ru_p,
                                const float* __restrict__ ru_avg, const float* __restrict__ rp_s,
                                const float* __restrict__ rho_pp, float* __restrict__ ru_out,
                                float* __restrict__ u_out, float* __restrict__ flux_u, int flux_mode,
                                float inv_steps, float inv_splits, int damp, int old_is_zero, float inv_dts,
                                const float* __restrict__ rtpp_new, const float* __restrict__ rtpp_old,
                                const float* __restrict__ theta_s) {
  HEX_VEC_PARALLEL(g.nE)
  const int e = ent, S = g.S;
  const int jj = e * S + k0;
  const int i0 = g.coe[2 * e] * S + k0, i1 = g.coe[2 * e + 1] * S + k0;
  V4 rp = ld4rw(ru_p + jj);
  if (damp) {
    const float damp_coef = g.smdiv_edge[e] * inv_dts;
    const V4 n0 = ld4(rtpp_new + i0), n1 = ld4(rtpp_new + i1);
    const V4 o0 = old_is_zero ? v4zero() : ld4(rtpp_old + i0);
    const V4 o1 = old_is_zero ? v4zero() : ld4(rtpp_old + i1);
    const V4 t0 = ld4(theta_s + i0), t1 = ld4(theta_s + i1);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float d0 = n0.a[j] - o0.a[j];
      const float d1 = n1.a[j] - o1.a[j];
      rp.a[j] = rp.a[j] + damp_coef * (d0 - d1) * (1.0f - 0.0f) / (t0.a[j] + t1.a[j]);
    }
    st4m(ru_p + jj, rp, k0, 0, g.L);
  }
  const V4 a0 = ld4(rp_s + i0), a1 = ld4(rp_s + i1), b0 = ld4(rho_pp + i0), b1 = ld4(rho_pp + i1);
  const V4 c0 = ld4(g.rho_base + i0), c1 = ld4(g.rho_base + i1);
  const V4 rs = ld4(ru_s + jj);
  V4 ru, uo;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float rho0 = a0.a[j] + b0.a[j] + c0.a[j];
    const float rho1 = a1.a[j] + b1.a[j] + c1.a[j];
    ru.a[j] = rs.a[j] + rp.a[j];
    uo.a[j] = 2.0f * ru.a[j] / (rho0 + rho1);
  }
  st4m(ru_out + jj, ru, k0, 0, g.L);
  st4m(u_out + jj, uo, k0, 0, g.L);
  if (flux_mode & 4) {
    const V4 av = ld4(ru_avg + jj);
    const V4 old = (flux_mode & 1) ? v4zero() : ld4rw(flux_u + jj);
    V4 acc;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float f = rs.a[j] + av.a[j] * inv_steps;
      float a = (flux_mode & 1) ? f : f + old.a[j];
      if (flux_mode & 2) a = a * inv_splits;
      acc.a[j] = a;
    }
    st4m(flux_u + jj, acc, k0, 0, g.L);
  }
}

// hexcore/driver.py:3166-3292 stage recovery, cell part: candidate state,
// rw end conditions, theta_m, Exner and p' at stage 3, w from
// hexcore/terrain.py:491 recover_velocities, and the split w-flux average.
__global__ void HEX_VEC_BOUNDS kv_recover_cell(HexGeo g, int stage3, const float* __restrict__ rp_s,
                                const float* __restrict__ rtp_s, const float* __restrict__ rw_s,
                                const float* __restrict__ rho_pp, const float* __restrict__ rtpp,
                                const float* __restrict__ rw_p, const float* __restrict__ ww_avg,
                                const float* __restrict__ ru_new, HexState out, HexSide side,
                                float* __restrict__ flux_w, int flux_mode, float inv_steps, float inv_splits,
                                int* flag, float* __restrict__ hdiv_next) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  const int ii = c * S + k0;
  // candidate density on the window k0-4 .. k0+7 (recomputed, not read back)
  const Win rpw = win(rp_s + c * S, k0, S), ppw = win(rho_pp + c * S, k0, S), rbw = win(g.rho_base + c * S, k0, S);
  float rho_w[12];
#pragma unroll
  for (int d = -4; d < 8; ++d) rho_w[d + 4] = rpw(d) + ppw(d) + rbw(d);
  {
    const V4 tp = ld4(rtp_s + ii), tq = ld4(rtpp + ii), tb = ld4(g.rtheta_base + ii);
    V4 rho, rt, rp, rtp, th;
    bool bad = false;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      rp.a[j] = rpw(j) + ppw(j);
      rtp.a[j] = tp.a[j] + tq.a[j];
      rho.a[j] = rp.a[j] + rbw(j);
      rt.a[j] = rtp.a[j] + tb.a[j];
      th.a[j] = rt.a[j] / rho.a[j];
      if (k0 + j < L && (!(rho.a[j] > 0.0f) || !(rt.a[j] > 0.0f))) bad = true;
    }
    if (bad) atomicOr(flag, HEX_FLAG_DENSITY);
    st4m(out.rho + ii, rho, k0, 0, g.L);
    st4m(out.rho_theta + ii, rt, k0, 0, g.L);
    st4m(side.rho_p + ii, rp, k0, 0, g.L);
    st4m(side.rtheta_p + ii, rtp, k0, 0, g.L);
    st4m(side.theta_m + ii, th, k0, 0, g.L);
    if (stage3) {
      const V4 zz = ld4(g.zz + ii), eb = ld4(g.exner_base + ii);
      V4 ex, pp;
      int badp = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (k0 + j < L) {
          int b = 0;
          ex.a[j] = hexdyn_powf::powf_gnu(zz.a[j] * g.r_over_p0 * rt.a[j], g.kappa, &b);
          badp |= b;
          pp.a[j] = zz.a[j] * g.rgas * (ex.a[j] * rtp.a[j] + tb.a[j] * (ex.a[j] - eb.a[j]));
        } else {
          ex.a[j] = 0.0f;
          pp.a[j] = 0.0f;
        }
      }
      if (badp) atomicOr(flag, HEX_FLAG_POWF);
      st4m(side.exner + ii, ex, k0, 0, g.L);
      st4m(side.pressure_p + ii, pp, k0, 0, g.L);
    }
  }
  // rw, w, split flux (interfaces)
  const V4 rs = ld4(rw_s + ii), rq = ld4(rw_p + ii);
  V4 rwv, wv;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    rwv.a[j] = (k == 0 || k == L || k > L) ? 0.0f : rs.a[j] + rq.a[j];
  }
  st4m(out.rho_w + ii, rwv, k0, 0, g.L + 1);
  const int n = g.deg[c];
  const Win zzw = win(g.zz + c * S, k0, S);
  float acc[4];
  bool bottom = k0 == 0;
  float bacc = 0.0f;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    acc[j] = 0.0f;
    if (k >= 1 && k < L) acc[j] = rwv.a[j] / (g.fzm[k] * zzw(j) + g.fzp[k] * zzw(j - 1));
  }
  // the next stage's mass-flux divergence of ru_new (mass_flux_div4, the
  // same operands in the same order) accumulates in the same edge loop
  V4 hd = v4zero();
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float sign = g.csign[c * g.maxE + s];
    const V4 r = ld4(ru_new + e * S + k0);
    const float sd = sign * g.dv[e];
#pragma unroll
    for (int j = 0; j < 4; ++j) hd.a[j] = hd.a[j] + sd * r.a[j];
    const float rm = k0 > 0 ? ru_new[e * S + k0 - 1] : 0.0f;
    const int zi = (c * g.maxE + s) * S + k0;
    const V4 zb = ld4(g.zb + zi), zb3 = ld4(g.zb3 + zi);
    if (bottom) {
      const float flux = g.cf1 * r.a[0] + g.cf2 * r.a[1] + g.cf3 * r.a[2];
      bacc = bacc + sign * (zb.a[0] + copysignf(1.0f, flux) * zb3.a[0]) * flux;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      if (k >= 1 && k < L) {
        const float rprev = j == 0 ? rm : r.a[j - 1];
        const float flux = g.fzm[k] * r.a[j] + g.fzp[k] * rprev;
        acc[j] = acc[j] + sign * (zb.a[j] + copysignf(1.0f, flux) * zb3.a[j]) * flux;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    float wk = 0.0f;
    if (k == 0) {
      const float bd = g.cf1 * rho_w[4] + g.cf2 * rho_w[5] + g.cf3 * rho_w[6];
      wk = bacc / bd;
    } else if (k < L) {
      const float irho = g.fzm[k] * rho_w[j + 4] + g.fzp[k] * rho_w[j + 3];
      wk = acc[j] / irho;
    }
    wv.a[j] = wk;
  }
  st4m(side.w + ii, wv, k0, 0, g.L + 1);
  {
    const float ia = g.inv_area[c];
#pragma unroll
    for (int j = 0; j < 4; ++j) hd.a[j] = hd.a[j] * ia;
    st4m(hdiv_next + ii, hd, k0, 0, g.L);
  }
  if (flux_mode & 4) {
    const V4 av = ld4(ww_avg + ii);
    const V4 old = (flux_mode & 1) ? v4zero() : ld4rw(flux_w + ii);
    V4 fa;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float f = rs.a[j] + av.a[j] * inv_steps;
      float a = (flux_mode & 1) ? f : f + old.a[j];
      if (flux_mode & 2) a = a * inv_splits;
      fa.a[j] = a;
    }
    st4m(flux_w + ii, fa, k0, 0, g.L + 1);
  }
}

// ------------------------------------------------------------ transport
// hexcore/transport.py:1461 third-order edge values.  A thread serves
// HEX_TR_GROUP tracers at its four levels: the stencil indices, the two
// coefficient tables and the per-level weights (coefficient + sign(u) x
// third-order coefficient) are loaded and formed once per stencil cell and
// applied to every tracer of the group; block b serves tracer group
// b % groups.  mono: the monotonic source flux (velocity folded in; the
// literal ten-term association for ten-cell stencils).
#ifndef HEX_TR_GROUP
#define HEX_TR_GROUP 3
#endif
__global__ void __launch_bounds__(256, HEX_TR_EDGE_MIN_BLOCKS) kv_tr_edge(HexGeo g, int nT, int mono, const float* __restrict__ q, const float* __restrict__ hv,
                           float* __restrict__ out) {
  HEX_VEC_TRACER(g.nE, (nT + HEX_TR_GROUP - 1) / HEX_TR_GROUP)
  constexpr int TG = HEX_TR_GROUP;
  const int e = ent, S = g.S;
  const int t0 = tr * TG;
  const size_t tstride = (size_t)g.nC * S;
  const float* qg = q + (size_t)t0 * tstride + k0;
  const int n = g.n_adv[e];
  const int* cells = g.adv_cells + (size_t)e * g.advW;
  const float* a1 = g.adv + (size_t)e * g.advW;
  const float* a3 = g.adv3 + (size_t)e * g.advW;
  const V4 vel = ld4(hv + e * S + k0);
#if HEX_PM_SELECT_TR_EDGE
  // A + (coef3 sign(vel)) B as A + X or A - X, X = coef3 B (see kv_edge_adv)
  bool neg[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) neg[j] = signbit(vel.a[j]);
#define HEX_TR_WEIGHTS(s_)                                   \
  const float A = a1[s_], X = g.coef3 * a3[s_];              \
  const float P = A + X, M = A - X;                          \
  float w[4];                                                \
  _Pragma("unroll") for (int j = 0; j < 4; ++j) w[j] = neg[j] ? M : P;
#else
  float cs[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) cs[j] = g.coef3 * copysignf(1.0f, vel.a[j]);
#define HEX_TR_WEIGHTS(s_)                                   \
  const float A = a1[s_], B = a3[s_];                        \
  float w[4];                                                \
  _Pragma("unroll") for (int j = 0; j < 4; ++j) w[j] = A + cs[j] * B;
#endif
  V4 res[TG];
  if (mono && n == 10) {
    {
      const float* qc = qg + cells[0] * S;
      HEX_TR_WEIGHTS(0)
#pragma unroll
      for (int t = 0; t < TG; ++t)
        if (t0 + t < nT) {
          const V4 qv = ld4(qc + t * tstride);
#pragma unroll
          for (int j = 0; j < 4; ++j) res[t].a[j] = w[j] * qv.a[j];
        }
    }
    HEX_UNROLL_N(HEX_TR_EDGE_UNROLL)
    for (int s = 1; s < 10; ++s) {
      const float* qc = qg + cells[s] * S;
      HEX_TR_WEIGHTS(s)
#pragma unroll
      for (int t = 0; t < TG; ++t)
        if (t0 + t < nT) {
          const V4 qv = ld4(qc + t * tstride);
#pragma unroll
          for (int j = 0; j < 4; ++j) res[t].a[j] = res[t].a[j] + w[j] * qv.a[j];
        }
    }
#pragma unroll
    for (int t = 0; t < TG; ++t)
#pragma unroll
      for (int j = 0; j < 4; ++j) res[t].a[j] = vel.a[j] * res[t].a[j];
  } else {
#pragma unroll
    for (int t = 0; t < TG; ++t) res[t] = v4zero();
    HEX_UNROLL_N(HEX_TR_EDGE_UNROLL)
    for (int s = 0; s < n; ++s) {
      const float* qc = qg + cells[s] * S;
      HEX_TR_WEIGHTS(s)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (mono) w[j] = vel.a[j] * w[j];
#pragma unroll
      for (int t = 0; t < TG; ++t)
        if (t0 + t < nT) {
          const V4 qv = ld4(qc + t * tstride);
#pragma unroll
          for (int j = 0; j < 4; ++j) res[t].a[j] = res[t].a[j] + w[j] * qv.a[j];
        }
    }
  }
#pragma unroll
  for (int t = 0; t < TG; ++t)
    if (t0 + t < nT) st4m(out + (size_t)(t0 + t) * g.nE * S + e * S + k0, res[t], k0, 0, g.L);
#undef HEX_TR_WEIGHTS
}

// transport vertical flux at interface j = k0 + d (hexcore/transport.py:1389).
__device__ __forceinline__ float tr_vflux_win(const HexGeo& g, const Win& q, const Win& ww, int k0, int d) {
  const int j = k0 + d, L = g.L;
  if (j <= 0 || j >= L) return 0.0f;
  if (j == 1 || j == L - 1) return ww(d) * (g.fzm[j] * q(d) + g.fzp[j] * q(d - 1));
  const float vel = ww(d);
  const float base = vel * (7.0f * (q(d) + q(d - 1)) - (q(d + 1) + q(d - 2))) / 12.0f;
  const float corr = g.coef3 * fabsf(vel) * ((q(d + 1) - q(d - 2)) - 3.0f * (q(d) - q(d - 1))) / 12.0f;
  return base + corr;
}

// hexcore/transport.py:1649 advance_scalars (RK1/RK2 of split transport).
__global__ void __launch_bounds__(256, HEX_TR_STD_MIN_BLOCKS) kv_tr_std(HexGeo g, int nT, float step, float wn, const float* __restrict__ q_old,
                          const float* __restrict__ q_stage, const float* __restrict__ rho_old,
                          const float* __restrict__ rho_new, const float* __restrict__ hv,
                          const float* __restrict__ ww, const float* __restrict__ edge_q,
                          float* __restrict__ q_out) {
  HEX_VEC_TRACER(g.nC, nT)
  const int c = ent, S = g.S;
  const int ii = c * S + k0;
  const size_t toff = (size_t)tr * g.nC * S;
  const float* ev = edge_q + (size_t)tr * g.nE * S;
  const int n = g.deg[c];
  V4 t = v4zero();
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float ts = -g.csign[c * g.maxE + s];
    const V4 h = ld4(hv + e * S + k0), x = ld4(ev + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) t.a[j] = t.a[j] + ts * h.a[j] * x.a[j];
  }
  const float ia = g.inv_area[c];
  const Win qw = win(q_stage + toff + c * S, k0, S), www = win(ww + c * S, k0, S);
  const V4 ro = ld4(rho_old + ii), rn = ld4(rho_new + ii), qo = ld4(q_old + toff + ii);
  float vf[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) vf[d] = tr_vflux_win(g, qw, www, k0, d);
  V4 out;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    const float tt = t.a[j] * ia + 0.0f;
    const float target = (1.0f - wn) * ro.a[j] + wn * rn.a[j];
    const float num = qo.a[j] * ro.a[j] + step * (tt - g.rdzw[k] * (vf[j + 1] - vf[j]));
    out.a[j] = num * (1.0f / target);
  }
  st4m(q_out + toff + ii, out, k0, 0, g.L);
}

// hexcore/transport.py:1887-1906 split-transport target density.
__global__ void HEX_VEC_BOUNDS kv_fct_target(HexGeo g, float step, const float* __restrict__ rho_old,
                              const float* __restrict__ hv, const float* __restrict__ ww,
                              float* __restrict__ target, int* flag) {
  HEX_VEC_PARALLEL(g.nC)
  const int c = ent, S = g.S, L = g.L;
  const int ii = c * S + k0;
  const int n = g.deg[c];
  const float ia = g.inv_area[c];
  V4 hd = v4zero();
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float ts = -g.csign[c * g.maxE + s];
    const float dv = g.dv[e];
    const V4 h = ld4(hv + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) hd.a[j] = hd.a[j] + ts * h.a[j] * dv * ia;
  }
  const Win www = win(ww + c * S, k0, S);
  const V4 ro = ld4(rho_old + ii);
  V4 td;
  bool bad = false;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    td.a[j] = ro.a[j] + step * (hd.a[j] - g.rdzw[k] * (www(j + 1) - www(j)));
    if (k < L && !(td.a[j] > 0.0f)) bad = true;
  }
  if (bad) atomicOr(flag, HEX_FLAG_TARGET);
  st4m(target + ii, td, k0, 0, g.L);
}

// low-order upwind vertical flux at interface j = k0 + d (old + 0 scalars)
__device__ __forceinline__ float fct_fcol_win(float step, const Win& o, const Win& ww, int d) {
  return step * (pos0(ww(d)) * (o(d - 1) + 0.0f) + neg0(ww(d)) * (o(d) + 0.0f));
}
__device__ __forceinline__ float fct_vres_win(const HexGeo& g, float step, const Win& q, const Win& o,
                                              const Win& ww, int k0, int d) {
  const float h = step * tr_vflux_win(g, q, ww, k0, d);
  const int j = k0 + d;
  if (j <= 0 || j >= g.L) return h;
  return h - fct_fcol_win(step, o, ww, d);
}

// hexcore/transport.py:1919-2118 (v8.4.1 order): bounds, low-order mass,
// incoming/outgoing antidiffusive totals and the scale factors.
// ACROSS: cellsOnCell[c][s] is the cell across edgesOnCell[c][s] for every
// slot (the MPAS convention, checked on the host), so the upwind flux of
// slot s takes its two cell values from this column and the neighbour column
// the bounds already load; the min/max over neighbours and the mass sums
// still run in slot order, so the words are those of the two-loop form.
template <bool ACROSS>
__global__ void HEX_VEC_BOUNDS kv_fct_cell1(HexGeo g, int nT, float step, const float* __restrict__ q_old,
                             const float* __restrict__ q_stage, const float* __restrict__ rho_old,
                             const float* __restrict__ hv, const float* __restrict__ ww,
                             const float* __restrict__ high_e, const float* __restrict__ target,
                             float* __restrict__ scale_in, float* __restrict__ scale_out, float* __restrict__ mass_out,
                             float* __restrict__ vres_out) {
  HEX_VEC_TRACER(g.nC, nT)
  const int c = ent, S = g.S, L = g.L;
  const int ii = c * S + k0;
  const size_t toff = (size_t)tr * g.nC * S;
  const float* ot = q_old + toff;
  const float* he = high_e + (size_t)tr * g.nE * S;
  const Win ow = win(ot + c * S, k0, S), qw = win(q_stage + toff + c * S, k0, S), www = win(ww + c * S, k0, S);
  float mn[4], mx[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    const float o = ow(j) + 0.0f;
    const float a = (k > 0 ? ow(j - 1) : ow(j)) + 0.0f;
    const float b = (k + 1 < L ? ow(j + 1) : ow(j)) + 0.0f;
    mn[j] = fminf(fminf(a, o), b);
    mx[j] = fmaxf(fmaxf(a, o), b);
  }
  const int n = g.deg[c];
  if (!ACROSS) {
    HEX_GATHER
    for (int s = 0; s < n; ++s) {
      const V4 on = ld4(ot + g.coc[c * g.maxE + s] * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        mn[j] = pymin(mn[j], on.a[j] + 0.0f);
        mx[j] = pymax(mx[j], on.a[j] + 0.0f);
      }
    }
  }
  const V4 ro = ld4(rho_old + ii), td = ld4(target + ii);
  float mass[4], s_in[4], s_out[4], vr[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) vr[d] = fct_vres_win(g, step, qw, ow, www, k0, d);
  // interfaces k0..k0+3 for the limited update (every interface of the
  // column is some thread's k0 + d, d < 4)
  st4(vres_out + toff + ii, V4{{vr[0], vr[1], vr[2], vr[3]}});
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    float m = (ow(j) + 0.0f) * ro.a[j];
    if (k < L - 1) m = m - fct_fcol_win(step, ow, www, j + 1) * g.rdzw[k];
    if (k >= 1) m = m + fct_fcol_win(step, ow, www, j) * g.rdzw[k];
    mass[j] = m;
    s_in[j] = -g.rdzw[k] * (neg0(vr[j + 1]) - pos0(vr[j]));
    s_out[j] = -g.rdzw[k] * (pos0(vr[j + 1]) - neg0(vr[j]));
  }
  const float ia = g.inv_area[c];
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float cs = g.csign[c * g.maxE + s];
    const float ts = -cs;
    const float dvs = g.dv[e] * step;
    const V4 vel = ld4(hv + e * S + k0), h = ld4(he + e * S + k0);
    V4 o0, o1;
    if (ACROSS) {
      // csign > 0: this cell is the edge's first cell
      const V4 on = ld4(ot + g.coc[c * g.maxE + s] * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        mn[j] = pymin(mn[j], on.a[j] + 0.0f);
        mx[j] = pymax(mx[j], on.a[j] + 0.0f);
        o0.a[j] = cs > 0.0f ? ow(j) : on.a[j];
        o1.a[j] = cs > 0.0f ? on.a[j] : ow(j);
      }
    } else {
      o0 = ld4(ot + g.coe[2 * e] * S + k0);
      o1 = ld4(ot + g.coe[2 * e + 1] * S + k0);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float upw = dvs * (pos0(vel.a[j]) * (o0.a[j] + 0.0f) + neg0(vel.a[j]) * (o1.a[j] + 0.0f));
      mass[j] = mass[j] + ts * upw * ia;
      const float hres = step * h.a[j] - upw;
      const float sr = -ts * hres;
      s_out[j] = s_out[j] - pos0(sr) * ia;
      s_in[j] = s_in[j] - neg0(sr) * ia;
    }
  }
  V4 si, so, ms;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    float sf = (mx[j] * td.a[j] - mass[j]) / (s_in[j] + 1.0e-20f);
    si.a[j] = pymin(1.0f, pos0(sf));
    sf = (mn[j] * td.a[j] - mass[j]) / (s_out[j] - 1.0e-20f);
    so.a[j] = pymin(1.0f, pos0(sf));
    ms.a[j] = mass[j];
  }
  st4m(scale_in + toff + ii, si, k0, 0, g.L);
  st4m(scale_out + toff + ii, so, k0, 0, g.L);
  st4m(mass_out + toff + ii, ms, k0, 0, g.L);
}

// hexcore/transport.py:1919-2118: the limited antidiffusive edge flux.
__global__ void __launch_bounds__(256, HEX_FCT_EDGE_MIN_BLOCKS) kv_fct_edge(HexGeo g, int nT, float step, const float* __restrict__ q_old, const float* __restrict__ hv,
                            const float* __restrict__ high_e, const float* __restrict__ scale_in,
                            const float* __restrict__ scale_out, float* __restrict__ hres_lim) {
  HEX_VEC_TRACER(g.nE, nT)
  const int e = ent, S = g.S;
  const size_t toff = (size_t)tr * g.nC * S;
  const size_t eoff = (size_t)tr * g.nE * S;
  const int i0 = g.coe[2 * e] * S + k0, i1 = g.coe[2 * e + 1] * S + k0;
  const V4 vel = ld4(hv + e * S + k0), h = ld4(high_e + eoff + e * S + k0);
  const V4 o0 = ld4(q_old + toff + i0), o1 = ld4(q_old + toff + i1);
  const V4 so0 = ld4(scale_out + toff + i0), si1 = ld4(scale_in + toff + i1);
  const V4 si0 = ld4(scale_in + toff + i0), so1 = ld4(scale_out + toff + i1);
  const float dvs = g.dv[e] * step;
  V4 out;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float upw = dvs * (pos0(vel.a[j]) * (o0.a[j] + 0.0f) + neg0(vel.a[j]) * (o1.a[j] + 0.0f));
    const float flux = step * h.a[j] - upw;
    out.a[j] = pos0(flux) * pymin(so0.a[j], si1.a[j]) + neg0(flux) * pymin(si0.a[j], so1.a[j]);
  }
  st4m(hres_lim + eoff + e * S + k0, out, k0, 0, g.L);
}

// hexcore/transport.py:1919-2118: limited update of the monotonic stage.
// The vertical residual fluxes are those kv_fct_cell1 formed (vres).
__global__ void HEX_VEC_BOUNDS kv_fct_cell2(HexGeo g, int nT, const float* __restrict__ vres,
                             const float* __restrict__ scale_in, const float* __restrict__ scale_out,
                             const float* __restrict__ mass_in, const float* __restrict__ hres_lim,
                             const float* __restrict__ target, float* __restrict__ q_out) {
  HEX_VEC_TRACER(g.nC, nT)
  const int c = ent, S = g.S;
  const int ii = c * S + k0;
  const size_t toff = (size_t)tr * g.nC * S;
  const float* hl = hres_lim + (size_t)tr * g.nE * S;
  V4 mass = ld4(mass_in + toff + ii);
  const int n = g.deg[c];
  const float ia = g.inv_area[c];
  HEX_GATHER
  for (int s = 0; s < n; ++s) {
    const int e = g.eoc[c * g.maxE + s];
    const float ts = -g.csign[c * g.maxE + s];
    const V4 h = ld4(hl + e * S + k0);
#pragma unroll
    for (int j = 0; j < 4; ++j) mass.a[j] = mass.a[j] + ts * h.a[j] * ia;
  }
  const Win siw = win(scale_in + toff + c * S, k0, S), sow = win(scale_out + toff + c * S, k0, S);
  // interface k0 + 4 belongs to the next chunk; past the column's last chunk
  // it only feeds a padding level, never stored
  const float* vc = vres + toff + c * S;
  const V4 f4 = ld4(vc + k0);
  const float fv[5] = {f4.a[0], f4.a[1], f4.a[2], f4.a[3], k0 + 4 < S ? vc[k0 + 4] : 0.0f};
  float vl[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const float f = fv[d];
    const int j = k0 + d;
    vl[d] = (j <= 0 || j >= g.L) ? f
                                 : pos0(f) * pymin(sow(d - 1), siw(d)) + neg0(f) * pymin(sow(d), siw(d - 1));
  }
  const V4 td = ld4(target + ii);
  V4 out;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = k0 + j;
    const float m = mass.a[j] - g.rdzw[k] * (vl[j + 1] - vl[j]);
    out.a[j] = pos0(m / td.a[j]);
  }
  st4m(q_out + toff + ii, out, k0, 0, g.L);
}

// ------------------------------------------------ column-sweep kernels
// The kernels with a sequential sweep down a column (the tridiagonal
// coefficients and the acoustic w solve) keep the S/4 threads of a column in
// G consecutive lanes of one warp (G = 8, 16 or 32: blockDim.x = G, the
// power of two >= S/4), so their phases synchronise with __syncwarp and a
// block holds 256/G columns.  Lanes with k0 >= S take part in the
// synchronisation and the shuffles only.  The sweeps run level by level on
// the column's first lane in level order (the order of the one-level forms
// k_vcoef and k_ac_cell), moving four levels per shared-memory access.

__device__ __forceinline__ V4 lds4(const float* p) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  return V4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ void sts4(float* p, const V4& v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.a[0], v.a[1], v.a[2], v.a[3]);
}

// Shared memory of the column sweeps: array a of column y at
// sm + (a * blockDim.y + y) * SP, with SP = S + 4 words per column (S is a
// multiple of 8, so every row stays 16-byte aligned, and the odd multiple
// of four words spreads the rows of consecutive columns over all 32 banks
// when one thread per column sweeps them).
#define HEX_SWEEP_PAD 4
__device__ __forceinline__ float* sweep_col(float* sm, int a, int S, int col) {
  return sm + ((size_t)a * blockDim.y + col) * (S + HEX_SWEEP_PAD);
}
__device__ __forceinline__ float* sweep_row(float* sm, int a, int S) { return sweep_col(sm, a, S, threadIdx.y); }

// The sequential sweep of every column of the block.  HEX_SWEEP_BLOCK 1:
// after a block barrier, thread t of the block sweeps column t (so one warp
// instruction advances up to 32 columns' recurrences), then a second barrier
// publishes the results; 0: the first lane of each column's group sweeps its
// own column between warp barriers.  Either way each column's recurrence
// runs in level order on one thread, so the words are the same.
#ifndef HEX_SWEEP_BLOCK
#define HEX_SWEEP_BLOCK 1
#endif
#if HEX_SWEEP_BLOCK
#define SWEEP_BEGIN(live, k0)                                                    \
  __syncthreads();                                                               \
  {                                                                              \
    const int sweep_c = threadIdx.y * blockDim.x + threadIdx.x;                  \
    if (sweep_c < (int)blockDim.y && blockIdx.x * blockDim.y + sweep_c < g.nC) {
#define SWEEP_END \
  }               \
  }               \
  __syncthreads();
#else
#define SWEEP_BEGIN(live, k0)     \
  __syncwarp();                   \
  {                               \
    const int sweep_c = threadIdx.y; \
    if ((live) && (k0) == 0) {
#define SWEEP_END \
  }               \
  }               \
  __syncwarp();
#endif

// Neighbour levels across a thread's chunk: the lane below in the column
// holds level k0-1 as its a[3], the lane above holds k0+4 as its a[0].  All
// lanes of the warp take part; a value is used only where the one-level form
// reads that level, which then lies in a live lane of the same column.
__device__ __forceinline__ float from_below(float a3) { return __shfl_up_sync(0xffffffffu, a3, 1); }
__device__ __forceinline__ float from_above(float a0) { return __shfl_down_sync(0xffffffffu, a0, 1); }

// hexcore/acoustic_v841.py:81 compute_vertical_implicit_coefficients_v841.
#define HEX_VCOEFV_SMEM_ARRAYS 3
__global__ void HEX_VEC_BOUNDS kv_vcoef(HexGeo g, float dts2, const float* __restrict__ exner, const float* __restrict__ theta,
                         const float* __restrict__ rtp, const float* __restrict__ cqw,
                         const float* __restrict__ qtot, float* __restrict__ cofwr, float* __restrict__ cofwz,
                         float* __restrict__ coftz, float* __restrict__ cofwt, float* __restrict__ a_tri,
                         float* __restrict__ alpha_tri, float* __restrict__ gamma_tri, int* flag) {
  extern __shared__ float sm[];
  const int S = g.S, L = g.L;
  const int k0 = threadIdx.x * 4;
  const int c = blockIdx.x * blockDim.y + threadIdx.y;
  const bool live = c < g.nC && k0 < S;
  float* s_a = sweep_row(sm, 0, S);
  float* s_b = sweep_row(sm, 1, S);
  float* s_c = sweep_row(sm, 2, S);
  const int ii = c * S + k0;
  V4 zz = v4zero(), ex = v4zero(), th = v4zero();
  V4 wr = v4zero(), wz = v4zero(), tz = v4zero(), wt = v4zero();
  if (live) {
    zz = ld4(g.zz + ii);
    ex = ld4(exner + ii);
    th = ld4(theta + ii);
  }
  const float zzm = from_below(zz.a[3]), exm = from_below(ex.a[3]), thm = from_below(th.a[3]);
  if (live) {
    const V4 cq = ld4(cqw + ii), qt = ld4(qtot + ii), rb = ld4(g.rho_base + ii), rtb = ld4(g.rtheta_base + ii);
    const V4 rp = ld4(rtp + ii), eb = ld4(g.exner_base + ii);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      const float zprev = j == 0 ? zzm : zz.a[j - 1];
      const float eprev = j == 0 ? exm : ex.a[j - 1];
      const float tprev = j == 0 ? thm : th.a[j - 1];
      if (k >= 1 && k < L) {
        const float izz = g.fzm[k] * zz.a[j] + g.fzp[k] * zprev;
        wr.a[j] = 0.5f * g.g * izz;
        wz.a[j] = g.c2 * izz * g.rdzu[k] * cq.a[j] * (g.fzm[k] * ex.a[j] + g.fzp[k] * eprev);
        tz.a[j] = g.fzm[k] * th.a[j] + g.fzp[k] * tprev;
      }
      if (k < L) {
        wt.a[j] = 0.5f * g.rcv * zz.a[j] * g.g * rb.a[j] / (1.0f + qt.a[j]) * ex.a[j]
                  / ((rtb.a[j] + rp.a[j]) * eb.a[j]);
      }
    }
  }
  const float tzm = from_below(tz.a[3]), wtm = from_below(wt.a[3]), tzp = from_above(tz.a[0]);
  V4 av = v4zero(), bv = v4zero(), cv = v4zero();
  if (live) {
    const float* rdzw = g.rdzw;
    const float* etp = g.etp;
    const float* ewp = g.ewp;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      float a = 0.0f, b = 0.0f, cc = 0.0f;
      if (k == 0) b = 1.0f;
      if (k >= 1 && k < L) {
        const float zzk = zz.a[j], zzb = j == 0 ? zzm : zz.a[j - 1];
        const float wz_k = wz.a[j], wr_k = wr.a[j], tz_k = tz.a[j], wt_k = wt.a[j];
        const float tz_m = j == 0 ? tzm : tz.a[j - 1], wt_m = j == 0 ? wtm : wt.a[j - 1];
        const float tz_p = j == 3 ? tzp : tz.a[j + 1];
        a = -wz_k * tz_m * rdzw[k - 1] * zzb + wr_k * rdzw[k - 1] - wt_m * tz_m * rdzw[k - 1];
        a = a * etp[k - 1] * ewp[k - 1];
        b = wz_k * tz_k * (etp[k] * rdzw[k] * zzk + etp[k - 1] * rdzw[k - 1] * zzb)
            - tz_k * (etp[k] * wt_k * rdzw[k] - etp[k - 1] * wt_m * rdzw[k - 1])
            + wr_k * (etp[k] * rdzw[k] - etp[k - 1] * rdzw[k - 1]);
        b = b * ewp[k];
        if (k < L - 1) {
          cc = -wz_k * tz_p * rdzw[k] * zzk - wr_k * rdzw[k] + wt_k * tz_p * rdzw[k];
          cc = cc * etp[k] * ewp[k + 1];
        }
      }
      av.a[j] = a;
      bv.a[j] = b;
      cv.a[j] = cc;
    }
    sts4(s_a + k0, av);
    sts4(s_b + k0, bv);
    sts4(s_c + k0, cv);
  }
  SWEEP_BEGIN(live, k0)
    // alpha overwrites b and gamma overwrites c; level 0 of both is zero
    const float* a_col = sweep_col(sm, 0, S, sweep_c);
    float* b_col = sweep_col(sm, 1, S, sweep_c);
    float* c_col = sweep_col(sm, 2, S, sweep_c);
    float gam = 0.0f;
    for (int q = 0; q < L; q += 4) {
      const V4 a4 = lds4(a_col + q);
      V4 b4 = lds4(b_col + q), c4 = lds4(c_col + q);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int kk = q + j;
        if (kk == 0) {
          b4.a[0] = 0.0f;
          c4.a[0] = 0.0f;
        } else if (kk < L) {
          const float den = 1.0f + dts2 * (b4.a[j] - a4.a[j] * gam);
          if (den == 0.0f) atomicOr(flag, HEX_FLAG_SINGULAR);
          const float alpha = 1.0f / den;
          gam = dts2 * c4.a[j] * alpha;
          b4.a[j] = alpha;
          c4.a[j] = gam;
        }
      }
      sts4(b_col + q, b4);
      sts4(c_col + q, c4);
    }
  SWEEP_END
  if (live) {
    st4m(coftz + ii, tz, k0, 0, L + 1);
    st4m(cofwr + ii, wr, k0, 0, L);
    st4m(cofwz + ii, wz, k0, 0, L);
    st4m(cofwt + ii, wt, k0, 0, L);
    st4m(a_tri + ii, av, k0, 0, L);
    st4m(alpha_tri + ii, lds4(s_b + k0), k0, 0, L);
    st4m(gamma_tri + ii, lds4(s_c + k0), k0, 0, L);
  }
}

// One acoustic cell pass (hexcore/acoustic_v841.py:461-567): the phases and
// expressions of k_ac_cell, four levels per thread; only the sweep's
// operands go through shared memory.
#define HEX_ACV_SMEM_ARRAYS 4
// With an all-zero damping profile the acoustic cell pass skips the
// damping's reads (1).
#ifndef HEX_AC_DSS_ZERO_SKIP
#define HEX_AC_DSS_ZERO_SKIP 1
#endif
__global__ void HEX_VEC_BOUNDS kv_ac_cell(HexGeo g, int first, float dts, float dts2, const float* __restrict__ ru_p,
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
  const int S = g.S, L = g.L;
  const int k0 = threadIdx.x * 4;
  const int c = blockIdx.x * blockDim.y + threadIdx.y;
  const bool live = c < g.nC && k0 < S;
  float* s_r = sweep_row(sm, 0, S);
  float* s_da = sweep_row(sm, 1, S);
  float* s_al = sweep_row(sm, 2, S);
  float* s_ga = sweep_row(sm, 3, S);
  const int ii = c * S + k0;
  const float* ewm = g.ewm;
  const float* ewp = g.ewp;
  const float* etp = g.etp;
  const float* etm = g.etm;
  // phase 1: old rw_p, the edge-flux sums, rs/ts and the ww_avg partial
  V4 rwp_old = v4zero(), ctz = v4zero(), wa = v4zero();
  V4 rs = v4zero(), ts = v4zero(), rho_old = v4zero(), rt_old = v4zero();
  if (live) {
    if (!first) {
      const V4 t = ld4rw(rw_p + ii);
#pragma unroll
      for (int j = 0; j < 4; ++j) rwp_old.a[j] = k0 + j <= L ? t.a[j] : 0.0f;
    }
    ctz = ld4(coftz + ii);
  }
  const float r4 = from_above(rwp_old.a[0]), ctz4 = from_above(ctz.a[0]);
  if (live) {
    const V4 at = ld4(a_tri + ii);
    V4 da;
#pragma unroll
    for (int j = 0; j < 4; ++j) da.a[j] = dts2 * at.a[j];
    sts4(s_da + k0, da);
    sts4(s_al + k0, ld4(alpha_tri + ii));
    sts4(s_ga + k0, ld4(gamma_tri + ii));
    if (!first) {
      rho_old = ld4rw(rho_pp + ii);
      rt_old = ld4(rtpp_old + ii);
    }
    const int n = g.deg[c];
    const float ia = g.inv_area[c];
    const V4 tc = ld4(theta_s + ii);
    HEX_GATHER
    for (int s = 0; s < n; ++s) {
      const int e = g.eoc[c * g.maxE + s];
      const int e0 = g.coe[2 * e], e1 = g.coe[2 * e + 1];
      const float sdd = g.csign[c * g.maxE + s] * dts * g.dv[e];
      const V4 r = ld4(ru_p + e * S + k0), tn = ld4(theta_s + (e0 == c ? e1 : e0) * S + k0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float flux = sdd * r.a[j] * ia;
        rs.a[j] = rs.a[j] - flux;
        // theta_s[e1] + theta_s[e0], one of the two being this cell (IEEE
        // addition commutes, so the order of the operands changes no bit)
        ts.a[j] = ts.a[j] - flux * 0.5f * (tn.a[j] + tc.a[j]);
      }
    }
    const V4 trho = ld4(tend_rho + ii), trt = ld4(tend_rt + ii);
    const V4 wav = first ? v4zero() : ld4rw(ww_avg + ii);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      if (k < L) {
        const float rnext = j == 3 ? r4 : rwp_old.a[j + 1];
        const float cnext = j == 3 ? ctz4 : ctz.a[j + 1];
        const float cofrz = g.rdzw[k];
        rs.a[j] = rho_old.a[j] + dts * trho.a[j] + rs.a[j]
                  - dts * cofrz * (ewm[k + 1] * rnext - ewm[k] * rwp_old.a[j]);
        ts.a[j] = rt_old.a[j] + dts * trt.a[j] + ts.a[j]
                  - dts * g.rdzw[k] * (ewm[k + 1] * cnext * rnext - ewm[k] * ctz.a[j] * rwp_old.a[j]);
      }
      if (k >= 1 && k < L) wa.a[j] = wav.a[j] + ewm[k] * rwp_old.a[j];
    }
  }
  // phase 2: right-hand side of the w system (levels k-1 from the lane below)
  V4 zz = v4zero(), cwt = v4zero();
  if (live) {
    zz = ld4(g.zz + ii);
    cwt = ld4(cofwt + ii);
  }
  const float ts_m = from_below(ts.a[3]), rt_m = from_below(rt_old.a[3]), rs_m = from_below(rs.a[3]);
  const float rho_m = from_below(rho_old.a[3]), zz_m = from_below(zz.a[3]), cwt_m = from_below(cwt.a[3]);
  V4 rhs = rwp_old;
  if (live) {
    const V4 trw = ld4(tend_rw + ii), cwz = ld4(cofwz + ii), cwr = ld4(cofwr + ii);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      if (k >= 1 && k < L) {
        const float zzk = zz.a[j], zzm = j == 0 ? zz_m : zz.a[j - 1];
        const float tsk = ts.a[j], tsm = j == 0 ? ts_m : ts.a[j - 1];
        const float rtk = rt_old.a[j], rtm = j == 0 ? rt_m : rt_old.a[j - 1];
        const float rsk = rs.a[j], rsm = j == 0 ? rs_m : rs.a[j - 1];
        const float rhk = rho_old.a[j], rhm = j == 0 ? rho_m : rho_old.a[j - 1];
        const float cwtm = j == 0 ? cwt_m : cwt.a[j - 1];
        rhs.a[j] = rwp_old.a[j] + dts * (trw.a[j]
                                         - cwz.a[j] * ((etp[k] * zzk * tsk - etp[k - 1] * zzm * tsm)
                                                       + (etm[k] * zzk * rtk - etm[k - 1] * zzm * rtm))
                                         - cwr.a[j] * ((etp[k] * rsk + etp[k - 1] * rsm)
                                                       + (etm[k] * rhk + etm[k - 1] * rhm))
                                         + cwt.a[j] * (etp[k] * tsk + etm[k] * rtk)
                                         + cwtm * (etp[k - 1] * tsm + etm[k - 1] * rtm));
      }
    }
    sts4(s_r + k0, rhs);
  }
  // phase 3: the dts^2 Thomas sweep (hexcore/acoustic_v841.py:236-257)
  SWEEP_BEGIN(live, k0)
    float* r_col = sweep_col(sm, 0, S, sweep_c);
    const float* da_col = sweep_col(sm, 1, S, sweep_c);
    const float* al_col = sweep_col(sm, 2, S, sweep_c);
    const float* ga_col = sweep_col(sm, 3, S, sweep_c);
    float prev = r_col[0];
    for (int q = 0; q < L; q += 4) {
      V4 r = lds4(r_col + q);
      const V4 d = lds4(da_col + q), al = lds4(al_col + q);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int kk = q + j;
        if (kk >= 1 && kk < L) {
          prev = (r.a[j] - d.a[j] * prev) * al.a[j];
          r.a[j] = prev;
        }
      }
      sts4(r_col + q, r);
    }
    float next = r_col[L];
    for (int q = ((L - 1) / 4) * 4; q >= 0; q -= 4) {
      V4 r = lds4(r_col + q);
      const V4 ga = lds4(ga_col + q);
#pragma unroll
      for (int j = 3; j >= 0; --j) {
        const int kk = q + j;
        if (kk < L) {
          next = r.a[j] - ga.a[j] * next;
          r.a[j] = next;
        }
      }
      sts4(r_col + q, r);
    }
  SWEEP_END
  // phase 4: implicit Rayleigh damping, ww_avg, rw_p
  V4 rwp = v4zero(), rz = v4zero();
  const bool damping = !(HEX_AC_DSS_ZERO_SKIP && g.dss_zero);
  if (live) {
    rwp = lds4(s_r + k0);
    if (damping) rz = ld4(rho_zz + ii);
  }
  const float rz_m = from_below(rz.a[3]);
  if (live) {
    const V4 rsv = ld4(rw_save + ii), rwv = ld4(rw + ii);
    V4 wo;
    if (damping) {
      const V4 dss = ld4(g.dss + ii), wv = ld4(w + ii);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + j;
        wo.a[j] = 0.0f;
        if (k >= 1 && k < L) {
          const float delta = rsv.a[j] - rwv.a[j];
          const float damp = dss.a[j];
          const float zzi = g.fzm[k] * zz.a[j] + g.fzp[k] * (j == 0 ? zz_m : zz.a[j - 1]);
          const float rhoi = g.fzm[k] * rz.a[j] + g.fzp[k] * (j == 0 ? rz_m : rz.a[j - 1]);
          rwp.a[j] = (rwp.a[j] + delta - dts * damp * zzi * rhoi * wv.a[j]) / (1.0f + dts * damp) - delta;
          wo.a[j] = wa.a[j] + ewp[k] * rwp.a[j];
        }
      }
    } else {
      // dss = +0 everywhere: the subtracted term dts (+0) zzi rhoi w is a
      // zero with w's sign (dts, zzi and rhoi positive and finite in any
      // state the step accepts) and the divisor is 1 + (+0) = 1, so the
      // result is t - delta with t = rw_p + delta, except for t = -0 with
      // w's sign bit set (then +0): w is read only there.
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + j;
        wo.a[j] = 0.0f;
        if (k >= 1 && k < L) {
          const float delta = rsv.a[j] - rwv.a[j];
          float t = rwp.a[j] + delta;
          if (__float_as_uint(t) == 0x80000000u && (__float_as_uint(w[ii + j]) & 0x80000000u)) t = 0.0f;
          rwp.a[j] = t - delta;
          wo.a[j] = wa.a[j] + ewp[k] * rwp.a[j];
        }
      }
    }
    st4m(ww_avg + ii, wo, k0, 0, L + 1);
    st4m(rw_p + ii, rwp, k0, 0, L + 1);
  }
  // phase 5: rho_pp and rtheta_pp from the new rw_p (level k+1 from the lane above)
  const float rwp4 = from_above(rwp.a[0]);
  if (live) {
    V4 rpo, rto;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      rpo.a[j] = 0.0f;
      rto.a[j] = 0.0f;
      if (k < L) {
        const float rnext = j == 3 ? rwp4 : rwp.a[j + 1];
        const float cnext = j == 3 ? ctz4 : ctz.a[j + 1];
        rpo.a[j] = rs.a[j] - dts * g.rdzw[k] * (ewp[k + 1] * rnext - ewp[k] * rwp.a[j]);
        rto.a[j] = ts.a[j] - dts * g.rdzw[k] * (ewp[k + 1] * cnext * rnext - ewp[k] * ctz.a[j] * rwp.a[j]);
      }
    }
    st4m(rho_pp + ii, rpo, k0, 0, L);
    st4m(rtpp_new + ii, rto, k0, 0, L);
  }
}
