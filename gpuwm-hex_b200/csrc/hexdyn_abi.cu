// C ABI of the dycore library: descriptor validation, device allocation,
// host-side preparation of derived FP32 fields (in the reference's FP32
// operation order), logical <-> padded layout transposes, stepping, CUDA
// graph capture and error reporting.  Declarations: include/hexdyn.h.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/hexdyn.h"
#include "hexdyn_ctx.h"

struct HexDynHandle {
  HexCtx ctx;
  float* staging[HEXDYN_NUM_FIELDS] = {};
  size_t staging_count[HEXDYN_NUM_FIELDS] = {};
  int* host_flag = nullptr;
  bool have_state[HEXDYN_NUM_FIELDS] = {};
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail((int)e, "%s: %s", what, cudaGetErrorString(e));
}

#define HEX_CUDA(call, what)                    \
  do {                                          \
    cudaError_t _e = (call);                    \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

template <class T>
cudaError_t dev_alloc(HexCtx& ctx, T** p, size_t count) {
  void* raw = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&raw, bytes);
  if (e != cudaSuccess) return e;
  ctx.allocations.push_back(raw);
  ctx.device_bytes += bytes;
  *p = (T*)raw;
  return cudaMemset(raw, 0, bytes);
}

template <class T>
cudaError_t upload(HexCtx& ctx, const T** dst, const std::vector<T>& host) {
  T* d = nullptr;
  cudaError_t e = dev_alloc(ctx, &d, host.size());
  if (e != cudaSuccess) return e;
  *dst = d;
  return cudaMemcpy(d, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// [rows][n] logical -> [n][S] padded
std::vector<float> pad_levels(const float* src, int rows, int n, int S) {
  std::vector<float> out((size_t)n * S, 0.0f);
  for (int r = 0; r < rows; ++r)
    for (int i = 0; i < n; ++i) out[(size_t)i * S + r] = src[(size_t)r * n + i];
  return out;
}

std::vector<float> pad_vector(const float* src, int n, int S) {
  std::vector<float> out(S, 0.0f);
  for (int i = 0; i < n; ++i) out[i] = src[i];
  return out;
}

// hexcore/offcentering_v841.py:47 build_v841_acoustic_offcentering, FP32 ops.
void offcentering(const HexDynDesc& d, const float* rdzw, int L, int S, std::vector<float>& etp,
                  std::vector<float>& etm, std::vector<float>& ewp, std::vector<float>& ewm) {
  const float lower = d.epssm_bottom_z, upper = d.epssm_top_z;
  const float mn = d.epssm_minimum, mx = d.epssm_maximum;
  std::vector<float> hw(L + 1, 0.0f), hu(L, 0.0f);
  for (int k = 0; k < L; ++k) {
    hw[k + 1] = hw[k] + 1.0f / rdzw[k];
    hu[k] = 0.5f * (hw[k + 1] + hw[k]);
  }
  const float width = upper - lower;
  const float pi = (float)acos(-1.0);
  auto coef = [&](float h) -> float {
    if (h <= lower) return mn;
    if (h >= upper) return mx;
    const float z = (h - lower) / width;
    const float s = (float)sin((double)(0.5f * pi * z));
    return mn + s * s * (mx - mn);
  };
  etp.assign(S, 0.0f);
  etm.assign(S, 0.0f);
  ewp.assign(S, 0.0f);
  ewm.assign(S, 0.0f);
  for (int k = 0; k < L; ++k) {
    const float e = coef(hu[k]);
    etp[k] = 0.5f * (1.0f + e);
    etm[k] = 0.5f * (1.0f - e);
  }
  for (int k = 0; k <= L; ++k) {
    const float e = coef(hw[k]);
    ewp[k] = 0.5f * (1.0f + e);
    ewm[k] = 0.5f * (1.0f - e);
  }
}

__global__ void k_fill(float* p, size_t n, float v) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// Logical [rows][n] -> padded [n][S] (and back) through a 32x32 tile.
__global__ void k_to_padded(const float* __restrict__ src, int rows, int n, int S, float* __restrict__ dst) {
  __shared__ float tile[32][33];
  const int i0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, i = i0 + threadIdx.x;
    if (r < rows && i < n) tile[y][threadIdx.x] = src[(size_t)r * n + i];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int i = i0 + y, r = r0 + threadIdx.x;
    if (r < rows && i < n) dst[(size_t)i * S + r] = tile[threadIdx.x][y];
  }
}

__global__ void k_from_padded(const float* __restrict__ src, int rows, int n, int S, float* __restrict__ dst) {
  __shared__ float tile[32][33];
  const int i0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int i = i0 + y, r = r0 + threadIdx.x;
    if (r < rows && i < n) tile[threadIdx.x][y] = src[(size_t)i * S + r];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, i = i0 + threadIdx.x;
    if (r < rows && i < n) dst[(size_t)r * n + i] = tile[y][threadIdx.x];
  }
}

struct FieldShape {
  int blocks;   // tracers (1 for ordinary fields)
  int rows;     // levels or interfaces
  int n;        // entities
};

FieldShape field_shape(const HexCtx& c, int field) {
  const HexGeo& g = c.geo;
  switch (field) {
    case HEXDYN_RHO_U:
    case HEXDYN_U:
      return {1, g.L, g.nE};
    case HEXDYN_RHO_W:
    case HEXDYN_W:
      return {1, g.L + 1, g.nC};
    case HEXDYN_SCALARS:
      return {c.n_scalars, g.L, g.nC};
    default:
      return {1, g.L, g.nC};
  }
}

float* field_ptr(const HexState& s, const HexSide& side, int field) {
  switch (field) {
    case HEXDYN_RHO: return s.rho;
    case HEXDYN_RHO_THETA: return s.rho_theta;
    case HEXDYN_RHO_U: return s.rho_u;
    case HEXDYN_RHO_W: return s.rho_w;
    case HEXDYN_SCALARS: return s.scalars;
    case HEXDYN_THETA_M: return side.theta_m;
    case HEXDYN_EXNER: return side.exner;
    case HEXDYN_RHO_P: return side.rho_p;
    case HEXDYN_RHO_THETA_P: return side.rtheta_p;
    case HEXDYN_PRESSURE_P: return side.pressure_p;
    case HEXDYN_U: return side.u;
    case HEXDYN_W: return side.w;
  }
  return nullptr;
}

cudaError_t alloc_state(HexCtx& c, HexState& s, bool scalars) {
  const HexGeo& g = c.geo;
  cudaError_t e;
  if ((e = dev_alloc(c, &s.rho, (size_t)g.nC * g.S))) return e;
  if ((e = dev_alloc(c, &s.rho_theta, (size_t)g.nC * g.S))) return e;
  if ((e = dev_alloc(c, &s.rho_u, (size_t)g.nE * g.S))) return e;
  if ((e = dev_alloc(c, &s.rho_w, (size_t)g.nC * g.S))) return e;
  s.scalars = nullptr;
  if (scalars && c.n_scalars > 0)
    if ((e = dev_alloc(c, &s.scalars, (size_t)c.n_scalars * g.nC * g.S))) return e;
  return cudaSuccess;
}

cudaError_t alloc_side(HexCtx& c, HexSide& s) {
  const HexGeo& g = c.geo;
  cudaError_t e;
  float** cell[] = {&s.theta_m, &s.exner, &s.rho_p, &s.rtheta_p, &s.pressure_p, &s.w};
  for (float** p : cell)
    if ((e = dev_alloc(c, p, (size_t)g.nC * g.S))) return e;
  return dev_alloc(c, &s.u, (size_t)g.nE * g.S);
}

int validate(const HexDynDesc* d) {
  if (!d) return fail(HEXDYN_E_ARG, "descriptor is NULL");
  if (d->n_cells <= 0 || d->n_edges <= 0 || d->n_vertices <= 0)
    return fail(HEXDYN_E_ARG, "mesh sizes must be positive");
  if (d->n_levels < 4)
    return fail(HEXDYN_E_ARG, "n_levels=%d: the third-order vertical fluxes need at least 4 levels", d->n_levels);
  if (d->n_levels > 1000)
    return fail(HEXDYN_E_ARG, "n_levels=%d: at most 1000 levels (a column's four-level chunks fill one block)",
                d->n_levels);
  if (d->max_edges <= 0 || d->max_edges2 <= 0 || d->adv_width <= 0 || d->n_scalars < 0)
    return fail(HEXDYN_E_ARG, "invalid slot widths or scalar count");
  if (d->max_edges > 8 || d->max_edges2 > 16 || d->adv_width > 16)
    return fail(HEXDYN_E_ARG, "slot widths (maxEdges %d, maxEdges2 %d, advection stencil %d) exceed the "
                "compiled maxima 8 / 16 / 16", d->max_edges, d->max_edges2, d->adv_width);
  if (!(d->dt > 0.0) || !isfinite(d->dt)) return fail(HEXDYN_E_ARG, "config_dt=%g must be finite and positive", d->dt);
  if (d->n_sub_steps < 1) return fail(HEXDYN_E_ARG, "config_number_of_sub_steps=%d must be positive", d->n_sub_steps);
  if (d->split_steps != 1 && d->split_steps != 3)
    return fail(HEXDYN_E_ARG, "config_dynamics_split_steps=%d: only 1 and 3 are implemented", d->split_steps);
  if (d->moist != 0 && d->moist != 1) return fail(HEXDYN_E_ARG, "moist=%d must be 0 or 1", d->moist);
  if (d->numerics != 0 && d->numerics != 1) return fail(HEXDYN_E_ARG, "numerics=%d must be 0 or 1", d->numerics);
  if (!(d->smdiv >= 0.0f)) return fail(HEXDYN_E_ARG, "config_smdiv must be non-negative");
  if (!(d->coef_3rd_order >= 0.0f)) return fail(HEXDYN_E_ARG, "config_coef_3rd_order must be non-negative");
  if (!(d->apvm_upwinding >= 0.0f)) return fail(HEXDYN_E_ARG, "config_apvm_upwinding must be non-negative");
  const void* ptrs[] = {d->cells_on_edge, d->edges_on_cell, d->cells_on_cell, d->vertices_on_cell,
                        d->n_edges_on_cell, d->vertices_on_edge, d->edges_on_vertex, d->cells_on_vertex,
                        d->edges_on_edge, d->n_edges_on_edge, d->adv_cells, d->n_adv_cells, d->dc_edge,
                        d->dv_edge, d->area_cell, d->area_triangle, d->kite_areas, d->weights_on_edge,
                        d->f_vertex, d->f_edge, d->cos_angle_edge, d->sin_angle_edge, d->adv_coefs,
                        d->adv_coefs_3rd, d->fzm, d->fzp, d->rdzw, d->rdzu, d->zz, d->zxu, d->dss, d->zb_cell,
                        d->zb3_cell, d->rho_base, d->rho_theta_base, d->exner_base, d->u_init, d->v_init};
  for (size_t i = 0; i < sizeof ptrs / sizeof ptrs[0]; ++i)
    if (!ptrs[i]) return fail(HEXDYN_E_ARG, "descriptor array %zu is NULL", i);
  // connectivity ranges
  for (int e = 0; e < d->n_edges; ++e)
    for (int j = 0; j < 2; ++j) {
      const int c = d->cells_on_edge[2 * e + j];
      if (c < 0 || c >= d->n_cells) return fail(HEXDYN_E_ARG, "cellsOnEdge[%d] out of range (closed meshes only)", e);
      const int v = d->vertices_on_edge[2 * e + j];
      if (v < 0 || v >= d->n_vertices) return fail(HEXDYN_E_ARG, "verticesOnEdge[%d] out of range", e);
    }
  for (int c = 0; c < d->n_cells; ++c) {
    const int n = d->n_edges_on_cell[c];
    if (n < 3 || n > d->max_edges) return fail(HEXDYN_E_ARG, "nEdgesOnCell[%d]=%d out of range", c, n);
    for (int s = 0; s < n; ++s) {
      const int e = d->edges_on_cell[c * d->max_edges + s];
      const int nb = d->cells_on_cell[c * d->max_edges + s];
      const int v = d->vertices_on_cell[c * d->max_edges + s];
      if (e < 0 || e >= d->n_edges || nb < 0 || nb >= d->n_cells || v < 0 || v >= d->n_vertices)
        return fail(HEXDYN_E_ARG, "cell %d slot %d connectivity out of range", c, s);
    }
  }
  for (int v = 0; v < d->n_vertices; ++v)
    for (int s = 0; s < 3; ++s) {
      const int e = d->edges_on_vertex[3 * v + s], c = d->cells_on_vertex[3 * v + s];
      if (e < 0 || e >= d->n_edges || c < 0 || c >= d->n_cells)
        return fail(HEXDYN_E_ARG, "vertex %d slot %d connectivity out of range", v, s);
    }
  for (int e = 0; e < d->n_edges; ++e) {
    const int n = d->n_edges_on_edge[e];
    if (n < 0 || n > d->max_edges2) return fail(HEXDYN_E_ARG, "nEdgesOnEdge[%d] out of range", e);
    for (int s = 0; s < n; ++s) {
      const int x = d->edges_on_edge[e * d->max_edges2 + s];
      if (x < 0 || x >= d->n_edges) return fail(HEXDYN_E_ARG, "edgesOnEdge[%d][%d] out of range", e, s);
    }
    const int na = d->n_adv_cells[e];
    if (na < 2 || na > d->adv_width) return fail(HEXDYN_E_ARG, "nAdvCellsForEdge[%d] out of range", e);
    for (int s = 0; s < na; ++s) {
      const int x = d->adv_cells[e * d->adv_width + s];
      if (x < 0 || x >= d->n_cells) return fail(HEXDYN_E_ARG, "advCellsForEdge[%d][%d] out of range", e, s);
    }
  }
  return HEXDYN_OK;
}

int build(HexDynHandle* h, const HexDynDesc& d) {
  HexCtx& c = h->ctx;
  HexGeo& g = c.geo;
  const int L = d.n_levels;
  const int S = ((L + 1) + 7) / 8 * 8;
  g.nC = d.n_cells;
  g.nE = d.n_edges;
  g.nV = d.n_vertices;
  g.L = L;
  g.S = S;
  g.maxE = d.max_edges;
  g.maxE2 = d.max_edges2;
  g.advW = d.adv_width;
  c.numerics = d.numerics;
  c.n_scalars = d.n_scalars;
  c.dt = d.dt;
  c.split_steps = d.split_steps;
  c.monotonic = d.monotonic;
  const int nC = g.nC, nE = g.nE, nV = g.nV, mE = g.maxE;

  // integer connectivity and derived slot data
  std::vector<int> coe(d.cells_on_edge, d.cells_on_edge + 2 * nE);
  std::vector<int> eoc(d.edges_on_cell, d.edges_on_cell + (size_t)nC * mE);
  std::vector<int> coc(d.cells_on_cell, d.cells_on_cell + (size_t)nC * mE);
  std::vector<int> voc(d.vertices_on_cell, d.vertices_on_cell + (size_t)nC * mE);
  std::vector<int> deg(d.n_edges_on_cell, d.n_edges_on_cell + nC);
  std::vector<int> voe(d.vertices_on_edge, d.vertices_on_edge + 2 * nE);
  std::vector<int> eov(d.edges_on_vertex, d.edges_on_vertex + 3 * nV);
  std::vector<int> eoe(d.edges_on_edge, d.edges_on_edge + (size_t)nE * g.maxE2);
  std::vector<int> neoe(d.n_edges_on_edge, d.n_edges_on_edge + nE);
  std::vector<int> advc(d.adv_cells, d.adv_cells + (size_t)nE * g.advW);
  std::vector<int> nadv(d.n_adv_cells, d.n_adv_cells + nE);
  std::vector<int> kite_slot((size_t)nC * mE, 0);
  std::vector<float> csign((size_t)nC * mE, 0.0f), vsign(3 * (size_t)nV, 0.0f);
  for (int ci = 0; ci < nC; ++ci)
    for (int s = 0; s < deg[ci]; ++s) {
      const int e = eoc[(size_t)ci * mE + s];
      csign[(size_t)ci * mE + s] = coe[2 * e] == ci ? 1.0f : -1.0f;         // hexcore/acoustic.py:224
      const int v = voc[(size_t)ci * mE + s];
      int slot = -1;
      for (int j = 0; j < 3; ++j)
        if (d.cells_on_vertex[3 * v + j] == ci) slot = j;
      if (slot < 0) return fail(HEXDYN_E_ARG, "cell %d is missing from vertex %d", ci, v);
      kite_slot[(size_t)ci * mE + s] = slot;                                // hexcore/diagnostics.py:64
    }
  for (int v = 0; v < nV; ++v)
    for (int j = 0; j < 3; ++j) {
      const int e = eov[3 * v + j];
      vsign[3 * v + j] = voe[2 * e + 1] == v ? 1.0f : -1.0f;                 // hexcore/diagnostics.py:49
    }
  // precomputed RKIND inverses (hexcore/dynamics_v841.py:28)
  auto recip = [](const float* x, int n) {
    std::vector<float> r(n);
    for (int i = 0; i < n; ++i) r[i] = 1.0f / x[i];
    return r;
  };
  cudaError_t e;
#define UP(dst, vec) \
  if ((e = upload(c, &(dst), vec)) != cudaSuccess) return cuda_fail(e, "upload " #dst);
  UP(g.coe, coe) UP(g.eoc, eoc) UP(g.coc, coc) UP(g.voc, voc) UP(g.deg, deg) UP(g.voe, voe) UP(g.eov, eov)
  UP(g.eoe, eoe) UP(g.neoe, neoe) UP(g.adv_cells, advc) UP(g.n_adv, nadv) UP(g.kite_slot, kite_slot)
  UP(g.csign, csign) UP(g.vsign, vsign)
  std::vector<float> tmp;
  tmp.assign(d.dc_edge, d.dc_edge + nE); UP(g.dc, tmp)
  tmp.assign(d.dv_edge, d.dv_edge + nE); UP(g.dv, tmp)
  UP(g.inv_dc, recip(d.dc_edge, nE)) UP(g.inv_dv, recip(d.dv_edge, nE))
  UP(g.inv_area, recip(d.area_cell, nC)) UP(g.inv_area_tri, recip(d.area_triangle, nV))
  tmp.assign(d.kite_areas, d.kite_areas + 3 * (size_t)nV); UP(g.kite, tmp)
  tmp.assign(d.weights_on_edge, d.weights_on_edge + (size_t)nE * g.maxE2); UP(g.weights, tmp)
  tmp.assign(d.f_vertex, d.f_vertex + nV); UP(g.f_vertex, tmp)
  tmp.assign(d.f_edge, d.f_edge + nE); UP(g.f_edge, tmp)
  tmp.assign(d.cos_angle_edge, d.cos_angle_edge + nE); UP(g.cos_angle, tmp)
  tmp.assign(d.sin_angle_edge, d.sin_angle_edge + nE); UP(g.sin_angle, tmp)
  tmp.assign(d.adv_coefs, d.adv_coefs + (size_t)nE * g.advW); UP(g.adv, tmp)
  tmp.assign(d.adv_coefs_3rd, d.adv_coefs_3rd + (size_t)nE * g.advW); UP(g.adv3, tmp)
  UP(g.fzm, pad_vector(d.fzm, L, S)) UP(g.fzp, pad_vector(d.fzp, L, S))
  UP(g.rdzw, pad_vector(d.rdzw, L, S)) UP(g.rdzu, pad_vector(d.rdzu, L, S))
  UP(g.u_init, pad_vector(d.u_init, L, S)) UP(g.v_init, pad_vector(d.v_init, L, S))
  {
    std::vector<float> etp, etm, ewp, ewm;
    offcentering(d, d.rdzw, L, S, etp, etm, ewp, ewm);
    UP(g.etp, etp) UP(g.etm, etm) UP(g.ewp, ewp) UP(g.ewm, ewm)
  }
  UP(g.zz, pad_levels(d.zz, L, nC, S)) UP(g.zxu, pad_levels(d.zxu, L, nE, S))
  UP(g.dss, pad_levels(d.dss, L, nC, S)) UP(g.rho_base, pad_levels(d.rho_base, L, nC, S))
  UP(g.rtheta_base, pad_levels(d.rho_theta_base, L, nC, S)) UP(g.exner_base, pad_levels(d.exner_base, L, nC, S))
  {
    // [L+1][C][maxE] -> [C][maxE][S]
    std::vector<float> zb((size_t)nC * mE * S, 0.0f), zb3((size_t)nC * mE * S, 0.0f);
    for (int k = 0; k <= L; ++k)
      for (int ci = 0; ci < nC; ++ci)
        for (int s = 0; s < mE; ++s) {
          const size_t src = ((size_t)k * nC + ci) * mE + s, dst = ((size_t)ci * mE + s) * S + k;
          zb[dst] = d.zb_cell[src];
          zb3[dst] = d.zb3_cell[src];
        }
    UP(g.zb, zb) UP(g.zb3, zb3)
  }
#undef UP
  g.cf1 = d.cf1;
  g.cf2 = d.cf2;
  g.cf3 = d.cf3;
  g.coef3 = d.coef_3rd_order;
  g.g = d.gravity;
  g.rgas = d.rgas;
  g.rcv = d.rgas / (d.cp - d.rgas);
  g.c2 = d.cp * g.rcv;
  g.r_over_p0 = (float)((double)d.rgas / (double)d.p0);
  g.kappa = (float)((double)d.rgas / ((double)d.cp - (double)d.rgas));
  g.apvm_on = d.apvm_upwinding > 0.0f ? 1 : 0;
  g.apvm_scale = d.apvm_upwinding * (float)d.dt;
  const float len = d.len_disp > 0.0f ? d.len_disp : d.nominal_min_dc;
  g.smdiv_base = 2.0f * d.smdiv * len;
  g.moist = d.moist;
  g.winds_zero = 1;
  for (int k = 0; k < L; ++k)
    if (d.u_init[k] != 0.0f || d.v_init[k] != 0.0f) g.winds_zero = 0;

  // schedules (hexcore/integration.py:104 RKSchedule.from_mpas, order 3)
  const double dt_dyn = d.dt / d.split_steps;
  const int n = d.n_sub_steps;
  const double large[3] = {dt_dyn / 3.0, dt_dyn / 2.0, dt_dyn};
  const double acoustic[3] = {dt_dyn / 3.0, dt_dyn / n, dt_dyn / n};
  const int counts[3] = {1, std::max(1, n / 2), n};
  const double slarge[3] = {d.dt / 3.0, d.dt / 2.0, d.dt};
  for (int i = 0; i < 3; ++i) {
    const float dts = (float)acoustic[i];
    const float dts2 = d.acoustic_dts2[i] != 0.0f ? d.acoustic_dts2[i] : dts * dts;
    c.dyn[i] = HexStage{i + 1, large[i], acoustic[i], counts[i], dts2};
    c.scal[i] = HexStage{i + 1, slarge[i], d.dt / 3.0, 1, 0.0f};
  }

  // state and work buffers
  if ((e = alloc_state(c, c.in, true))) return cuda_fail(e, "alloc state");
  if ((e = alloc_state(c, c.out, true))) return cuda_fail(e, "alloc state");
  for (auto& t : c.tmp)
    if ((e = alloc_state(c, t, false))) return cuda_fail(e, "alloc state");
  if ((e = alloc_side(c, c.side_in)) || (e = alloc_side(c, c.side_out))) return cuda_fail(e, "alloc sidecar");
  for (auto& t : c.side_tmp)
    if ((e = alloc_side(c, t))) return cuda_fail(e, "alloc sidecar");
  HexWork& w = c.w;
  const size_t CS = (size_t)nC * S, ES = (size_t)nE * S, VS = (size_t)nV * S;
  const size_t T = std::max(1, c.n_scalars);
  struct { float** p; size_t n; } bufs[] = {
      {&w.qtot, CS}, {&w.cqw, CS}, {&w.cqu, ES}, {&w.pv_vertex, VS}, {&w.ke_vertex, VS}, {&w.ke, CS},
      {&w.pv_cell, CS}, {&w.v, ES}, {&w.pv_edge, ES}, {&w.euler_ru, ES}, {&w.tend_rho, CS}, {&w.euler_rw, CS},
      {&w.hdiv, CS}, {&w.edge_theta, ES}, {&w.edge_w, ES}, {&w.tend_ru, ES}, {&w.tend_rt, CS}, {&w.tend_rw, CS},
      {&w.cofwr, CS}, {&w.cofwz, CS}, {&w.coftz, CS}, {&w.cofwt, CS}, {&w.a_tri, CS}, {&w.alpha_tri, CS},
      {&w.gamma_tri, CS}, {&w.ru_p, ES}, {&w.ru_avg, ES}, {&w.rw_p, CS}, {&w.ww_avg, CS}, {&w.rho_pp, CS},
      {&w.rtpp[0], CS}, {&w.rtpp[1], CS}, {&w.flux_u, ES}, {&w.flux_w, CS}, {&w.q_stage[0], T * CS},
      {&w.q_stage[1], T * CS}, {&w.edge_q, T * ES}, {&w.target, CS}, {&w.scale_in, T * CS},
      {&w.scale_out, T * CS}, {&w.mass, T * CS}, {&w.hres_lim, T * ES}};
  for (auto& b : bufs)
    if ((e = dev_alloc(c, b.p, b.n))) return cuda_fail(e, "alloc work");
  if ((e = dev_alloc(c, &w.flag, 1))) return cuda_fail(e, "alloc flag");
  // dry coefficients: qtot = 0, cqw = cqu = 1 (hexcore/driver.py:2573,2787)
  k_fill<<<(unsigned)((CS + 255) / 256), 256>>>(w.cqw, CS, 1.0f);
  k_fill<<<(unsigned)((ES + 255) / 256), 256>>>(w.cqu, ES, 1.0f);
  HEX_CUDA(cudaGetLastError(), "fill");
  for (int f = 0; f < HEXDYN_NUM_FIELDS; ++f) {
    const FieldShape fs = field_shape(c, f);
    h->staging_count[f] = (size_t)fs.blocks * fs.rows * fs.n;
    if (h->staging_count[f] && (e = dev_alloc(c, &h->staging[f], h->staging_count[f])))
      return cuda_fail(e, "alloc staging");
  }
  HEX_CUDA(cudaMallocHost(&h->host_flag, sizeof(int)), "host flag");
  *h->host_flag = 0;
  HEX_CUDA(cudaDeviceSynchronize(), "create");
  return HEXDYN_OK;
}

HexState cur_state(HexDynHandle* h) { return h->ctx.parity ? h->ctx.out : h->ctx.in; }
HexSide cur_side(HexDynHandle* h) { return h->ctx.parity ? h->ctx.side_out : h->ctx.side_in; }

cudaError_t enqueue_step(HexDynHandle* h, cudaStream_t st, std::vector<HexProfEvent>* prof = nullptr) {
  HexCtx& c = h->ctx;
  const int p = c.parity;
  if (c.graph_exec[p] && !prof) return cudaGraphLaunch(c.graph_exec[p], st);
  const HexState& in = p ? c.out : c.in;
  const HexState& out = p ? c.in : c.out;
  const HexSide& si = p ? c.side_out : c.side_in;
  const HexSide& so = p ? c.side_in : c.side_out;
  long long launches = 0;
  cudaError_t e = c.numerics ? hexdyn_fast::run_step(c, in, si, out, so, st, &launches, prof)
                             : hexdyn_strict::run_step(c, in, si, out, so, st, &launches, prof);
  c.launches_per_step = launches;
  return e;
}

}  // namespace

extern "C" {

int hexdyn_abi_version(void) { return HEXDYN_ABI_VERSION; }

int hexdyn_create(const HexDynDesc* desc, HexDynHandle** out) {
  if (!out) return fail(HEXDYN_E_ARG, "out is NULL");
  *out = nullptr;
  int rc = validate(desc);
  if (rc) return rc;
  HexDynHandle* h = new HexDynHandle();
  rc = build(h, *desc);
  if (rc) {
    hexdyn_destroy(h);
    return rc;
  }
  *out = h;
  return HEXDYN_OK;
}

int hexdyn_set_state(HexDynHandle* h, int field, const float* host, size_t count, void* stream) {
  if (!h || !host) return fail(HEXDYN_E_ARG, "NULL handle or host pointer");
  if (field < 0 || field >= HEXDYN_NUM_FIELDS) return fail(HEXDYN_E_ARG, "unknown field %d", field);
  if (count != h->staging_count[field])
    return fail(HEXDYN_E_ARG, "field %d expects %zu values, got %zu", field, h->staging_count[field], count);
  if (count == 0) return HEXDYN_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const FieldShape fs = field_shape(h->ctx, field);
  float* dst = field_ptr(cur_state(h), cur_side(h), field);
  HEX_CUDA(cudaMemcpyAsync(h->staging[field], host, count * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
  for (int b = 0; b < fs.blocks; ++b) {
    dim3 grid((fs.n + 31) / 32, (fs.rows + 31) / 32), block(32, 8);
    k_to_padded<<<grid, block, 0, st>>>(h->staging[field] + (size_t)b * fs.rows * fs.n, fs.rows, fs.n, h->ctx.geo.S,
                                        dst + (size_t)b * fs.n * h->ctx.geo.S);
  }
  HEX_CUDA(cudaGetLastError(), "set_state transpose");
  h->have_state[field] = true;
  return HEXDYN_OK;
}

int hexdyn_get_state(HexDynHandle* h, int field, float* host, size_t count, void* stream) {
  if (!h || !host) return fail(HEXDYN_E_ARG, "NULL handle or host pointer");
  if (field < 0 || field >= HEXDYN_NUM_FIELDS) return fail(HEXDYN_E_ARG, "unknown field %d", field);
  if (count != h->staging_count[field])
    return fail(HEXDYN_E_ARG, "field %d holds %zu values, got %zu", field, h->staging_count[field], count);
  if (count == 0) return HEXDYN_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const FieldShape fs = field_shape(h->ctx, field);
  const float* src = field_ptr(cur_state(h), cur_side(h), field);
  for (int b = 0; b < fs.blocks; ++b) {
    dim3 grid((fs.n + 31) / 32, (fs.rows + 31) / 32), block(32, 8);
    k_from_padded<<<grid, block, 0, st>>>(src + (size_t)b * fs.n * h->ctx.geo.S, fs.rows, fs.n, h->ctx.geo.S,
                                          h->staging[field] + (size_t)b * fs.rows * fs.n);
  }
  HEX_CUDA(cudaGetLastError(), "get_state transpose");
  HEX_CUDA(cudaMemcpyAsync(host, h->staging[field], count * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H");
  return HEXDYN_OK;
}

int hexdyn_rebuild_sidecar(HexDynHandle* h, void* stream) {
  if (!h) return fail(HEXDYN_E_ARG, "NULL handle");
  for (int f = HEXDYN_RHO; f <= HEXDYN_RHO_W; ++f)
    if (!h->have_state[f]) return fail(HEXDYN_E_STATE, "state field %d was never set", f);
  cudaStream_t st = (cudaStream_t)stream;
  const HexState s = cur_state(h);
  const HexSide side = cur_side(h);
  cudaError_t e = h->ctx.numerics ? hexdyn_fast::rebuild_sidecar(h->ctx, s, side, st)
                                  : hexdyn_strict::rebuild_sidecar(h->ctx, s, side, st);
  if (e != cudaSuccess) return cuda_fail(e, "rebuild_sidecar");
  for (int f = HEXDYN_THETA_M; f < HEXDYN_NUM_FIELDS; ++f) h->have_state[f] = true;
  return HEXDYN_OK;
}

int hexdyn_step_async(HexDynHandle* h, void* stream, int nsteps) {
  if (!h) return fail(HEXDYN_E_ARG, "NULL handle");
  if (nsteps < 0) return fail(HEXDYN_E_ARG, "nsteps must be non-negative");
  for (int f = 0; f < HEXDYN_NUM_FIELDS; ++f)
    if (!h->have_state[f] && !(f == HEXDYN_SCALARS && h->ctx.n_scalars == 0))
      return fail(HEXDYN_E_STATE, "state field %d was never set (set it or rebuild the sidecar)", f);
  cudaStream_t st = (cudaStream_t)stream;
  for (int i = 0; i < nsteps; ++i) {
    cudaError_t e = enqueue_step(h, st);
    if (e != cudaSuccess) return cuda_fail(e, "step");
    h->ctx.parity ^= 1;
    h->ctx.steps_done++;
  }
  return HEXDYN_OK;
}

int hexdyn_profile_steps(HexDynHandle* h, void* stream, int nsteps, char* out, size_t len) {
  if (!h || !out || len == 0) return fail(HEXDYN_E_ARG, "NULL argument");
  if (nsteps <= 0) return fail(HEXDYN_E_ARG, "nsteps must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<HexProfEvent> prof;
  prof.reserve(4096);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < nsteps && e == cudaSuccess; ++i) {
    e = enqueue_step(h, st, &prof);
    h->ctx.parity ^= 1;
    h->ctx.steps_done++;
  }
  cudaError_t se = cudaStreamSynchronize(st);
  std::vector<std::string> names;
  std::vector<double> total;
  std::vector<long long> count;
  for (auto& ev : prof) {
    float ms = 0.0f;
    if (e == cudaSuccess && se == cudaSuccess) cudaEventElapsedTime(&ms, ev.start, ev.stop);
    size_t i = 0;
    while (i < names.size() && names[i] != ev.name) ++i;
    if (i == names.size()) {
      names.push_back(ev.name);
      total.push_back(0.0);
      count.push_back(0);
    }
    total[i] += ms;
    count[i] += 1;
    cudaEventDestroy(ev.start);
    cudaEventDestroy(ev.stop);
  }
  if (e != cudaSuccess) return cuda_fail(e, "profile step");
  if (se != cudaSuccess) return cuda_fail(se, "profile sync");
  std::string text;
  char line[256];
  for (size_t i = 0; i < names.size(); ++i) {
    snprintf(line, sizeof line, "%s %lld %.6f\n", names[i].c_str(), count[i], total[i]);
    text += line;
  }
  snprintf(out, len, "%s", text.c_str());
  return text.size() < len ? HEXDYN_OK : fail(HEXDYN_E_CAPACITY, "profile text needs %zu bytes", text.size() + 1);
}

int hexdyn_read_flag(HexDynHandle* h, void* stream, int* flag_out) {
  if (!h) return fail(HEXDYN_E_ARG, "NULL handle");
  cudaStream_t st = (cudaStream_t)stream;
  HEX_CUDA(cudaMemcpyAsync(h->host_flag, h->ctx.w.flag, sizeof(int), cudaMemcpyDeviceToHost, st), "flag D2H");
  HEX_CUDA(cudaMemsetAsync(h->ctx.w.flag, 0, sizeof(int), st), "flag clear");
  HEX_CUDA(cudaStreamSynchronize(st), "flag sync");
  if (flag_out) *flag_out = *h->host_flag;
  if (*h->host_flag) return fail(HEXDYN_E_NUMERIC, "device validation flag 0x%x set (density, singular system, powf "
                                 "domain or FCT target; reduce config_dt)", *h->host_flag);
  return HEXDYN_OK;
}

int hexdyn_step(HexDynHandle* h, void* stream, int nsteps, int* flag_out, int* completed) {
  if (completed) *completed = 0;
  int rc = hexdyn_step_async(h, stream, nsteps);
  if (rc) return rc;
  if (completed) *completed = nsteps;
  return hexdyn_read_flag(h, stream, flag_out);
}

int hexdyn_capture_graph(HexDynHandle* h, void* stream) {
  if (!h) return fail(HEXDYN_E_ARG, "NULL handle");
  HexCtx& c = h->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  bool own = false;
  if (!st) {
    HEX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "capture stream");
    own = true;
  }
  const int saved_parity = c.parity;
  for (int p = 0; p < 2; ++p) {
    if (c.graph_exec[p]) {
      cudaGraphExecDestroy(c.graph_exec[p]);
      c.graph_exec[p] = nullptr;
    }
    if (c.graph[p]) {
      cudaGraphDestroy(c.graph[p]);
      c.graph[p] = nullptr;
    }
    c.parity = p;
    HEX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t e = enqueue_step(h, st);
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) return cuda_fail(e, "capture step");
    if (e2 != cudaSuccess) return cuda_fail(e2, "end capture");
    c.graph[p] = graph;
    HEX_CUDA(cudaGraphInstantiate(&c.graph_exec[p], graph, 0), "instantiate");
  }
  c.parity = saved_parity;
  if (own) cudaStreamDestroy(st);
  return HEXDYN_OK;
}

int hexdyn_device_field(HexDynHandle* h, int field, void** dev_ptr) {
  if (!h || !dev_ptr) return fail(HEXDYN_E_ARG, "NULL argument");
  if (field < 0 || field >= HEXDYN_NUM_FIELDS) return fail(HEXDYN_E_ARG, "unknown field %d", field);
  *dev_ptr = field_ptr(cur_state(h), cur_side(h), field);
  return HEXDYN_OK;
}

int hexdyn_level_stride(HexDynHandle* h) { return h ? h->ctx.geo.S : 0; }
long long hexdyn_launches_per_step(HexDynHandle* h) { return h ? h->ctx.launches_per_step : 0; }
size_t hexdyn_device_bytes(HexDynHandle* h) { return h ? h->ctx.device_bytes : 0; }

int hexdyn_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return HEXDYN_E_ARG;
  snprintf(buf, len, "%s", g_last_error.c_str());
  return HEXDYN_OK;
}

int hexdyn_destroy(HexDynHandle* h) {
  if (!h) return HEXDYN_OK;
  HexCtx& c = h->ctx;
  for (int p = 0; p < 2; ++p) {
    if (c.graph_exec[p]) cudaGraphExecDestroy(c.graph_exec[p]);
    if (c.graph[p]) cudaGraphDestroy(c.graph[p]);
  }
  for (void* p : c.allocations) cudaFree(p);
  if (h->host_flag) cudaFreeHost(h->host_flag);
  delete h;
  return HEXDYN_OK;
}

}  // extern "C"

// ------------------------------------------------------------ no-alloc step
// hexdyn_step_noalloc: the large step with its scratch in a file-scope device
// array instead of the handle's workspace (declaration and contract in
// include/hexdyn.h).

#include <mutex>

#define HEXDYN_NOALLOC_SCRATCH_BYTES (64u << 20)
#define HEXDYN_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) float g_noalloc_scratch[HEXDYN_NOALLOC_SCRATCH_BYTES / sizeof(float)];

namespace {

std::mutex g_noalloc_mutex;
float* g_noalloc_ptr[HEXDYN_NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on the current device, looked up once
// per device with that device current.
int noalloc_scratch(float** out) {
  int dev = 0;
  HEX_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= HEXDYN_NOALLOC_MAX_DEVICES)
    return fail(HEXDYN_E_CAPACITY, "device %d beyond the %d devices the no-alloc step tracks", dev,
                HEXDYN_NOALLOC_MAX_DEVICES);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    HEX_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
    g_noalloc_ptr[dev] = (float*)p;
  }
  *out = g_noalloc_ptr[dev];
  return HEXDYN_OK;
}

// Bump carver over the scratch array; every buffer starts on 256 bytes.
struct Carver {
  float* base;
  size_t used = 0;  // words
  float* take(size_t words) {
    float* p = base ? base + used : nullptr;
    used += (words + 63) / 64 * 64;
    return p;
  }
};

// Lays out the step's intermediates; with base == nullptr only counts.
void carve(Carver& cv, const HexCtx& src, HexCtx& c) {
  const HexGeo& g = src.geo;
  const size_t CS = (size_t)g.nC * g.S, ES = (size_t)g.nE * g.S, VS = (size_t)g.nV * g.S;
  const size_t T = std::max(1, src.n_scalars);
  HexWork& w = c.w;
  float** cell[] = {&w.qtot, &w.cqw, &w.ke, &w.pv_cell, &w.tend_rho, &w.euler_rw, &w.hdiv, &w.tend_rt,
                    &w.tend_rw, &w.cofwr, &w.cofwz, &w.coftz, &w.cofwt, &w.a_tri, &w.alpha_tri, &w.gamma_tri,
                    &w.rw_p, &w.ww_avg, &w.rho_pp, &w.rtpp[0], &w.rtpp[1], &w.flux_w, &w.target};
  for (float** p : cell) *p = cv.take(CS);
  float** edge[] = {&w.cqu, &w.v, &w.pv_edge, &w.euler_ru, &w.edge_theta, &w.edge_w, &w.tend_ru, &w.ru_p,
                    &w.ru_avg, &w.flux_u};
  for (float** p : edge) *p = cv.take(ES);
  w.pv_vertex = cv.take(VS);
  w.ke_vertex = cv.take(VS);
  float** tcell[] = {&w.q_stage[0], &w.q_stage[1], &w.scale_in, &w.scale_out, &w.mass};
  for (float** p : tcell) *p = cv.take(T * CS);
  w.edge_q = cv.take(T * ES);
  w.hres_lim = cv.take(T * ES);
  w.flag = (int*)cv.take(1);
  for (int i = 0; i < 2; ++i) {
    HexState& t = c.tmp[i];
    t.rho = cv.take(CS);
    t.rho_theta = cv.take(CS);
    t.rho_w = cv.take(CS);
    t.rho_u = cv.take(ES);
    t.scalars = nullptr;
    HexSide& sd = c.side_tmp[i];
    float** sc[] = {&sd.theta_m, &sd.exner, &sd.rho_p, &sd.rtheta_p, &sd.pressure_p, &sd.w};
    for (float** p : sc) *p = cv.take(CS);
    sd.u = cv.take(ES);
  }
}

bool fields_of(const HexDynFields* f, int n_scalars, HexState& s, HexSide& side) {
  for (int i = 0; i < HEXDYN_NUM_FIELDS; ++i)
    if (!f->field[i] && !(i == HEXDYN_SCALARS && n_scalars == 0)) return false;
  s = HexState{f->field[HEXDYN_RHO], f->field[HEXDYN_RHO_THETA], f->field[HEXDYN_RHO_U], f->field[HEXDYN_RHO_W],
               f->field[HEXDYN_SCALARS]};
  side = HexSide{f->field[HEXDYN_THETA_M], f->field[HEXDYN_EXNER], f->field[HEXDYN_RHO_P],
                 f->field[HEXDYN_RHO_THETA_P], f->field[HEXDYN_PRESSURE_P], f->field[HEXDYN_U],
                 f->field[HEXDYN_W]};
  return true;
}

}  // namespace

extern "C" int hexdyn_step_noalloc(HexDynHandle* h, const HexDynFields* in, const HexDynFields* out, void* stream,
                                   int* flag_out) {
  if (!h || !in || !out) return fail(HEXDYN_E_ARG, "NULL handle or field set");
  const HexCtx& src = h->ctx;
  HexState s_in, s_out;
  HexSide d_in, d_out;
  if (!fields_of(in, src.n_scalars, s_in, d_in) || !fields_of(out, src.n_scalars, s_out, d_out))
    return fail(HEXDYN_E_ARG, "every state and sidecar field needs a device pointer");
  for (int i = 0; i < HEXDYN_NUM_FIELDS; ++i)
    for (int j = 0; j < HEXDYN_NUM_FIELDS; ++j)
      if (in->field[i] && in->field[i] == out->field[j])
        return fail(HEXDYN_E_ARG, "input field %d and output field %d are the same buffer", i, j);
  // Size check before touching the device.
  HexCtx c;
  Carver count{nullptr};
  carve(count, src, c);
  const size_t need = count.used * sizeof(float);
  if (need > HEXDYN_NOALLOC_SCRATCH_BYTES)
    return fail(HEXDYN_E_CAPACITY, "this mesh needs %zu bytes of step scratch; the no-alloc step holds %u "
                "(use hexdyn_step)", need, (unsigned)HEXDYN_NOALLOC_SCRATCH_BYTES);
  float* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  Carver cv{base};
  carve(cv, src, c);
  c.numerics = src.numerics;
  c.n_scalars = src.n_scalars;
  c.dt = src.dt;
  c.split_steps = src.split_steps;
  c.monotonic = src.monotonic;
  c.geo = src.geo;
  for (int i = 0; i < 3; ++i) {
    c.dyn[i] = src.dyn[i];
    c.scal[i] = src.scal[i];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const HexGeo& g = c.geo;
  const size_t CS = (size_t)g.nC * g.S, ES = (size_t)g.nE * g.S;
  // what must start at zero (or one): the flag and the dry coefficients
  HEX_CUDA(cudaMemsetAsync(c.w.flag, 0, sizeof(int), st), "clear flag");
  if (!g.moist) {
    HEX_CUDA(cudaMemsetAsync(c.w.qtot, 0, CS * sizeof(float), st), "clear qtot");
    k_fill<<<(unsigned)((CS + 255) / 256), 256, 0, st>>>(c.w.cqw, CS, 1.0f);
    k_fill<<<(unsigned)((ES + 255) / 256), 256, 0, st>>>(c.w.cqu, ES, 1.0f);
    HEX_CUDA(cudaGetLastError(), "fill dry coefficients");
  }
  long long launches = 0;
  cudaError_t e = c.numerics ? hexdyn_fast::run_step(c, s_in, d_in, s_out, d_out, st, &launches, nullptr)
                             : hexdyn_strict::run_step(c, s_in, d_in, s_out, d_out, st, &launches, nullptr);
  if (e != cudaSuccess) return cuda_fail(e, "no-alloc step");
  int flag = 0;
  HEX_CUDA(cudaMemcpyAsync(&flag, c.w.flag, sizeof(int), cudaMemcpyDeviceToHost, st), "flag D2H");
  HEX_CUDA(cudaStreamSynchronize(st), "no-alloc step sync");
  if (flag_out) *flag_out = flag;
  if (flag) return fail(HEXDYN_E_NUMERIC, "device validation flag 0x%x set in the no-alloc step", flag);
  return HEXDYN_OK;
}

