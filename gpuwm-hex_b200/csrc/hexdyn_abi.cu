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
  // ensemble members: first cell / edge / vertex and counts of each member in
  // the concatenated mesh (one member for a single instance), and the fields
  // each member has been given
  std::vector<int> m_c0, m_e0, m_v0, m_nc, m_ne, m_nv;
  std::vector<unsigned> m_have;
  // the library's own buffers of the parity-0 state while caller buffers are
  // bound (hexdyn_bind_state)
  bool bound = false;
  HexState own_in{};
  HexSide own_side_in{};
  // private stream and events of hexdyn_step_batched
  cudaStream_t batch_stream = nullptr;
  cudaEvent_t batch_fork = nullptr, batch_done = nullptr;
  // downloads of hexdyn_step_host that overlap the scalar transport
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_done = nullptr;
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
  if (d->time_integration_order != 0 && d->time_integration_order != 2 && d->time_integration_order != 3)
    return fail(HEXDYN_E_ARG, "config_time_integration_order=%d: only 2 and 3 exist", d->time_integration_order);
  if (d->split_steps != 1 && d->split_steps != 3)
    return fail(HEXDYN_E_ARG, "config_dynamics_split_steps=%d: only 1 and 3 are implemented", d->split_steps);
  if (d->moist != 0 && d->moist != 1) return fail(HEXDYN_E_ARG, "moist=%d must be 0 or 1", d->moist);
  if (d->numerics != 0 && d->numerics != 1) return fail(HEXDYN_E_ARG, "numerics=%d must be 0 or 1", d->numerics);
  if (!(d->smdiv >= 0.0f)) return fail(HEXDYN_E_ARG, "config_smdiv must be non-negative");
  if (!(d->coef_3rd_order >= 0.0f)) return fail(HEXDYN_E_ARG, "config_coef_3rd_order must be non-negative");
  if (!(d->apvm_upwinding >= 0.0f)) return fail(HEXDYN_E_ARG, "config_apvm_upwinding must be non-negative");
  if (d->rayleigh_levels < 0 || d->rayleigh_levels > d->n_levels || d->cam_levels < 0 ||
      d->cam_levels > d->n_levels)
    return fail(HEXDYN_E_ARG, "upper damping level counts (%d, %d) must lie in 0..n_levels", d->rayleigh_levels,
                d->cam_levels);
  if (d->cam_levels && !d->horiz_mixing)
    return fail(HEXDYN_E_ARG, "the CAM floor applies to the Smagorinsky diffusivity: mixing must be on");
  if (d->clamp_negative_scalars != 0 && d->clamp_negative_scalars != 1)
    return fail(HEXDYN_E_ARG, "clamp_negative_scalars=%d must be 0 or 1", d->clamp_negative_scalars);
  if (d->horiz_mixing != 0 && d->horiz_mixing != 1)
    return fail(HEXDYN_E_ARG, "horiz_mixing=%d must be 0 (off) or 1 (2-D Smagorinsky)", d->horiz_mixing);
  if (d->horiz_mixing) {
    if (!d->deform_c2 || !d->deform_s2 || !d->deform_cs || !d->mix_del2 || !d->mix_del4)
      return fail(HEXDYN_E_ARG, "2-D Smagorinsky mixing needs the deformation weights and mesh scalings");
    if (!(d->smag_strain_scale >= 0.0f) || !(d->smag_ceiling >= 0.0f) || !(d->smag_h4 >= 0.0f) ||
        !(d->smag_div_factor > 0.0f))
      return fail(HEXDYN_E_ARG, "invalid Smagorinsky constants");
  }
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

// smdiv_edge: per-edge 2*smdiv*len_disp for ensembles of several meshes;
// NULL gives every edge the descriptor's value.
int build(HexDynHandle* h, const HexDynDesc& d, const std::vector<float>* smdiv_edge = nullptr) {
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
  g.coc_across = 1;
  for (int ci = 0; ci < nC; ++ci)
    for (int s = 0; s < deg[ci]; ++s) {
      const int e = eoc[(size_t)ci * mE + s];
      csign[(size_t)ci * mE + s] = coe[2 * e] == ci ? 1.0f : -1.0f;         // hexcore/acoustic.py:224
      if (coc[(size_t)ci * mE + s] != (coe[2 * e] == ci ? coe[2 * e + 1] : coe[2 * e])) g.coc_across = 0;
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
  {
    const std::vector<float> sm = smdiv_edge ? *smdiv_edge : std::vector<float>((size_t)nE, g.smdiv_base);
    if ((e = upload(c, &g.smdiv_edge, sm)) != cudaSuccess) return cuda_fail(e, "upload smdiv_edge");
  }
  g.moist = d.moist;
  g.smag_on = d.horiz_mixing ? 1 : 0;
  if (g.smag_on) {
    // hexcore/mixing_v841.py:495 weights, hexcore/mixing.py:271 scalings and
    // the limited inverse dvEdge of hexcore/mixing.py:440
    std::vector<float> tmp;
    const size_t slots = (size_t)nC * g.maxE;
    tmp.assign(d.deform_c2, d.deform_c2 + slots);
    if ((e = upload(c, &g.deform_c2, tmp)) != cudaSuccess) return cuda_fail(e, "upload deform_c2");
    tmp.assign(d.deform_s2, d.deform_s2 + slots);
    if ((e = upload(c, &g.deform_s2, tmp)) != cudaSuccess) return cuda_fail(e, "upload deform_s2");
    tmp.assign(d.deform_cs, d.deform_cs + slots);
    if ((e = upload(c, &g.deform_cs, tmp)) != cudaSuccess) return cuda_fail(e, "upload deform_cs");
    tmp.assign(d.mix_del2, d.mix_del2 + nE);
    if ((e = upload(c, &g.mix_del2, tmp)) != cudaSuccess) return cuda_fail(e, "upload mix_del2");
    tmp.assign(d.mix_del4, d.mix_del4 + nE);
    if ((e = upload(c, &g.mix_del4, tmp)) != cudaSuccess) return cuda_fail(e, "upload mix_del4");
    tmp.resize(nE);
    for (int ei = 0; ei < nE; ++ei) {
      const float idv = 1.0f / d.dv_edge[ei], lim = 4.0f * (1.0f / d.dc_edge[ei]);
      tmp[ei] = idv < lim ? idv : lim;
    }
    if ((e = upload(c, &g.inv_dv_lim, tmp)) != cudaSuccess) return cuda_fail(e, "upload inv_dv_lim");
    g.smag_strain_scale = d.smag_strain_scale;
    g.smag_ceiling = d.smag_ceiling;
    g.smag_h4 = d.smag_h4;
    g.smag_div_factor = d.smag_div_factor;
  }
  g.clamp_scalars = d.clamp_negative_scalars;
  g.rayleigh_levels = d.rayleigh_levels;
  g.rayleigh_inverse = d.rayleigh_inverse;
  g.cam_levels = d.cam_levels;
  g.cam_base = d.cam_base;
  g.winds_zero = 1;
  for (int k = 0; k < L; ++k)
    if (d.u_init[k] != 0.0f || d.v_init[k] != 0.0f) g.winds_zero = 0;
  g.dss_zero = 1;
  for (size_t i = 0; i < (size_t)L * nC && g.dss_zero; ++i) {
    uint32_t bits;
    memcpy(&bits, d.dss + i, sizeof bits);
    if (bits != 0u) g.dss_zero = 0;
  }

  // schedules (hexcore/integration.py:104 RKSchedule.from_mpas): order 3
  // (dt/3, dt/2, dt; one substep of dt/3, then n/2 and n of dt/n) or order
  // 2 (dt/2, dt/2, dt; n/2, n/2 and n substeps of dt/n)
  c.order = d.time_integration_order == 2 ? 2 : 3;
  const double dt_dyn = d.dt / d.split_steps;
  const int n = d.n_sub_steps;
  const bool rk2 = c.order == 2;
  const double large[3] = {dt_dyn / (rk2 ? 2.0 : 3.0), dt_dyn / 2.0, dt_dyn};
  const double acoustic[3] = {rk2 ? dt_dyn / n : dt_dyn / 3.0, dt_dyn / n, dt_dyn / n};
  const int counts[3] = {rk2 ? std::max(1, n / 2) : 1, std::max(1, n / 2), n};
  const double slarge[3] = {d.dt / (rk2 ? 2.0 : 3.0), d.dt / 2.0, d.dt};
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
      {&w.scale_out, T * CS}, {&w.mass, T * CS}, {&w.hres_lim, T * ES}, {&w.vres, T * CS}};
  for (auto& b : bufs)
    if ((e = dev_alloc(c, b.p, b.n))) return cuda_fail(e, "alloc work");
  if ((e = dev_alloc(c, &w.flag, 1))) return cuda_fail(e, "alloc flag");
  if (c.geo.smag_on) {
    struct { float** p; size_t n; } mix[] = {
        {&w.vorticity, VS}, {&w.divergence, CS}, {&w.kdiff, CS}, {&w.delsq_u, ES}, {&w.delsq_div, CS},
        {&w.delsq_vort, VS}, {&w.w_mix, CS}, {&w.delsq_w, CS}, {&w.theta_mix, CS}, {&w.delsq_theta, CS},
        {&w.mix_u, ES}, {&w.mix_w, CS}};
    for (auto& b : mix)
      if ((e = dev_alloc(c, b.p, b.n))) return cuda_fail(e, "alloc mixing");
  }
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
  // HEXDYN_CONCURRENT=0 keeps every launch of a step on the caller's stream
  const char* conc = getenv("HEXDYN_CONCURRENT");
  if (conc) c.concurrent_regions = atoi(conc);
  if (c.concurrent_regions != 0) {
    HEX_CUDA(cudaStreamCreateWithFlags(&c.side_stream, cudaStreamNonBlocking), "side stream");
    for (auto& ev : c.fork_events) HEX_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "fork event");
  }
  HEX_CUDA(cudaEventCreateWithFlags(&c.dynamics_done, cudaEventDisableTiming), "dynamics event");
  HEX_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking), "copy stream");
  HEX_CUDA(cudaEventCreateWithFlags(&h->copy_done, cudaEventDisableTiming), "copy event");
  HEX_CUDA(cudaDeviceSynchronize(), "create");
  return HEXDYN_OK;
}

HexState cur_state(HexDynHandle* h) { return h->ctx.parity ? h->ctx.out : h->ctx.in; }
HexSide cur_side(HexDynHandle* h) { return h->ctx.parity ? h->ctx.side_out : h->ctx.side_in; }

cudaError_t enqueue_step(HexDynHandle* h, cudaStream_t st, std::vector<HexProfEvent>* prof = nullptr) {
  HexCtx& c = h->ctx;
  const int p = c.parity;
  // a physics stage hook runs on the host between the stage launches: eager
  if (c.graph_exec[p] && !prof && !c.stage_hook && !c.exchange_hook) return cudaGraphLaunch(c.graph_exec[p], st);
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
  h->m_c0 = {0};
  h->m_e0 = {0};
  h->m_v0 = {0};
  h->m_nc = {desc->n_cells};
  h->m_ne = {desc->n_edges};
  h->m_nv = {desc->n_vertices};
  h->m_have = {0u};
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
    if (h->ctx.phys_failed) {
      h->ctx.phys_failed = 0;
      return fail(HEXDYN_E_STATE, "a physics or halo exchange hook aborted step %d (nothing was published)", i + 1);
    }
    if (e != cudaSuccess) return cuda_fail(e, "step");
    h->ctx.parity ^= 1;
    h->ctx.steps_done++;
  }
  return HEXDYN_OK;
}

int hexdyn_step_host(HexDynHandle* h, const float* const* in, float* const* out, void* stream) {
  if (!h || !in || !out) return fail(HEXDYN_E_ARG, "NULL argument");
  for (int f = 0; f < HEXDYN_NUM_FIELDS; ++f)
    if (h->staging_count[f] && (!in[f] || !out[f])) return fail(HEXDYN_E_ARG, "NULL host buffer of field %d", f);
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  for (int f = 0; f < HEXDYN_NUM_FIELDS; ++f)
    if (h->staging_count[f] && (rc = hexdyn_set_state(h, f, in[f], h->staging_count[f], stream)) != HEXDYN_OK)
      return rc;
  if ((rc = hexdyn_step_async(h, stream, 1)) != HEXDYN_OK) return rc;
  // every field but the scalars leaves on the copy stream once the step's
  // dynamics end (beside the scalar transport); the scalars after the step
  HEX_CUDA(cudaStreamWaitEvent(h->copy_stream, h->ctx.dynamics_done, 0), "copy wait");
  for (int f = 0; f < HEXDYN_NUM_FIELDS; ++f)
    if (f != HEXDYN_SCALARS && h->staging_count[f] &&
        (rc = hexdyn_get_state(h, f, out[f], h->staging_count[f], h->copy_stream)) != HEXDYN_OK)
      return rc;
  if (h->staging_count[HEXDYN_SCALARS] &&
      (rc = hexdyn_get_state(h, HEXDYN_SCALARS, out[HEXDYN_SCALARS], h->staging_count[HEXDYN_SCALARS], stream)) !=
          HEXDYN_OK)
    return rc;
  HEX_CUDA(cudaEventRecord(h->copy_done, h->copy_stream), "copy record");
  HEX_CUDA(cudaStreamWaitEvent(st, h->copy_done, 0), "copy join");
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

// Per-label mean launch time (ms) of nsteps eager steps, one CUDA event pair
// per launch.
static cudaError_t profile_means(HexDynHandle* h, cudaStream_t st, int nsteps,
                                 std::vector<std::pair<std::string, double>>& out) {
  std::vector<HexProfEvent> prof;
  prof.reserve(4096);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < nsteps && e == cudaSuccess; ++i) {
    e = enqueue_step(h, st, &prof);
    h->ctx.parity ^= 1;
  }
  cudaError_t se = cudaStreamSynchronize(st);
  std::vector<long long> count;
  out.clear();
  for (auto& ev : prof) {
    float ms = 0.0f;
    if (e == cudaSuccess && se == cudaSuccess) cudaEventElapsedTime(&ms, ev.start, ev.stop);
    size_t i = 0;
    while (i < out.size() && out[i].first != ev.name) ++i;
    if (i == out.size()) {
      out.emplace_back(ev.name, 0.0);
      count.push_back(0);
    }
    out[i].second += ms;
    count[i] += 1;
    cudaEventDestroy(ev.start);
    cudaEventDestroy(ev.stop);
  }
  for (size_t i = 0; i < out.size(); ++i) out[i].second /= (double)count[i];
  return e != cudaSuccess ? e : se;
}

int hexdyn_autotune(HexDynHandle* h, void* stream, int steps_per_candidate, char* report, size_t len) {
  if (!h || steps_per_candidate < 1) return fail(HEXDYN_E_ARG, "NULL handle or steps_per_candidate < 1");
  for (int f = 0; f < HEXDYN_NUM_FIELDS; ++f)
    if (!h->have_state[f] && !(f == HEXDYN_SCALARS && h->ctx.n_scalars == 0))
      return fail(HEXDYN_E_STATE, "state field %d was never set", f);
  HexCtx& c = h->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  // save the current state and sidecar; every candidate starts from it
  struct Saved { float* dev; float* copy; size_t bytes; };
  std::vector<Saved> saved;
  const HexState s0 = cur_state(h);
  const HexSide d0 = cur_side(h);
  for (int f = 0; f < HEXDYN_NUM_FIELDS; ++f) {
    const FieldShape fs = field_shape(c, f);
    const size_t words = (size_t)fs.blocks * fs.n * c.geo.S;
    float* dev = field_ptr(s0, d0, f);
    if (!dev || words == 0) continue;
    void* copy = nullptr;
    cudaError_t e = cudaMalloc(&copy, words * sizeof(float));
    if (e != cudaSuccess) {
      for (auto& x : saved) cudaFree(x.copy);
      return cuda_fail(e, "autotune state copy");
    }
    saved.push_back({dev, (float*)copy, words * sizeof(float)});
    cudaMemcpyAsync(copy, dev, words * sizeof(float), cudaMemcpyDeviceToDevice, st);
  }
  const int parity0 = c.parity;
  auto restore = [&]() {
    c.parity = parity0;
    for (auto& x : saved) cudaMemcpyAsync(x.dev, x.copy, x.bytes, cudaMemcpyDeviceToDevice, st);
  };
  // block sizes tried per launch label (a level-vector block holds
  // threads / (S/4) cells or edges, a column-group block threads / G columns)
#ifndef HEX_TUNE_CANDIDATES
#if HEX_TUNE_THREE
#define HEX_TUNE_CANDIDATES 64, 128, 256
#else
#define HEX_TUNE_CANDIDATES 64, 96, 128, 160, 192, 224, 256
#endif
#endif
  const int candidates[] = {HEX_TUNE_CANDIDATES};
  constexpr int NC = (int)(sizeof(candidates) / sizeof(candidates[0]));
  std::vector<std::pair<std::string, double>> times[NC];
  cudaError_t err = cudaSuccess;
  for (int ci = 0; ci < NC && err == cudaSuccess; ++ci) {
    restore();
    c.force_threads = candidates[ci];
    err = profile_means(h, st, steps_per_candidate, times[ci]);
  }
  c.force_threads = 0;
  restore();
  cudaError_t se = cudaStreamSynchronize(st);
  for (auto& x : saved) cudaFree(x.copy);
  cudaMemsetAsync(c.w.flag, 0, sizeof(int), st);
  if (err != cudaSuccess) return cuda_fail(err, "autotune step");
  if (se != cudaSuccess) return cuda_fail(se, "autotune restore");
  // the fastest block size of every label; the report's first line lists
  // the candidates, then one line per label: its mean microseconds at each
  // candidate and the choice
  std::string text = "threads";
  for (int ci = 0; ci < NC; ++ci) text += " " + std::to_string(candidates[ci]);
  text += "\n";
  std::vector<std::pair<std::string, int>> tuned;
  for (const auto& lab : times[NC - 1]) {
    double best = 1e30;
    int best_t = candidates[NC - 1];
    std::string line = lab.first;
    for (int ci = 0; ci < NC; ++ci) {
      double t = 0.0;
      for (const auto& x : times[ci])
        if (x.first == lab.first) t = x.second;
      if (t > 0.0 && t < best) {
        best = t;
        best_t = candidates[ci];
      }
      char num[32];
      snprintf(num, sizeof num, " %.3f", 1000.0 * t);
      line += num;
    }
    line += " " + std::to_string(best_t) + "\n";
    tuned.emplace_back(lab.first, best_t);
    text += line;
  }
  c.tuned_threads = tuned;
  // captured graphs hold the old launch shapes
  if (c.graph_exec[0] || c.graph_exec[1]) {
    const int rc = hexdyn_capture_graph(h, stream);
    if (rc) return rc;
  }
  if (report && len) snprintf(report, len, "%s", text.c_str());
  return (report && len && text.size() >= len) ? fail(HEXDYN_E_CAPACITY, "report needs %zu bytes", text.size() + 1)
                                               : HEXDYN_OK;
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
  if (c.stage_hook || c.exchange_hook)
    return fail(HEXDYN_E_STATE, "a physics or halo exchange hook runs on the host between stages: the step stays "
                "eager");
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

int hexdyn_acoustic_field(HexDynHandle* h, int which, void** dev_ptr) {
  if (!h || !dev_ptr) return fail(HEXDYN_E_ARG, "NULL argument");
  if (which == HEXDYN_WORK_RU_P) *dev_ptr = h->ctx.w.ru_p;
  else if (which == HEXDYN_WORK_RW_P) *dev_ptr = h->ctx.w.rw_p;
  else return fail(HEXDYN_E_ARG, "unknown acoustic field %d", which);
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
  for (auto& ev : c.fork_events)
    if (ev) cudaEventDestroy(ev);
  if (c.side_stream) cudaStreamDestroy(c.side_stream);
  if (c.dynamics_done) cudaEventDestroy(c.dynamics_done);
  if (h->copy_done) cudaEventDestroy(h->copy_done);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->host_flag) cudaFreeHost(h->host_flag);
  if (h->batch_fork) cudaEventDestroy(h->batch_fork);
  if (h->batch_done) cudaEventDestroy(h->batch_done);
  if (h->batch_stream) cudaStreamDestroy(h->batch_stream);
  delete h;
  return HEXDYN_OK;
}

}  // extern "C"

// ------------------------------------------------------------ ensembles
// An ensemble handle holds several members as one mesh: member m's cells,
// edges and vertices are a contiguous range of the concatenated mesh, its
// connectivity is offset into that range, and no stencil reaches across
// members.  Every kernel of the step therefore computes each member exactly
// as a handle of its own would, in one launch for all members.

namespace {

template <class T>
bool same_bits(const T* a, const T* b, size_t n) {
  return memcmp(a, b, n * sizeof(T)) == 0;
}

// Owns the arrays of the concatenated descriptor.
struct MergedDesc {
  HexDynDesc d{};
  std::vector<int32_t> coe, eoc, coc, voc, deg, voe, eov, cov, eoe, neoe, advc, nadv;
  std::vector<float> dc, dv, area, area_tri, kite, weights, fv, fe, cosa, sina, adv, adv3;
  std::vector<float> zz, zxu, dss, zb, zb3, rb, rtb, eb;
  std::vector<float> smdiv_edge;
  std::vector<float> deform_c2, deform_s2, deform_cs, mix_del2, mix_del4;
};

int check_compatible(const HexDynDesc& a, const HexDynDesc& b, int m) {
  const int L = a.n_levels;
  auto bad = [&](const char* what) {
    return fail(HEXDYN_E_ARG, "ensemble member %d differs from member 0 in %s (members of one ensemble share "
                "the configuration, levels, tracers and vertical coordinate)", m, what);
  };
  if (b.n_levels != L) return bad("n_levels");
  if (b.n_scalars != a.n_scalars) return bad("n_scalars");
  if (b.dt != a.dt) return bad("dt");
  if (b.n_sub_steps != a.n_sub_steps || b.split_steps != a.split_steps ||
      (b.time_integration_order == 2) != (a.time_integration_order == 2))
    return bad("the schedule");
  if (b.monotonic != a.monotonic || b.moist != a.moist || b.numerics != a.numerics ||
      b.clamp_negative_scalars != a.clamp_negative_scalars)
    return bad("the options");
  const float fa[] = {a.coef_3rd_order, a.apvm_upwinding, a.smdiv, a.len_disp, a.epssm_minimum, a.epssm_maximum,
                      a.epssm_bottom_z, a.epssm_top_z, a.rgas, a.cp, a.gravity, a.p0, a.cf1, a.cf2, a.cf3,
                      a.acoustic_dts2[0], a.acoustic_dts2[1], a.acoustic_dts2[2]};
  const float fb[] = {b.coef_3rd_order, b.apvm_upwinding, b.smdiv, b.len_disp, b.epssm_minimum, b.epssm_maximum,
                      b.epssm_bottom_z, b.epssm_top_z, b.rgas, b.cp, b.gravity, b.p0, b.cf1, b.cf2, b.cf3,
                      b.acoustic_dts2[0], b.acoustic_dts2[1], b.acoustic_dts2[2]};
  if (!same_bits(fa, fb, sizeof fa / sizeof fa[0])) return bad("a configuration constant");
  if (!same_bits(a.fzm, b.fzm, L) || !same_bits(a.fzp, b.fzp, L) || !same_bits(a.rdzw, b.rdzw, L) ||
      !same_bits(a.rdzu, b.rdzu, L))
    return bad("the vertical coordinate");
  if (!same_bits(a.u_init, b.u_init, L) || !same_bits(a.v_init, b.v_init, L)) return bad("the reference winds");
  if (b.horiz_mixing != a.horiz_mixing || b.rayleigh_levels != a.rayleigh_levels || b.cam_levels != a.cam_levels)
    return bad("the mixing or upper-damping options");
  const float ma[] = {a.rayleigh_inverse, a.horiz_mixing ? a.cam_base : 0.0f,
                      a.horiz_mixing ? a.smag_strain_scale : 0.0f, a.horiz_mixing ? a.smag_ceiling : 0.0f,
                      a.horiz_mixing ? a.smag_h4 : 0.0f, a.horiz_mixing ? a.smag_div_factor : 0.0f};
  const float mb[] = {b.rayleigh_inverse, b.horiz_mixing ? b.cam_base : 0.0f,
                      b.horiz_mixing ? b.smag_strain_scale : 0.0f, b.horiz_mixing ? b.smag_ceiling : 0.0f,
                      b.horiz_mixing ? b.smag_h4 : 0.0f, b.horiz_mixing ? b.smag_div_factor : 0.0f};
  // the Smagorinsky length scales with the mesh (config_len_disp or
  // nominalMinDc), so a mixing ensemble holds meshes of one filter length
  if (!same_bits(ma, mb, sizeof ma / sizeof ma[0])) return bad("the mixing or upper-damping constants");
  return HEXDYN_OK;
}

// [rows][n_m] blocks of every member -> [rows][sum n]
void cat_rows(std::vector<float>& out, const HexDynDesc* ds, int n, int rows, const float* HexDynDesc::*field,
              const std::vector<int>& off, const std::vector<int>& cnt, size_t total) {
  out.assign((size_t)rows * total, 0.0f);
  for (int m = 0; m < n; ++m)
    for (int r = 0; r < rows; ++r)
      memcpy(&out[(size_t)r * total + off[m]], ds[m].*field + (size_t)r * cnt[m], cnt[m] * sizeof(float));
}

// [n_m][w_m] rows of every member -> [sum n][w], entries + shift (ints)
void cat_slots(std::vector<int32_t>& out, const HexDynDesc* ds, int n, const int32_t* const HexDynDesc::*field,
               const std::vector<int>& cnt, const std::vector<int>& wm, int w, const std::vector<int>& shift,
               size_t total) {
  out.assign(total * w, 0);
  size_t row = 0;
  for (int m = 0; m < n; ++m)
    for (int i = 0; i < cnt[m]; ++i, ++row)
      for (int s = 0; s < wm[m]; ++s) out[row * w + s] = (ds[m].*field)[(size_t)i * wm[m] + s] + shift[m];
}

void cat_slots_f(std::vector<float>& out, const HexDynDesc* ds, int n, const float* HexDynDesc::*field,
                 const std::vector<int>& cnt, const std::vector<int>& wm, int w, size_t total) {
  out.assign(total * w, 0.0f);
  size_t row = 0;
  for (int m = 0; m < n; ++m)
    for (int i = 0; i < cnt[m]; ++i, ++row)
      for (int s = 0; s < wm[m]; ++s) out[row * w + s] = (ds[m].*field)[(size_t)i * wm[m] + s];
}

int merge_members(const HexDynDesc* ds, int n, MergedDesc& M, HexDynHandle* h) {
  const HexDynDesc& a = ds[0];
  const int L = a.n_levels;
  std::vector<int> nc(n), ne(n), nv(n), c0(n), e0(n), v0(n), wE(n), wE2(n), wA(n), w3(n, 3), w2(n, 2), w1(n, 1);
  size_t C = 0, E = 0, V = 0;
  int mE = 0, mE2 = 0, mA = 0;
  for (int m = 0; m < n; ++m) {
    nc[m] = ds[m].n_cells;
    ne[m] = ds[m].n_edges;
    nv[m] = ds[m].n_vertices;
    c0[m] = (int)C;
    e0[m] = (int)E;
    v0[m] = (int)V;
    C += nc[m];
    E += ne[m];
    V += nv[m];
    wE[m] = ds[m].max_edges;
    wE2[m] = ds[m].max_edges2;
    wA[m] = ds[m].adv_width;
    mE = std::max(mE, wE[m]);
    mE2 = std::max(mE2, wE2[m]);
    mA = std::max(mA, wA[m]);
  }
  if (C > (size_t)INT32_MAX / 64 || E > (size_t)INT32_MAX / 64)
    return fail(HEXDYN_E_CAPACITY, "ensemble of %zu cells / %zu edges exceeds the int32 index range", C, E);
  std::vector<int> zero(n, 0);
  cat_slots(M.coe, ds, n, &HexDynDesc::cells_on_edge, ne, w2, 2, c0, E);
  cat_slots(M.eoc, ds, n, &HexDynDesc::edges_on_cell, nc, wE, mE, e0, C);
  cat_slots(M.coc, ds, n, &HexDynDesc::cells_on_cell, nc, wE, mE, c0, C);
  cat_slots(M.voc, ds, n, &HexDynDesc::vertices_on_cell, nc, wE, mE, v0, C);
  cat_slots(M.deg, ds, n, &HexDynDesc::n_edges_on_cell, nc, w1, 1, zero, C);
  cat_slots(M.voe, ds, n, &HexDynDesc::vertices_on_edge, ne, w2, 2, v0, E);
  cat_slots(M.eov, ds, n, &HexDynDesc::edges_on_vertex, nv, w3, 3, e0, V);
  cat_slots(M.cov, ds, n, &HexDynDesc::cells_on_vertex, nv, w3, 3, c0, V);
  cat_slots(M.eoe, ds, n, &HexDynDesc::edges_on_edge, ne, wE2, mE2, e0, E);
  cat_slots(M.neoe, ds, n, &HexDynDesc::n_edges_on_edge, ne, w1, 1, zero, E);
  cat_slots(M.advc, ds, n, &HexDynDesc::adv_cells, ne, wA, mA, c0, E);
  cat_slots(M.nadv, ds, n, &HexDynDesc::n_adv_cells, ne, w1, 1, zero, E);
  cat_slots_f(M.dc, ds, n, &HexDynDesc::dc_edge, ne, w1, 1, E);
  cat_slots_f(M.dv, ds, n, &HexDynDesc::dv_edge, ne, w1, 1, E);
  cat_slots_f(M.area, ds, n, &HexDynDesc::area_cell, nc, w1, 1, C);
  cat_slots_f(M.area_tri, ds, n, &HexDynDesc::area_triangle, nv, w1, 1, V);
  cat_slots_f(M.kite, ds, n, &HexDynDesc::kite_areas, nv, w3, 3, V);
  cat_slots_f(M.weights, ds, n, &HexDynDesc::weights_on_edge, ne, wE2, mE2, E);
  cat_slots_f(M.fv, ds, n, &HexDynDesc::f_vertex, nv, w1, 1, V);
  cat_slots_f(M.fe, ds, n, &HexDynDesc::f_edge, ne, w1, 1, E);
  cat_slots_f(M.cosa, ds, n, &HexDynDesc::cos_angle_edge, ne, w1, 1, E);
  cat_slots_f(M.sina, ds, n, &HexDynDesc::sin_angle_edge, ne, w1, 1, E);
  cat_slots_f(M.adv, ds, n, &HexDynDesc::adv_coefs, ne, wA, mA, E);
  cat_slots_f(M.adv3, ds, n, &HexDynDesc::adv_coefs_3rd, ne, wA, mA, E);
  if (a.horiz_mixing) {
    cat_slots_f(M.deform_c2, ds, n, &HexDynDesc::deform_c2, nc, wE, mE, C);
    cat_slots_f(M.deform_s2, ds, n, &HexDynDesc::deform_s2, nc, wE, mE, C);
    cat_slots_f(M.deform_cs, ds, n, &HexDynDesc::deform_cs, nc, wE, mE, C);
    cat_slots_f(M.mix_del2, ds, n, &HexDynDesc::mix_del2, ne, w1, 1, E);
    cat_slots_f(M.mix_del4, ds, n, &HexDynDesc::mix_del4, ne, w1, 1, E);
  }
  cat_rows(M.zz, ds, n, L, &HexDynDesc::zz, c0, nc, C);
  cat_rows(M.zxu, ds, n, L, &HexDynDesc::zxu, e0, ne, E);
  cat_rows(M.dss, ds, n, L, &HexDynDesc::dss, c0, nc, C);
  cat_rows(M.rb, ds, n, L, &HexDynDesc::rho_base, c0, nc, C);
  cat_rows(M.rtb, ds, n, L, &HexDynDesc::rho_theta_base, c0, nc, C);
  cat_rows(M.eb, ds, n, L, &HexDynDesc::exner_base, c0, nc, C);
  // terrain metrics [L+1][C][maxEdges]
  M.zb.assign((size_t)(L + 1) * C * mE, 0.0f);
  M.zb3.assign((size_t)(L + 1) * C * mE, 0.0f);
  for (int m = 0; m < n; ++m)
    for (int k = 0; k <= L; ++k)
      for (int i = 0; i < nc[m]; ++i)
        for (int sl = 0; sl < wE[m]; ++sl) {
          const size_t src = ((size_t)k * nc[m] + i) * wE[m] + sl, dst = ((size_t)k * C + c0[m] + i) * mE + sl;
          M.zb[dst] = ds[m].zb_cell[src];
          M.zb3[dst] = ds[m].zb3_cell[src];
        }
  // divergence damping length of each member's mesh (hexcore/mixing.py:851)
  M.smdiv_edge.assign(E, 0.0f);
  for (int m = 0; m < n; ++m) {
    const float len = ds[m].len_disp > 0.0f ? ds[m].len_disp : ds[m].nominal_min_dc;
    const float base = 2.0f * ds[m].smdiv * len;
    std::fill(M.smdiv_edge.begin() + e0[m], M.smdiv_edge.begin() + e0[m] + ne[m], base);
  }
  HexDynDesc& d = M.d;
  d = a;
  d.n_cells = (int)C;
  d.n_edges = (int)E;
  d.n_vertices = (int)V;
  d.max_edges = mE;
  d.max_edges2 = mE2;
  d.adv_width = mA;
  if (a.horiz_mixing) {
    d.deform_c2 = M.deform_c2.data();
    d.deform_s2 = M.deform_s2.data();
    d.deform_cs = M.deform_cs.data();
    d.mix_del2 = M.mix_del2.data();
    d.mix_del4 = M.mix_del4.data();
  }
  d.cells_on_edge = M.coe.data();
  d.edges_on_cell = M.eoc.data();
  d.cells_on_cell = M.coc.data();
  d.vertices_on_cell = M.voc.data();
  d.n_edges_on_cell = M.deg.data();
  d.vertices_on_edge = M.voe.data();
  d.edges_on_vertex = M.eov.data();
  d.cells_on_vertex = M.cov.data();
  d.edges_on_edge = M.eoe.data();
  d.n_edges_on_edge = M.neoe.data();
  d.adv_cells = M.advc.data();
  d.n_adv_cells = M.nadv.data();
  d.dc_edge = M.dc.data();
  d.dv_edge = M.dv.data();
  d.area_cell = M.area.data();
  d.area_triangle = M.area_tri.data();
  d.kite_areas = M.kite.data();
  d.weights_on_edge = M.weights.data();
  d.f_vertex = M.fv.data();
  d.f_edge = M.fe.data();
  d.cos_angle_edge = M.cosa.data();
  d.sin_angle_edge = M.sina.data();
  d.adv_coefs = M.adv.data();
  d.adv_coefs_3rd = M.adv3.data();
  d.zz = M.zz.data();
  d.zxu = M.zxu.data();
  d.dss = M.dss.data();
  d.zb_cell = M.zb.data();
  d.zb3_cell = M.zb3.data();
  d.rho_base = M.rb.data();
  d.rho_theta_base = M.rtb.data();
  d.exner_base = M.eb.data();
  h->m_c0 = c0;
  h->m_e0 = e0;
  h->m_v0 = v0;
  h->m_nc = nc;
  h->m_ne = ne;
  h->m_nv = nv;
  h->m_have.assign(n, 0u);
  return HEXDYN_OK;
}

// Member m's slice of a field: entity offset and count.
void member_slice(const HexDynHandle* h, int field, int m, int* off, int* cnt) {
  const bool edge = field == HEXDYN_RHO_U || field == HEXDYN_U;
  *off = edge ? h->m_e0[m] : h->m_c0[m];
  *cnt = edge ? h->m_ne[m] : h->m_nc[m];
}

int member_io(HexDynHandle* h, int member, int field, float* host, size_t count, void* stream, bool upload) {
  if (!h || !host) return fail(HEXDYN_E_ARG, "NULL handle or host pointer");
  if (field < 0 || field >= HEXDYN_NUM_FIELDS) return fail(HEXDYN_E_ARG, "unknown field %d", field);
  if (member < 0 || member >= (int)h->m_c0.size())
    return fail(HEXDYN_E_ARG, "member %d out of range (%zu members)", member, h->m_c0.size());
  const FieldShape fs = field_shape(h->ctx, field);
  int off = 0, n = 0;
  member_slice(h, field, member, &off, &n);
  const size_t want = (size_t)fs.blocks * fs.rows * n;
  if (count != want) return fail(HEXDYN_E_ARG, "member %d field %d has %zu values, got %zu", member, field, want, count);
  if (count == 0) return HEXDYN_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int S = h->ctx.geo.S;
  float* base = field_ptr(cur_state(h), cur_side(h), field);
  float* stage = h->staging[field];
  if (upload) HEX_CUDA(cudaMemcpyAsync(stage, host, count * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
  for (int b = 0; b < fs.blocks; ++b) {
    dim3 grid((n + 31) / 32, (fs.rows + 31) / 32), block(32, 8);
    float* dev = base + ((size_t)b * fs.n + off) * S;
    float* sb = stage + (size_t)b * fs.rows * n;
    if (upload)
      k_to_padded<<<grid, block, 0, st>>>(sb, fs.rows, n, S, dev);
    else
      k_from_padded<<<grid, block, 0, st>>>(dev, fs.rows, n, S, sb);
  }
  HEX_CUDA(cudaGetLastError(), "member transpose");
  if (!upload) {
    HEX_CUDA(cudaMemcpyAsync(host, stage, count * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H");
    return HEXDYN_OK;
  }
  h->m_have[member] |= 1u << field;
  bool all = true;
  for (unsigned bits : h->m_have) all = all && (bits >> field & 1u);
  if (all) h->have_state[field] = true;
  return HEXDYN_OK;
}

}  // namespace

extern "C" {

int hexdyn_create_ensemble(const HexDynDesc* members, int n_members, HexDynHandle** out) {
  if (!out) return fail(HEXDYN_E_ARG, "out is NULL");
  *out = nullptr;
  if (!members || n_members < 1) return fail(HEXDYN_E_ARG, "an ensemble needs at least one member");
  for (int m = 0; m < n_members; ++m) {
    int rc = validate(&members[m]);
    if (rc) return fail(rc, "ensemble member %d: %s", m, g_last_error.c_str());
    if (m > 0 && (rc = check_compatible(members[0], members[m], m))) return rc;
  }
  HexDynHandle* h = new HexDynHandle();
  MergedDesc M;
  int rc = merge_members(members, n_members, M, h);
  if (!rc) rc = validate(&M.d);
  if (!rc) rc = build(h, M.d, &M.smdiv_edge);
  if (rc) {
    hexdyn_destroy(h);
    return rc;
  }
  *out = h;
  return HEXDYN_OK;
}

int hexdyn_member_count(HexDynHandle* h) { return h ? (int)h->m_c0.size() : 0; }

int hexdyn_set_stage_hook(HexDynHandle* h, HexDynStageHook hook, void* user) {
  if (!h) return fail(HEXDYN_E_ARG, "NULL handle");
  HexCtx& c = h->ctx;
  if (hook && h->m_c0.size() > 1)
    return fail(HEXDYN_E_ARG, "the physics stage hook is for single instances, not ensembles");
  if (hook && !c.phys_ru) {
    const HexGeo& g = c.geo;
    const size_t CS = (size_t)g.nC * g.S, ES = (size_t)g.nE * g.S;
    cudaError_t e;
    if ((e = dev_alloc(c, &c.phys_ru, ES)) || (e = dev_alloc(c, &c.phys_rt, CS)) ||
        (e = dev_alloc(c, &c.phys_rho, CS)) || (e = dev_alloc(c, &c.phys_dth, CS)) ||
        (e = dev_alloc(c, &c.mod_rate, CS)) || (e = dev_alloc(c, &c.tend_rho_dyn, CS)))
      return cuda_fail(e, "physics buffers");
  }
  c.stage_hook = hook;
  c.stage_user = user;
  c.phys_held_rho = 0;
  c.phys_failed = 0;
  return HEXDYN_OK;
}

int hexdyn_set_exchange_hook(HexDynHandle* h, HexDynExchangeHook hook, void* user) {
  if (!h) return fail(HEXDYN_E_ARG, "NULL handle");
  if (hook && h->m_c0.size() > 1)
    return fail(HEXDYN_E_ARG, "the halo exchange hook is for single instances, not ensembles");
  h->ctx.exchange_hook = hook;
  h->ctx.exchange_user = user;
  h->ctx.phys_failed = 0;
  return HEXDYN_OK;
}

// Halo rows of a partitioned instance: one launch moves the chosen rows of
// every buffer of an exchange point into one packed array or back.  Packed
// layout: buffer by buffer, block by block (tracer blocks), row by row, the
// S words of each row.
#define HEX_HALO_MAX 24
struct HexHaloBufs {
  float* p[HEX_HALO_MAX];
  const int* idx[HEX_HALO_MAX];
  int rows[HEX_HALO_MAX];    // rows of one block of the buffer (cells or edges)
  int nrows[HEX_HALO_MAX];   // rows moved
  long long off[HEX_HALO_MAX + 1];  // start of each buffer in the packed array (16-byte units)
  int n;
};

__global__ void k_halo_rows(HexHaloBufs hb, int S4, float4* packed, int unpack) {
  const long long total = hb.off[hb.n];
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int b = 0;
    while (t >= hb.off[b + 1]) ++b;
    const long long u = t - hb.off[b];
    const int l = (int)(u % S4);
    const long long r = u / S4;
    const int i = (int)(r % hb.nrows[b]);
    const long long blk = r / hb.nrows[b];
    const int row = hb.idx[b][i];
    if (row < 0 || row >= hb.rows[b]) continue;  // the host checked the lists; never touch memory outside
    float4* cell = reinterpret_cast<float4*>(hb.p[b]) + (blk * hb.rows[b] + row) * S4 + l;
    if (unpack)
      *cell = packed[t];
    else
      packed[t] = *cell;
  }
}

static int halo_setup(HexDynHandle* h, int nbuf, float* const* bufs, const int* kinds, const int* cell_rows,
                      int n_cell_rows, const int* edge_rows, int n_edge_rows, HexHaloBufs& hb) {
  if (!h || (nbuf > 0 && (!bufs || !kinds))) return fail(HEXDYN_E_ARG, "NULL argument");
  if (nbuf < 0 || nbuf > HEX_HALO_MAX) return fail(HEXDYN_E_ARG, "nbuf %d outside [0, %d]", nbuf, HEX_HALO_MAX);
  if (n_cell_rows < 0 || n_edge_rows < 0) return fail(HEXDYN_E_ARG, "negative row count");
  if ((n_cell_rows > 0 && !cell_rows) || (n_edge_rows > 0 && !edge_rows)) return fail(HEXDYN_E_ARG, "NULL row list");
  const HexCtx& c = h->ctx;
  hb = HexHaloBufs{};
  hb.n = nbuf;
  for (int b = 0; b < nbuf; ++b) {
    const int k = kinds[b];
    if (k != HEXDYN_KIND_CELL && k != HEXDYN_KIND_EDGE && k != HEXDYN_KIND_TRACER)
      return fail(HEXDYN_E_ARG, "buffer %d: unknown kind %d", b, k);
    if (!bufs[b] || (reinterpret_cast<uintptr_t>(bufs[b]) & 15))
      return fail(HEXDYN_E_ARG, "buffer %d: NULL or not 16-byte aligned", b);
    const bool edge = k == HEXDYN_KIND_EDGE;
    const int blocks = k == HEXDYN_KIND_TRACER ? std::max(1, c.n_scalars) : 1;
    hb.p[b] = bufs[b];
    hb.idx[b] = edge ? edge_rows : cell_rows;
    hb.rows[b] = edge ? c.geo.nE : c.geo.nC;
    hb.nrows[b] = edge ? n_edge_rows : n_cell_rows;
    hb.off[b + 1] = hb.off[b] + (long long)blocks * hb.nrows[b] * (c.geo.S / 4);
  }
  return HEXDYN_OK;
}

size_t hexdyn_halo_words(HexDynHandle* h, int nbuf, const int* kinds, int n_cell_rows, int n_edge_rows) {
  if (!h || nbuf < 0 || nbuf > HEX_HALO_MAX || (nbuf > 0 && !kinds)) return 0;
  size_t words = 0;
  for (int b = 0; b < nbuf; ++b) {
    const int blocks = kinds[b] == HEXDYN_KIND_TRACER ? std::max(1, h->ctx.n_scalars) : 1;
    words += (size_t)blocks * (kinds[b] == HEXDYN_KIND_EDGE ? n_edge_rows : n_cell_rows) * h->ctx.geo.S;
  }
  return words;
}

static int halo_move(HexDynHandle* h, int nbuf, float* const* bufs, const int* kinds, const int* cell_rows,
                     int n_cell_rows, const int* edge_rows, int n_edge_rows, float* packed, void* stream,
                     int unpack) {
  HexHaloBufs hb;
  const int rc = halo_setup(h, nbuf, bufs, kinds, cell_rows, n_cell_rows, edge_rows, n_edge_rows, hb);
  if (rc != HEXDYN_OK) return rc;
  const long long total = hb.off[nbuf];
  if (total == 0) return HEXDYN_OK;
  if (!packed || (reinterpret_cast<uintptr_t>(packed) & 15))
    return fail(HEXDYN_E_ARG, "packed array NULL or not 16-byte aligned");
  const int threads = 256;
  const long long want = (total + threads - 1) / threads;
  const int grid = (int)std::min<long long>(want, 148LL * 8);
  k_halo_rows<<<grid, threads, 0, (cudaStream_t)stream>>>(hb, h->ctx.geo.S / 4, reinterpret_cast<float4*>(packed),
                                                            unpack);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "halo rows");
  return HEXDYN_OK;
}

int hexdyn_halo_pack(HexDynHandle* h, int nbuf, float* const* bufs, const int* kinds, const int* cell_rows,
                     int n_cell_rows, const int* edge_rows, int n_edge_rows, float* packed, void* stream) {
  return halo_move(h, nbuf, bufs, kinds, cell_rows, n_cell_rows, edge_rows, n_edge_rows, packed, stream, 0);
}

int hexdyn_halo_unpack(HexDynHandle* h, int nbuf, float* const* bufs, const int* kinds, const int* cell_rows,
                       int n_cell_rows, const int* edge_rows, int n_edge_rows, const float* packed, void* stream) {
  return halo_move(h, nbuf, bufs, kinds, cell_rows, n_cell_rows, edge_rows, n_edge_rows,
                   const_cast<float*>(packed), stream, 1);
}

int hexdyn_physics_buffer(HexDynHandle* h, int which, void** device_ptr) {
  if (!h || !device_ptr) return fail(HEXDYN_E_ARG, "NULL argument");
  HexCtx& c = h->ctx;
  if (!c.phys_ru) return fail(HEXDYN_E_STATE, "no physics stage hook was set on this handle");
  float* p = which == HEXDYN_PHYS_RHO_U ? c.phys_ru : which == HEXDYN_PHYS_RHO_THETA ? c.phys_rt
           : which == HEXDYN_PHYS_RHO ? c.phys_rho : which == HEXDYN_PHYS_DIABATIC_THETA ? c.phys_dth
           : which == HEXDYN_PHYS_MODIFIED_RATE ? c.mod_rate : nullptr;
  if (!p) return fail(HEXDYN_E_ARG, "unknown physics buffer %d", which);
  *device_ptr = p;
  return HEXDYN_OK;
}

int hexdyn_set_member_state(HexDynHandle* h, int member, int field, const float* host, size_t count, void* stream) {
  return member_io(h, member, field, const_cast<float*>(host), count, stream, true);
}

int hexdyn_get_member_state(HexDynHandle* h, int member, int field, float* host, size_t count, void* stream) {
  return member_io(h, member, field, host, count, stream, false);
}

int hexdyn_step_batched(const HexDynBatch* batch, void* stream) {
  if (!batch || batch->n_groups < 1 || !batch->groups || !batch->steps)
    return fail(HEXDYN_E_ARG, "batch needs n_groups >= 1, groups and steps");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = batch->n_groups;
  for (int i = 0; i < n; ++i) {
    HexDynHandle* h = batch->groups[i];
    if (!h) return fail(HEXDYN_E_ARG, "batch group %d is NULL", i);
    if (batch->steps[i] < 0) return fail(HEXDYN_E_ARG, "batch group %d: negative step count", i);
    for (int j = 0; j < i; ++j)
      if (batch->groups[j] == h) return fail(HEXDYN_E_ARG, "batch groups %d and %d are the same handle", j, i);
    if (!h->batch_stream) {
      HEX_CUDA(cudaStreamCreateWithFlags(&h->batch_stream, cudaStreamNonBlocking), "batch stream");
      HEX_CUDA(cudaEventCreateWithFlags(&h->batch_fork, cudaEventDisableTiming), "batch event");
      HEX_CUDA(cudaEventCreateWithFlags(&h->batch_done, cudaEventDisableTiming), "batch event");
    }
  }
  // fork: every group waits for the caller's stream, then steps on its own
  // stream so that the groups run concurrently; join back into the caller's
  // stream
  for (int i = 0; i < n; ++i) {
    HexDynHandle* h = batch->groups[i];
    HEX_CUDA(cudaEventRecord(h->batch_fork, st), "fork record");
    HEX_CUDA(cudaStreamWaitEvent(h->batch_stream, h->batch_fork, 0), "fork wait");
    int rc = hexdyn_step_async(h, h->batch_stream, batch->steps[i]);
    if (rc) return fail(rc, "batch group %d: %s", i, g_last_error.c_str());
    HEX_CUDA(cudaEventRecord(h->batch_done, h->batch_stream), "join record");
    HEX_CUDA(cudaStreamWaitEvent(st, h->batch_done, 0), "join wait");
  }
  if (!batch->flags) return HEXDYN_OK;
  int bad = -1;
  for (int i = 0; i < n; ++i) {
    int f = 0;
    int rc = hexdyn_read_flag(batch->groups[i], st, &f);
    batch->flags[i] = f;
    if (rc == HEXDYN_E_NUMERIC) {
      if (bad < 0) bad = i;
    } else if (rc) {
      return rc;
    }
  }
  if (bad >= 0)
    return fail(HEXDYN_E_NUMERIC, "batch group %d: device validation flag 0x%x set", bad, batch->flags[bad]);
  return HEXDYN_OK;
}

}  // extern "C"

// ------------------------------------------------------ learned corrector
// State access of the learned corrector (no counterpart in the reference):
// raw input features of the column and edge networks, the application of
// their output increments to the prognostic state, and the total energy
// that decides whether a corrected step is accepted.

namespace {

// Column features [C][6L]: theta_m, rho_zz, w (interfaces 0..L-1), the first
// scalar (qv), the mean of u over the cell's edges, and the mean of theta_m
// over the neighbouring cells, each for levels 0..L-1.
__global__ void k_col_features(HexGeo g, HexState s, HexSide d, float* __restrict__ X, int ld) {
  const int c = blockIdx.x, L = g.L, S = g.S;
  const int n = g.deg[c];
  float* row = X + (size_t)c * ld;
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const int i = c * S + k;
    float um = 0.0f, tm = 0.0f;
    for (int q = 0; q < n; ++q) {
      um += d.u[g.eoc[c * g.maxE + q] * S + k];
      tm += d.theta_m[g.coc[c * g.maxE + q] * S + k];
    }
    row[k] = d.theta_m[i];
    row[L + k] = s.rho[i];
    row[2 * L + k] = d.w[i];
    row[3 * L + k] = s.scalars ? s.scalars[i] : 0.0f;
    row[4 * L + k] = um / (float)n;
    row[5 * L + k] = tm / (float)n;
  }
}

// Edge features [E][4L]: u, theta_m of both cells, mean rho_zz of both cells.
__global__ void k_edge_features(HexGeo g, HexState s, HexSide d, float* __restrict__ X, int ld) {
  const int e = blockIdx.x, L = g.L, S = g.S;
  const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
  float* row = X + (size_t)e * ld;
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    row[k] = d.u[e * S + k];
    row[L + k] = d.theta_m[c0 * S + k];
    row[2 * L + k] = d.theta_m[c1 * S + k];
    row[3 * L + k] = 0.5f * (s.rho[c0 * S + k] + s.rho[c1 * S + k]);
  }
}

// Column increments (denormalised y * scale + shift of theta_m, rho_zz, w)
// applied to the prognostic state: rho' = rho + drho, rho_theta' = rho' *
// (theta_m + dtheta), rho_w' = rho_w + dw * zz_k * rho'_k at the interfaces
// 1..L-1 (the interface weights of w recovery).
__global__ void k_apply_col(HexGeo g, HexState s, HexSide d, const float* __restrict__ Y, int ld,
                            const float* __restrict__ scale, const float* __restrict__ shift) {
  const int c = blockIdx.x, L = g.L, S = g.S;
  const float* y = Y + (size_t)c * ld;
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const int i = c * S + k;
    const float dth = y[k] * scale[k] + shift[k];
    const float drho = y[L + k] * scale[L + k] + shift[L + k];
    const float rho = s.rho[i] + drho;
    s.rho[i] = rho;
    s.rho_theta[i] = rho * (d.theta_m[i] + dth);
  }
  __syncthreads();
  for (int k = 1 + threadIdx.x; k < L; k += blockDim.x) {
    const int i = c * S + k;
    const float dw = y[2 * L + k] * scale[2 * L + k] + shift[2 * L + k];
    const float zzi = g.fzm[k] * g.zz[i] + g.fzp[k] * g.zz[i - 1];
    const float rhoi = g.fzm[k] * s.rho[i] + g.fzp[k] * s.rho[i - 1];
    s.rho_w[i] = s.rho_w[i] + dw * zzi * rhoi;
  }
}

// Edge increments of u: rho_u' = rho_u + du * (rho_zz at the edge).
__global__ void k_apply_edge(HexGeo g, HexState s, const float* __restrict__ Y, int ld,
                             const float* __restrict__ scale, const float* __restrict__ shift) {
  const int e = blockIdx.x, L = g.L, S = g.S;
  const int c0 = g.coe[2 * e], c1 = g.coe[2 * e + 1];
  const float* y = Y + (size_t)e * ld;
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const float du = y[k] * scale[k] + shift[k];
    s.rho_u[e * S + k] += du * 0.5f * (s.rho[c0 * S + k] + s.rho[c1 * S + k]);
  }
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
  if (threadIdx.x < 32)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Total energy: sum over cells and levels of the mass rho_zz * area * dzw
// times (cv T + g z) with T = theta_m * exner, plus the vertical kinetic
// energy rho_w * w / 2 * area / rdzu at the interior interfaces, plus sum
// over edges and levels of rho_u * u * (dc dv / 2) * dzw / 2.
__global__ void k_energy(HexGeo g, HexState s, HexSide d, const float* __restrict__ z, float cv,
                         double* __restrict__ out) {
  const int L = g.L, S = g.S;
  double acc = 0.0, w2 = 0.0;
  const size_t nc = (size_t)g.nC * L, ne = (size_t)g.nE * L;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nc + ne; t += (size_t)gridDim.x * blockDim.x) {
    if (t < nc) {
      const int c = (int)(t / L), k = (int)(t % L);
      const int i = c * S + k;
      const double mass = (double)s.rho[i] / ((double)g.inv_area[c] * (double)g.rdzw[k]);
      acc += mass * ((double)cv * d.theta_m[i] * d.exner[i] + (double)g.g * z[i]);
      if (k >= 1) {
        const double vol = 1.0 / ((double)g.inv_area[c] * (double)g.rdzu[k]);
        acc += 0.5 * (double)s.rho_w[i] * d.w[i] * vol;
        w2 += (double)d.w[i] * d.w[i] * vol;
      }
    } else {
      const size_t te = t - nc;
      const int e = (int)(te / L), k = (int)(te % L);
      const int j = e * S + k;
      acc += 0.25 * (double)s.rho_u[j] * d.u[j] * g.dc[e] * g.dv[e] / (double)g.rdzw[k];
    }
  }
  acc = block_sum(acc);
  __syncthreads();
  w2 = block_sum(w2);
  if (threadIdx.x == 0) {
    atomicAdd(out, acc);
    atomicAdd(out + 1, w2);
  }
}

}  // namespace

extern "C" {

int hexdyn_column_features(HexDynHandle* h, float* X, int ld, void* stream) {
  if (!h || !X || ld < 6 * h->ctx.geo.L) return fail(HEXDYN_E_ARG, "column features need ld >= 6 L");
  k_col_features<<<h->ctx.geo.nC, 64, 0, (cudaStream_t)stream>>>(h->ctx.geo, cur_state(h), cur_side(h), X, ld);
  HEX_CUDA(cudaGetLastError(), "column features");
  return HEXDYN_OK;
}

int hexdyn_edge_features(HexDynHandle* h, float* X, int ld, void* stream) {
  if (!h || !X || ld < 4 * h->ctx.geo.L) return fail(HEXDYN_E_ARG, "edge features need ld >= 4 L");
  k_edge_features<<<h->ctx.geo.nE, 64, 0, (cudaStream_t)stream>>>(h->ctx.geo, cur_state(h), cur_side(h), X, ld);
  HEX_CUDA(cudaGetLastError(), "edge features");
  return HEXDYN_OK;
}

int hexdyn_apply_increments(HexDynHandle* h, const float* Ycol, int ldc, const float* col_scale,
                            const float* col_shift, const float* Yedge, int lde, const float* edge_scale,
                            const float* edge_shift, void* stream) {
  if (!h) return fail(HEXDYN_E_ARG, "NULL handle");
  const HexGeo& g = h->ctx.geo;
  cudaStream_t st = (cudaStream_t)stream;
  if (Ycol) {
    if (ldc < 3 * g.L || !col_scale || !col_shift) return fail(HEXDYN_E_ARG, "column increments need ld >= 3 L");
    k_apply_col<<<g.nC, 64, 0, st>>>(g, cur_state(h), cur_side(h), Ycol, ldc, col_scale, col_shift);
  }
  if (Yedge) {
    if (lde < g.L || !edge_scale || !edge_shift) return fail(HEXDYN_E_ARG, "edge increments need ld >= L");
    k_apply_edge<<<g.nE, 64, 0, st>>>(g, cur_state(h), Yedge, lde, edge_scale, edge_shift);
  }
  HEX_CUDA(cudaGetLastError(), "apply increments");
  return HEXDYN_OK;
}

int hexdyn_total_energy(HexDynHandle* h, const float* z_mid, double* dev_out, void* stream) {
  if (!h || !z_mid || !dev_out) return fail(HEXDYN_E_ARG, "NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  HEX_CUDA(cudaMemsetAsync(dev_out, 0, 2 * sizeof(double), st), "energy clear");
  const float cv = h->ctx.geo.c2 / h->ctx.geo.rcv - h->ctx.geo.rgas;
  k_energy<<<4 * 148, 256, 0, st>>>(h->ctx.geo, cur_state(h), cur_side(h), z_mid, cv, dev_out);
  HEX_CUDA(cudaGetLastError(), "energy");
  return HEXDYN_OK;
}

}  // extern "C"

// ------------------------------------------------------------- bind state

extern "C" int hexdyn_bind_state(HexDynHandle* h, const HexDynFields* fields, void* stream) {
  if (!h) return fail(HEXDYN_E_ARG, "NULL handle");
  HexCtx& c = h->ctx;
  if (!fields) {
    if (h->bound) {
      if (c.parity == 0) return fail(HEXDYN_E_STATE, "the current state is in the bound buffers; step once more "
                                     "(or copy it) before unbinding");
      c.in = h->own_in;
      c.side_in = h->own_side_in;
      h->bound = false;
    }
  } else {
    for (int i = 0; i < HEXDYN_NUM_FIELDS; ++i) {
      const float* p = fields->field[i];
      if (!p && !(i == HEXDYN_SCALARS && c.n_scalars == 0))
        return fail(HEXDYN_E_ARG, "bound field %d is NULL", i);
      if ((uintptr_t)p & 15u)
        return fail(HEXDYN_E_ARG, "bound field %d is not 16-byte aligned (the kernels move four levels per "
                    "128-bit access)", i);
      if (p && p == field_ptr(c.out, c.side_out, i))
        return fail(HEXDYN_E_ARG, "bound field %d is the handle's own output buffer", i);
    }
    if (!h->bound) {
      h->own_in = c.in;
      h->own_side_in = c.side_in;
    }
    c.in = HexState{fields->field[HEXDYN_RHO], fields->field[HEXDYN_RHO_THETA], fields->field[HEXDYN_RHO_U],
                    fields->field[HEXDYN_RHO_W], fields->field[HEXDYN_SCALARS]};
    c.side_in = HexSide{fields->field[HEXDYN_THETA_M], fields->field[HEXDYN_EXNER], fields->field[HEXDYN_RHO_P],
                        fields->field[HEXDYN_RHO_THETA_P], fields->field[HEXDYN_PRESSURE_P], fields->field[HEXDYN_U],
                        fields->field[HEXDYN_W]};
    c.parity = 0;
    h->bound = true;
    for (int f = 0; f < HEXDYN_NUM_FIELDS; ++f) h->have_state[f] = true;
  }
  // captured graphs hold the old buffer addresses
  if (c.graph_exec[0] || c.graph_exec[1]) return hexdyn_capture_graph(h, stream);
  return HEXDYN_OK;
}

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
  float** tcell[] = {&w.q_stage[0], &w.q_stage[1], &w.scale_in, &w.scale_out, &w.mass, &w.vres};
  for (float** p : tcell) *p = cv.take(T * CS);
  w.edge_q = cv.take(T * ES);
  w.hres_lim = cv.take(T * ES);
  w.flag = (int*)cv.take(1);
  if (g.smag_on) {
    // 2-D Smagorinsky work arrays, one contiguous run (cleared per call)
    struct { float** p; size_t n; } mix[] = {
        {&w.vorticity, VS}, {&w.divergence, CS}, {&w.kdiff, CS}, {&w.delsq_u, ES}, {&w.delsq_div, CS},
        {&w.delsq_vort, VS}, {&w.w_mix, CS}, {&w.delsq_w, CS}, {&w.theta_mix, CS}, {&w.delsq_theta, CS},
        {&w.mix_u, ES}, {&w.mix_w, CS}};
    for (auto& b : mix) *b.p = cv.take(b.n);
  }
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
    if (((uintptr_t)in->field[i] | (uintptr_t)out->field[i]) & 15u)
      return fail(HEXDYN_E_ARG, "field %d is not 16-byte aligned (the kernels move four levels per 128-bit access)",
                  i);
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
  c.order = src.order;
  c.monotonic = src.monotonic;
  c.geo = src.geo;
  for (int i = 0; i < 3; ++i) {
    c.dyn[i] = src.dyn[i];
    c.scal[i] = src.scal[i];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const HexGeo& g = c.geo;
  const size_t CS = (size_t)g.nC * g.S, ES = (size_t)g.nE * g.S;
  // The array keeps the previous call's words (possibly of another mesh and
  // layout): clear every word this step uses, as the allocating path's
  // workspace starts cleared, then set what starts at one (dry coefficients).
  HEX_CUDA(cudaMemsetAsync(base, 0, need, st), "clear no-alloc scratch");
  if (!g.moist) {
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

