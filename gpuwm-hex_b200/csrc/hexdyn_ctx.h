// Host-side context of one dycore instance (shared by the strict and fast
// kernel builds and by the C ABI layer).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/hexdyn.h"
#include "dycore_geo.cuh"

struct HexState {       // prognostic state, [entity][level] padded
  float* rho;           // C
  float* rho_theta;     // C
  float* rho_u;         // E
  float* rho_w;         // C (interfaces)
  float* scalars;       // [T][C][S] (only the step in/out states own one)
};

struct HexSide {        // DrySavedDiagnostics
  float* theta_m;
  float* exner;
  float* rho_p;
  float* rtheta_p;
  float* pressure_p;
  float* u;             // E
  float* w;             // C (interfaces)
};

struct HexWork {
  // moist coefficients
  float *qtot, *cqw, *cqu;
  // diagnostics
  float *pv_vertex, *ke_vertex, *ke, *pv_cell, *v, *pv_edge;
  // saved Euler + stage tendencies
  float *euler_ru, *tend_rho, *euler_rw, *hdiv, *edge_theta, *edge_w, *tend_ru, *tend_rt, *tend_rw;
  // vertical implicit coefficients
  float *cofwr, *cofwz, *coftz, *cofwt, *a_tri, *alpha_tri, *gamma_tri;
  // acoustic
  float *ru_p, *ru_avg, *rw_p, *ww_avg, *rho_pp, *rtpp[2];
  // split mass flux (time-averaged over the dynamics subcycles)
  float *flux_u, *flux_w;
  // transport
  float *q_stage[2], *edge_q, *target, *scale_in, *scale_out, *mass, *hres_lim;
  float* vres;  // [T][C][S] the limiter's vertical residual flux at interfaces 0..S-1
  int* flag;            // device validation flag (bit set, see HEX_FLAG_*)
  // 2-D Smagorinsky mixing (allocated when on): diagnostics of the
  // subcycle's start, diffusivity, Laplacians and the saved mixed terms
  float *vorticity = nullptr, *divergence = nullptr, *kdiff = nullptr, *delsq_u = nullptr;
  float *delsq_div = nullptr, *delsq_vort = nullptr, *w_mix = nullptr, *delsq_w = nullptr;
  float *theta_mix = nullptr, *delsq_theta = nullptr, *mix_u = nullptr, *mix_w = nullptr;
};

struct HexProfEvent {   // one profiled launch: kernel name and its bracketing events
  const char* name;
  cudaEvent_t start, stop;
};

struct HexStage {
  int stage;            // 1..3
  double large_dt;
  double acoustic_dt;
  int acoustic_steps;
  float dts2;           // FP32 dts^2 used by the implicit solve
};

struct HexCtx {
  int numerics;         // 0 strict, 1 fast
  int n_scalars;
  double dt;
  int split_steps;
  int order = 3;        // config_time_integration_order (2 or 3)
  int monotonic;
  HexGeo geo;
  HexStage dyn[3];      // dynamics subcycle schedule
  HexStage scal[3];     // scalar transport schedule
  HexState in, out, tmp[2];
  HexSide side_in, side_out, side_tmp[2];
  HexWork w;
  std::vector<void*> allocations;
  size_t device_bytes = 0;
  cudaStream_t bound_stream = nullptr;
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
  int parity = 0;       // 0: state in `in`, 1: state in `out`
  long long steps_done = 0;
  long long launches_per_step = 0;
  // Autotuned block size (threads) per launch label; labels not listed use
  // 256 threads, and `force_threads` (when non-zero) overrides every label
  // while the autotuner times a candidate.
  std::vector<std::pair<std::string, int>> tuned_threads;
  int force_threads = 0;
  // Second stream for independent kernels of a stage (fork/join by events,
  // captured into the step graph as parallel branches); null: one stream.
  cudaStream_t side_stream = nullptr;
  cudaEvent_t fork_events[4] = {nullptr, nullptr, nullptr, nullptr};
  int concurrent_regions = 7;  // bit mask of the forked regions of a step
  // Recorded on the step's stream once the last recovery of a step has
  // written every output field but the scalars (an external event node of
  // the step graph when captured); hexdyn_step_host starts the downloads of
  // those fields on it while the scalar transport runs.
  cudaEvent_t dynamics_done = nullptr;
  // Per-stage physics hand-off (hexdyn_set_stage_hook): the hook, its
  // argument, the physics buffers it fills ([E][S] ru, [C][S] the others),
  // the stage-3 modified theta rate, the density tendency without physics,
  // and whether the last hook of the previous subcycle gave a density
  // tendency (held into the next subcycle's saved density tendency).
  HexDynStageHook stage_hook = nullptr;
  void* stage_user = nullptr;
  float *phys_ru = nullptr, *phys_rt = nullptr, *phys_rho = nullptr, *phys_dth = nullptr;
  float *mod_rate = nullptr, *tend_rho_dyn = nullptr;
  int phys_held_rho = 0;
  int phys_failed = 0;  // a hook returned a negative value
  // Halo exchange hook of a partitioned instance (hexdyn_set_exchange_hook)
  HexDynExchangeHook exchange_hook = nullptr;
  void* exchange_user = nullptr;
  int threads_for(const char* label) const {
    if (force_threads) return force_threads;
    for (const auto& t : tuned_threads)
      if (t.first == label) return t.second;
    return 256;
  }
};

namespace hexdyn_strict {
cudaError_t run_step(HexCtx& ctx, const HexState& in, const HexSide& side_in, const HexState& out,
                     const HexSide& side_out, cudaStream_t stream, long long* launches,
                     std::vector<HexProfEvent>* prof);
cudaError_t rebuild_sidecar(HexCtx& ctx, const HexState& s, const HexSide& side, cudaStream_t stream);
cudaError_t diagnostics_only(HexCtx& ctx, const HexState& s, const HexSide& side, cudaStream_t stream);
}  // namespace hexdyn_strict
namespace hexdyn_fast {
cudaError_t run_step(HexCtx& ctx, const HexState& in, const HexSide& side_in, const HexState& out,
                     const HexSide& side_out, cudaStream_t stream, long long* launches,
                     std::vector<HexProfEvent>* prof);
cudaError_t rebuild_sidecar(HexCtx& ctx, const HexState& s, const HexSide& side, cudaStream_t stream);
cudaError_t diagnostics_only(HexCtx& ctx, const HexState& s, const HexSide& side, cudaStream_t stream);
}  // namespace hexdyn_fast
