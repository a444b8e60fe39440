#include <initializer_list>
#include <utility>
// The first acoustic substep's start values (ru_p = ru_avg = dts tend_ru)
// formed by the momentum tendency, and the last substep's divergence
// damping applied by the edge recovery, instead of two kv_ac_edge launches
// per RK stage (the same operations on the same words).
#ifndef HEX_FUSE_AC_FIRST
#define HEX_FUSE_AC_FIRST 1
#endif
#ifndef HEX_FUSE_AC_DAMP
#define HEX_FUSE_AC_DAMP 1
#endif
#ifndef HEX_SKIP_FINAL_DIAG
#define HEX_SKIP_FINAL_DIAG 1
#endif
// Step orchestration: hexcore/driver.py:3314 DryDycoreDriver.step with the
// v8.4.1 subcycle of hexcore/driver.py:2710, as a fixed sequence of kernel
// launches on one stream (capturable into one CUDA graph).

struct Launcher {
  HexCtx& ctx;
  cudaStream_t st;
  std::vector<HexProfEvent>* prof = nullptr;  // per-launch CUDA events when profiling
  long long count = 0;
  cudaError_t err = cudaSuccess;
  cudaStream_t main_st = nullptr;  // the caller's stream while launches go to the side stream
  bool on_side = false;            // (the caller's stream may be the legacy stream, handle 0)
  int next_event = 0;
  // Independent kernels: fork() makes the side stream wait for everything
  // launched so far, side() sends the following launches there, and
  // join() makes the caller's stream wait for them.  Serial (no-ops) when
  // the context has no side stream or launches are being profiled.
  int region = 0;  // the forked region being launched (bit of ctx.concurrent_regions)
  bool concurrent() const {
    return ctx.side_stream != nullptr && prof == nullptr && (ctx.concurrent_regions & region);
  }
  void signal(cudaStream_t from, cudaStream_t to) {
    if (err != cudaSuccess) return;
    cudaEvent_t ev = ctx.fork_events[next_event++ & 3];
    err = cudaEventRecord(ev, from);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(to, ev, 0);
  }
  void fork() {
    if (concurrent()) signal(st, ctx.side_stream);
  }
  void side() {
    if (concurrent() && !on_side) {
      main_st = st;
      st = ctx.side_stream;
      on_side = true;
    }
  }
  void main() {
    if (on_side) {
      st = main_st;
      main_st = nullptr;
      on_side = false;
    }
  }
  void join() {
    if (!concurrent()) return;
    main();
    signal(ctx.side_stream, st);
  }
  // entities per block for tpe threads per entity under the label's block size
  int epb(const char* name, int tpe) const {
    const int threads = ctx.threads_for(name);
    return tpe >= threads ? 1 : threads / tpe;
  }
  template <class K, class... A>
  void lp(const char* name, int n, int nz, size_t smem_per_entity, K kernel, A... args) {
    launch(name, ctx.geo.S, n, nz, smem_per_entity, kernel, args...);
  }
  // level-vector form: S/4 threads per entity, four levels each
  template <class K, class... A>
  void lpv(const char* name, int n, int nz, K kernel, A... args) {
    launch(name, ctx.geo.S / 4, n, nz, 0, kernel, args...);
  }
  // column-group form: G lanes of one warp per column (0 when S/4 > 32)
  int group() const {
    const int q = ctx.geo.S / 4;
    return q <= 8 ? 8 : q <= 16 ? 16 : q <= 32 ? 32 : 0;
  }
  template <class K, class... A>
  void lpg(const char* name, int n, size_t smem_per_entity, K kernel, A... args) {
    launch(name, group(), n, 1, smem_per_entity, kernel, args...);
  }
  // level-vector form over nz tracers folded into the block index: block b
  // serves tracer b % nz (the kernel takes nz as its argument after the
  // geometry)
  template <class K, class... A>
  void lpvt(const char* name, int n, int nz, K kernel, A... args) {
    launch_impl(name, ctx.geo.S / 4, n, nz, 0, true, kernel, args...);
  }
  template <class K, class... A>
  void launch(const char* name, int tpe, int n, int nz, size_t smem_per_entity, K kernel, A... args) {
    launch_impl(name, tpe, n, nz, smem_per_entity, false, kernel, args...);
  }
  template <class K, class... A>
  void launch_impl(const char* name, int tpe, int n, int nz, size_t smem_per_entity, bool fold, K kernel,
                   A... args) {
    if (err != cudaSuccess || n <= 0 || nz <= 0) return;
    const int e = epb(name, tpe);
    const unsigned nb = (unsigned)((n + e - 1) / e);
    dim3 block(tpe, e), grid(fold ? nb * (unsigned)nz : nb, 1, fold ? 1 : nz);
    run(name, grid, block, smem_per_entity * e, kernel, args...);
  }
  template <class K, class... A>
  void run(const char* name, dim3 grid, dim3 block, size_t smem, K kernel, A... args) {
    HexProfEvent ev{name, nullptr, nullptr};
    if (prof) {
      cudaEventCreate(&ev.start);
      cudaEventCreate(&ev.stop);
      cudaEventRecord(ev.start, st);
    }
    kernel<<<grid, block, smem, st>>>(args...);
    ++count;
    err = cudaGetLastError();
    if (prof) {
      cudaEventRecord(ev.stop, st);
      prof->push_back(ev);
    }
  }
};
#define LP(L, n, nz, smem, kernel, ...) (L).lp(#kernel, n, nz, smem, kernel, __VA_ARGS__)
// Stencil kernel kv_<name> (four levels per thread), profiled as k_<name>.
#define LPS(L, n, nz, name, ...) (L).lpv("k_" #name, n, nz, kv_##name, __VA_ARGS__)
#define LPSN(L, label, n, nz, name, ...) (L).lpv(label, n, nz, kv_##name, __VA_ARGS__)
// Transport kernel kv_<name> over nT tracers (tracer folded into the block index).
#define LPST(L, n, nT, name, g, ...) (L).lpvt("k_" #name, n, nT, kv_##name, g, nT, __VA_ARGS__)
// Column-sweep kernel: the column-group form kv_<name> when a column fits in
// one warp (S/4 <= 32), else the one-level form k_<name> (shared memory per
// column: smem_v and smem respectively).
#define LPG(L, label, n, smem, smem_v, name, ...)                      \
  do {                                                                 \
    if ((L).group())                                                   \
      (L).lpg(label, n, smem_v, kv_##name, __VA_ARGS__);               \
    else                                                               \
      (L).lp(label, n, 1, smem, k_##name, __VA_ARGS__);                \
  } while (0)

static void diagnostics(Launcher& L, const float* u, int recompute_v) {
  HexCtx& c = L.ctx;
  const HexGeo& g = c.geo;
  HexWork& w = c.w;
  // (vorticity and divergence are kept only for the horizontal mixing)
  LPS(L, g.nV, 1, diag_vertex, g, u, w.pv_vertex, w.ke_vertex, w.vorticity);
  L.lpv("k_diag_cell", g.nC, 1, w.divergence ? kv_diag_cell<true> : kv_diag_cell<false>, g, u,
        (const float*)w.pv_vertex, (const float*)w.ke_vertex, w.ke, w.pv_cell, w.divergence);
  LPSN(L, recompute_v ? "k_diag_edge_v" : "k_diag_edge", g.nE, 1, diag_edge, g, u, (const float*)w.pv_vertex,
       (const float*)w.pv_cell, w.v, w.pv_edge, recompute_v);
}

cudaError_t diagnostics_only(HexCtx& ctx, const HexState& s, const HexSide& side, cudaStream_t stream) {
  Launcher L{ctx, stream};
  (void)s;
  diagnostics(L, side.u, 1);
  return L.err;
}

cudaError_t rebuild_sidecar(HexCtx& ctx, const HexState& s, const HexSide& side, cudaStream_t stream) {
  Launcher L{ctx, stream};
  const HexGeo& g = ctx.geo;
  LP(L, g.nE, 1, 0, k_recover_u, g, (const float*)s.rho, (const float*)s.rho_u, side.u);
  LP(L, g.nC, 1, 0, k_rebuild_cell, g, (const float*)s.rho, (const float*)s.rho_theta, (const float*)s.rho_u,
       (const float*)s.rho_w, side, ctx.w.flag);
  return L.err;
}

cudaError_t run_step(HexCtx& ctx, const HexState& in, const HexSide& side_in, const HexState& out,
                     const HexSide& side_out, cudaStream_t stream, long long* launches,
                     std::vector<HexProfEvent>* prof) {
  Launcher L{ctx, stream, prof};
  const HexGeo& g = ctx.geo;
  HexWork& w = ctx.w;
  const int nT = ctx.n_scalars;
  const bool hooked = ctx.stage_hook != nullptr;
  if (hooked) ctx.phys_held_rho = 0;  // no held physics at the step's start
  // halo exchange at a named point (a partitioned instance): the buffers and
  // their kinds; a failing hook stops the launches
  auto exchange = [&](int point, std::initializer_list<std::pair<const float*, int>> list) {
    if (!ctx.exchange_hook || L.err != cudaSuccess) return;
    float* bufs[24];
    int kinds[24];
    int n = 0;
    for (const auto& b : list)
      if (b.first && n < 24) {
        bufs[n] = const_cast<float*>(b.first);
        kinds[n++] = b.second;
      }
    if (ctx.exchange_hook(ctx.exchange_user, point, n, bufs, kinds) < 0) {
      ctx.phys_failed = 1;
      L.err = cudaErrorLaunchFailure;
    }
  };
  const int KC = HEXDYN_KIND_CELL, KE = HEXDYN_KIND_EDGE, KT = HEXDYN_KIND_TRACER;
  exchange(HEXDYN_XCH_STATE, {{in.rho, KC}, {in.rho_theta, KC}, {in.rho_u, KE}, {in.rho_w, KC}, {in.scalars, KT},
                              {side_in.theta_m, KC}, {side_in.exner, KC}, {side_in.rho_p, KC}, {side_in.rtheta_p, KC},
                              {side_in.pressure_p, KC}, {side_in.u, KE}, {side_in.w, KC}});
  const size_t sm_vcoef = sizeof(float) * g.S * 7, sm_ac = sizeof(float) * g.S * HEX_AC_SMEM_ARRAYS;
  const size_t sm_vcoef_v = sizeof(float) * (g.S + HEX_SWEEP_PAD) * HEX_VCOEFV_SMEM_ARRAYS;
  const size_t sm_ac_v = sizeof(float) * (g.S + HEX_SWEEP_PAD) * HEX_ACV_SMEM_ARRAYS;

  if (g.moist) {
    L.lpv("k_moist_cell", g.nC, 1, kv_moist_cell, g, (const float*)in.scalars, nT, w.qtot, w.cqw);
    L.lpv("k_moist_edge", g.nE, 1, kv_moist_edge, g, (const float*)in.scalars, nT, w.cqu);
  }
  // initial solve diagnostics with v reconstructed (rk_step=3)
  diagnostics(L, side_in.u, 1);
  exchange(HEXDYN_XCH_DIAG, {{w.pv_edge, KE}, {w.ke, KC}, {w.v, KE}});

  const HexState* saved = &in;
  const HexSide* s_in = &side_in;
  for (int sub = 0; sub < ctx.split_steps; ++sub) {
    const bool last = sub == ctx.split_steps - 1;
    const HexState& o = last ? out : ctx.tmp[sub & 1];
    const HexSide& so = last ? side_out : ctx.side_tmp[sub & 1];
    // split-flux accumulation: bit 2 active, bit 0 first subcycle (copy),
    // bit 1 last subcycle (multiply by 1/splits after the sum)
    const int flux_mode = 4 | (sub == 0 ? 1 : 0) | (last ? 2 : 0);
    // vertical coefficients before RK (stage-1 acoustic dts, saved theta)
    // (the saved Euler terms on the side stream: they share no array with
    // the coefficients)
    L.region = 1;
    L.fork();
    {
      LPG(L, "k_vcoef", g.nC, sm_vcoef, sm_vcoef_v, vcoef, g, ctx.dyn[0].dts2, (const float*)s_in->exner, (const float*)s_in->theta_m,
           (const float*)s_in->rtheta_p, (const float*)w.cqw, (const float*)w.qtot, w.cofwr, w.cofwz, w.coftz,
           w.cofwt, w.a_tri, w.alpha_tri, w.gamma_tri, w.flag);
    }
    L.side();
    LPS(L, g.nE, 1, euler_edge, g, (const float*)s_in->pressure_p, (const float*)s_in->rho_p,
         (const float*)w.qtot, (const float*)w.cqu, w.euler_ru);
    LPS(L, g.nC, 1, euler_cell, g, (const float*)saved->rho_u, (const float*)saved->rho_w,
         (const float*)s_in->pressure_p, (const float*)s_in->rho_p, (const float*)w.qtot, (const float*)w.cqw,
         w.tend_rho, w.euler_rw, (const float*)(hooked && ctx.phys_held_rho ? ctx.phys_rho : nullptr),
         hooked ? ctx.tend_rho_dyn : nullptr);
    L.join();
    if (g.smag_on) {
      // 2-D Smagorinsky mixing of the subcycle's start state, saved with the
      // Euler terms for its three RK stages (hexcore/driver.py:2826-2880)
      LPS(L, g.nC, 1, smag_kdiff, g, (const float*)s_in->u, (const float*)w.v, w.kdiff);
      LPS(L, g.nE, 1, mix_edge2, g, (const float*)w.divergence, (const float*)w.vorticity, (const float*)w.kdiff,
          (const float*)saved->rho, (const float*)w.euler_ru, w.delsq_u, w.mix_u);
      LPS(L, g.nC, 1, mix_cell2, g, (const float*)w.kdiff, (const float*)saved->rho, (const float*)s_in->w,
          (const float*)s_in->theta_m, w.w_mix, w.delsq_w, w.theta_mix, w.delsq_theta);
      if (g.smag_h4 > 0.0f) {
        LPS(L, g.nV, 1, mix_lap_vertex, g, (const float*)w.delsq_u, w.delsq_vort);
        LPS(L, g.nC, 1, mix_lap_cell, g, (const float*)w.delsq_u, w.delsq_div);
        LPS(L, g.nE, 1, mix_edge4, g, (const float*)saved->rho, (const float*)w.delsq_div,
            (const float*)w.delsq_vort, w.mix_u);
      }
      LPS(L, g.nC, 1, mix_cell4, g, (const float*)w.delsq_w, (const float*)w.delsq_theta, (const float*)w.euler_rw,
          (const float*)w.w_mix, w.theta_mix, w.mix_w);
    }
    const float* saved_ru = g.smag_on ? w.mix_u : w.euler_ru;
    const float* saved_rw = g.smag_on ? w.mix_w : w.euler_rw;
    const float* saved_theta = g.smag_on ? w.theta_mix : nullptr;

    const HexState* cur = saved;
    const HexSide* cs = s_in;
    for (int si = 0; si < 3; ++si) {
      const HexStage& stg = ctx.dyn[si];
      const float dts = (float)stg.acoustic_dt;
      // physics hand-off before the stage's tendencies (the host hook runs
      // in stream order: what it enqueues on the stream precedes the stage)
      int phys = 0;
      if (hooked && L.err == cudaSuccess) {
        HexDynFields cur_fields{};
        const float* f[HEXDYN_NUM_FIELDS] = {cur->rho, cur->rho_theta, cur->rho_u, cur->rho_w, in.scalars,
                                             cs->theta_m, cs->exner, cs->rho_p, cs->rtheta_p, cs->pressure_p,
                                             cs->u, cs->w};
        for (int i = 0; i < HEXDYN_NUM_FIELDS; ++i) cur_fields.field[i] = const_cast<float*>(f[i]);
        phys = ctx.stage_hook(ctx.stage_user, sub + 1, stg.stage, &cur_fields);
        if (phys < 0) {
          ctx.phys_failed = 1;
          L.err = cudaErrorLaunchFailure;
          break;
        }
      }
      // the mass-flux divergence of cur->rho_u: computed by the previous
      // stage's recovery, except for the first stage of the step
      if (sub == 0 && si == 0) LPS(L, g.nC, 1, hdiv, g, (const float*)cur->rho_u, w.hdiv);
      // edge values, the momentum tendency and (stage 2) the coefficients
      // are independent: the first on this stream, the others on the side
      L.region = 2;
      L.fork();
      LPS(L, g.nE, 1, edge_adv, g, (const float*)cur->rho_u, (const float*)cs->theta_m, (const float*)cs->w,
           w.edge_theta, w.edge_w);
      L.side();
      L.lpv("k_tend_u", g.nE, 1, g.rayleigh_levels ? kv_tend_u<true> : kv_tend_u<false>, g, (const float*)cs->u,
            (const float*)cur->rho_w, (const float*)cur->rho, (const float*)w.pv_edge, (const float*)w.ke,
            (const float*)w.hdiv, saved_ru, w.tend_ru,
            (const float*)((phys & HEXDYN_PHYS_RHO_U) ? ctx.phys_ru : nullptr), dts,
            HEX_FUSE_AC_FIRST ? w.ru_p : nullptr, HEX_FUSE_AC_FIRST ? w.ru_avg : nullptr);
      if (stg.stage == 2 && ctx.order == 3) {  // hexcore/driver.py:2894
        LPG(L, "k_vcoef", g.nC, sm_vcoef, sm_vcoef_v, vcoef, g, stg.dts2, (const float*)s_in->exner, (const float*)cs->theta_m,
             (const float*)cs->rtheta_p, (const float*)w.cqw, (const float*)w.qtot, w.cofwr, w.cofwz, w.coftz,
             w.cofwt, w.a_tri, w.alpha_tri, w.gamma_tri, w.flag);
      }
      L.join();
      LPS(L, g.nC, 1, tend_cell, g, (const float*)cur->rho_u, (const float*)saved->rho_u,
           (const float*)cur->rho_w, (const float*)saved->rho_w, (const float*)cs->theta_m,
           (const float*)s_in->theta_m, (const float*)cs->w, (const float*)w.edge_theta, (const float*)w.edge_w,
           saved_rw, (const float*)w.tend_ru, w.tend_rt, w.tend_rw, stg.stage, saved_theta,
           HexPhysCell{hooked ? 1 : 0, (phys & HEXDYN_PHYS_RHO_THETA) ? ctx.phys_rt : nullptr,
                       (phys & HEXDYN_PHYS_DIABATIC_THETA) ? ctx.phys_dth : nullptr, cur->rho,
                       ctx.tend_rho_dyn, hooked && stg.stage == 3 ? ctx.mod_rate : nullptr});
      // acoustic substeps
      const float inv_dts = 1.0f / dts;
      const float dts2 = stg.dts2;
      for (int n = 1; n <= stg.acoustic_steps; ++n) {
        const float* old_rt = w.rtpp[(n - 1) & 1];
        float* new_rt = w.rtpp[n & 1];
        if (n == 1) {
          // (with HEX_FUSE_AC_FIRST the momentum tendency already formed them)
          if (!HEX_FUSE_AC_FIRST)
          LPSN(L, "k_ac_edge_first", g.nE, 1, ac_edge, g, 0, 1, dts, inv_dts, (const float*)w.tend_ru, (const float*)new_rt,
               old_rt, (const float*)w.rho_pp, (const float*)s_in->theta_m, (const float*)s_in->exner,
               (const float*)w.cqu, w.ru_p, w.ru_avg);
        } else {
          // damping of substep n-1 (new = its output, old = its input), then update n
          const float* prev_new = w.rtpp[(n - 1) & 1];
          const float* prev_old = w.rtpp[(n - 2) & 1];
          LPSN(L, "k_ac_edge", g.nE, 1, ac_edge, g, 1, n - 1 == 1 ? 1 : 0, dts, inv_dts, (const float*)w.tend_ru, prev_new,
               prev_old, (const float*)w.rho_pp, (const float*)s_in->theta_m, (const float*)s_in->exner,
               (const float*)w.cqu, w.ru_p, w.ru_avg);
        }
        LPG(L, n == 1 ? "k_ac_cell_first" : "k_ac_cell", g.nC, sm_ac, sm_ac_v, ac_cell, g, n == 1 ? 1 : 0, dts, dts2, (const float*)w.ru_p,
             (const float*)s_in->theta_m, (const float*)w.tend_rho, (const float*)w.tend_rt,
             (const float*)w.tend_rw, (const float*)w.cofwr, (const float*)w.cofwz, (const float*)w.coftz,
             (const float*)w.cofwt, (const float*)w.a_tri, (const float*)w.alpha_tri, (const float*)w.gamma_tri,
             (const float*)cur->rho, (const float*)cs->w, (const float*)cur->rho_w, (const float*)saved->rho_w,
             old_rt, new_rt, w.rho_pp, w.rw_p, w.ww_avg);
        exchange(HEXDYN_XCH_ACOUSTIC, {{w.rho_pp, KC}, {new_rt, KC}, {w.rw_p, KC}, {w.ww_avg, KC}, {w.ru_p, KE},
                                       {w.ru_avg, KE}});
      }
      const int n_last = stg.acoustic_steps;
      if (!HEX_FUSE_AC_DAMP) {
        LPSN(L, "k_ac_edge_damp", g.nE, 1, ac_edge, g, 2, n_last == 1 ? 1 : 0, dts, inv_dts, (const float*)w.tend_ru,
             (const float*)w.rtpp[n_last & 1], (const float*)w.rtpp[(n_last - 1) & 1], (const float*)w.rho_pp,
             (const float*)s_in->theta_m, (const float*)s_in->exner, (const float*)w.cqu, w.ru_p, w.ru_avg);
      }
      const float* rtpp_final = w.rtpp[stg.acoustic_steps & 1];
      const float inv_steps = 1.0f / (float)stg.acoustic_steps;
      const float inv_splits = 1.0f / (float)ctx.split_steps;
      const int fm = stg.stage == 3 ? flux_mode : 0;
      // (with HEX_FUSE_AC_DAMP the last substep's divergence damping of
      // ru_p runs inside the edge recovery)
      LPS(L, g.nE, 1, recover_edge, g, (const float*)saved->rho_u, w.ru_p,
           (const float*)w.ru_avg, (const float*)s_in->rho_p, (const float*)w.rho_pp, o.rho_u, so.u, w.flux_u,
           fm, inv_steps, inv_splits, HEX_FUSE_AC_DAMP, n_last == 1 ? 1 : 0, inv_dts,
           (const float*)w.rtpp[n_last & 1], (const float*)w.rtpp[(n_last - 1) & 1], (const float*)s_in->theta_m);
      // the cell recovery and the diagnostics of the new u share no array
      L.region = 4;
      L.fork();
      LPS(L, g.nC, 1, recover_cell, g, stg.stage == 3 ? 1 : 0, (const float*)s_in->rho_p,
           (const float*)s_in->rtheta_p, (const float*)saved->rho_w, (const float*)w.rho_pp, rtpp_final,
           (const float*)w.rw_p, (const float*)w.ww_avg, (const float*)o.rho_u, o, so, w.flux_w, fm, inv_steps,
           inv_splits, w.flag, w.hdiv);
      L.side();
      // the step's last stage needs none: nothing after it reads them, and
      // the next step forms them from the same u at its start
      if (!(last && si == 2) || !HEX_SKIP_FINAL_DIAG) diagnostics(L, so.u, stg.stage == 3 ? 1 : 0);
      L.join();
      exchange(HEXDYN_XCH_STATE, {{o.rho, KC}, {o.rho_theta, KC}, {o.rho_u, KE}, {o.rho_w, KC}, {so.theta_m, KC},
                                  {so.exner, KC}, {so.rho_p, KC}, {so.rtheta_p, KC}, {so.pressure_p, KC},
                                  {so.u, KE}, {so.w, KC}, {w.pv_edge, KE}, {w.ke, KC}, {w.v, KE}, {w.hdiv, KC}});
      cur = &o;
      cs = &so;
      // the next subcycle's saved density tendency takes this stage's density
      // physics when this is the subcycle's last stage
      if (hooked && si == 2) ctx.phys_held_rho = (phys & HEXDYN_PHYS_RHO) ? 1 : 0;
    }
    if (L.err != cudaSuccess) break;
    saved = &o;
    s_in = &so;
  }

  // every output field but the scalars is final here (captured as an
  // external event node, so that work outside the graph can wait on it)
  if (ctx.dynamics_done && L.err == cudaSuccess) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    L.err = cudaStreamIsCapturing(L.st, &cap);
    if (L.err == cudaSuccess)
      L.err = cap == cudaStreamCaptureStatusActive
                  ? cudaEventRecordWithFlags(ctx.dynamics_done, L.st, cudaEventRecordExternal)
                  : cudaEventRecord(ctx.dynamics_done, L.st);
  }
  // split scalar transport: RK1, RK2 standard, RK3 monotonic FCT
  if (nT > 0) {
    const float* q_prev = in.scalars;
    for (int si = 0; si < 3; ++si) {
      const HexStage& stg = ctx.scal[si];
      const float step = (float)stg.large_dt;
      float* q_next = si == 2 ? out.scalars : w.q_stage[si];
      if (si == 0)
        exchange(HEXDYN_XCH_SCALARS, {{q_prev, KT}, {w.flux_u, KE}, {w.flux_w, KC}});
      else
        exchange(HEXDYN_XCH_SCALARS, {{q_prev, KT}});
      if (si < 2 || !ctx.monotonic) {
        // hexcore/transport.py:1749-1755 time-interpolation weight of rho_new
        const float wn = si == 0 ? (ctx.order == 3 ? (float)(1.0 / 3.0) : 0.5f) : (si == 1 ? 0.5f : 1.0f);
        L.lpvt("k_tr_edge", g.nE, (nT + HEX_TR_GROUP - 1) / HEX_TR_GROUP, kv_tr_edge, g, nT, 0, q_prev,
               (const float*)w.flux_u, w.edge_q);
        LPST(L, g.nC, nT, tr_std, g, step, wn, (const float*)in.scalars, q_prev, (const float*)in.rho,
             (const float*)out.rho, (const float*)w.flux_u, (const float*)w.flux_w, (const float*)w.edge_q, q_next);
      } else {
        LPS(L, g.nC, 1, fct_target, g, step, (const float*)in.rho, (const float*)w.flux_u,
             (const float*)w.flux_w, w.target, w.flag);
        L.lpvt("k_tr_edge", g.nE, (nT + HEX_TR_GROUP - 1) / HEX_TR_GROUP, kv_tr_edge, g, nT, 1, q_prev,
               (const float*)w.flux_u, w.edge_q);
        L.lpvt("k_fct_cell1", g.nC, nT, g.coc_across ? kv_fct_cell1<true> : kv_fct_cell1<false>, g, nT, step,
             (const float*)in.scalars, q_prev, (const float*)in.rho, (const float*)w.flux_u, (const float*)w.flux_w, (const float*)w.edge_q, (const float*)w.target,
             w.scale_in, w.scale_out, w.mass, w.vres);
        exchange(HEXDYN_XCH_FCT, {{w.scale_in, KT}, {w.scale_out, KT}});
        LPST(L, g.nE, nT, fct_edge, g, step, (const float*)in.scalars, (const float*)w.flux_u,
             (const float*)w.edge_q, (const float*)w.scale_in, (const float*)w.scale_out, w.hres_lim);
        LPST(L, g.nC, nT, fct_cell2, g, (const float*)w.vres, (const float*)w.scale_in, (const float*)w.scale_out, (const float*)w.mass, (const float*)w.hres_lim,
             (const float*)w.target, q_next);
      }
      q_prev = q_next;
    }
    if (g.clamp_scalars) L.lpv("k_clamp_scalars", g.nC, nT, kv_clamp_scalars, g, out.scalars);
  }
  if (launches) *launches = L.count;
  return L.err;
}
