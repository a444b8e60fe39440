/*
 * hexdyn: B200-native MPAS-A v8.4.2 dry-plus-tracer dycore step, C ABI.
 *
 * The entry points are the drop-in boundary for the reference's dycore step
 * path (gpuwm-hex 0.5.0, tree/src/hexcore/).  Each declaration names the
 * reference interface it replaces:
 *
 *   hexdyn_abi_version      <- hexcore/native/step_submit.c:33 hex_step_abi_version
 *   hexdyn_create           <- hexcore/cuda_driver.py:2826 CudaDryDycoreDriver.from_host
 *                              (upload of mesh, vertical grid, reference state,
 *                              terrain and advection coefficients; validation
 *                              as in hexcore/cuda_driver.py:3096 _validate_config)
 *   hexdyn_set_state        <- from_host's DeviceAtmosphere upload
 *                              (hexcore/cuda_backend/containers.py:1098)
 *   hexdyn_get_state        <- hexcore/cuda_driver.py:6112 step() host download
 *   hexdyn_step             <- hexcore/cuda_driver.py:5751 step_device /
 *                              :4854 _step_device_v841 (flag read :5355-5402)
 *   hexdyn_capture_graph    <- hexcore/cuda_subcycle_graphs.py:64 attach_subcycle_graphs
 *                              (here the whole large step is one graph)
 *   hexdyn_create_ensemble,
 *   hexdyn_set/get_member_state,
 *   hexdyn_step_batched     <- hexcore/multi_member.py (members on private
 *                              streams); batched stepping of uneven ensembles
 *   hexdyn_last_error       <- the refusal / FloatingPointError text of the driver
 *   hexdyn_destroy          <- driver teardown
 *
 * Conventions (hexcore/native/step_submit.c:33-90): every call returns an
 * int status, 0 on success, a negative HEXDYN_E_* code for a refused
 * argument, or a positive CUDA error code; nothing is retried.  Host arrays
 * use the reference's logical layout: [level][entity] for fields, row-major
 * [entity][slot] for connectivity, zero-based indices, int32 and float32.
 * One handle is bound to one stream at a time and steps one state at a time.
 */
#ifndef HEXDYN_H
#define HEXDYN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HEXDYN_ABI_VERSION 5

#define HEXDYN_OK 0
#define HEXDYN_E_ARG (-1)        /* invalid argument or descriptor */
#define HEXDYN_E_STATE (-2)      /* call out of order (no state bound, ...) */
#define HEXDYN_E_NUMERIC (-3)    /* device validation flag set (see flag_out) */
#define HEXDYN_E_CAPACITY (-4)   /* size beyond a stated maximum */

/* Validation-flag bits reported by hexdyn_step (hexcore/cuda_driver.py:4885). */
#define HEXDYN_FLAG_DENSITY 1    /* rho or rho_theta became non-positive */
#define HEXDYN_FLAG_SINGULAR 2   /* singular vertical acoustic system */
#define HEXDYN_FLAG_POWF 4       /* Exner argument outside positive normals */
#define HEXDYN_FLAG_TARGET 8     /* non-positive FCT target density */

/* Field identifiers for hexdyn_set_state / hexdyn_get_state. */
enum HexDynField {
  HEXDYN_RHO = 0,             /* rho_zz      [L][C]   */
  HEXDYN_RHO_THETA = 1,       /* rho_theta_m [L][C]   */
  HEXDYN_RHO_U = 2,           /* ru          [L][E]   */
  HEXDYN_RHO_W = 3,           /* rw          [L+1][C] */
  HEXDYN_SCALARS = 4,         /* scalars     [T][L][C] */
  HEXDYN_THETA_M = 5,         /* saved diagnostics (DrySavedDiagnostics) */
  HEXDYN_EXNER = 6,
  HEXDYN_RHO_P = 7,
  HEXDYN_RHO_THETA_P = 8,
  HEXDYN_PRESSURE_P = 9,
  HEXDYN_U = 10,              /* [L][E]   */
  HEXDYN_W = 11,              /* [L+1][C] */
  HEXDYN_NUM_FIELDS = 12
};

typedef struct HexDynDesc {
  /* sizes */
  int32_t n_cells, n_edges, n_vertices, n_levels;
  int32_t max_edges, max_edges2, adv_width, n_scalars;
  /* connectivity */
  const int32_t* cells_on_edge;     /* [E][2] */
  const int32_t* edges_on_cell;     /* [C][max_edges] */
  const int32_t* cells_on_cell;     /* [C][max_edges] */
  const int32_t* vertices_on_cell;  /* [C][max_edges] */
  const int32_t* n_edges_on_cell;   /* [C] */
  const int32_t* vertices_on_edge;  /* [E][2] */
  const int32_t* edges_on_vertex;   /* [V][3] */
  const int32_t* cells_on_vertex;   /* [V][3] */
  const int32_t* edges_on_edge;     /* [E][max_edges2] */
  const int32_t* n_edges_on_edge;   /* [E] */
  const int32_t* adv_cells;         /* [E][adv_width] advCellsForEdge */
  const int32_t* n_adv_cells;       /* [E] */
  /* FP32 geometry (the float64 static fields rounded to float32) */
  const float *dc_edge, *dv_edge, *area_cell, *area_triangle;
  const float* kite_areas;          /* [V][3] */
  const float* weights_on_edge;     /* [E][max_edges2] */
  const float *f_vertex, *f_edge;
  const float *cos_angle_edge, *sin_angle_edge; /* cos/sin of FP32 angleEdge */
  const float *adv_coefs, *adv_coefs_3rd;       /* [E][adv_width] */
  /* vertical grid */
  const float *fzm, *fzp, *rdzw, *rdzu;         /* [L] */
  const float* zz;                  /* [L][C] */
  const float* zxu;                 /* [L][E] */
  const float* dss;                 /* [L][C] implicit w damping */
  const float* zb_cell;             /* [L+1][C][max_edges] */
  const float* zb3_cell;            /* [L+1][C][max_edges], x coef_3rd_order */
  const float *rho_base, *rho_theta_base, *exner_base; /* [L][C] */
  const float *u_init, *v_init;     /* [L] */
  float cf1, cf2, cf3;
  float nominal_min_dc;
  /* configuration (V841DryDycoreConfig, hexcore/config_v841.py:114) */
  double dt;
  int32_t n_sub_steps;              /* config_number_of_sub_steps */
  int32_t split_steps;              /* config_dynamics_split_steps (1 or 3) */
  int32_t monotonic;                /* config_monotonic */
  int32_t moist;                    /* 0: dry coefficients, 1: native (all scalars load) */
  int32_t numerics;                 /* 0: strict (bitwise), 1: fast (FMA) */
  float coef_3rd_order, apvm_upwinding, smdiv, len_disp;
  float epssm_minimum, epssm_maximum, epssm_bottom_z, epssm_top_z;
  float rgas, cp, gravity, p0;
  /* dts^2 of the three dynamics RK stages as the host computes FP32
   * dts**2 (NumPy's scalar power, which is powf and not always dts*dts);
   * zero selects dts*dts. */
  float acoustic_dts2[3];
  /* config_time_integration_order: 3, or 2 (stages dt/2, dt/2, dt with
   * n/2, n/2, n substeps of dt/n; hexcore/integration.py:104-160); 0 = 3 */
  int32_t time_integration_order;
  /* 2-D Smagorinsky horizontal mixing, v8.4.1 deformation form
   * (hexcore/mixing_v841.py, hexcore/mixing.py:391-736; config_horiz_mixing
   * '2d_smagorinsky'): 0 = off.  The host supplies the deformation weights
   * of every cell slot (atm_initialize_deformation_weights), the per-edge
   * mesh scalings meshScalingDel2/Del4 and the FP32 constants of
   * smagorinsky_2d: (c_s len)^2, the diffusivity ceiling 0.01 len^2 / dt,
   * the fourth-order viscosity visc4 len^3 and config_del4u_div_factor. */
  int32_t horiz_mixing;
  const float *deform_c2, *deform_s2, *deform_cs; /* [C][max_edges] */
  const float *mix_del2, *mix_del4;                /* [E] */
  float smag_strain_scale, smag_ceiling, smag_h4, smag_div_factor;
  /* Upper damping (hexcore/native/upper_damping.rs, the reference's native
   * operators): Rayleigh damping of u over the top rayleigh_levels levels
   * (0 = off; config_rayleigh_damp_u) with rayleigh_inverse =
   * 1/(levels (days 86400)) in FP32; the CAM floor of the Smagorinsky
   * diffusivity over the top cam_levels levels (0 = off;
   * config_mpas_cam_coef > 0) with cam_base = ((4 x 2.0833) len) coef. */
  int32_t rayleigh_levels;
  float rayleigh_inverse;
  int32_t cam_levels;
  float cam_base;
  /* 1: set negative mixing ratios to zero at the end of the step (where
   * q < 0: q = 0; -0 and NaN kept), as the reference's CUDA driver does on
   * the global path without physics (hexcore/cuda_driver.py:5306-5311,
   * atm_srk3 2798-2800); its NumPy authority does so only with
   * config_moist_physics (hexcore/driver.py:3531-3534).  0: no clamp. */
  int32_t clamp_negative_scalars;
} HexDynDesc;

typedef struct HexDynHandle HexDynHandle;

int hexdyn_abi_version(void);

/* Validate the descriptor, allocate device memory, upload the static
 * fields.  Runs on the current CUDA device. */
int hexdyn_create(const HexDynDesc* desc, HexDynHandle** out);

/* Upload one field of the current state from host memory (logical layout),
 * enqueued on `stream` (asynchronous when `host` is pinned; the caller must
 * keep `host` alive until the stream reaches the copy). */
int hexdyn_set_state(HexDynHandle* h, int field, const float* host, size_t count, void* stream);

/* Rebuild the saved diagnostics from the current prognostic state, as the
 * reference does when no sidecar is supplied (hexcore/driver.py:2655). */
int hexdyn_rebuild_sidecar(HexDynHandle* h, void* stream);

/* Download one field of the current state into host memory, enqueued on
 * `stream` (synchronise the stream before reading `host`). */
int hexdyn_get_state(HexDynHandle* h, int field, float* host, size_t count, void* stream);

/* Advance nsteps large steps on `stream` (a cudaStream_t; NULL = default).
 * Reads the validation flag once at the end; *flag_out receives it and a
 * non-zero flag returns HEXDYN_E_NUMERIC.  *completed counts the steps
 * enqueued. */
int hexdyn_step(HexDynHandle* h, void* stream, int nsteps, int* flag_out, int* completed);

/* Enqueue nsteps large steps without reading the flag (asynchronous). */
int hexdyn_step_async(HexDynHandle* h, void* stream, int nsteps);

/* One large step from host buffers to host buffers, enqueued on `stream`:
 * the reference's from_host upload, step_device and step() download
 * (hexcore/cuda_driver.py:2826, :5751, :6112) in one call.  `in` and `out`
 * hold HEXDYN_NUM_FIELDS host pointers indexed by field identifier (logical
 * layout as hexdyn_set_state / hexdyn_get_state; pinned memory for
 * asynchronous copies; NULL allowed for an empty field).  Every field but
 * the scalars is final when the step's dynamics end, so those downloads run
 * on a private stream beside the scalar transport; the call returns with
 * all of it ordered before later work on `stream` (synchronise `stream`
 * before reading `out`). */
int hexdyn_step_host(HexDynHandle* h, const float* const* in, float* const* out, void* stream);

/* Read and clear the validation flag (synchronises `stream`). */
int hexdyn_read_flag(HexDynHandle* h, void* stream, int* flag_out);

/* Run nsteps eager steps with a CUDA event pair around every kernel launch
 * and write one line per kernel, "name launches total_ms", into out.
 * (Profiling entry point; the reference's launch_timed,
 * hexcore/cuda_subcycle_graphs.py:45-62.) */
int hexdyn_profile_steps(HexDynHandle* h, void* stream, int nsteps, char* out, size_t len);

/* Autotuner of launch shapes (no counterpart in the reference, whose
 * kernels launch fixed shapes): times every kernel of `steps_per_candidate`
 * eager steps with 64, 96, 128, 160, 192, 224 and 256 threads per block
 * (CUDA events per launch; a block holds threads / (S/4) cells or edges, or
 * threads / 16 columns in the column sweeps), keeps the fastest block size of
 * every launch label, and restores the state and sidecar the steps started
 * from; captured graphs are captured again with the tuned shapes.  Results
 * do not depend on the block size (every entity is computed by the same
 * code).  `report` receives "threads <candidates>" and then one line per
 * label: "label <us at each candidate> chosen". */
int hexdyn_autotune(HexDynHandle* h, void* stream, int steps_per_candidate, char* report, size_t len);

/* Capture the whole large step into CUDA graphs (one per buffer parity);
 * later hexdyn_step calls replay them. */
int hexdyn_capture_graph(HexDynHandle* h, void* stream);

/* Device pointer of a field of the current state ([entity][level] padded
 * layout, level stride from hexdyn_level_stride) for zero-copy consumers. */
int hexdyn_device_field(HexDynHandle* h, int field, void** dev_ptr);

/* The final acoustic words of the last step: the perturbation momenta
 * ru_p ([edge][level], L levels) and rw_p ([cell][level], L+1 interfaces)
 * after the last substep of RK stage 3 of the last dynamics subcycle, in
 * the padded layout.  They are the restart words the reference hands to its
 * acoustic_output_callback (hexcore/cuda_driver.py:4707-4711; MPAS
 * Registry.xml restart stream) and stay valid until the next step. */
#define HEXDYN_WORK_RU_P 0
#define HEXDYN_WORK_RW_P 1
int hexdyn_acoustic_field(HexDynHandle* h, int which, void** dev_ptr);
int hexdyn_level_stride(HexDynHandle* h);
long long hexdyn_launches_per_step(HexDynHandle* h);
size_t hexdyn_device_bytes(HexDynHandle* h);

/* Caller-owned device buffers of one state and sidecar, in the library's
 * padded [entity][level] layout (level stride from hexdyn_level_stride;
 * scalars [tracer][cell][level]), indexed by HexDynField. */
typedef struct HexDynFields {
  float* field[HEXDYN_NUM_FIELDS];
} HexDynFields;

/* Per-stage physics hand-off: `physics_stage_callback` of the reference's
 * `_step_device_v841` (hexcore/cuda_driver.py:4393-4400, called by
 * hexcore/mpasphys/runtime_v842.py:2310).  With a hook set, every large
 * step runs eagerly (no graph) and calls the hook on the host before the
 * tendencies of each RK stage of each dynamics subcycle, in stream order,
 * with `current` holding device pointers (padded layout) of the stage's
 * state and saved diagnostics.  The hook fills the physics buffers of
 * hexdyn_physics_buffer on the step's stream and returns a bit set of what
 * it gave (HEXDYN_PHYS_*), or a negative value to abort the step (the step
 * returns HEXDYN_E_STATE).  The tendencies enter as the reference adds them:
 * tend_ru = (tend_ru + saved Euler u term) + rho_u; tend_rt gains, after its
 * stage-3 modified-rate snapshot, rho x diabatic_theta, the saved mixing
 * term, then rho_theta; the density tendency that the hook gave at the last
 * stage of a subcycle is added to the next subcycle's saved density
 * tendency.  At RK stage 3 of every subcycle the step stores the modified
 * theta dynamics rate (tend_rt - tend_rho theta_m) / rho, before any
 * physics term, in buffer HEXDYN_PHYS_MODIFIED_RATE.  Single instances only;
 * `hook` NULL removes it. */
#define HEXDYN_PHYS_RHO_U 1
#define HEXDYN_PHYS_RHO_THETA 2
#define HEXDYN_PHYS_RHO 4
#define HEXDYN_PHYS_DIABATIC_THETA 8
#define HEXDYN_PHYS_MODIFIED_RATE 16
typedef int (*HexDynStageHook)(void* user, int dynamics_substep, int rk_step, const struct HexDynFields* current);
int hexdyn_set_stage_hook(HexDynHandle* h, HexDynStageHook hook, void* user);
/* Device pointer of a physics buffer ([E][S] for HEXDYN_PHYS_RHO_U, [C][S]
 * otherwise; padded layout, zeroed when the hook is set). */
int hexdyn_physics_buffer(HexDynHandle* h, int which, void** device_ptr);

/* Halo exchange hook of a partitioned instance (one rank's local mesh:
 * owned entities first, halo entities last; hexdyn.partition builds the
 * meshes and the plan).  With a hook set, every step runs eagerly and calls
 * it on the host, in stream order and with both streams joined, at the
 * points where owner values must reach the halo -- the reference's rounds
 * (hexcore/partition_executor_v841.py:35-50):
 *   HEXDYN_XCH_STATE     the step's start (state, saved diagnostics and
 *                        scalars) and the end of every RK stage after the
 *                        recovery and the solve diagnostics (state, saved
 *                        diagnostics, pv_edge, ke, v and the mass-flux
 *                        divergence);
 *   HEXDYN_XCH_DIAG      after the step's initial solve diagnostics (pv_edge,
 *                        ke, v);
 *   HEXDYN_XCH_ACOUSTIC  after every acoustic cell pass (rho_pp, rtheta_pp,
 *                        rw_p, ww_avg, ru_p, ru_avg);
 *   HEXDYN_XCH_SCALARS   at the entry of every transport stage (the stage's
 *                        input scalars; at the first also the split mass
 *                        fluxes);
 *   HEXDYN_XCH_FCT       after the monotonic limiter's scale factors.
 * `bufs[i]` is a device buffer in the padded layout of kind `kinds[i]`
 * (HEXDYN_KIND_*); the hook overwrites its halo rows with the owners'
 * values on the step's stream and returns 0, or a negative value to abort
 * the step.  Single instances only; `hook` NULL removes it. */
#define HEXDYN_XCH_STATE 1
#define HEXDYN_XCH_DIAG 2
#define HEXDYN_XCH_ACOUSTIC 3
#define HEXDYN_XCH_SCALARS 4
#define HEXDYN_XCH_FCT 5
#define HEXDYN_KIND_CELL 0    /* [nCells][S] */
#define HEXDYN_KIND_EDGE 1    /* [nEdges][S] */
#define HEXDYN_KIND_TRACER 2  /* [n_scalars][nCells][S] */
typedef int (*HexDynExchangeHook)(void* user, int point, int nbufs, float* const* bufs, const int* kinds);
int hexdyn_set_exchange_hook(HexDynHandle* h, HexDynExchangeHook hook, void* user);

/* Halo rows of an exchange point in one launch (no counterpart in the
 * reference, whose executor packs each field with a NumPy/CuPy fancy index,
 * hexcore/partition_executor_v841.py): hexdyn_halo_pack copies the rows
 * `cell_rows` (cell and tracer buffers) and `edge_rows` (edge buffers) --
 * device int32 lists of local row indices -- of the `nbuf` (<= 24) buffers of
 * a hook call, padded layout and shapes of handle `h`, into `packed`;
 * hexdyn_halo_unpack writes them back from `packed`.  Packed layout: buffer
 * by buffer, tracer block by block, row by row, S words per row;
 * hexdyn_halo_words gives its size in floats.  `packed` and every buffer
 * 16-byte aligned; row indices outside the buffer are skipped.  A rank packs
 * the owned rows its peer needs (with its own handle), the peer unpacks them
 * into its halo rows (with its handle), in the same buffer order. */
size_t hexdyn_halo_words(HexDynHandle* h, int nbuf, const int* kinds, int n_cell_rows, int n_edge_rows);
int hexdyn_halo_pack(HexDynHandle* h, int nbuf, float* const* bufs, const int* kinds, const int* cell_rows,
                     int n_cell_rows, const int* edge_rows, int n_edge_rows, float* packed, void* stream);
int hexdyn_halo_unpack(HexDynHandle* h, int nbuf, float* const* bufs, const int* kinds, const int* cell_rows,
                       int n_cell_rows, const int* edge_rows, int n_edge_rows, const float* packed, void* stream);

/* Bind caller-owned device buffers (padded layout, 16-byte aligned, every
 * field; replaces the reference's DeviceAtmosphere handed to the driver,
 * hexcore/cuda_driver.py:5419) as the current state
 * and sidecar; the handle steps from them without a copy.  Each step
 * publishes the new state in the other buffer set, as the reference does, so
 * after an odd number of steps the state is in the library's own buffers and
 * after an even number back in the bound ones (hexdyn_device_field always
 * points at the current state).  fields == NULL unbinds (when the current
 * state is in the library's buffers).  Captured graphs are captured again. */
int hexdyn_bind_state(HexDynHandle* h, const HexDynFields* fields, void* stream);

/* No counterpart in the reference: one large step that allocates nothing.
 * For callers that cannot call cudaMalloc when they step -- host frameworks
 * whose device memory is owned by a pool that must not be bypassed (an
 * allocation outside it breaks their accounting or fails under their memory
 * limit), or ensembles that keep every member's state in their own buffers
 * and cannot give each member a private workspace.  The caller passes the
 * input state and sidecar and the output buffers (`in` and `out` must not
 * overlap); the mesh and configuration come from `h`.  Every intermediate of
 * the step (tendencies, acoustic perturbations, coefficients, subcycle
 * states, transport limiter fields) lives in one file-scope device array of
 * 64 MiB that each GPU loading the library holds until exit; a step needing
 * more returns HEXDYN_E_CAPACITY and names the size (2562 cells x 55 levels
 * with 6 scalars is already too large).  The first call on a device looks up
 * that array's address (cudaGetSymbolAddress, with that device current, in
 * its primary context).  All calls share the array and it keeps the last
 * call's contents: each call clears the words it uses before the step, and
 * calls that overlap on the GPU (different streams, or concurrent host
 * threads) race on it, so issue them on one stream.  Kernels run on `stream`
 * alone (no second stream) at 256 threads per block (the handle's autotuned
 * block sizes are not used).  Reads the flag at the end like hexdyn_step
 * (synchronises `stream`). */
int hexdyn_step_noalloc(HexDynHandle* h, const HexDynFields* in, const HexDynFields* out, void* stream,
                        int* flag_out);

/* Ensembles (hexcore/multi_member.py:1-7 runs members on private streams,
 * one launch sequence each).  hexdyn_create_ensemble concatenates several
 * members into one handle: member m keeps its own mesh (meshes may differ in
 * size), terrain, reference state and state, all members share the
 * configuration, levels, tracer count and vertical coordinate (refused with
 * HEXDYN_E_ARG otherwise), and every kernel of the step runs once for all
 * members.  No stencil crosses members, so each member's result equals, bit
 * for bit, the step of a handle created from its descriptor alone.  The
 * whole-field calls (hexdyn_set_state, hexdyn_get_state, hexdyn_step,
 * hexdyn_capture_graph, ...) act on the concatenation; the member calls move
 * one member's field in its own logical layout ([level][entity] of that
 * member). */
int hexdyn_create_ensemble(const HexDynDesc* members, int n_members, HexDynHandle** out);
int hexdyn_member_count(HexDynHandle* h);
int hexdyn_set_member_state(HexDynHandle* h, int member, int field, const float* host, size_t count,
                            void* stream);
int hexdyn_get_member_state(HexDynHandle* h, int member, int field, float* host, size_t count, void* stream);

/* Groups of an uneven batch: handles (single instances or ensembles) whose
 * members differ in time step, each advanced by its own number of large
 * steps per call (for instance 1 step of 1440 s and 2 steps of 720 s). */
typedef struct HexDynBatch {
  int32_t n_groups;
  HexDynHandle* const* groups;   /* distinct handles */
  const int32_t* steps;          /* large steps of each group */
  int32_t* flags;                /* out: validation flag of each group; NULL = do not read */
} HexDynBatch;

/* Advance every group of the batch, each on the handle's private stream
 * after the work already on `stream`, and make `stream` wait for all of them
 * (the groups run concurrently).  With flags != NULL the flags are read and
 * cleared (synchronises `stream`) and a set flag returns HEXDYN_E_NUMERIC
 * naming the first group; with flags == NULL nothing synchronises. */
int hexdyn_step_batched(const HexDynBatch* batch, void* stream);

/* Learned-corrector state access (no counterpart in the reference: the
 * corrector is this library's own).  All act on the current state of `h`
 * and are enqueued on `stream`; arrays are device pointers.
 *   hexdyn_column_features: X [n_cells][ld] floats, ld >= 6 L: theta_m,
 *     rho_zz, w (interfaces 0..L-1), first scalar, mean u over the cell's
 *     edges, mean theta_m over the neighbouring cells, each over L levels.
 *   hexdyn_edge_features: X [n_edges][ld], ld >= 4 L: u, theta_m of both
 *     cells, mean rho_zz of both cells.
 *   hexdyn_apply_increments: adds y * scale + shift (per feature) of the
 *     column outputs (theta_m, rho_zz, w; [n_cells][ldc]) and of the edge
 *     outputs (u; [n_edges][lde]) to the prognostic state; either may be
 *     NULL.  Rebuild the saved diagnostics afterwards.
 *   hexdyn_total_energy: dev_out[0] (device double) = internal + potential
 *     + kinetic energy, dev_out[1] = the volume integral of w^2, with z_mid
 *     the height of every cell level in the padded [cell][level] layout. */
int hexdyn_column_features(HexDynHandle* h, float* X, int ld, void* stream);
int hexdyn_edge_features(HexDynHandle* h, float* X, int ld, void* stream);
int hexdyn_apply_increments(HexDynHandle* h, const float* Ycol, int ldc, const float* col_scale,
                            const float* col_shift, const float* Yedge, int lde, const float* edge_scale,
                            const float* edge_shift, void* stream);
int hexdyn_total_energy(HexDynHandle* h, const float* z_mid, double* dev_out, void* stream);

/* Copy the last error message of this thread into buf. */
int hexdyn_last_error(char* buf, size_t len);

int hexdyn_destroy(HexDynHandle* h);

#ifdef __cplusplus
}
#endif
#endif /* HEXDYN_H */
