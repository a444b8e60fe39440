// Device-side mesh / vertical-grid descriptor and layout helpers.
//
// HBM layout: every cell, edge and vertex field is [entity][level] with a
// padded level stride S (multiple of 8 floats, S >= nlev+1), so that a column
// is one contiguous 32-byte-aligned run and the threads of a warp that cover
// consecutive levels of one entity read consecutive words.  Interface fields
// (nlev+1 levels) use the same stride.  Tracers are [tracer][cell][level].
// Level vectors (fzm, rdzw, etp ...) are length S.  Cell-slot fields are
// [cell][slot] and the terrain metrics are [cell][slot][level].
#pragma once
#include <stdint.h>

struct HexGeo {
  int nC, nE, nV, L, S, maxE, maxE2, advW;
  // connectivity (int32)
  const int* coe;        // [E][2]
  const int* eoc;        // [C][maxE]
  const int* coc;        // [C][maxE]
  const int* voc;        // [C][maxE]
  const int* deg;        // [C]
  const int* voe;        // [E][2]
  const int* eov;        // [V][3]
  const int* eoe;        // [E][maxE2]
  const int* neoe;       // [E]
  const int* adv_cells;  // [E][advW]
  const int* n_adv;      // [E]
  const int* kite_slot;  // [C][maxE]
  // per-entity FP32 (already rounded to RKIND exactly as the reference does)
  const float* csign;     // [C][maxE] edgesOnCell_sign (+1 cell1, -1 cell2)
  const float* vsign;     // [V][3]
  const float* dc;
  const float* dv;
  const float* inv_dc;
  const float* inv_dv;
  const float* inv_area;
  const float* inv_area_tri;
  const float* kite;      // [V][3]
  const float* weights;   // [E][maxE2]
  const float* f_vertex;
  const float* f_edge;
  const float* cos_angle;
  const float* sin_angle;
  const float* adv;       // [E][advW]
  const float* adv3;      // [E][advW]
  // level vectors [S]
  const float* fzm;
  const float* fzp;
  const float* rdzw;
  const float* rdzu;
  const float* etp;
  const float* etm;
  const float* ewp;
  const float* ewm;
  const float* u_init;
  const float* v_init;
  // [entity][level] fields
  const float* zz;        // C
  const float* zxu;       // E
  const float* dss;       // C
  const float* zb;        // [C][maxE][S]
  const float* zb3;       // [C][maxE][S]
  const float* rho_base;  // C
  const float* rtheta_base;
  const float* exner_base;
  // scalars
  float cf1, cf2, cf3;
  float coef3;        // config_coef_3rd_order
  float g;            // gravity
  float rgas;
  float rcv;          // R/(cp-R) in FP32 operations
  float c2;           // cp*rcv
  float r_over_p0;    // FP32(R/p0)
  float kappa;        // FP32(R/(cp-R)) computed in double then rounded
  float apvm_scale;   // FP32(apvm)*FP32(dt)
  float smdiv_base;   // 2*smdiv*len_disp in FP32 operations
  const float* smdiv_edge;  // [E] smdiv_base of the edge's mesh (ensembles mix meshes)
  int apvm_on;
  int moist;          // 0 = dry coefficients, 1 = native (all scalars load)
  int winds_zero;     // u_init and v_init are zero at every level
  int dss_zero;       // the implicit w damping profile dss is +0 in every word (config_xnutr = 0)
  int coc_across;     // cells_on_cell[c][s] is the cell across edges_on_cell[c][s] everywhere
  int clamp_scalars;  // negative mixing ratios set to zero at the end of the step
  // 2-D Smagorinsky mixing (hexcore/mixing_v841.py), when smag_on
  int smag_on;
  const float* deform_c2;   // [C][maxE] deformation weights
  const float* deform_s2;
  const float* deform_cs;
  const float* mix_del2;    // [E] meshScalingDel2
  const float* mix_del4;    // [E] meshScalingDel4
  const float* inv_dv_lim;  // [E] min(1/dvEdge, 4/dcEdge)
  float smag_strain_scale, smag_ceiling, smag_h4, smag_div_factor;
  // upper damping (hexcore/native/upper_damping.rs): Rayleigh damping of u
  // over the top rayleigh_levels levels, CAM floor of kdiff over the top
  // cam_levels levels (0 = off)
  int rayleigh_levels;
  float rayleigh_inverse;
  int cam_levels;
  float cam_base;
};

#define HEX_FLAG_DENSITY 1
#define HEX_FLAG_SINGULAR 2
#define HEX_FLAG_POWF 4
#define HEX_FLAG_TARGET 8

// Physics hand-off inputs of the cell tendency kernel (all NULL when off):
// the physics rho-theta tendency, the lagged diabatic theta, the stage's
// density, the density tendency without physics and, at RK stage 3, the
// modified theta dynamics rate output.
struct HexPhysCell {
  int on;
  const float* rt;
  const float* dth;
  const float* rho;
  const float* tend_rho_dyn;
  float* mod_rate;
};
