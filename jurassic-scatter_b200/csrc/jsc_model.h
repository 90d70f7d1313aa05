// Definitions of the opaque handles declared in jurassic_b200.h (CUDA side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "jsc_internal.h"

struct jsc_model {
  int device;
  int ng, nd, nw;
  int n_grid;
  int grid_np0;  // pressure levels of grid 0 (host copy)
  int64_t n_nodes;
  size_t table_bytes;
  double nu[NDMAX];
  jsc_dev_model dv;  // device view passed to kernels
  int *d_grid_np, *d_grid_nt, *d_tab_grid, *d_window;
  double *d_grid_p, *d_grid_t, *d_planck_b, *d_planck_s, *d_nu;
  jsc_row *d_rows;
  jsc_node *d_nodes;
  jsc_ctm_coef *d_ctm;
};

// Forward-model switches copied from ctl_t when a batch is created.
struct jsc_run_cfg {
  int ng, nd, nw;
  double transs;
  int ctm_co2, ctm_h2o, ctm_n2, ctm_o2;
  int refrac;
  double rayds, raydz, hydz;
  int sca_n, sca_mult, sca_ext_beta_a;
};

// LOS point record for the radiative transfer (doubles): pressure,
// temperature, step length, H2O VMR, packed (p, T) table bracket of the
// shared grid (-1 when tables use several grids), Planck table index,
// aerosol/cloud scaling factor and layer index (0 and -999 in clear air),
// the window extinctions, then the column densities (volume mixing ratios
// in the raw records the aerosol refinement reads).
enum { REC_P = 0, REC_T, REC_DS, REC_QH2O, REC_GRID, REC_PLK, REC_AF, REC_AI, REC_K };
#define JSC_REC_W(nw, ng) (REC_K + (nw) + (ng))

// Arguments of the EGA + radiative-transfer kernel.
struct EgaArgs {
  jsc_dev_model m;
  jsc_run_cfg cfg;
  int n_rays, W, ndp, single_grid;
  const int *nlos;
  const int64_t *los_off;
  const double *pts, *tsurf;
  double *rad, *tau;
  unsigned long long *counters;
  unsigned long long *digest;  // optional [n_rays][nd] EGA index checksums
  const double *beta;          // aerosol beta_e/beta_s/beta_a [3][nl][nd]
  int aero_nl;
  // Scattering source at the scattering points (LOS points with aerosol
  // factor > 0) when the batch scatters: [n_sp][nd], points of ray r from
  // sp_off[r] on, in LOS order.  Null: extinction only.
  const double *src_sca;
  const int64_t *sp_off;
  // Continuum extinction and Planck source per (LOS point, channel),
  // [n_points][nd] (read by the lane kernel).
  const double *beta_ctm, *src_pl;
  // Ray order of the ray-tile kernel: tile t holds rays order[32 t ..
  // 32 t + 31] (rays of one profile and similar geometry side by side).
  const int *order;
};

// Kernel timers of a batch.
enum { JSC_T_HYDRO = 0, JSC_T_RAYTRACE, JSC_T_EGA, JSC_T_SCATTER, JSC_T_CTM, JSC_T_SUR, JSC_T_N };

#define JSC_NALPHA_REF 28  // secondary pencils per scattering point (src/scatter.c:673)
#define JSC_MAX_DEPTH 7    // deepest scattering order with its own pencil count
#define JSC_WAIT_BUDGET (1u << 22)  // default polls of a device wait (each >= 64 ns)
#define JSC_FIXED_POINTS_PER_RAY 40  // default scattering-point capacity per primary ray
#define JSC_FIXED_PENCIL_LOS 144     // LOS capacity per secondary pencil (fixed runs)
#define JSC_FIXED_SUN_LOS 256        // LOS capacity per solar pencil (fixed runs)

struct jsc_batch {
  jsc_model *m;
  jsc_run_cfg cfg;
  int max_atm, max_levels, max_rays;
  int64_t max_seg;
  int n_atm, n_levels, n_rays;
  int W;  // doubles per LOS point record for the radiative transfer

  // Inputs.
  int *d_atm_off;
  double *d_z, *d_lon, *d_lat, *d_p_in, *d_t, *d_q, *d_k;
  double *d_p;              // pressure after hydrostatic balance
  double *d_zmin, *d_zmax;  // per profile
  int ip;                   // atmosphere interpolation (1 profile, 2, 3)
  double cz, cx;            // IP 3 influence lengths [km]
  double *d_psurf;          // IP 2/3 surface positions [profiles or levels][3]
  int *d_ray_atm;
  double *d_ray;            // [9][max_rays]: time obsz obslon obslat vpz vplon vplat + 2 spare

  // Aerosol/cloud layers (sca_n > 0): layer geometry, optics [nl][nd],
  // phase functions [nl][nd][NTHETA], edge altitudes of the refinement.
  int aero_nl, n_alti;
  double altimax, altimin;
  double *d_aero;           // top[NLMAX] bottom[NLMAX] trans[NLMAX] alti[...]
  double *d_beta;           // beta_e, beta_s, beta_a: [3][nl][nd]
  double *d_phase;          // [nl][nd][NTHETA]
  int *d_nlos_b;            // LOS points before the refinement
  int64_t *d_los_off_b;
  double *d_geo_b, *d_pts_b;
  int64_t max_seg_b;
  aero_t *h_aero;           // host copy for child batches

  // Scattering (depth > 0): the scattering order of this batch's rays
  // (ctl->sca_mult for the caller's batch, one less for each generation of
  // secondary pencils), the secondary pencils per point and their zenith
  // angles, the scattering points and their source, and the child batches
  // that run the secondary and the solar pencils.
  int depth, nalpha;
  double alpha[32];
  int nalpha_at[JSC_MAX_DEPTH + 1];  // per-depth pencil counts (0: inherit nalpha)
  int *d_nsp;               // [max_rays]
  int64_t *d_sp_off;        // [max_rays+1]
  double *d_sp;             // [max_sp][JSC_SP_REC]
  int *d_sp_atm;            // [max_sp]
  double *d_src;            // [max_sp][nd]
  int64_t max_sp, n_sp;
  double *d_theta2;         // [n_theta2] solar scattering angles
  int n_theta2;
  double *d_planck_sun;     // [nd]
  jsc_batch *child, *sun_child;
  ctl_t *ctl;               // copy for child batches

  // Scattering-source surrogate (caller's batch only): the network, the
  // relative tolerance of the sampled check and its stride, per-point
  // features and marks, the plain-path subset, and the last run's counts.
  struct jsc_surrogate *sur;
  int sur_on, sur_stride;
  float sur_tol;
  // surrogates for the points of other scattering orders (descendants)
  struct jsc_surrogate *sur_at[JSC_MAX_DEPTH + 1];
  float sur_tol_at[JSC_MAX_DEPTH + 1];
  int sur_stride_at[JSC_MAX_DEPTH + 1];
  int64_t sur_cap;
  float *d_feat;
  int *d_mark, *d_idx, *d_atm_sub;
  double *d_sp_sub, *d_src_sub;
  int64_t sur_points, sur_fallback, sur_checked, sur_rejected;
  float sur_maxerr;
  double sur_errsum;            // checked deviations summed over (point, channel) pairs
  int64_t sur_errn;             // ... and their number
  int inner;                    // secondary-pencil batch of a deeper recursion
  int sur_runs, sur_used_runs;  // chunks of the last run with points / from the surrogate

  // Fixed-capacity mode (no host read-backs; graph capture) and the
  // captured upload + run + download graph.  With scattering (depth 1):
  // the scattering-point capacity and the points per round of secondary
  // pencils (fx_max_sp = fx_rounds * fx_chunk).
  int fixed;
  int64_t fx_points_req;    // requested point capacity (0: max_rays * JSC_FIXED_POINTS_PER_RAY)
  int64_t fx_max_sp, fx_chunk;
  int fx_rounds;
  unsigned long long *d_sp_listed;  // points listed by the last fixed-capacity run
  // Pencil batches of a fixed-capacity round: their rays form a device work
  // queue (live count and head on the device) pulled by persistent tracing.
  int *d_live;
  unsigned *d_qhead;
  unsigned *h_status;       // pinned: status word of the last asynchronous download
  cudaGraphExec_t gexec;
  jsc_batch_input gin;      // host inputs the graph copies from
  int graph_ready, graph_kernels;

  // Line of sight.
  int *d_nlos;
  int64_t *d_los_off;       // [max_rays+1]
  double *d_geo;            // [max_seg][4]: z lon lat raw-ds
  double *d_pts;            // [max_seg][W]: p t ds qh2o k[nw] u[ng]
  double *d_ctm, *d_srcp;   // [max_seg][nd]: continuum extinction, Planck source
  int64_t n_points;         // LOS points of the current run
  double *d_tsurf;          // [max_rays]
  double *d_tp;             // [3][max_rays]
  unsigned long long *d_rkeys;  // [2][max_rays] ray sort keys (ray-tile EGA variants)
  int *d_rorder;                // [2][max_rays] ray order of the tiles
  void *d_rtmp;                 // sort scratch
  size_t rtmp_bytes;

  // Outputs and status.
  double *d_rad, *d_tau;    // [max_rays][nd]
  unsigned *d_status;
  unsigned long long *d_counters;  // [0] LOS points, [1] EGA evaluations
  int64_t *h_total;         // pinned: LOS points of the current batch

  // Multi-block prefix scans: ticket (word 0) and one flag word per tile,
  // and the polls a device wait may spend before it gives up.
  unsigned long long *d_scan;
  int scan_tiles;
  unsigned wait_budget;

  unsigned long long *d_digest;  // [max_rays][nd] when index digests are on
  int digest;
  int timing;
  int ega_variant;          // launch variant of ega_rt (autotuned), -1 = default
  EgaArgs last_ega;         // arguments of the last ega_rt launch
  float ega_variant_ms[32];  // autotuner timings (room for every variant)
  cudaEvent_t ev[2 * JSC_T_N];
  int ran[JSC_T_N];
};
