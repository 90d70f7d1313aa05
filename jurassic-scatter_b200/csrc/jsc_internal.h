/*
 * Internal interface between the C host code (tables, filters, continua,
 * formod drop-in) and the CUDA layer (model upload, kernels, batches).
 * Not installed; the public interface is include/jurassic_b200.h.
 */
#ifndef JSC_INTERNAL_H
#define JSC_INTERNAL_H

#include <math.h>

#include "jurassic_b200.h"

#ifdef __CUDACC__
#define JSC_HD __host__ __device__ __forceinline__
#define JSC_ALIGN(n) __align__(n)
#else
#define JSC_HD static inline
#define JSC_ALIGN(n) __attribute__((aligned(n)))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Planck source table: 1201 temperatures from 100 K to 400 K in 0.25 K
 * steps (src/forwardmodel.c:747-784). */
#define JSC_NPLANCK 1201
#define JSC_PLANCK_TMIN 100.0
#define JSC_PLANCK_TMAX 400.0

/* ------------------------------------------------------------------------
 * Small numerical helpers shared by host and device.  They keep the exact
 * operation order of the reference macros, so results agree bit for bit
 * when no FMA contraction is applied (device code is built --fmad=false).
 * ------------------------------------------------------------------------ */

/* LIN macro of src/jurassic.h:72-73. */
JSC_HD double jsc_lin(double x0, double y0, double x1, double y1, double x) {
  return y0 + (y1 - y0) / (x1 - x0) * (x - x0);
}

/* GSL_MAX(GSL_MIN(x, 1), 0) with GSL's ternary semantics (NaN -> 1). */
JSC_HD double jsc_clamp01(double x) {
  double m = (x < 1.0 ? x : 1.0);
  return (m > 0.0 ? m : 0.0);
}

/* Bisection of src/misc.c:237-265 on an ascending or descending double
 * array; n >= 2 (n < 2 returns 0 without reading). */
JSC_HD int jsc_locate(const double *xx, int n, double x) {
  int ilo = 0, ihi = n - 1, i;
  if (n < 2) return 0;
  i = (ihi + ilo) >> 1;
  if (xx[i] < xx[i + 1]) {
    while (ihi > ilo + 1) {
      i = (ihi + ilo) >> 1;
      if (xx[i] > x) ihi = i; else ilo = i;
    }
  } else {
    while (ihi > ilo + 1) {
      i = (ihi + ilo) >> 1;
      if (xx[i] <= x) ihi = i; else ilo = i;
    }
  }
  return ilo;
}

/* ------------------------------------------------------------------------
 * Host staging of the emissivity tables (what read_tbl produces, but only
 * for the tables that exist, in compact arrays).
 * ------------------------------------------------------------------------ */
typedef struct {
  int np;                                  /* pressure levels, < 2: no table */
  double p[TBLNPMAX];
  int nt[TBLNPMAX];
  double t[TBLNPMAX][TBLNTMAX];
  int nu[TBLNPMAX][TBLNTMAX];              /* points per (p, T) row */
  int64_t off[TBLNPMAX][TBLNTMAX];         /* first point in u[]/eps[] */
} jsc_host_table;

typedef struct {
  int ng, nd;
  jsc_host_table *tab;                     /* [nd][ng] (index id*ng+ig) */
  float *u, *eps;                          /* all rows back to back */
  int64_t n_points, cap_points;
} jsc_host_tables;

/* Per-channel continuum coefficients (ctmco2/ctmh2o/ctmn2/ctmo2 of
 * src/continua.c with the wavenumber interpolation done once per channel). */
typedef struct {
  int co2_on;      /* CO2 continuum active for this channel */
  double co2_c230, co2_c260, co2_c296;
  int h2o_on;
  double h2o_self296;   /* sfac * cw296 */
  double h2o_ratio;     /* cw260 / cw296 */
  double h2o_frn;       /* cwfrn * fscal */
  int n2_on;
  double n2_b, n2_beta;
  int o2_on;
  double o2_b, o2_beta;
} jsc_ctm_coef;

/* Continuum extinction of one channel at one LOS point
 * (src/forwardmodel.c:120-152 with src/continua.c:5-2049): the window
 * extinction kwin, the CO2 and H2O continua over the segment's columns u
 * (per emitter; emitter indices ig_co2/ig_h2o, -1 when absent) divided by
 * the segment length DS, and the N2 and O2 collision-induced bands; c holds
 * the channel's coefficients (jsc_ctm_coefficients), ctm_* the CTM_*
 * switches.  Shared by the GPU kernels and the host helper formod_continua. */
JSC_HD double jsc_continuum(const jsc_ctm_coef *c, int ig_co2, int ig_h2o, int ctm_co2,
                            int ctm_h2o, int ctm_n2, int ctm_o2, double nu, double kwin,
                            double P, double T, double DS, double qh2o, const double *u) {
  double beta = kwin;
  if (ctm_co2) {
    double ctm = 0;
    if (ig_co2 >= 0 && c->co2_on) {
      const double dt230 = T - 230, dt260 = T - 260, dt296 = T - 296;
      const double ctw = dt260 * 5.050505e-4 * dt296 * c->co2_c230 -
                         dt230 * 9.259259e-4 * dt296 * c->co2_c260 +
                         dt230 * 4.208754e-4 * dt260 * c->co2_c296;
      ctm = u[ig_co2] / JSC_AVOGADRO / 1000 * P / JSC_P0 * ctw;
    }
    beta += ctm / DS;
  }
  if (ctm_h2o) {
    double ctm = 0;
    if (ig_h2o >= 0 && c->h2o_on) {
      const double ctwslf = c->h2o_self296 * pow(c->h2o_ratio, (296 - T) / (296 - 260));
      const double a1 = nu * u[ig_h2o] * tanh(.7193876 / T * nu);
      const double a2 = 296 / T;
      const double a3 = P / JSC_P0 * (qh2o * ctwslf + (1 - qh2o) * c->h2o_frn) * 1e-20;
      ctm = a1 * a2 * a3;
    }
    beta += ctm / DS;
  }
  if (ctm_n2 && c->n2_on) {
    const double t0 = 273, tr = 296, q_n2 = 0.79;
    const double pp = P / JSC_P0, tt = t0 / T;
    beta += 0.1 * (pp * pp) * (tt * tt) * q_n2 * c->n2_b *
            exp(c->n2_beta * (1 / tr - 1 / T)) *
            (q_n2 + (1 - q_n2) * (1.294 - 0.4545 * T / tr));
  }
  if (ctm_o2 && c->o2_on) {
    const double t0 = 273, tr = 296, q_o2 = 0.21;
    const double pp = P / JSC_P0, tt = t0 / T;
    beta += 0.1 * (pp * pp) * (tt * tt) * q_o2 * c->o2_b *
            exp(c->o2_beta * (1 / tr - 1 / T));
  }
  return beta;
}

/* Everything the host reads or derives before upload. */
typedef struct {
  int ng, nd, nw;
  double nu[NDMAX];
  int window[NDMAX];
  int ig_co2, ig_h2o;          /* emitter indices, -1 when absent */
  int ctm_co2, ctm_h2o, ctm_n2, ctm_o2;
  jsc_host_tables tables;
  double *planck_b;            /* [nd][JSC_NPLANCK] */
  double *planck_s;            /* [nd][JSC_NPLANCK] slope to the next node */
  jsc_ctm_coef ctm[NDMAX];
} jsc_host_model;

/* Readers and derived data (model_host.c).  Return JSC_* status. */
int jsc_host_model_load(const ctl_t *ctl, jsc_host_model *hm);
void jsc_host_model_free(jsc_host_model *hm);
int jsc_read_filter(const char *filename, double *nu, double *f, int *n);
int jsc_read_tables(const ctl_t *ctl, jsc_host_tables *ht);
int jsc_planck_only(const ctl_t *ctl, jsc_host_model *hm);
void jsc_ctm_coefficients(const ctl_t *ctl, jsc_ctm_coef *c, int id);
double jsc_gsl_expm1(double x);
double jsc_gsl_log1p(double x);
int jsc_find_emitter(const ctl_t *ctl, const char *name);

/* Error reporting shared by C and CUDA parts. */
void jsc_set_error(int status, const char *fmt, ...);
/* End of a drop-in call (formod.c): records the status, and prints and
 * exits like the reference's ERRMSG unless jsc_set_exit_on_error(0). */
int jsc_finish_call(int st, const char *func);

/* Mie efficiencies and phase functions of n (size parameter, refractive
 * index) tasks on GPU `device` (mie.cu): out[i][0] = Q_ext,
 * out[i][1] = Q_sca, out[i][2 + j] = phase function at j degrees. */
int jsc_mie_eval(int device, int n, const double *x, const double *nr, const double *ni,
                 double *out);

/* ------------------------------------------------------------------------
 * Device layout of a model (device pointers; passed by value to kernels).
 * ------------------------------------------------------------------------ */

/* One point k of an emissivity-table row: column density and emissivity
 * as the table stores them (float).  The reference's LIN on float table
 * entries evaluates the slope (y1-y0)/(x1-x0) in single precision
 * (src/forwardmodel.c:519-541 with the LIN macro of src/jurassic.h:72);
 * the kernels compute it from the two nodes of an interval with the same
 * IEEE single-precision operations. */
typedef struct JSC_ALIGN(8) {
  float u, e;
} jsc_node;

/* Row descriptor: first node of the row and n | flags << 16, where n is
 * the number of points of the row. */
typedef struct JSC_ALIGN(8) {
  int off;
  int nf;
} jsc_row;

/* Row descriptor flags. */
#define JSC_ROW_STRICT 1   /* u and eps strictly increasing */

typedef struct {
  int ng, nd, nw;
  int ig_co2, ig_h2o;
  int n_grid;
  /* (p, T) grids shared by tables; grid g occupies
   * p[g*TBLNPMAX], nt[g*TBLNPMAX], t[(g*TBLNPMAX+ip)*TBLNTMAX+it]. */
  const int *grid_np;
  const double *grid_p;
  const int *grid_nt;
  const double *grid_t;
  const int *tab_grid;       /* [nd*ng] grid id, -1: table unusable (np<2) */
  const jsc_row *rows;       /* [TBLNPMAX][TBLNTMAX][ng][nd] */
  const jsc_node *nodes;
  const double *planck_b, *planck_s;   /* [nd][JSC_NPLANCK] */
  const jsc_ctm_coef *ctm;             /* [nd] */
  const double *nu;                    /* [nd] */
  const int *window;                   /* [nd] */
} jsc_dev_model;

#ifdef __cplusplus
}
#endif

#endif /* JSC_INTERNAL_H */
