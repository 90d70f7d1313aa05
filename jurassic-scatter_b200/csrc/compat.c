/*
 * The non-hot helpers of the reference's forwardmodel.h that work on its
 * host-side structs: read_tbl, srcfunc_planck, formod_continua, intpol_tbl,
 * intpol_tbl_eps, intpol_tbl_u, locate_tbl.  They exist so that a program
 * or object written against forwardmodel.h links this library in place of
 * forwardmodel.o and gets the same answers from them.  The caller's tbl_t
 * (about 12.5 GB) and los_t live in host memory, so these run on the host;
 * the GPU forward model (formod, formod_pencil, the jsc_* batches) never
 * calls them.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "jsc_internal.h"

/* ------------------------------------------------------------ read_tbl -- */

static int read_tbl_impl(ctl_t *ctl, tbl_t *tbl) {
  jsc_host_tables ht;
  int st = jsc_read_tables(ctl, &ht);
  for (int id = 0; id < ctl->nd && !st; id++)
    for (int ig = 0; ig < ctl->ng; ig++) {
      const jsc_host_table *tb = &ht.tab[id * ctl->ng + ig];
      tbl->np[ig][id] = tb->np;
      for (int ip = 0; ip < tb->np; ip++) {
        tbl->p[ig][id][ip] = tb->p[ip];
        tbl->nt[ig][id][ip] = tb->nt[ip];
        for (int it = 0; it < tb->nt[ip]; it++) {
          const int n = tb->nu[ip][it];
          tbl->t[ig][id][ip][it] = tb->t[ip][it];
          tbl->nu[ig][id][ip][it] = n;
          memcpy(tbl->u[ig][id][ip][it], ht.u + tb->off[ip][it], (size_t)n * sizeof(float));
          memcpy(tbl->eps[ig][id][ip][it], ht.eps + tb->off[ip][it], (size_t)n * sizeof(float));
        }
      }
    }
  free(ht.tab);
  free(ht.u);
  free(ht.eps);
  return st;
}

void read_tbl(ctl_t *ctl, tbl_t *tbl) { jsc_finish_call(read_tbl_impl(ctl, tbl), "read_tbl"); }

/* ------------------------------------------------------ srcfunc_planck -- */

/* Planck tables of the last channel set asked for (tblbase and
 * wavenumbers), rebuilt when it changes. */
static pthread_mutex_t g_planck_lock = PTHREAD_MUTEX_INITIALIZER;
static jsc_host_model g_planck;
static char g_planck_base[LEN];
static double g_planck_nu[NDMAX];

static int planck_impl(ctl_t *ctl, double t, double *src) {
  int st = JSC_OK;
  pthread_mutex_lock(&g_planck_lock);
  int same = g_planck.planck_b && g_planck.nd == ctl->nd && !strcmp(g_planck_base, ctl->tblbase);
  for (int id = 0; same && id < ctl->nd; id++) same = g_planck_nu[id] == ctl->nu[id];
  if (!same) {
    jsc_host_model_free(&g_planck);
    st = jsc_planck_only(ctl, &g_planck);
    if (!st) {
      snprintf(g_planck_base, LEN, "%s", ctl->tblbase);
      memcpy(g_planck_nu, ctl->nu, (size_t)ctl->nd * sizeof(double));
    } else {
      jsc_host_model_free(&g_planck);
    }
  }
  if (!st) {
    /* locate() on the uniform temperature grid, then LIN (src/forwardmodel.c:788-793) */
    double temp[JSC_NPLANCK];
    for (int i = 0; i < JSC_NPLANCK; i++)
      temp[i] = jsc_lin(0.0, JSC_PLANCK_TMIN, JSC_NPLANCK - 1.0, JSC_PLANCK_TMAX, (double)i);
    const int it = jsc_locate(temp, JSC_NPLANCK, t);
    for (int id = 0; id < ctl->nd; id++) {
      const double *b = g_planck.planck_b + (size_t)id * JSC_NPLANCK;
      src[id] = jsc_lin(temp[it], b[it], temp[it + 1], b[it + 1], t);
    }
  }
  pthread_mutex_unlock(&g_planck_lock);
  return st;
}

void srcfunc_planck(ctl_t *ctl, double t, double *src) {
  jsc_finish_call(planck_impl(ctl, t, src), "srcfunc_planck");
}

/* ----------------------------------------------------- formod_continua -- */

void formod_continua(ctl_t *ctl, los_t *los, int ip, double *beta) {
  const int ig_co2 = jsc_find_emitter(ctl, "CO2"), ig_h2o = jsc_find_emitter(ctl, "H2O");
  const double qh2o = ig_h2o >= 0 ? los->q[ip][ig_h2o] : 0.0;
  for (int id = 0; id < ctl->nd; id++) {
    jsc_ctm_coef c;
    jsc_ctm_coefficients(ctl, &c, id);
    beta[id] = jsc_continuum(&c, ig_co2, ig_h2o, ctl->ctm_co2, ctl->ctm_h2o, ctl->ctm_n2,
                             ctl->ctm_o2, ctl->nu[id], los->k[ip][ctl->window[id]], los->p[ip],
                             los->t[ip], los->ds[ip], qh2o, los->u[ip]);
  }
}

/* ---------------------------------------------------------- intpol_tbl -- */

int locate_tbl(float *xx, int n, double x) {
  int lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    const int mid = (lo + hi) >> 1;
    if (xx[mid] > x) hi = mid;
    else lo = mid;
  }
  return lo;
}

/* LIN on float table entries: the slope is a float expression, promoted to
 * double when it meets the double abscissa. */
static double lin_float(float x0, float y0, float x1, float y1, double x) {
  const float slope = (y1 - y0) / (x1 - x0);
  return y0 + slope * (x - x0);
}

double intpol_tbl_eps(tbl_t *tbl, int ig, int id, int ip, int it, double u) {
  const float *x = tbl->u[ig][id][ip][it], *y = tbl->eps[ig][id][ip][it];
  const int i = locate_tbl((float *)x, tbl->nu[ig][id][ip][it], u);
  return lin_float(x[i], y[i], x[i + 1], y[i + 1], u);
}

double intpol_tbl_u(tbl_t *tbl, int ig, int id, int ip, int it, double eps) {
  const float *x = tbl->eps[ig][id][ip][it], *y = tbl->u[ig][id][ip][it];
  const int i = locate_tbl((float *)x, tbl->nu[ig][id][ip][it], eps);
  return lin_float(x[i], y[i], x[i + 1], y[i + 1], eps);
}

/* Emissivity of the extended path at table node (ig, id, ip, it): the path
 * emissivity x1 turned into a column density on the row, the segment's
 * column added, looked up again, clamped to [0, 1]. */
static double node_eps(tbl_t *tbl, int ig, int id, int ip, int it, double x1, double useg) {
  const double u = intpol_tbl_u(tbl, ig, id, ip, it, x1);
  return jsc_clamp01(intpol_tbl_eps(tbl, ig, id, ip, it, u + useg));
}

void intpol_tbl(ctl_t *ctl, tbl_t *tbl, los_t *los, int ip, double tau_path[NGMAX][NDMAX],
                double tau_seg[NDMAX]) {
  if (ip <= 0)
    for (int ig = 0; ig < ctl->ng; ig++)
      for (int id = 0; id < ctl->nd; id++) tau_path[ig][id] = 1;
  const double P = los->p[ip], T = los->t[ip];
  for (int id = 0; id < ctl->nd; id++) {
    tau_seg[id] = 1;
    for (int ig = 0; ig < ctl->ng; ig++) {
      double eps = 0;
      const int np = tbl->np[ig][id];
      if (np >= 2 && tau_path[ig][id] < 1e-9) {
        eps = 1;
      } else if (np >= 2) {
        const int ipr = jsc_locate(tbl->p[ig][id], np, P);
        const int *nt = tbl->nt[ig][id];
        const int it0 = jsc_locate(tbl->t[ig][id][ipr], nt[ipr], T);
        const int it1 = jsc_locate(tbl->t[ig][id][ipr + 1], nt[ipr + 1], T);
        const int(*nu)[TBLNTMAX] = tbl->nu[ig][id];
        if (nt[ipr] >= 2 && nt[ipr + 1] >= 2 && nu[ipr][it0] >= 2 && nu[ipr][it0 + 1] >= 2 &&
            nu[ipr + 1][it1] >= 2 && nu[ipr + 1][it1 + 1] >= 2) {
          const double x1 = 1 - tau_path[ig][id], useg = los->u[ip][ig];
          const double e00 = node_eps(tbl, ig, id, ipr, it0, x1, useg);
          const double e01 = node_eps(tbl, ig, id, ipr, it0 + 1, x1, useg);
          const double e10 = node_eps(tbl, ig, id, ipr + 1, it1, x1, useg);
          const double e11 = node_eps(tbl, ig, id, ipr + 1, it1 + 1, x1, useg);
          const double *t0 = tbl->t[ig][id][ipr], *t1 = tbl->t[ig][id][ipr + 1];
          const double ea = jsc_clamp01(jsc_lin(t0[it0], e00, t0[it0 + 1], e01, T));
          const double eb = jsc_clamp01(jsc_lin(t1[it1], e10, t1[it1 + 1], e11, T));
          const double e = jsc_clamp01(
              jsc_lin(tbl->p[ig][id][ipr], ea, tbl->p[ig][id][ipr + 1], eb, P));
          eps = 1 - (1 - e) / tau_path[ig][id];
        }
      }
      tau_path[ig][id] *= (1 - eps);
      tau_seg[id] *= (1 - eps);
    }
  }
}
