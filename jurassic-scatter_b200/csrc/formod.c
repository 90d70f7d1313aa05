/*
 * Drop-in forward model: formod(), brightness() and the plumbing between the
 * reference's structs and the batch C-ABI.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "jsc_internal.h"
#include "physics.h"

/* Aerosol optical properties for RETNN/RETRR/RETSS retrievals come from the
 * program's own get_opt_prop (the reference's scatter.o) when it is linked. */
extern void get_opt_prop(ctl_t *ctl, aero_t *aero) __attribute__((weak));

static int g_exit_on_error = 1;
static __thread int g_last_status = JSC_OK;
static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;

/* Cached model and batch, rebuilt when the table set or switches change. */
static jsc_model *g_model;
static jsc_batch *g_batch;
static ctl_t *g_key;          /* ctl the cache was built for */

void jsc_set_exit_on_error(int on) { g_exit_on_error = on; }
int jsc_last_status(void) { return g_last_status; }

double brightness(double rad, double nu) {
  return JSC_C2 * nu / jsc_gsl_log1p(JSC_C1 * (nu * nu * nu) / rad);
}

static int same_tables(const ctl_t *a, const ctl_t *b) {
  if (a->ng != b->ng || a->nd != b->nd || a->nw != b->nw) return 0;
  if (strcmp(a->tblbase, b->tblbase)) return 0;
  for (int ig = 0; ig < a->ng; ig++)
    if (strcmp(a->emitter[ig], b->emitter[ig])) return 0;
  for (int id = 0; id < a->nd; id++)
    if (a->nu[id] != b->nu[id] || a->window[id] != b->window[id]) return 0;
  return 1;
}

static int same_switches(const ctl_t *a, const ctl_t *b) {
  return a->ctm_co2 == b->ctm_co2 && a->ctm_h2o == b->ctm_h2o &&
         a->ctm_n2 == b->ctm_n2 && a->ctm_o2 == b->ctm_o2 &&
         a->refrac == b->refrac && a->rayds == b->rayds &&
         a->raydz == b->raydz && a->sca_n == b->sca_n &&
         a->sca_mult == b->sca_mult && a->ip == b->ip &&
         a->transs == b->transs && !strcmp(a->sca_ext, b->sca_ext);
}

static int device_from_env(void) {
  const char *s = getenv("JURASSIC_GPU_DEVICE");
  return s ? atoi(s) : 0;
}

/* Model and batch for this ctl; the batch never re-applies hydrostatic
 * balance because formod() does it on the host, in place, like the
 * reference. */
static int ensure_cache(const ctl_t *ctl) {
  int st;
  if (g_key && !same_tables(g_key, ctl)) {
    jsc_batch_destroy(g_batch);
    jsc_model_destroy(g_model);
    g_batch = NULL;
    g_model = NULL;
  }
  if (g_batch && g_key && !same_switches(g_key, ctl)) {
    jsc_batch_destroy(g_batch);
    g_batch = NULL;
  }
  if (!g_key) {
    g_key = (ctl_t *)malloc(sizeof(ctl_t));
    if (!g_key) return JSC_ERR_NOMEM;
  }
  memcpy(g_key, ctl, sizeof(ctl_t));
  if (!g_model && (st = jsc_model_create(ctl, device_from_env(), &g_model))) return st;
  if (!g_batch) {
    ctl_t c2;
    memcpy(&c2, ctl, sizeof(ctl_t));
    c2.hydz = -999;
    if ((st = jsc_batch_create(g_model, &c2, 1, NPMAX, NRMAX, 0, &g_batch))) return st;
  }
  return JSC_OK;
}

static int formod_impl(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero) {
  const int nd = ctl->nd, nr = obs->nr, np = atm->np, ng = ctl->ng, nw = ctl->nw;
  int st = JSC_OK;
  if (nd < 1 || nd > NDMAX || ng < 0 || ng > NGMAX || nw < 0 || nw > NWMAX ||
      nr < 0 || nr > NRMAX || np < 2 || np > NPMAX) {
    jsc_set_error(JSC_ERR_ARG, "formod: invalid sizes (nd=%d ng=%d nw=%d nr=%d np=%d)",
                  nd, ng, nw, nr, np);
    return JSC_ERR_ARG;
  }
  if (ctl->fov[0] != '-') {
    jsc_set_error(JSC_ERR_UNSUPPORTED, "field-of-view convolution (FOV=%s)", ctl->fov);
    return JSC_ERR_UNSUPPORTED;
  }
  if (ctl->sca_n > 0 && !aero) {
    jsc_set_error(JSC_ERR_ARG, "formod: SCA_N=%d needs the aerosol/cloud data", ctl->sca_n);
    return JSC_ERR_ARG;
  }

  /* Observation mask (src/forwardmodel.c:25-28). */
  unsigned char *mask = (unsigned char *)malloc((size_t)nd * (nr > 0 ? nr : 1));
  double *buf = NULL;
  if (!mask) return JSC_ERR_NOMEM;
  for (int id = 0; id < nd; id++)
    for (int ir = 0; ir < nr; ir++) mask[(size_t)id * nr + ir] = !isfinite(obs->rad[id][ir]);

  /* Hydrostatic balance on the caller's atmosphere (src/atmosphere.c:163). */
  {
    const int ig_h2o = jsc_find_emitter(ctl, "H2O");
    jsc_hydrostatic(ctl->hydz, np, atm->z, atm->lon, atm->lat, atm->t,
                    ig_h2o >= 0 ? atm->q[ig_h2o] : NULL, atm->p);
  }

  /* Optical properties for aerosol retrievals (src/forwardmodel.c:34-36). */
  if (ctl->retnn || ctl->retrr || ctl->retss) {
    if (!get_opt_prop) {
      free(mask);
      jsc_set_error(JSC_ERR_UNSUPPORTED, "RETNN/RETRR/RETSS need get_opt_prop");
      return JSC_ERR_UNSUPPORTED;
    }
    get_opt_prop(ctl, aero);
  }

  pthread_mutex_lock(&g_lock);
  st = ensure_cache(ctl);
  if (!st && nr > 0) {
    /* Pack the atmosphere as one profile and the rays. */
    size_t nbuf = (size_t)np * (size_t)(ng + nw) + 2 * (size_t)nr * nd + 3 * (size_t)nr;
    buf = (double *)malloc(nbuf * sizeof(double));
    int *ray_atm = (int *)calloc((size_t)nr, sizeof(int));
    if (!buf || !ray_atm) {
      st = JSC_ERR_NOMEM;
    } else {
      double *q = buf, *k = q + (size_t)np * ng, *rad = k + (size_t)np * nw;
      double *tau = rad + (size_t)nr * nd, *tp = tau + (size_t)nr * nd;
      for (int ig = 0; ig < ng; ig++) memcpy(q + (size_t)ig * np, atm->q[ig], np * sizeof(double));
      for (int iw = 0; iw < nw; iw++) memcpy(k + (size_t)iw * np, atm->k[iw], np * sizeof(double));
      int off[2] = {0, np};
      jsc_batch_input in;
      memset(&in, 0, sizeof(in));
      in.n_atm = 1;
      in.n_levels = np;
      in.atm_off = off;
      in.z = atm->z;
      in.lon = atm->lon;
      in.lat = atm->lat;
      in.p = atm->p;
      in.t = atm->t;
      in.q = q;
      in.k = k;
      in.n_rays = nr;
      in.ray_atm = ray_atm;
      in.time = obs->time;
      in.obsz = obs->obsz;
      in.obslon = obs->obslon;
      in.obslat = obs->obslat;
      in.vpz = obs->vpz;
      in.vplon = obs->vplon;
      in.vplat = obs->vplat;
      jsc_batch_output out;
      memset(&out, 0, sizeof(out));
      out.rad = rad;
      out.tau = tau;
      out.tpz = tp;
      out.tplon = tp + nr;
      out.tplat = tp + 2 * nr;
      /* Aerosol/cloud layers and optical properties (read_aero +
       * get_opt_prop of the caller, or of this call for retrievals). */
      if (ctl->sca_n > 0) st = jsc_batch_set_aero(g_batch, aero);
      if (!st) st = jsc_batch_upload(g_batch, &in, NULL);
      if (!st) st = jsc_batch_run(g_batch, NULL);
      if (!st) st = jsc_batch_download(g_batch, &out, NULL);
      if (!st) {
        for (int ir = 0; ir < nr; ir++) {
          obs->tpz[ir] = tp[ir];
          obs->tplon[ir] = tp[nr + ir];
          obs->tplat[ir] = tp[2 * nr + ir];
          for (int id = 0; id < nd; id++) {
            obs->rad[id][ir] = rad[(size_t)ir * nd + id];
            obs->tau[id][ir] = tau[(size_t)ir * nd + id];
          }
        }
      }
    }
    free(ray_atm);
  }
  pthread_mutex_unlock(&g_lock);
  free(buf);

  if (!st) {
    /* Brightness temperature (src/forwardmodel.c:106-109). */
    if (ctl->write_bbt)
      for (int ir = 0; ir < nr; ir++)
        for (int id = 0; id < nd; id++)
          obs->rad[id][ir] = brightness(obs->rad[id][ir], ctl->nu[id]);
    /* Re-apply the mask (src/forwardmodel.c:112-115). */
    for (int id = 0; id < nd; id++)
      for (int ir = 0; ir < nr; ir++)
        if (mask[(size_t)id * nr + ir]) obs->rad[id][ir] = NAN;
  }
  free(mask);
  return st;
}

void formod(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero) {
  int st = formod_impl(ctl, atm, obs, aero);
  g_last_status = st;
  if (st && g_exit_on_error) {
    printf("\nError (%s, %s, l%d): %s: %s\n\n", __FILE__, __func__, __LINE__,
           jsc_status_string(st), jsc_last_error_message());
    exit(EXIT_FAILURE);
  }
}

/* Release the cached model and batch (tests and long-running hosts). */
void jsc_release_cache(void) {
  pthread_mutex_lock(&g_lock);
  jsc_batch_destroy(g_batch);
  jsc_model_destroy(g_model);
  g_batch = NULL;
  g_model = NULL;
  free(g_key);
  g_key = NULL;
  pthread_mutex_unlock(&g_lock);
}
