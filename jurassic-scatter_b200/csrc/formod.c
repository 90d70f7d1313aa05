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

static int g_exit_on_error = 1;
static __thread int g_last_status = JSC_OK;
static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;

/* Cached model and batch, rebuilt when the table set or switches change. */
static jsc_model *g_model;
static jsc_batch *g_batch;
static ctl_t *g_key;          /* ctl the cache was built for */
/* Batch of formod_pencil (one ray; its scattering order in sca_mult). */
static jsc_batch *g_pbatch;
static ctl_t *g_pkey;
/* Batch of jsc_kernel (undisturbed + disturbed profiles) and its capacity. */
static jsc_batch *g_jbatch;
static int g_jcap_atm, g_jcap_lev, g_jcap_rays;

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
         a->sca_mult == b->sca_mult && a->ip == b->ip && a->cz == b->cz && a->cx == b->cx &&
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
    jsc_batch_destroy(g_jbatch);
    jsc_batch_destroy(g_pbatch);
    jsc_model_destroy(g_model);
    g_batch = NULL;
    g_jbatch = NULL;
    g_pbatch = NULL;
    g_model = NULL;
  }
  if (g_key && !same_switches(g_key, ctl)) {
    jsc_batch_destroy(g_batch);
    jsc_batch_destroy(g_jbatch);
    g_batch = NULL;
    g_jbatch = NULL;
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
    /* up to NPMAX / 2 profiles: an IP=2 atmosphere of two-level profiles */
    if ((st = jsc_batch_create(g_model, &c2, NPMAX / 2, NPMAX, NRMAX, 0, &g_batch))) return st;
  }
  return JSC_OK;
}

/* Field-of-view shape of the last FOV file read (read_shape,
 * src/forwardmodel.c:577-606): offsets dz [km] and weights. */
static pthread_mutex_t g_fov_lock = PTHREAD_MUTEX_INITIALIZER;
static char g_fov_file[LEN];
static double g_fov_dz[NSHAPE + 1], g_fov_w[NSHAPE + 1];
static int g_fov_n;

static int fov_shape(const char *file) {
  if (g_fov_n > 0 && !strcmp(g_fov_file, file)) return JSC_OK;
  FILE *in = fopen(file, "r");
  if (!in) {
    jsc_set_error(JSC_ERR_FILE, "cannot open field-of-view file %s", file);
    return JSC_ERR_FILE;
  }
  char *line = (char *)malloc(LEN);
  int n = 0, st = JSC_OK;
  if (!line) st = JSC_ERR_NOMEM;
  while (!st && fgets(line, LEN, in))
    if (sscanf(line, "%lg %lg", &g_fov_dz[n], &g_fov_w[n]) == 2)
      if (++n > NSHAPE) {
        jsc_set_error(JSC_ERR_ARG, "too many points in %s", file);
        st = JSC_ERR_ARG;
      }
  fclose(in);
  free(line);
  if (!st && n < 1) {
    jsc_set_error(JSC_ERR_FILE, "could not read any data from %s", file);
    st = JSC_ERR_FILE;
  }
  g_fov_n = st ? 0 : n;
  if (!st) snprintf(g_fov_file, LEN, "%s", file);
  return st;
}

/* Field-of-view convolution of the pencil-beam results (formod_fov,
 * src/forwardmodel.c:156-220): per ray, the radiance and transmittance
 * profiles over tangent height of the up to NFOV rays on either side with
 * the same observation time, interpolated at tangent height + dz of every
 * shape point and averaged with the shape's weights. */
static int fov_convolve(const ctl_t *ctl, obs_t *obs) {
  pthread_mutex_lock(&g_fov_lock);
  int st = fov_shape(ctl->fov);
  const int nd = ctl->nd, nr = obs->nr, nf = 2 * NFOV + 1;
  double *rad = NULL, *tau = NULL, *buf = NULL;
  if (!st) {
    rad = (double *)malloc(2 * (size_t)nd * nr * sizeof(double) + 1);
    buf = (double *)malloc((size_t)nf * (2 * nd + 1) * sizeof(double));
    if (!rad || !buf) st = JSC_ERR_NOMEM;
  }
  if (!st) {
    tau = rad + (size_t)nd * nr;
    /* the profiles come from the unconvolved results */
    for (int id = 0; id < nd; id++) {
      memcpy(rad + (size_t)id * nr, obs->rad[id], nr * sizeof(double));
      memcpy(tau + (size_t)id * nr, obs->tau[id], nr * sizeof(double));
    }
    double *z = buf, *pr = z + nf, *pt = pr + (size_t)nd * nf;
    for (int ir = 0; ir < nr && !st; ir++) {
      int nz = 0;
      const int lo = ir - NFOV > 0 ? ir - NFOV : 0, hi = ir + 1 + NFOV < nr ? ir + 1 + NFOV : nr;
      for (int ir2 = lo; ir2 < hi; ir2++)
        if (obs->time[ir2] == obs->time[ir]) {
          z[nz] = obs->tpz[ir2];
          for (int id = 0; id < nd; id++) {
            pr[(size_t)id * nf + nz] = rad[(size_t)id * nr + ir2];
            pt[(size_t)id * nf + nz] = tau[(size_t)id * nr + ir2];
          }
          nz++;
        }
      if (nz < 2) {
        jsc_set_error(JSC_ERR_ARG, "cannot apply FOV convolution to ray %d", ir);
        st = JSC_ERR_ARG;
        break;
      }
      double wsum = 0;
      for (int id = 0; id < nd; id++) obs->rad[id][ir] = obs->tau[id][ir] = 0;
      for (int i = 0; i < g_fov_n; i++) {
        const double zf = obs->tpz[ir] + g_fov_dz[i];
        const int k = jsc_locate(z, nz, zf);
        for (int id = 0; id < nd; id++) {
          const double *r = pr + (size_t)id * nf, *t = pt + (size_t)id * nf;
          obs->rad[id][ir] += g_fov_w[i] * jsc_lin(z[k], r[k], z[k + 1], r[k + 1], zf);
          obs->tau[id][ir] += g_fov_w[i] * jsc_lin(z[k], t[k], z[k + 1], t[k + 1], zf);
        }
        wsum += g_fov_w[i];
      }
      for (int id = 0; id < nd; id++) {
        obs->rad[id][ir] /= wsum;
        obs->tau[id][ir] /= wsum;
      }
    }
  }
  pthread_mutex_unlock(&g_fov_lock);
  free(rad);
  free(buf);
  return st;
}

/* Host arrays of one packed batch input; they must live until the stream
 * has passed the upload. */
typedef struct {
  double *buf;   /* q [ng][np], k [nw][np], then room for rad, tau, tp of nr rays */
  int *ray_atm;
  int *off;
} packed_t;

static void packed_free(packed_t *pk) {
  free(pk->buf);
  free(pk->ray_atm);
  free(pk->off);
  memset(pk, 0, sizeof(*pk));
}

/* Pack atm and rays [r0, r0 + nr) of obs as the input of batch b and upload
 * it (the aerosol layers first when ctl->sca_n > 0): one profile (IP 1 and
 * IP 3, whose points are weighted one by one) or, for IP 2, a new profile
 * wherever lon/lat change, as intpol_atm_2d groups them
 * (src/atmosphere.c:343-356). */
static int upload_atm(jsc_batch *b, const ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero,
                      int r0, int nr, packed_t *pk) {
  const int nd = ctl->nd, np = atm->np, ng = ctl->ng, nw = ctl->nw;
  size_t nbuf = (size_t)np * (size_t)(ng + nw) + 2 * (size_t)nr * nd + 3 * (size_t)nr + 1;
  memset(pk, 0, sizeof(*pk));
  pk->buf = (double *)malloc(nbuf * sizeof(double));
  pk->ray_atm = (int *)calloc((size_t)nr + 1, sizeof(int));
  pk->off = (int *)malloc(((size_t)np + 1) * sizeof(int));
  if (!pk->buf || !pk->ray_atm || !pk->off) {
    packed_free(pk);
    return JSC_ERR_NOMEM;
  }
  double *q = pk->buf, *k = q + (size_t)np * ng;
  int *off = pk->off, n_atm = 1;
  for (int ig = 0; ig < ng; ig++) memcpy(q + (size_t)ig * np, atm->q[ig], np * sizeof(double));
  for (int iw = 0; iw < nw; iw++) memcpy(k + (size_t)iw * np, atm->k[iw], np * sizeof(double));
  off[0] = 0;
  if (ctl->ip == 2)
    for (int ip = 1; ip < np; ip++)
      if (atm->lon[ip] != atm->lon[ip - 1] || atm->lat[ip] != atm->lat[ip - 1])
        off[n_atm++] = ip;
  off[n_atm] = np;
  jsc_batch_input in;
  memset(&in, 0, sizeof(in));
  in.n_atm = n_atm;
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
  in.ray_atm = pk->ray_atm;
  in.time = obs->time + r0;
  in.obsz = obs->obsz + r0;
  in.obslon = obs->obslon + r0;
  in.obslat = obs->obslat + r0;
  in.vpz = obs->vpz + r0;
  in.vplon = obs->vplon + r0;
  in.vplat = obs->vplat + r0;
  /* Aerosol/cloud layers and optical properties (read_aero +
   * get_opt_prop of the caller, or of this call for retrievals). */
  int st = JSC_OK;
  if (ctl->sca_n > 0) st = jsc_batch_set_aero(b, aero);
  if (!st) st = jsc_batch_upload(b, &in, NULL);
  return st;
}

/* Run rays [r0, r0 + nr) of obs through atm on batch b (held under g_lock)
 * and write their radiances, transmittances and tangent points into obs. */
static int run_rays(jsc_batch *b, const ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero,
                    int r0, int nr) {
  const int nd = ctl->nd, np = atm->np, ng = ctl->ng, nw = ctl->nw;
  packed_t pk;
  int st = upload_atm(b, ctl, atm, obs, aero, r0, nr, &pk);
  if (st) return st;
  double *rad = pk.buf + (size_t)np * (size_t)(ng + nw);
  double *tau = rad + (size_t)nr * nd, *tp = tau + (size_t)nr * nd;
  jsc_batch_output out;
  memset(&out, 0, sizeof(out));
  out.rad = rad;
  out.tau = tau;
  out.tpz = tp;
  out.tplon = tp + nr;
  out.tplat = tp + 2 * nr;
  st = jsc_batch_run(b, NULL);
  if (!st) st = jsc_batch_download(b, &out, NULL);
  if (!st) {
    for (int i = 0; i < nr; i++) {
      const int ir = r0 + i;
      obs->tpz[ir] = tp[i];
      obs->tplon[ir] = tp[nr + i];
      obs->tplat[ir] = tp[2 * nr + i];
      for (int id = 0; id < nd; id++) {
        obs->rad[id][ir] = rad[(size_t)i * nd + id];
        obs->tau[id][ir] = tau[(size_t)i * nd + id];
      }
    }
  }
  packed_free(&pk);
  return st;
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
  if (ctl->sca_n > 0 && !aero) {
    jsc_set_error(JSC_ERR_ARG, "formod: SCA_N=%d needs the aerosol/cloud data", ctl->sca_n);
    return JSC_ERR_ARG;
  }

  /* Observation mask (src/forwardmodel.c:25-28). */
  unsigned char *mask = (unsigned char *)malloc((size_t)nd * (nr > 0 ? nr : 1));
  if (!mask) return JSC_ERR_NOMEM;
  for (int id = 0; id < nd; id++)
    for (int ir = 0; ir < nr; ir++) mask[(size_t)id * nr + ir] = !isfinite(obs->rad[id][ir]);

  /* Hydrostatic balance on the caller's atmosphere (src/atmosphere.c:163). */
  {
    const int ig_h2o = jsc_find_emitter(ctl, "H2O");
    jsc_hydrostatic(ctl->hydz, np, atm->z, atm->lon, atm->lat, atm->t,
                    ig_h2o >= 0 ? atm->q[ig_h2o] : NULL, atm->p);
  }

  /* Optical properties for aerosol retrievals (src/forwardmodel.c:34-36),
   * with the Mie series on the GPU. */
  if ((ctl->retnn || ctl->retrr || ctl->retss) && (st = jsc_get_opt_prop(ctl, aero))) {
    free(mask);
    return st;
  }

  pthread_mutex_lock(&g_lock);
  st = ensure_cache(ctl);
  if (!st && nr > 0) st = run_rays(g_batch, ctl, atm, obs, aero, 0, nr);
  pthread_mutex_unlock(&g_lock);

  /* Field-of-view convolution (src/forwardmodel.c:102). */
  if (!st && ctl->fov[0] != '-') st = fov_convolve(ctl, obs);
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

/* End of a drop-in call: record the status for jsc_last_status() and, with
 * exit-on-error (the default), print the message and exit like the
 * reference's ERRMSG (src/jurassic.h:48-52). */
int jsc_finish_call(int st, const char *func) {
  g_last_status = st;
  if (st && g_exit_on_error) {
    printf("\nError (%s, %s, l%d): %s: %s\n\n", __FILE__, func, __LINE__,
           jsc_status_string(st), jsc_last_error_message());
    exit(EXIT_FAILURE);
  }
  return st;
}

void formod(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero) {
  jsc_finish_call(formod_impl(ctl, atm, obs, aero), "formod");
}

/* Batch of formod_pencil for the switches of c (hydrostatic balance off,
 * scattering order in c->sca_mult), one ray; held under g_lock after
 * ensure_cache. */
static int ensure_pencil(const ctl_t *c) {
  if (g_pbatch && same_switches(g_pkey, c)) return JSC_OK;
  jsc_batch_destroy(g_pbatch);
  g_pbatch = NULL;
  if (!g_pkey && !(g_pkey = (ctl_t *)malloc(sizeof(ctl_t)))) return JSC_ERR_NOMEM;
  memcpy(g_pkey, c, sizeof(ctl_t));
  return jsc_batch_create(g_model, c, NPMAX / 2, NPMAX, 1, 0, &g_pbatch);
}

static int pencil_impl(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero, int scattering,
                       int ir) {
  const int nd = ctl->nd, np = atm->np, ng = ctl->ng, nw = ctl->nw;
  if (nd < 1 || nd > NDMAX || ng < 0 || ng > NGMAX || nw < 0 || nw > NWMAX || np < 2 ||
      np > NPMAX || ir < 0 || ir >= obs->nr || obs->nr > NRMAX || scattering < 0) {
    jsc_set_error(JSC_ERR_ARG, "formod_pencil: invalid sizes or ray (nd=%d ng=%d np=%d "
                  "ir=%d nr=%d scattering=%d)", nd, ng, np, ir, obs->nr, scattering);
    return JSC_ERR_ARG;
  }
  if (ctl->sca_n > 0 && !aero) {
    jsc_set_error(JSC_ERR_ARG, "formod_pencil: SCA_N=%d needs the aerosol/cloud data",
                  ctl->sca_n);
    return JSC_ERR_ARG;
  }
  ctl_t *c = (ctl_t *)malloc(sizeof(ctl_t));
  if (!c) return JSC_ERR_NOMEM;
  memcpy(c, ctl, sizeof(ctl_t));
  c->hydz = -999;          /* the pencil takes atm as it is */
  c->sca_mult = scattering;
  pthread_mutex_lock(&g_lock);
  int st = ensure_cache(ctl);
  if (!st) st = ensure_pencil(c);
  if (!st) st = run_rays(g_pbatch, c, atm, obs, aero, ir, 1);
  pthread_mutex_unlock(&g_lock);
  free(c);
  return st;
}

/* Replaces formod_pencil (src/forwardmodel.c:224-405): ray ir of obs through
 * atm as it is (no hydrostatic balance, no mask, no field of view), traced,
 * refined at aerosol/cloud layer edges and integrated on the GPU with
 * scattering sources of order `scattering` (0: none); writes
 * obs->rad[*][ir], obs->tau[*][ir] and obs->tp*[ir]. */
void formod_pencil(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero, int scattering, int ir) {
  jsc_finish_call(pencil_impl(ctl, atm, obs, aero, scattering, ir), "formod_pencil");
}

static int srcfunc_impl(ctl_t *ctl, atm_t *atm, aero_t *aero, int n, const double *x,
                        const double *dx, const int *layer, const double *sec, int scattering,
                        double *src) {
  const int nd = ctl->nd, np = atm->np, ng = ctl->ng, nw = ctl->nw;
  if (nd < 1 || nd > NDMAX || ng < 0 || ng > NGMAX || nw < 0 || nw > NWMAX || np < 2 ||
      np > NPMAX || n < 0 || scattering < 1 || ctl->sca_n < 1 || !aero) {
    jsc_set_error(JSC_ERR_ARG, "jsc_srcfunc_sca: invalid sizes (nd=%d np=%d n=%d "
                  "scattering=%d sca_n=%d) or no aerosol data", nd, np, n, scattering,
                  ctl->sca_n);
    return JSC_ERR_ARG;
  }
  ctl_t *c = (ctl_t *)malloc(sizeof(ctl_t));
  if (!c) return JSC_ERR_NOMEM;
  memcpy(c, ctl, sizeof(ctl_t));
  c->hydz = -999;          /* atm as given, as srcfunc_sca takes it */
  c->sca_mult = scattering;
  int st;
  pthread_mutex_lock(&g_lock);
  st = ensure_cache(ctl);
  jsc_batch *b = NULL;
  if (!st) st = jsc_batch_create(g_model, c, NPMAX / 2, NPMAX, 1, 0, &b);
  packed_t pk;
  memset(&pk, 0, sizeof(pk));
  if (!st) {
    /* the atmosphere as formod packs it, no rays */
    obs_t *none = (obs_t *)calloc(1, sizeof(obs_t));
    if (!none) st = JSC_ERR_NOMEM;
    if (!st) st = upload_atm(b, c, atm, none, aero, 0, 0, &pk);
    free(none);
  }
  /* synchronises its stream before it returns: the upload has passed */
  if (!st) st = jsc_batch_scatter_points(b, n, x, dx, layer, sec, NULL, src, NULL);
  packed_free(&pk);
  jsc_batch_destroy(b);
  pthread_mutex_unlock(&g_lock);
  free(c);
  return st;
}

int jsc_srcfunc_sca(ctl_t *ctl, atm_t *atm, aero_t *aero, int n, const double *x,
                    const double *dx, const int *layer, const double *sec, int scattering,
                    double *src) {
  const int st = srcfunc_impl(ctl, atm, aero, n, x, dx, layer, sec, scattering, src);
  g_last_status = st;
  return st;
}

/* Replaces formod_fov (src/forwardmodel.c:156-220): the field-of-view
 * convolution of obs over tangent height, nothing when ctl->fov is "-". */
void formod_fov(ctl_t *ctl, obs_t *obs) {
  if (ctl->fov[0] == '-') return;
  jsc_finish_call(fov_convolve(ctl, obs), "formod_fov");
}

/* Replaces read_shape (src/forwardmodel.c:577-606): two columns x, y of a
 * filter or field-of-view file, *n points (at most NSHAPE). */
void read_shape(const char *filename, double *x, double *y, int *n) {
  jsc_finish_call(jsc_read_filter(filename, x, y, n), "read_shape");
}

/* Release the cached model and batches (tests and long-running hosts). */
void jsc_release_cache(void) {
  pthread_mutex_lock(&g_lock);
  jsc_batch_destroy(g_batch);
  jsc_batch_destroy(g_jbatch);
  jsc_batch_destroy(g_pbatch);
  jsc_model_destroy(g_model);
  g_batch = NULL;
  g_jbatch = NULL;
  g_pbatch = NULL;
  g_model = NULL;
  free(g_key);
  g_key = NULL;
  free(g_pkey);
  g_pkey = NULL;
  pthread_mutex_unlock(&g_lock);
}

/* ---------------------------------------------------------------- kernel -- */

/* Elements of one quantity at the levels inside [zmin, zmax]
 * (atm2x_help, src/atmosphere.c:72-97). */
static void atm2x_help(const atm_t *atm, double zmin, double zmax, const double *value,
                       int idx, double *x, int *iqa, int *ipa, size_t *n) {
  for (int ip = 0; ip < atm->np; ip++)
    if (atm->z[ip] >= zmin && atm->z[ip] <= zmax) {
      if (x) x[*n] = value[ip];
      if (iqa) iqa[*n] = idx;
      if (ipa) ipa[*n] = ip;
      (*n)++;
    }
}

static void atm2x_aero(double v, int idx, double *x, int *iqa, int *ipa, size_t *n) {
  if (x) x[*n] = v;
  if (iqa) iqa[*n] = idx;
  if (ipa) ipa[*n] = -1;
  (*n)++;
}

size_t jsc_atm2x(const ctl_t *ctl, const atm_t *atm, const aero_t *aero, double *x,
                 int *iqa, int *ipa) {
  size_t n = 0;
  atm2x_help(atm, ctl->retp_zmin, ctl->retp_zmax, atm->p, JSC_IDXP, x, iqa, ipa, &n);
  atm2x_help(atm, ctl->rett_zmin, ctl->rett_zmax, atm->t, JSC_IDXT, x, iqa, ipa, &n);
  for (int ig = 0; ig < ctl->ng; ig++)
    atm2x_help(atm, ctl->retq_zmin[ig], ctl->retq_zmax[ig], atm->q[ig], JSC_IDXQ(ig), x, iqa,
               ipa, &n);
  for (int iw = 0; iw < ctl->nw; iw++)
    atm2x_help(atm, ctl->retk_zmin[iw], ctl->retk_zmax[iw], atm->k[iw], JSC_IDXK(ctl, iw), x,
               iqa, ipa, &n);
  if (ctl->retnn) atm2x_aero(aero ? aero->nn[0] : 0, JSC_IDXNN(ctl), x, iqa, ipa, &n);
  if (ctl->retrr) atm2x_aero(aero ? aero->rr[0] : 0, JSC_IDXRR(ctl), x, iqa, ipa, &n);
  if (ctl->retss) atm2x_aero(aero ? aero->ss[0] : 0, JSC_IDXSS(ctl), x, iqa, ipa, &n);
  return n;
}

/* x2atm_help, src/retrievalmodel.c:1147-1163. */
static void x2atm_help(atm_t *atm, double zmin, double zmax, double *value, const double *x,
                       size_t *n) {
  for (int ip = 0; ip < atm->np; ip++)
    if (atm->z[ip] >= zmin && atm->z[ip] <= zmax) value[ip] = x[(*n)++];
}

void jsc_x2atm(const ctl_t *ctl, const double *x, atm_t *atm, aero_t *aero) {
  size_t n = 0;
  x2atm_help(atm, ctl->retp_zmin, ctl->retp_zmax, atm->p, x, &n);
  x2atm_help(atm, ctl->rett_zmin, ctl->rett_zmax, atm->t, x, &n);
  for (int ig = 0; ig < ctl->ng; ig++)
    x2atm_help(atm, ctl->retq_zmin[ig], ctl->retq_zmax[ig], atm->q[ig], x, &n);
  for (int iw = 0; iw < ctl->nw; iw++)
    x2atm_help(atm, ctl->retk_zmin[iw], ctl->retk_zmax[iw], atm->k[iw], x, &n);
  if (ctl->retnn) {
    if (aero) aero->nn[0] = x[n];
    n++;
  }
  if (ctl->retrr) {
    if (aero) aero->rr[0] = x[n];
    n++;
  }
  if (ctl->retss) {
    if (aero) aero->ss[0] = x[n];
    n++;
  }
}

size_t jsc_obs2y(const ctl_t *ctl, const obs_t *obs, double *y, int *ida, int *ira) {
  size_t m = 0;
  for (int ir = 0; ir < obs->nr; ir++)
    for (int id = 0; id < ctl->nd; id++)
      if (isfinite(obs->rad[id][ir])) {
        if (y) y[m] = obs->rad[id][ir];
        if (ida) ida[m] = id;
        if (ira) ira[m] = ir;
        m++;
      }
  return m;
}

/* GSL_MAX as the reference evaluates it. */
static double gmax(double a, double b) { return a > b ? a : b; }

/* Perturbation size of a state-vector element of quantity iqa and value x
 * (src/retrievalmodel.c:241-273); -999 where the reference has none. */
static double perturbation(const ctl_t *ctl, int iqa, double x) {
  double h = -999;
  if (iqa == JSC_IDXP) h = gmax(fabs(0.01 * x), 1e-7);
  if (iqa == JSC_IDXT) h = 1;
  if (iqa >= JSC_IDXQ(0) && iqa < JSC_IDXQ(ctl->ng)) h = gmax(fabs(0.01 * x), 1e-15);
  if (iqa >= JSC_IDXK(ctl, 0) && iqa < JSC_IDXK(ctl, ctl->nw)) h = 1e-4;
  return h;
}

/* Pointer to the profile value a state-vector element of quantity iqa sets
 * at level ip of a packed profile set (p, t, q [ng][nl], k [nw][nl]). */
static double *element(const ctl_t *ctl, int iqa, int ip, double *p, double *t, double *q,
                       double *k, size_t nl) {
  if (iqa == JSC_IDXP) return p + ip;
  if (iqa == JSC_IDXT) return t + ip;
  if (iqa >= JSC_IDXQ(0) && iqa < JSC_IDXQ(ctl->ng)) return q + (size_t)(iqa - JSC_IDXQ(0)) * nl + ip;
  return k + (size_t)(iqa - JSC_IDXK(ctl, 0)) * nl + ip;
}

/* Jacobian batch with room for natm profiles of np levels and nrays rays. */
static int ensure_jbatch(const ctl_t *ctl, int natm, int nlev, int nrays) {
  if (g_jbatch && natm <= g_jcap_atm && nlev <= g_jcap_lev && nrays <= g_jcap_rays)
    return JSC_OK;
  jsc_batch_destroy(g_jbatch);
  g_jbatch = NULL;
  ctl_t c2;
  memcpy(&c2, ctl, sizeof(ctl_t));
  c2.hydz = -999;  /* hydrostatic balance is applied per profile on the host */
  int st = jsc_batch_create(g_model, &c2, natm, nlev, nrays, 0, &g_jbatch);
  if (st) return st;
  g_jcap_atm = natm;
  g_jcap_lev = nlev;
  g_jcap_rays = nrays;
  return JSC_OK;
}

/* Radiance of ray ir, channel id of a batch output as formod leaves it in
 * obs->rad (brightness temperature when ctl->write_bbt). */
static double out_rad(const ctl_t *ctl, const double *rad, size_t ray, int id) {
  const double v = rad[ray * ctl->nd + id];
  return ctl->write_bbt ? brightness(v, ctl->nu[id]) : v;
}

/* Jacobian with one forward model per column, the reference's own scheme
 * (kernel, src/retrievalmodel.c:201-298), for atmospheres a batch cannot
 * hold several disturbed copies of (IP 2/3: all profiles form one
 * horizontally varying atmosphere).  Each column runs formod_impl on a
 * copy of the undisturbed atm/obs/aero with one state element moved. */
static int kernel_columns(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero, double *k,
                          size_t m, size_t n, size_t tda) {
  aero_t *empty = NULL;  /* aero_t is ~2 MB: never on the stack */
  if (!aero) {
    empty = (aero_t *)calloc(1, sizeof(aero_t));
    if (!empty) return JSC_ERR_NOMEM;
    aero = empty;
  }
  int st = formod_impl(ctl, atm, obs, aero);
  if (st) {
    free(empty);
    return st;
  }
  const size_t n0 = jsc_atm2x(ctl, atm, aero, NULL, NULL, NULL);
  const size_t m0 = jsc_obs2y(ctl, obs, NULL, NULL, NULL);
  if (n0 != n || m0 != m) {
    jsc_set_error(JSC_ERR_ARG, "jsc_kernel: %zu x %zu matrix for %zu measurements and %zu "
                  "state elements", m, n, m0, n0);
    free(empty);
    return JSC_ERR_ARG;
  }
  if ((m > 0 && n > 0 && !k) || tda < n) {
    jsc_set_error(JSC_ERR_ARG, "jsc_kernel: no matrix, or row stride %zu below %zu columns",
                  tda, n);
    free(empty);
    return JSC_ERR_ARG;
  }
  double *x0 = (double *)malloc((n + 1) * sizeof(double));
  double *x1 = (double *)malloc((n + 1) * sizeof(double));
  double *y = (double *)malloc((2 * m + 1) * sizeof(double));
  int *iqa = (int *)malloc((n + 1) * sizeof(int));
  atm_t *atm1 = (atm_t *)malloc(sizeof(atm_t));
  obs_t *obs1 = (obs_t *)malloc(sizeof(obs_t));
  aero_t *aero1 = (aero_t *)malloc(sizeof(aero_t));
  if (!x0 || !x1 || !y || !iqa || !atm1 || !obs1 || !aero1) {
    st = JSC_ERR_NOMEM;
  } else {
    jsc_atm2x(ctl, atm, aero, x0, iqa, NULL);
    jsc_obs2y(ctl, obs, y, NULL, NULL);
    for (size_t j = 0; j < n && !st; j++) {
      double h = perturbation(ctl, iqa[j], x0[j]);
      if (iqa[j] == JSC_IDXNN(ctl)) h = gmax(fabs(0.5 * x0[j]), 0.1);
      if (iqa[j] == JSC_IDXRR(ctl)) h = gmax(fabs(0.25 * x0[j]), 0.1);
      if (iqa[j] == JSC_IDXSS(ctl)) h = gmax(fabs(0.1 * x0[j]), 0.01);
      if (h <= 0) {
        jsc_set_error(JSC_ERR_ARG, "jsc_kernel: cannot set perturbation size");
        st = JSC_ERR_ARG;
        break;
      }
      memcpy(x1, x0, n * sizeof(double));
      x1[j] += h;
      memcpy(atm1, atm, sizeof(atm_t));
      memcpy(obs1, obs, sizeof(obs_t));
      memcpy(aero1, aero, sizeof(aero_t));
      jsc_x2atm(ctl, x1, atm1, aero1);
      if ((st = formod_impl(ctl, atm1, obs1, aero1))) break;
      double *y1 = y + m;
      size_t c = 0;
      for (int ir = 0; ir < obs1->nr; ir++)
        for (int id = 0; id < ctl->nd; id++)
          if (isfinite(obs1->rad[id][ir])) {
            if (c < m) y1[c] = obs1->rad[id][ir];
            c++;
          }
      if (c != m) {
        jsc_set_error(JSC_ERR_ARG,
                      "jsc_kernel: disturbed forward model %zu has %zu finite radiances, "
                      "the undisturbed one %zu", j, c, m);
        st = JSC_ERR_ARG;
        break;
      }
      for (size_t i = 0; i < m; i++) k[i * tda + j] = (y1[i] - y[i]) / h;
    }
  }
  free(x0);
  free(x1);
  free(y);
  free(iqa);
  free(atm1);
  free(obs1);
  free(aero1);
  free(empty);
  return st;
}

/* Aerosol parameter of a state-vector element (the value x2atm sets). */
static double *aero_element(const ctl_t *ctl, int iqa, aero_t *aero) {
  if (iqa == JSC_IDXNN(ctl)) return &aero->nn[0];
  if (iqa == JSC_IDXRR(ctl)) return &aero->rr[0];
  return &aero->ss[0];
}

int jsc_kernel(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero, double *k, size_t m,
               size_t n, size_t tda) {
  const int nd = ctl->nd, nr = obs->nr, np = atm->np, ng = ctl->ng, nw = ctl->nw;
  if (nd < 1 || nd > NDMAX || ng < 0 || ng > NGMAX || nw < 0 || nw > NWMAX ||
      nr < 0 || nr > NRMAX || np < 2 || np > NPMAX) {
    jsc_set_error(JSC_ERR_ARG, "jsc_kernel: invalid sizes (nd=%d ng=%d nw=%d nr=%d np=%d)",
                  nd, ng, nw, nr, np);
    return JSC_ERR_ARG;
  }
  if (ctl->ip != 1) return kernel_columns(ctl, atm, obs, aero, k, m, n, tda);
  const int aero_ret = ctl->retnn || ctl->retrr || ctl->retss;
  if ((ctl->sca_n > 0 || aero_ret) && !aero) {
    jsc_set_error(JSC_ERR_ARG, "jsc_kernel: SCA_N=%d needs the aerosol/cloud data", ctl->sca_n);
    return JSC_ERR_ARG;
  }
  if ((m > 0 && n > 0 && !k) || tda < n) {
    jsc_set_error(JSC_ERR_ARG, "jsc_kernel: no matrix, or row stride %zu below %zu columns",
                  tda, n);
    return JSC_ERR_ARG;
  }

  /* Hydrostatic balance on the caller's atmosphere and, for aerosol
   * retrievals, fresh optical properties, as formod does. */
  const int ig_h2o = jsc_find_emitter(ctl, "H2O");
  jsc_hydrostatic(ctl->hydz, np, atm->z, atm->lon, atm->lat, atm->t,
                  ig_h2o >= 0 ? atm->q[ig_h2o] : NULL, atm->p);
  const size_t n0 = jsc_atm2x(ctl, atm, aero, NULL, NULL, NULL);
  if (n0 != n) {
    jsc_set_error(JSC_ERR_ARG, "jsc_kernel: the state vector has %zu elements, k %zu columns",
                  n0, n);
    return JSC_ERR_ARG;
  }

  int st = JSC_OK;
  if (aero_ret && (st = jsc_get_opt_prop(ctl, aero))) return st;
  double *x0 = (double *)malloc((n + 1) * sizeof(double));
  double *h = (double *)malloc((n + 1) * sizeof(double));
  int *iqa = (int *)malloc((n + 1) * sizeof(int)), *ipa = (int *)malloc((n + 1) * sizeof(int));
  /* source of column j: disturbed profile col[j] >= 1 of the main batch, or
   * -1 - a for the a-th aerosol parameter (its own run) */
  long *col = (long *)malloc((n + 1) * sizeof(long));
  unsigned char *mask = (unsigned char *)malloc((size_t)nd * (nr > 0 ? nr : 1));
  double *prof = NULL, *rays = NULL, *res = NULL, *ares = NULL, *bq = NULL, *bk = NULL;
  int *atm_off = NULL, *ray_atm = NULL;
  aero_t *aero1 = NULL;
  obs_t *fobs = NULL;
  size_t natm = 1, naero = 0;
  if (!x0 || !h || !iqa || !ipa || !col || !mask) {
    st = JSC_ERR_NOMEM;
    goto done;
  }
  jsc_atm2x(ctl, atm, aero, x0, iqa, ipa);
  for (size_t j = 0; j < n; j++) {
    h[j] = perturbation(ctl, iqa[j], x0[j]);
    if (iqa[j] == JSC_IDXNN(ctl)) h[j] = gmax(fabs(0.5 * x0[j]), 0.1);
    if (iqa[j] == JSC_IDXRR(ctl)) h[j] = gmax(fabs(0.25 * x0[j]), 0.1);
    if (iqa[j] == JSC_IDXSS(ctl)) h[j] = gmax(fabs(0.1 * x0[j]), 0.01);
    if (h[j] <= 0) {
      jsc_set_error(JSC_ERR_ARG, "jsc_kernel: cannot set perturbation size");
      st = JSC_ERR_ARG;
      goto done;
    }
    col[j] = iqa[j] >= JSC_IDXNN(ctl) ? -1 - (long)naero++ : (long)natm++;
  }
  const size_t nl = natm * (size_t)np, nrays = natm * (size_t)nr;
  if (nl > 0x7fffffff || nrays > 0x7fffffff) {
    jsc_set_error(JSC_ERR_ARG, "jsc_kernel: %zu profiles x %d rays exceed the batch limits",
                  natm, nr);
    st = JSC_ERR_ARG;
    goto done;
  }
  /* packed profiles: z lon lat p t [nl], q [ng][nl], k [nw][nl] */
  prof = (double *)malloc(nl * (5 + (size_t)ng + nw) * sizeof(double));
  atm_off = (int *)malloc((natm + 1) * sizeof(int));
  /* rays: time obsz obslon obslat vpz vplon vplat [nrays]; outputs */
  rays = (double *)malloc(nrays * 7 * sizeof(double) + 1);
  ray_atm = (int *)malloc(nrays * sizeof(int) + 1);
  res = (double *)malloc((nrays * (2 * (size_t)nd + 3) + 2 * m + 1) * sizeof(double));
  /* aerosol columns: rad, tau [nr][nd] and tpz, tplon, tplat [nr] each */
  ares = (double *)malloc((naero * (size_t)nr * (2 * (size_t)nd + 3) + 1) * sizeof(double));
  if (naero) {
    aero1 = (aero_t *)malloc(sizeof(aero_t));
    bq = (double *)malloc(((size_t)(ng + nw) * np + 1) * sizeof(double));
    if (bq) {
      bk = bq + (size_t)ng * np;
      for (int ig = 0; ig < ng; ig++) memcpy(bq + (size_t)ig * np, atm->q[ig], np * sizeof(double));
      for (int iw = 0; iw < nw; iw++) memcpy(bk + (size_t)iw * np, atm->k[iw], np * sizeof(double));
    }
  }
  if (ctl->fov[0] != '-') fobs = (obs_t *)malloc(sizeof(obs_t));
  if (!prof || !atm_off || !rays || !ray_atm || !res || !ares || (naero && (!aero1 || !bq)) ||
      (ctl->fov[0] != '-' && !fobs)) {
    st = JSC_ERR_NOMEM;
    goto done;
  }
  for (int id = 0; id < nd; id++)
    for (int ir = 0; ir < nr; ir++) mask[(size_t)id * nr + ir] = !isfinite(obs->rad[id][ir]);

  {
    double *z = prof, *lon = z + nl, *lat = lon + nl, *p = lat + nl, *t = p + nl;
    double *q = t + nl, *kx = q + (size_t)ng * nl;
    for (size_t a = 0; a < natm; a++) {
      const size_t o = a * np;
      atm_off[a] = (int)o;
      memcpy(z + o, atm->z, np * sizeof(double));
      memcpy(lon + o, atm->lon, np * sizeof(double));
      memcpy(lat + o, atm->lat, np * sizeof(double));
      memcpy(p + o, atm->p, np * sizeof(double));
      memcpy(t + o, atm->t, np * sizeof(double));
      for (int ig = 0; ig < ng; ig++) memcpy(q + (size_t)ig * nl + o, atm->q[ig], np * sizeof(double));
      for (int iw = 0; iw < nw; iw++) memcpy(kx + (size_t)iw * nl + o, atm->k[iw], np * sizeof(double));
    }
    /* disturbed profiles: state element + h, then the hydrostatic balance
     * formod applies to them */
    for (size_t j = 0; j < n; j++) {
      if (col[j] < 1) continue;
      const size_t o = (size_t)col[j] * np;
      *element(ctl, iqa[j], ipa[j], p + o, t + o, q + o, kx + o, nl) = x0[j] + h[j];
      jsc_hydrostatic(ctl->hydz, np, z + o, lon + o, lat + o, t + o,
                      ig_h2o >= 0 ? q + (size_t)ig_h2o * nl + o : NULL, p + o);
    }
    atm_off[natm] = (int)nl;
    for (size_t a = 0; a < natm; a++)
      for (int ir = 0; ir < nr; ir++) {
        const size_t r = a * nr + ir;
        ray_atm[r] = (int)a;
        rays[r] = obs->time[ir];
        rays[nrays + r] = obs->obsz[ir];
        rays[2 * nrays + r] = obs->obslon[ir];
        rays[3 * nrays + r] = obs->obslat[ir];
        rays[4 * nrays + r] = obs->vpz[ir];
        rays[5 * nrays + r] = obs->vplon[ir];
        rays[6 * nrays + r] = obs->vplat[ir];
      }
    jsc_batch_input in;
    memset(&in, 0, sizeof(in));
    in.n_atm = (int)natm;
    in.n_levels = (int)nl;
    in.atm_off = atm_off;
    in.z = z;
    in.lon = lon;
    in.lat = lat;
    in.p = p;
    in.t = t;
    in.q = q;
    in.k = kx;
    in.n_rays = (int)nrays;
    in.ray_atm = ray_atm;
    in.time = rays;
    in.obsz = rays + nrays;
    in.obslon = rays + 2 * nrays;
    in.obslat = rays + 3 * nrays;
    in.vpz = rays + 4 * nrays;
    in.vplon = rays + 5 * nrays;
    in.vplat = rays + 6 * nrays;
    double *rad = res, *tau = rad + nrays * nd, *tp = tau + nrays * nd;
    jsc_batch_output out;
    memset(&out, 0, sizeof(out));
    out.rad = rad;
    out.tau = tau;
    out.tpz = tp;
    out.tplon = tp + nrays;
    out.tplat = tp + 2 * nrays;
    if (nr > 0) {
      pthread_mutex_lock(&g_lock);
      st = ensure_cache(ctl);
      if (!st) st = ensure_jbatch(ctl, (int)natm, (int)nl, (int)nrays);
      if (!st && ctl->sca_n > 0) st = jsc_batch_set_aero(g_jbatch, aero);
      if (!st) st = jsc_batch_upload(g_jbatch, &in, NULL);
      if (!st) st = jsc_batch_run(g_jbatch, NULL);
      if (!st) st = jsc_batch_download(g_jbatch, &out, NULL);
      /* aerosol parameters: the undisturbed profile with the optical
       * properties of the disturbed parameter, one run each */
      for (size_t j = 0; j < n && !st; j++) {
        if (col[j] >= 0) continue;
        memcpy(aero1, aero, sizeof(aero_t));
        *aero_element(ctl, iqa[j], aero1) = x0[j] + h[j];
        st = jsc_get_opt_prop(ctl, aero1);
        double *ar = ares + (size_t)(-1 - col[j]) * nr * (2 * (size_t)nd + 3);
        jsc_batch_input in1 = in;
        int off1[2] = {0, np};
        in1.n_atm = 1;
        in1.n_levels = np;
        in1.atm_off = off1;
        in1.q = bq;       /* the undisturbed profile's blocks, [ng][np], [nw][np] */
        in1.k = bk;
        in1.n_rays = nr;  /* the first profile's rays, all on profile 0 */
        jsc_batch_output out1;
        memset(&out1, 0, sizeof(out1));
        out1.rad = ar;
        out1.tau = ar + (size_t)nr * nd;
        out1.tpz = ar + 2 * (size_t)nr * nd;
        out1.tplon = out1.tpz + nr;
        out1.tplat = out1.tplon + nr;
        if (!st) st = jsc_batch_set_aero(g_jbatch, aero1);
        if (!st) st = jsc_batch_upload(g_jbatch, &in1, NULL);
        if (!st) st = jsc_batch_run(g_jbatch, NULL);
        if (!st) st = jsc_batch_download(g_jbatch, &out1, NULL);
      }
      pthread_mutex_unlock(&g_lock);
    }
    if (st) goto done;

    /* The undisturbed forward model into obs (formod's outputs: field-of-
     * view convolution, brightness temperature, mask). */
    const int fov = ctl->fov[0] != '-';
    for (int ir = 0; ir < nr; ir++) {
      obs->tpz[ir] = tp[ir];
      obs->tplon[ir] = tp[nrays + ir];
      obs->tplat[ir] = tp[2 * nrays + ir];
      for (int id = 0; id < nd; id++) {
        obs->rad[id][ir] = rad[(size_t)ir * nd + id];
        obs->tau[id][ir] = tau[(size_t)ir * nd + id];
      }
    }
    if (fov && (st = fov_convolve(ctl, obs))) goto done;
    for (int ir = 0; ir < nr; ir++)
      for (int id = 0; id < nd; id++) {
        const double v = obs->rad[id][ir];
        obs->rad[id][ir] = mask[(size_t)id * nr + ir] ? NAN
                           : ctl->write_bbt ? brightness(v, ctl->nu[id]) : v;
      }
    double *y0 = tp + 3 * nrays, *y1 = y0 + m;
    const size_t m0 = jsc_obs2y(ctl, obs, NULL, NULL, NULL);
    if (m0 != m) {
      jsc_set_error(JSC_ERR_ARG, "jsc_kernel: %zu finite radiances, k has %zu rows", m0, m);
      st = JSC_ERR_ARG;
      goto done;
    }
    jsc_obs2y(ctl, obs, y0, NULL, NULL);
    /* Disturbed columns: the measurement vector of each disturbed forward
     * model (obs2y of a copy of obs, whose non-finite entries stay masked). */
    for (size_t j = 0; j < n; j++) {
      const double *cr, *ct, *cz;  /* column's rad, tau [nr][nd], tpz [nr] */
      if (col[j] >= 1) {
        cr = rad + (size_t)col[j] * nr * nd;
        ct = tau + (size_t)col[j] * nr * nd;
        cz = tp + (size_t)col[j] * nr;
      } else {
        cr = ares + (size_t)(-1 - col[j]) * nr * (2 * (size_t)nd + 3);
        ct = cr + (size_t)nr * nd;
        cz = ct + (size_t)nr * nd;
      }
      if (fov) {
        /* the disturbed results through the same convolution */
        fobs->nr = nr;
        for (int ir = 0; ir < nr; ir++) {
          fobs->time[ir] = obs->time[ir];
          fobs->tpz[ir] = cz[ir];
          for (int id = 0; id < nd; id++) {
            fobs->rad[id][ir] = cr[(size_t)ir * nd + id];
            fobs->tau[id][ir] = ct[(size_t)ir * nd + id];
          }
        }
        if ((st = fov_convolve(ctl, fobs))) goto done;
      }
      size_t c = 0;
      for (int ir = 0; ir < nr; ir++)
        for (int id = 0; id < nd; id++) {
          if (!isfinite(obs->rad[id][ir])) continue;
          const double v = fov ? (ctl->write_bbt ? brightness(fobs->rad[id][ir], ctl->nu[id])
                                                 : fobs->rad[id][ir])
                               : out_rad(ctl, cr, (size_t)ir, id);
          if (!isfinite(v)) continue;
          if (c < m) y1[c] = v;
          c++;
        }
      if (c != m) {
        jsc_set_error(JSC_ERR_ARG,
                      "jsc_kernel: disturbed forward model %zu has %zu finite radiances, "
                      "the undisturbed one %zu", j, c, m);
        st = JSC_ERR_ARG;
        goto done;
      }
      for (size_t i = 0; i < m; i++) k[i * tda + j] = (y1[i] - y0[i]) / h[j];
    }
  }

done:
  free(x0);
  free(h);
  free(iqa);
  free(ipa);
  free(col);
  free(mask);
  free(prof);
  free(atm_off);
  free(rays);
  free(ray_atm);
  free(res);
  free(ares);
  free(bq);
  free(aero1);
  free(fobs);
  return st;
}
