/*
 * CPU restatement of the reference forward-model hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * test and bench.py's CPU baseline load it; the product never does.  It
 * restates, in plain sequential-per-ray C with OpenMP over rays, the
 * algorithm of the reference files cited at each function, keeping their
 * operation order so that results agree with the reference bit for bit
 * where libm agrees.  Built by oracle/Makefile (no FMA contraction).
 *
 * Entry points (C ABI, structs of include/jurassic_b200.h):
 *   oracle_formod(ctl, atm, obs, aero)    formod() restated (clear air)
 *   oracle_diagnostics(...)               LOS point counts and EGA index
 *                                         checksums per (ray, channel)
 *   oracle_raytrace(...)                  one ray's line of sight
 *   oracle_hydrostatic, oracle_planck, oracle_brightness, oracle_srcfunc
 *   oracle_reset()                        drop cached tables
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "jurassic_b200.h"
#include "ckd_tables.h"

#define JSC_NPLANCK_O 1201   /* Planck table nodes, 100..400 K */
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#define LINV(x0, y0, x1, y1, x) ((y0) + ((y1) - (y0)) / ((x1) - (x0)) * ((x) - (x0)))
#define DOT(a, b) ((a)[0] * (b)[0] + (a)[1] * (b)[1] + (a)[2] * (b)[2])
#define NRM(a) sqrt(DOT(a, a))

static int g_err = 0;            /* first error code of the last call */

static void fail(int code) {
#pragma omp critical(oracle_err)
  if (!g_err) g_err = code;
}

/* ------------------------------------------------------------- misc.c -- */

/* src/misc.c:5-16 */
static void o_cart2geo(const double *x, double *z, double *lon, double *lat) {
  double radius = NRM(x);
  *lat = asin(x[2] / radius) * 180 / M_PI;
  *lon = atan2(x[1], x[0]) * 180 / M_PI;
  *z = radius - JSC_RE;
}

/* src/misc.c:61-72 */
static void o_geo2cart(double z, double lon, double lat, double *x) {
  double radius = z + JSC_RE;
  x[0] = radius * cos(lat / 180 * M_PI) * cos(lon / 180 * M_PI);
  x[1] = radius * cos(lat / 180 * M_PI) * sin(lon / 180 * M_PI);
  x[2] = radius * sin(lat / 180 * M_PI);
}

/* src/misc.c:237-265 */
static int o_locate(const double *xx, int n, double x) {
  int i, ilo = 0, ihi = n - 1;
  if (n < 2) return 0;
  i = (ihi + ilo) >> 1;
  if (xx[i] < xx[i + 1])
    while (ihi > ilo + 1) {
      i = (ihi + ilo) >> 1;
      if (xx[i] > x) ihi = i; else ilo = i;
    }
  else
    while (ihi > ilo + 1) {
      i = (ihi + ilo) >> 1;
      if (xx[i] <= x) ihi = i; else ilo = i;
    }
  return ilo;
}

/* src/forwardmodel.c:546-565 */
static int o_locate_tbl(const float *xx, int n, double x) {
  int i, ilo = 0, ihi = n - 1;
  while (ihi > ilo + 1) {
    i = (ihi + ilo) >> 1;
    if (xx[i] > x) ihi = i; else ilo = i;
  }
  return ilo;
}

static int o_find_emitter(const ctl_t *ctl, const char *name) {
  for (int ig = 0; ig < ctl->ng; ig++)
    if (strcasecmp(ctl->emitter[ig], name) == 0) return ig;
  return -1;
}

/* GSL 1.15 sys/expm1.c and sys/log1p.c */
static double o_expm1(double x) {
  if (fabs(x) < M_LN2) {
    double i = 1.0, sum = x, term = x / 1.0;
    do {
      i++;
      term *= x / i;
      sum += term;
    } while (fabs(term) > fabs(sum) * 2.2204460492503131e-16);
    return sum;
  }
  return exp(x) - 1;
}

static double o_log1p(double x) {
  volatile double y = 1 + x, z = y - 1;
  return log(y) - (z - x) / y;
}

double oracle_planck(double t, double nu) {   /* src/forwardmodel.c:569-573 */
  return JSC_C1 * (nu * nu * nu) / o_expm1(JSC_C2 * nu / t);
}

double oracle_brightness(double rad, double nu) {   /* src/forwardmodel.c:7-11 */
  return JSC_C2 * nu / o_log1p(JSC_C1 * (nu * nu * nu) / rad);
}

/* ------------------------------------------------------- atmosphere.c -- */

/* src/atmosphere.c:153-159 */
static double o_gravity(double z, double lat) {
  double a = sin(lat / 180 * M_PI), b = sin(2 * lat / 180 * M_PI);
  return 9.780318 * (1 + 0.0053024 * (a * a) - 0.0000058 * (b * b)) - 3.086e-3 * z;
}

/* src/atmosphere.c:188-243 */
static void o_hydrostatic_1d(const ctl_t *ctl, atm_t *atm, int ip0, int ip1) {
  double dzmin = 1e99, e = 0, mean, mmair = 28.96456e-3, mmh2o = 18.0153e-3, z;
  int ipref = 0, ipts = 20, ig_h2o = o_find_emitter(ctl, "H2O");
  for (int ip = ip0; ip < ip1; ip++)
    if (fabs(atm->z[ip] - ctl->hydz) < dzmin) {
      dzmin = fabs(atm->z[ip] - ctl->hydz);
      ipref = ip;
    }
  for (int ip = ipref + 1; ip < ip1; ip++) {
    mean = 0;
    for (int i = 0; i < ipts; i++) {
      z = LINV(0.0, atm->z[ip - 1], ipts - 1.0, atm->z[ip], (double)i);
      if (ig_h2o >= 0)
        e = LINV(0.0, atm->q[ig_h2o][ip - 1], ipts - 1.0, atm->q[ig_h2o][ip], (double)i);
      mean += (e * mmh2o + (1 - e) * mmair) * o_gravity(z, atm->lat[ipref]) / JSC_RGAS /
              LINV(0.0, atm->t[ip - 1], ipts - 1.0, atm->t[ip], (double)i) / ipts;
    }
    atm->p[ip] = exp(log(atm->p[ip - 1]) - mean * 1000 * (atm->z[ip] - atm->z[ip - 1]));
  }
  for (int ip = ipref - 1; ip >= ip0; ip--) {
    mean = 0;
    for (int i = 0; i < ipts; i++) {
      z = LINV(0.0, atm->z[ip + 1], ipts - 1.0, atm->z[ip], (double)i);
      if (ig_h2o >= 0)
        e = LINV(0.0, atm->q[ig_h2o][ip + 1], ipts - 1.0, atm->q[ig_h2o][ip], (double)i);
      mean += (e * mmh2o + (1 - e) * mmair) * o_gravity(z, atm->lat[ipref]) / JSC_RGAS /
              LINV(0.0, atm->t[ip + 1], ipts - 1.0, atm->t[ip], (double)i) / ipts;
    }
    atm->p[ip] = exp(log(atm->p[ip + 1]) - mean * 1000 * (atm->z[ip] - atm->z[ip + 1]));
  }
}

/* src/atmosphere.c:163-184 */
static void o_hydrostatic(const ctl_t *ctl, atm_t *atm) {
  double lat0 = -999, lon0 = -999;
  int ip0 = -999;
  if (ctl->hydz < 0 || atm->np < 1) return;
  for (int ip = 0; ip < atm->np; ip++)
    if (atm->lon[ip] != lon0 || atm->lat[ip] != lat0) {
      if (ip > 0) o_hydrostatic_1d(ctl, atm, ip0, ip);
      lon0 = atm->lon[ip];
      lat0 = atm->lat[ip];
      ip0 = ip;
    }
  o_hydrostatic_1d(ctl, atm, ip0, atm->np);
}

/* src/atmosphere.c:298-320 (IP=1, the only mode of the hot path) */
static void o_intpol_atm(const ctl_t *ctl, const atm_t *atm, double z0,
                         double *p, double *t, double *q, double *k) {
  int ip = o_locate(atm->z, atm->np, z0);
  double y0 = atm->p[ip], y1 = atm->p[ip + 1], x0 = atm->z[ip], x1 = atm->z[ip + 1];
  *p = (y0 > 0 && y1 > 0) ? (y0 * exp(log(y1 / y0) / (x1 - x0) * (z0 - x0)))
                          : LINV(x0, y0, x1, y1, z0);
  *t = LINV(x0, atm->t[ip], x1, atm->t[ip + 1], z0);
  if (q)
    for (int ig = 0; ig < ctl->ng; ig++)
      q[ig] = LINV(x0, atm->q[ig][ip], x1, atm->q[ig][ip + 1], z0);
  if (k)
    for (int iw = 0; iw < ctl->nw; iw++)
      k[iw] = LINV(x0, atm->k[iw][ip], x1, atm->k[iw][ip + 1], z0);
}

/* ------------------------------------------------------ lineofsight.c -- */

typedef struct {
  int np;
  double tsurf;
  double *z, *lon, *lat, *p, *t, *ds, *aerofac;
  int *aeroi;
  double (*q)[NGMAX], (*k)[NWMAX], (*u)[NGMAX];
} olos_t;

static olos_t *los_new(void) {
  olos_t *l = (olos_t *)calloc(1, sizeof(olos_t));
  l->z = (double *)malloc(sizeof(double) * NLOS);
  l->lon = (double *)malloc(sizeof(double) * NLOS);
  l->lat = (double *)malloc(sizeof(double) * NLOS);
  l->p = (double *)malloc(sizeof(double) * NLOS);
  l->t = (double *)malloc(sizeof(double) * NLOS);
  l->ds = (double *)malloc(sizeof(double) * NLOS);
  l->aerofac = (double *)calloc(NLOS, sizeof(double));
  l->aeroi = (int *)calloc(NLOS, sizeof(int));
  l->q = malloc(sizeof(double) * NLOS * NGMAX);
  l->k = malloc(sizeof(double) * NLOS * NWMAX);
  l->u = malloc(sizeof(double) * NLOS * NGMAX);
  return l;
}

static void los_free(olos_t *l) {
  if (!l) return;
  free(l->z); free(l->lon); free(l->lat); free(l->p); free(l->t); free(l->ds);
  free(l->aerofac); free(l->aeroi); free(l->q); free(l->k); free(l->u);
  free(l);
}

/* src/lineofsight.c:385-407 */
static void o_intersection(const ctl_t *ctl, const atm_t *atm, double znew,
                           const olos_t *los, int ip, olos_t *dst, int jp) {
  double x1[3], x2[3];
  double frac = (los->z[ip - 1] - znew) / (los->z[ip - 1] - los->z[ip]);
  o_geo2cart(los->z[ip - 1], los->lon[ip - 1], los->lat[ip - 1], x1);
  o_geo2cart(los->z[ip], los->lon[ip], los->lat[ip], x2);
  for (int i = 0; i < 3; i++) x2[i] = x1[i] + frac * (x2[i] - x1[i]);
  o_cart2geo(x2, &dst->z[jp], &dst->lon[jp], &dst->lat[jp]);
  o_intpol_atm(ctl, atm, dst->z[jp], &dst->p[jp], &dst->t[jp], dst->q[jp], dst->k[jp]);
}

/* src/lineofsight.c:411-452 */
static void o_tangent_point(const olos_t *los, double *tpz, double *tplon, double *tplat) {
  size_t ip = 0;
  double mn = los->z[0];
  for (size_t i = 0; i < (size_t)los->np; i++) {
    if (los->z[i] < mn) { mn = los->z[i]; ip = i; }
    if (isnan(los->z[i])) { ip = i; break; }
  }
  if (ip <= 0 || ip >= (size_t)los->np - 1) {
    *tpz = los->z[los->np - 1];
    *tplon = los->lon[los->np - 1];
    *tplat = los->lat[los->np - 1];
  } else {
    double yy0 = los->z[ip - 1], yy1 = los->z[ip], yy2 = los->z[ip + 1], dummy;
    double x1 = sqrt(los->ds[ip] * los->ds[ip] - (yy1 - yy0) * (yy1 - yy0));
    double x2 = x1 + sqrt(los->ds[ip + 1] * los->ds[ip + 1] - (yy2 - yy1) * (yy2 - yy1));
    double a = 1 / (x1 - x2) * (-(yy0 - yy1) / x1 + (yy0 - yy2) / x2);
    double b = -(yy0 - yy1) / x1 - a * x1, c = yy0, x = -b / (2 * a);
    double v[3], v0[3], v2[3];
    *tpz = a * x * x + b * x + c;
    o_geo2cart(los->z[ip - 1], los->lon[ip - 1], los->lat[ip - 1], v0);
    o_geo2cart(los->z[ip + 1], los->lon[ip + 1], los->lat[ip + 1], v2);
    for (int i = 0; i < 3; i++) v[i] = LINV(0.0, v0[i], x2, v2[i], x);
    o_cart2geo(v, &dummy, tplon, tplat);
  }
}

static int o_add_aerosol_layers(const ctl_t *ctl, const atm_t *atm, olos_t *los,
                                const aero_t *aero);

/* src/lineofsight.c:5-190 */
static int o_raytrace(const ctl_t *ctl, const atm_t *atm, obs_t *obs, const aero_t *aero,
                      olos_t *los, int ir) {
  double cosa, d, dmax, dmin = 0, ds, ex0[3], ex1[3], h = 0.02, k[NWMAX], lat, lon,
         n, naux, ng[3], norm, p = 0, q[NGMAX], t = 0, x[3], xh[3], xobs[3], xvp[3],
         z = 1e99, zmax, zmin, zrefrac = 60;
  int stop = 0;
  los->np = 0;
  los->tsurf = -999;
  obs->tpz[ir] = obs->vpz[ir];
  obs->tplon[ir] = obs->vplon[ir];
  obs->tplat[ir] = obs->vplat[ir];
  zmin = zmax = atm->z[0];
  for (int i = 0; i < atm->np; i++) {
    if (atm->z[i] < zmin) zmin = atm->z[i];
    if (atm->z[i] > zmax) zmax = atm->z[i];
  }
  if (obs->obsz[ir] < zmin) return JSC_ERR_OBSERVER;
  if (obs->vpz[ir] > zmax - 0.001) return 0;
  o_geo2cart(obs->obsz[ir], obs->obslon[ir], obs->obslat[ir], xobs);
  o_geo2cart(obs->vpz[ir], obs->vplon[ir], obs->vplat[ir], xvp);
  for (int i = 0; i < 3; i++) ex0[i] = xvp[i] - xobs[i];
  norm = NRM(ex0);
  for (int i = 0; i < 3; i++) ex0[i] /= norm;
  for (int i = 0; i < 3; i++) x[i] = xobs[i];
  if (obs->obsz[ir] > zmax) {
    dmax = norm;
    while (fabs(dmin - dmax) > 0.001) {
      d = (dmax + dmin) / 2;
      for (int i = 0; i < 3; i++) x[i] = xobs[i] + d * ex0[i];
      o_cart2geo(x, &z, &lon, &lat);
      if (z <= zmax && z > zmax - 0.001) break;
      if (z < zmax - 0.0005) dmax = d; else dmin = d;
    }
  }
  while (1) {
    ds = ctl->rayds;
    if (ctl->raydz > 0) {
      norm = NRM(x);
      for (int i = 0; i < 3; i++) xh[i] = x[i] / norm;
      cosa = fabs(DOT(ex0, xh));
      if (cosa != 0) ds = MIN(ctl->rayds, ctl->raydz / cosa);
    }
    o_cart2geo(x, &z, &lon, &lat);
    if (los->np >= NLOS) return JSC_ERR_NLOS;
    if (z < zmin + 0.001 || z > zmax + 0.001) {
      stop = (z < zmin + 0.001 ? 2 : 1);
      los->z[los->np] = z;
      los->lon[los->np] = lon;
      los->lat[los->np] = lat;
      if (los->np > 0)
        o_intersection(ctl, atm, (stop == 2 ? zmin : zmax), los, los->np, los, los->np);
      else  /* the reference reads before the LOS here; keep the point */
        o_intpol_atm(ctl, atm, z, &los->p[0], &los->t[0], los->q[0], los->k[0]);
      los->ds[los->np] = 0.;
    }
    if (stop == 0) {
      o_intpol_atm(ctl, atm, z, &p, &t, q, k);
      los->lon[los->np] = lon;
      los->lat[los->np] = lat;
      los->z[los->np] = z;
      los->p[los->np] = p;
      los->t[los->np] = t;
      for (int ig = 0; ig < ctl->ng; ig++) los->q[los->np][ig] = q[ig];
      for (int iw = 0; iw < ctl->nw; iw++) los->k[los->np][iw] = k[iw];
      los->ds[los->np] = ds;
    }
    los->np++;
    if (stop) {
      los->tsurf = (stop == 2 ? t : -999);
      break;
    }
    n = (ctl->refrac && z <= zrefrac) ? 1 + 7.753e-05 * p / t : 1;
    for (int i = 0; i < 3; i++) ex1[i] = ex0[i] * n;
    if (ctl->refrac && z <= zrefrac) {
      for (int i = 0; i < 3; i++) xh[i] = x[i] + 0.5 * ds * ex0[i];
      o_cart2geo(xh, &z, &lon, &lat);
      o_intpol_atm(ctl, atm, z, &p, &t, NULL, NULL);
      n = 7.753e-05 * p / t;
      for (int i = 0; i < 3; i++) {
        xh[i] += h;
        o_cart2geo(xh, &z, &lon, &lat);
        o_intpol_atm(ctl, atm, z, &p, &t, NULL, NULL);
        naux = 7.753e-05 * p / t;
        ng[i] = (naux - n) / h;
        xh[i] -= h;
      }
    } else
      for (int i = 0; i < 3; i++) ng[i] = 0;
    for (int i = 0; i < 3; i++) ex1[i] += ds * ng[i];
    norm = NRM(ex1);
    for (int i = 0; i < 3; i++) ex1[i] /= norm;
    for (int i = 0; i < 3; i++) x[i] += 0.5 * ds * (ex0[i] + ex1[i]);
    for (int i = 0; i < 3; i++) ex0[i] = ex1[i];
  }
  if (los->np > 2 && los->ds[los->np - 2] < 1e-3) los->np--;
  o_tangent_point(los, &obs->tpz[ir], &obs->tplon[ir], &obs->tplat[ir]);
  los->ds[0] = 0.5 * los->ds[0];
  for (int ip = 1; ip < los->np; ip++) los->ds[ip] = 0.5 * (los->ds[ip - 1] + los->ds[ip]);
  for (int ip = 0; ip < los->np; ip++)
    for (int ig = 0; ig < ctl->ng; ig++)
      los->u[ip][ig] = 10 * los->q[ip][ig] * los->p[ip] / (JSC_KBOLTZ * los->t[ip]) * los->ds[ip];
  for (int ip = 0; ip < los->np; ip++) {
    los->aerofac[ip] = 0;   /* the reference leaves these unset in clear air */
    los->aeroi[ip] = -999;
  }
  if (ctl->sca_n > 0) return o_add_aerosol_layers(ctl, atm, los, aero);
  return 0;
}

static int cmp_desc(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return (x < y) - (x > y);
}

#define DIST3(a, b) sqrt(((a)[0] - (b)[0]) * ((a)[0] - (b)[0]) + ((a)[1] - (b)[1]) * ((a)[1] - (b)[1]) + \
                         ((a)[2] - (b)[2]) * ((a)[2] - (b)[2]))

/* Extra LOS points at the aerosol/cloud layer edges and through the
 * transition layers, chord step lengths, layer index and scaling factor
 * per point (src/lineofsight.c:193-372). */
static int o_add_aerosol_layers(const ctl_t *ctl, const atm_t *atm, olos_t *los,
                                const aero_t *aero) {
  double alti[4 * NLMAX + 2 * 1000], altimax, altimin, x1[3], x2[3], x3[3], eps = 0.005;
  int jl = 0;
  for (int il = 0; il < aero->nl; il++) {
    alti[jl] = aero->top[il] + eps;
    alti[jl + 1] = aero->top[il] - eps;
    alti[jl + 2] = aero->bottom[il] + eps;
    alti[jl + 3] = aero->bottom[il] - eps;
    jl += 4;
    if (aero->trans[il] > ctl->transs) {
      double tt = aero->trans[il] / ctl->transs;
      alti[jl] = aero->top[il] + aero->trans[il] + eps;
      alti[jl + 1] = aero->top[il] + aero->trans[il] - eps;
      alti[jl + 2] = aero->bottom[il] - aero->trans[il] + eps;
      alti[jl + 3] = aero->bottom[il] - aero->trans[il] - eps;
      jl += 4;
      for (int it = 1; it < (int)tt; it++) {
        if (jl + 2 > (int)(sizeof(alti) / sizeof(alti[0]))) return JSC_ERR_NLOS;
        alti[jl++] = aero->top[il] + aero->trans[il] - eps - it * ctl->transs;
        alti[jl++] = aero->bottom[il] - aero->trans[il] + eps + it * ctl->transs;
      }
    }
  }
  /* top-down order (the reference negates, sorts ascending, negates) */
  qsort(alti, (size_t)jl, sizeof(double), cmp_desc);
  altimax = alti[0];
  altimin = alti[0];
  for (int i = 0; i < jl; i++) {
    if (alti[i] > altimax) altimax = alti[i];
    if (alti[i] < altimin) altimin = alti[i];
  }
  olos_t *la = los_new();
  la->tsurf = los->tsurf;
  la->z[0] = los->z[0];
  la->lat[0] = los->lat[0];
  la->lon[0] = los->lon[0];
  la->ds[0] = los->ds[0];
  la->t[0] = los->t[0];
  la->p[0] = los->p[0];
  for (int ig = 0; ig < ctl->ng; ig++) la->q[0][ig] = los->q[0][ig];
  for (int iw = 0; iw < ctl->nw; iw++) la->k[0][iw] = los->k[0][iw];
  la->np = 1;
  for (int ip = 1; ip < los->np; ip++) {
    if ((los->z[ip - 1] < altimax || los->z[ip] < altimax) &&
        (los->z[ip - 1] > altimin || los->z[ip] > altimin)) {
      for (int il = 0; il < jl; il++) {
        if (los->z[ip - 1] > alti[il] && los->z[ip] < alti[il]) {
          if (la->np >= NLOS) { los_free(la); return JSC_ERR_NLOS; }
          o_intersection(ctl, atm, alti[il], los, ip, la, la->np);
          la->np++;
        }
        if (los->z[ip - 1] < alti[jl - il - 1] && los->z[ip] > alti[jl - il - 1]) {
          if (la->np >= NLOS) { los_free(la); return JSC_ERR_NLOS; }
          o_intersection(ctl, atm, alti[jl - il - 1], los, ip, la, la->np);
          la->np++;
        }
      }
    }
    if (la->np >= NLOS) { los_free(la); return JSC_ERR_NLOS; }
    la->z[la->np] = los->z[ip];
    la->lat[la->np] = los->lat[ip];
    la->lon[la->np] = los->lon[ip];
    la->t[la->np] = los->t[ip];
    la->p[la->np] = los->p[ip];
    for (int ig = 0; ig < ctl->ng; ig++) la->q[la->np][ig] = los->q[ip][ig];
    for (int iw = 0; iw < ctl->nw; iw++) la->k[la->np][iw] = los->k[ip][iw];
    la->np++;
  }
  o_geo2cart(la->z[0], la->lon[0], la->lat[0], x1);
  o_geo2cart(la->z[1], la->lon[1], la->lat[1], x2);
  la->ds[0] = 0.5 * (DIST3(x1, x2));
  for (int ip = 1; ip < la->np - 1; ip++) {
    o_geo2cart(la->z[ip - 1], la->lon[ip - 1], la->lat[ip - 1], x1);
    o_geo2cart(la->z[ip], la->lon[ip], la->lat[ip], x2);
    o_geo2cart(la->z[ip + 1], la->lon[ip + 1], la->lat[ip + 1], x3);
    la->ds[ip] = 0.5 * (DIST3(x1, x2) + DIST3(x2, x3));
  }
  o_geo2cart(la->z[la->np - 1], la->lon[la->np - 1], la->lat[la->np - 1], x1);
  o_geo2cart(la->z[la->np - 2], la->lon[la->np - 2], la->lat[la->np - 2], x2);
  la->ds[la->np - 1] = 0.5 * (DIST3(x1, x2));
  for (int ip = 0; ip < la->np; ip++) {
    for (int ig = 0; ig < ctl->ng; ig++)
      la->u[ip][ig] = 10 * la->q[ip][ig] * la->p[ip] / (JSC_KBOLTZ * la->t[ip]) * la->ds[ip];
    la->aeroi[ip] = -999;
    la->aerofac[ip] = 0.;
    /* at ip = 0 the reference reads z[-1]; z[0] stands in (the first
     * point lies at the top of the atmosphere, outside every layer) */
    double zprev = la->z[ip > 0 ? ip - 1 : 0];
    if ((zprev < altimax || la->z[ip] < altimax) && (zprev > altimin || la->z[ip] > altimin)) {
      for (int il = 0; il < aero->nl; il++) {
        if (la->z[ip] <= aero->top[il] && la->z[ip] >= aero->bottom[il]) {
          la->aeroi[ip] = il;
          la->aerofac[ip] = 1.;
        }
        if (aero->trans[il] > ctl->transs && la->z[ip] <= (aero->top[il] + aero->trans[il]) &&
            la->z[ip] > aero->top[il]) {
          la->aeroi[ip] = il;
          la->aerofac[ip] = (aero->top[il] + aero->trans[il] - la->z[ip]) / aero->trans[il];
        }
        if (aero->trans[il] > ctl->transs && la->z[ip] < aero->bottom[il] &&
            la->z[ip] >= (aero->bottom[il] - aero->trans[il])) {
          la->aeroi[ip] = il;
          la->aerofac[ip] = fabs(aero->bottom[il] - aero->trans[il] - la->z[ip]) / aero->trans[il];
        }
      }
    }
  }
  /* copy back */
  los->np = la->np;
  los->tsurf = la->tsurf;
  memcpy(los->z, la->z, sizeof(double) * NLOS);
  memcpy(los->lon, la->lon, sizeof(double) * NLOS);
  memcpy(los->lat, la->lat, sizeof(double) * NLOS);
  memcpy(los->p, la->p, sizeof(double) * NLOS);
  memcpy(los->t, la->t, sizeof(double) * NLOS);
  memcpy(los->ds, la->ds, sizeof(double) * NLOS);
  memcpy(los->aerofac, la->aerofac, sizeof(double) * NLOS);
  memcpy(los->aeroi, la->aeroi, sizeof(int) * NLOS);
  memcpy(los->q, la->q, sizeof(double) * NLOS * NGMAX);
  memcpy(los->k, la->k, sizeof(double) * NLOS * NWMAX);
  memcpy(los->u, la->u, sizeof(double) * NLOS * NGMAX);
  los_free(la);
  return 0;
}

/* ------------------------------------------------------------- tables -- */

typedef struct {
  int np;
  double p[TBLNPMAX];
  int nt[TBLNPMAX];
  double t[TBLNPMAX][TBLNTMAX];
  int nu[TBLNPMAX][TBLNTMAX];
  float *u[TBLNPMAX][TBLNTMAX], *eps[TBLNPMAX][TBLNTMAX];
} otab_t;

static otab_t *g_tab;            /* [nd][ng] */
static double *g_planck;         /* [nd][1201] */
static ctl_t g_key;
static int g_init;

/* Binary table (src/forwardmodel.c:630-656). */
static int read_bin(FILE *in, otab_t *tb) {
#define RDN(p, s, n) if (fread((p), (s), (size_t)(n), in) != (size_t)(n)) return JSC_ERR_FILE
  RDN(&tb->np, sizeof(int), 1);
  if (tb->np > TBLNPMAX) return JSC_ERR_TABLE;
  RDN(tb->p, sizeof(double), tb->np);
  RDN(tb->nt, sizeof(int), tb->np);
  for (int ip = 0; ip < tb->np; ip++) {
    if (tb->nt[ip] > TBLNTMAX) return JSC_ERR_TABLE;
    RDN(tb->t[ip], sizeof(double), tb->nt[ip]);
    RDN(tb->nu[ip], sizeof(int), tb->nt[ip]);
    for (int it = 0; it < tb->nt[ip]; it++) {
      int n = tb->nu[ip][it];
      if (n > TBLNUMAX) return JSC_ERR_TABLE;
      tb->u[ip][it] = (float *)malloc(sizeof(float) * (n > 0 ? n : 1));
      tb->eps[ip][it] = (float *)malloc(sizeof(float) * (n > 0 ? n : 1));
      RDN(tb->u[ip][it], sizeof(float), n);
      RDN(tb->eps[ip][it], sizeof(float), n);
    }
  }
  return 0;
#undef RDN
}

/* ASCII table (src/forwardmodel.c:661-733). */
static int read_tab(FILE *in, otab_t *tb) {
  char line[LEN];
  double press, temp, u, eps, eps_old = -999, press_old = -999, temp_old = -999, u_old = -999;
  static float bu[TBLNPMAX][TBLNTMAX][TBLNUMAX], be[TBLNPMAX][TBLNTMAX][TBLNUMAX];
  tb->np = -1;
  while (fgets(line, LEN, in)) {
    if (sscanf(line, "%lg %lg %lg %lg", &press, &temp, &u, &eps) != 4) continue;
    if (press != press_old) {
      press_old = press;
      if (++tb->np >= TBLNPMAX) return JSC_ERR_TABLE;
      tb->nt[tb->np] = -1;
    }
    if (temp != temp_old || tb->nt[tb->np] < 0) {
      temp_old = temp;
      if (++tb->nt[tb->np] >= TBLNTMAX) return JSC_ERR_TABLE;
      tb->nu[tb->np][tb->nt[tb->np]] = -1;
    }
    int *nu = &tb->nu[tb->np][tb->nt[tb->np]];
    if ((eps > eps_old && u > u_old) || *nu < 0) {
      eps_old = eps;
      u_old = u;
      if (++(*nu) >= TBLNUMAX) {
        (*nu)--;
        continue;
      }
    }
    tb->p[tb->np] = press;
    tb->t[tb->np][tb->nt[tb->np]] = temp;
    bu[tb->np][tb->nt[tb->np]][*nu] = (float)u;
    be[tb->np][tb->nt[tb->np]][*nu] = (float)eps;
  }
  tb->np++;
  for (int ip = 0; ip < tb->np; ip++) {
    tb->nt[ip]++;
    for (int it = 0; it < tb->nt[ip]; it++) {
      int n = ++tb->nu[ip][it];
      tb->u[ip][it] = (float *)malloc(sizeof(float) * (n > 0 ? n : 1));
      tb->eps[ip][it] = (float *)malloc(sizeof(float) * (n > 0 ? n : 1));
      memcpy(tb->u[ip][it], bu[ip][it], sizeof(float) * n);
      memcpy(tb->eps[ip][it], be[ip][it], sizeof(float) * n);
    }
  }
  return 0;
}

void oracle_reset(void) {
  if (g_tab) {
    for (int i = 0; i < g_key.nd * g_key.ng; i++)
      for (int ip = 0; ip < g_tab[i].np; ip++)
        for (int it = 0; it < g_tab[i].nt[ip]; it++) {
          free(g_tab[i].u[ip][it]);
          free(g_tab[i].eps[ip][it]);
        }
    free(g_tab);
  }
  free(g_planck);
  g_tab = NULL;
  g_planck = NULL;
  g_init = 0;
}

/* read_tbl (src/forwardmodel.c:610-739) and the Planck table of
 * srcfunc_planck (src/forwardmodel.c:757-786). */
static int load_tables(const ctl_t *ctl) {
  char fn[2 * LEN + 64];
  if (g_init && g_key.nd == ctl->nd && g_key.ng == ctl->ng &&
      !strcmp(g_key.tblbase, ctl->tblbase) &&
      !memcmp(g_key.nu, ctl->nu, sizeof(ctl->nu)) &&
      !memcmp(g_key.emitter, ctl->emitter, sizeof(ctl->emitter)))
    return 0;
  oracle_reset();
  memcpy(&g_key, ctl, sizeof(ctl_t));
  g_tab = (otab_t *)calloc((size_t)(ctl->nd * ctl->ng + 1), sizeof(otab_t));
  for (int id = 0; id < ctl->nd; id++)
    for (int ig = 0; ig < ctl->ng; ig++) {
      otab_t *tb = &g_tab[id * ctl->ng + ig];
      int st;
      snprintf(fn, sizeof(fn), "%s_%.4f_%s.bin", ctl->tblbase, ctl->nu[id], ctl->emitter[ig]);
      FILE *in = fopen(fn, "r");
      if (in) {
        st = read_bin(in, tb);
        fclose(in);
      } else {
        snprintf(fn, sizeof(fn), "%s_%.4f_%s.tab", ctl->tblbase, ctl->nu[id], ctl->emitter[ig]);
        in = fopen(fn, "r");
        if (!in) {
          tb->np = -1;
          continue;
        }
        st = read_tab(in, tb);
        fclose(in);
      }
      if (st) return st;
    }
  g_planck = (double *)malloc(sizeof(double) * (size_t)ctl->nd * JSC_NPLANCK_O);
  for (int id = 0; id < ctl->nd; id++) {
    static double fx[NSHAPE], fy[NSHAPE];
    char line[LEN];
    int n = 0;
    snprintf(fn, sizeof(fn), "%s_%.4f.filt", ctl->tblbase, ctl->nu[id]);
    FILE *in = fopen(fn, "r");
    if (!in) return JSC_ERR_FILE;
    while (fgets(line, LEN, in))
      if (n < NSHAPE && sscanf(line, "%lg %lg", &fx[n], &fy[n]) == 2) n++;
    fclose(in);
    if (n < 1) return JSC_ERR_FILE;
    for (int it = 0; it < JSC_NPLANCK_O; it++) {
      double temp = LINV(0.0, 100.0, JSC_NPLANCK_O - 1.0, 400.0, (double)it), fsum = 0, acc = 0;
      for (int i = 0; i < n; i++) {
        fsum += fy[i];
        acc += fy[i] * oracle_planck(temp, fx[i]);
      }
      g_planck[(size_t)id * JSC_NPLANCK_O + it] = acc / fsum;
    }
  }
  g_init = 1;
  return 0;
}

/* srcfunc_planck lookup (src/forwardmodel.c:788-793). */
static void o_srcfunc_planck(const ctl_t *ctl, double t, double *src) {
  static double temp[JSC_NPLANCK_O];
  static int tinit = 0;
  if (!tinit) {
    for (int it = 0; it < JSC_NPLANCK_O; it++)
      temp[it] = LINV(0.0, 100.0, JSC_NPLANCK_O - 1.0, 400.0, (double)it);
    tinit = 1;
  }
  int it = o_locate(temp, JSC_NPLANCK_O, t);
  for (int id = 0; id < ctl->nd; id++) {
    const double *b = g_planck + (size_t)id * JSC_NPLANCK_O;
    src[id] = LINV(temp[it], b[it], temp[it + 1], b[it + 1], t);
  }
}

/* --------------------------------------------------------- intpol_tbl -- */

/* LIN on float table entries: C evaluates (y1-y0)/(x1-x0) in single
 * precision before the product with the double (x-x0) promotes it. */
static double o_lin_f(float x0, float y0, float x1, float y1, double x) {
  float slope = (y1 - y0) / (x1 - x0);
  return (double)y0 + (double)slope * (x - (double)x0);
}

/* intpol_tbl_eps / intpol_tbl_u (src/forwardmodel.c:506-542). */
static double o_tbl_eps(const otab_t *tb, int ip, int it, double u, uint64_t *dig) {
  int idx = o_locate_tbl(tb->u[ip][it], tb->nu[ip][it], u);
  if (dig) *dig = *dig * 1000003u + (uint64_t)idx;
  return o_lin_f(tb->u[ip][it][idx], tb->eps[ip][it][idx],
                 tb->u[ip][it][idx + 1], tb->eps[ip][it][idx + 1], u);
}

static double o_tbl_u(const otab_t *tb, int ip, int it, double eps, uint64_t *dig) {
  int idx = o_locate_tbl(tb->eps[ip][it], tb->nu[ip][it], eps);
  if (dig) *dig = *dig * 1000003u + (uint64_t)idx;
  return o_lin_f(tb->eps[ip][it][idx], tb->u[ip][it][idx],
                 tb->eps[ip][it][idx + 1], tb->u[ip][it][idx + 1], eps);
}

#define CLAMP01(e) MAX(MIN((e), 1), 0)

/* src/forwardmodel.c:409-502.  digs (optional, [nd][ng]) accumulate, per
 * channel and emitter, every table index the interpolation selects. */
static void o_intpol_tbl(const ctl_t *ctl, const olos_t *los, int ip,
                         double tau_path[NGMAX][NDMAX], double *tau_seg, uint64_t *digs) {
  if (ip <= 0)
    for (int ig = 0; ig < ctl->ng; ig++)
      for (int id = 0; id < ctl->nd; id++) tau_path[ig][id] = 1;
  for (int id = 0; id < ctl->nd; id++) {
    tau_seg[id] = 1;
    for (int ig = 0; ig < ctl->ng; ig++) {
      uint64_t *dig = digs ? &digs[id * ctl->ng + ig] : NULL;
      const otab_t *tb = &g_tab[id * ctl->ng + ig];
      double eps;
      if (tb->np < 2)
        eps = 0;
      else if (tau_path[ig][id] < 1e-9)
        eps = 1;
      else {
        int ipr = o_locate(tb->p, tb->np, los->p[ip]);
        int it0 = o_locate(tb->t[ipr], tb->nt[ipr], los->t[ip]);
        int it1 = o_locate(tb->t[ipr + 1], tb->nt[ipr + 1], los->t[ip]);
        if (tb->nt[ipr] < 2 || tb->nt[ipr + 1] < 2 || tb->nu[ipr][it0] < 2 ||
            tb->nu[ipr][it0 + 1] < 2 || tb->nu[ipr + 1][it1] < 2 || tb->nu[ipr + 1][it1 + 1] < 2)
          eps = 0;
        else {
          if (dig) *dig = *dig * 1000003u + (uint64_t)(ipr * 961 + it0 * 31 + it1);
          double x = 1 - tau_path[ig][id], us = los->u[ip][ig], u, e00, e01, e10, e11;
          /* assign, then clamp (the clamp macro evaluates its argument
           * more than once) */
          u = o_tbl_u(tb, ipr, it0, x, dig);
          e00 = o_tbl_eps(tb, ipr, it0, u + us, dig);
          e00 = CLAMP01(e00);
          u = o_tbl_u(tb, ipr, it0 + 1, x, dig);
          e01 = o_tbl_eps(tb, ipr, it0 + 1, u + us, dig);
          e01 = CLAMP01(e01);
          u = o_tbl_u(tb, ipr + 1, it1, x, dig);
          e10 = o_tbl_eps(tb, ipr + 1, it1, u + us, dig);
          e10 = CLAMP01(e10);
          u = o_tbl_u(tb, ipr + 1, it1 + 1, x, dig);
          e11 = o_tbl_eps(tb, ipr + 1, it1 + 1, u + us, dig);
          e11 = CLAMP01(e11);
          e00 = LINV(tb->t[ipr][it0], e00, tb->t[ipr][it0 + 1], e01, los->t[ip]);
          e00 = CLAMP01(e00);
          e11 = LINV(tb->t[ipr + 1][it1], e10, tb->t[ipr + 1][it1 + 1], e11, los->t[ip]);
          e11 = CLAMP01(e11);
          e00 = LINV(tb->p[ipr], e00, tb->p[ipr + 1], e11, los->p[ip]);
          e00 = CLAMP01(e00);
          eps = 1 - (1 - e00) / tau_path[ig][id];
        }
      }
      tau_path[ig][id] *= (1 - eps);
      tau_seg[id] *= (1 - eps);
    }
  }
}

/* ----------------------------------------------------------- continua -- */

/* src/continua.c:5-872 */
static double o_ctmco2(const ctl_t *ctl, double nu, double p, double t, const double *u) {
  int ig = o_find_emitter(ctl, "CO2");
  if (ig < 0) return 0;
  double xw = nu / 2 + 1;
  if (!(xw >= 1 && xw < 2001)) return 0;
  int iw = (int)xw, jw = iw + 1;
  double dw = xw - iw, ew = 1 - dw;
  double cw296 = ew * jsc_ckd_co2_t296[iw - 1] + dw * jsc_ckd_co2_t296[jw - 1];
  double cw260 = ew * jsc_ckd_co2_t260[iw - 1] + dw * jsc_ckd_co2_t260[jw - 1];
  double cw230 = ew * jsc_ckd_co2_t230[iw - 1] + dw * jsc_ckd_co2_t230[jw - 1];
  double dt230 = t - 230, dt260 = t - 260, dt296 = t - 296;
  double ctw = dt260 * 5.050505e-4 * dt296 * cw230 - dt230 * 9.259259e-4 * dt296 * cw260 +
               dt230 * 4.208754e-4 * dt260 * cw296;
  return u[ig] / JSC_AVOGADRO / 1000 * p / JSC_P0 * ctw;
}

/* src/continua.c:876-1931 */
static double o_ctmh2o(const ctl_t *ctl, double nu, double p, double t, const double *q,
                       const double *u) {
  int ig = o_find_emitter(ctl, "H2O");
  if (ig < 0) return 0;
  double xw = nu / 10 + 1;
  if (!(xw >= 1 && xw < 2001)) return 0;
  int iw = (int)xw, jw = iw + 1;
  double dw = xw - iw, ew = 1 - dw, sfac;
  double cw296 = ew * jsc_ckd_h2o_t296[iw - 1] + dw * jsc_ckd_h2o_t296[jw - 1];
  double cw260 = ew * jsc_ckd_h2o_t260[iw - 1] + dw * jsc_ckd_h2o_t260[jw - 1];
  double cwfrn = ew * jsc_ckd_h2o_frn[iw - 1] + dw * jsc_ckd_h2o_frn[jw - 1];
  if (nu <= 820 || nu >= 960)
    sfac = 1;
  else {
    double xx = (nu - 820) / 10, dx;
    int ix = (int)xx;
    dx = xx - ix;
    sfac = (1 - dx) * jsc_ckd_h2o_xfc[ix] + dx * jsc_ckd_h2o_xfc[ix + 1];
  }
  double ctwslf = sfac * cw296 * pow(cw260 / cw296, (296 - t) / (296 - 260));
  double vf2 = (nu - 370) * (nu - 370), vf6 = vf2 * vf2 * vf2;
  double fscal = 36100 / (vf2 + vf6 * 1e-8 + 36100) * -.25 + 1;
  double ctwfrn = cwfrn * fscal;
  double a1 = nu * u[ig] * tanh(.7193876 / t * nu), a2 = 296 / t;
  double a3 = p / JSC_P0 * (q[ig] * ctwslf + (1 - q[ig]) * ctwfrn) * 1e-20;
  return a1 * a2 * a3;
}

/* src/continua.c:1935-1993 and :1997-2049 */
static double o_ctmn2o2(double nu, double p, double t, int o2) {
  const double *nua = o2 ? jsc_o2_nu : jsc_n2_nu, *ba = o2 ? jsc_o2_b : jsc_n2_b,
               *betaa = o2 ? jsc_o2_beta : jsc_n2_beta;
  int n = o2 ? 90 : 98;
  double t0 = 273, tr = 296, qx = o2 ? 0.21 : 0.79;
  if (nu < nua[0] || nu > nua[n - 1]) return 0;
  int idx = o_locate(nua, n, nu);
  double b = LINV(nua[idx], ba[idx], nua[idx + 1], ba[idx + 1], nu);
  double beta = LINV(nua[idx], betaa[idx], nua[idx + 1], betaa[idx + 1], nu);
  double pp = p / JSC_P0, tt = t0 / t;
  if (o2) return 0.1 * (pp * pp) * (tt * tt) * qx * b * exp(beta * (1 / tr - 1 / t));
  return 0.1 * (pp * pp) * (tt * tt) * qx * b * exp(beta * (1 / tr - 1 / t)) *
         (qx + (1 - qx) * (1.294 - 0.4545 * t / tr));
}

/* src/forwardmodel.c:120-152 */
static void o_continua(const ctl_t *ctl, const olos_t *los, int ip, double *beta) {
  for (int id = 0; id < ctl->nd; id++) beta[id] = los->k[ip][ctl->window[id]];
  if (ctl->ctm_co2)
    for (int id = 0; id < ctl->nd; id++)
      beta[id] += o_ctmco2(ctl, ctl->nu[id], los->p[ip], los->t[ip], los->u[ip]) / los->ds[ip];
  if (ctl->ctm_h2o)
    for (int id = 0; id < ctl->nd; id++)
      beta[id] += o_ctmh2o(ctl, ctl->nu[id], los->p[ip], los->t[ip], los->q[ip], los->u[ip]) /
                  los->ds[ip];
  if (ctl->ctm_n2)
    for (int id = 0; id < ctl->nd; id++) beta[id] += o_ctmn2o2(ctl->nu[id], los->p[ip], los->t[ip], 0);
  if (ctl->ctm_o2)
    for (int id = 0; id < ctl->nd; id++) beta[id] += o_ctmn2o2(ctl->nu[id], los->p[ip], los->t[ip], 1);
}

/* ------------------------------------------------------------ formod -- */

static int o_pencil(const ctl_t *ctl, const atm_t *atm, obs_t *obs, const aero_t *aero,
                    int scattering, int ir, uint64_t *dig, int *nlos);

/* Orthonormal basis with ez along dz (src/scatter.c:6-52). */
static void o_bascoord(const double *dz, const double *dy, double *ex, double *ey, double *ez) {
  double dotp, norm = NRM(dz);
  for (int i = 0; i < 3; i++) ez[i] = dz[i] / norm;
  norm = NRM(dy);
  for (int i = 0; i < 3; i++) ey[i] = dy[i] / norm;
  dotp = DOT(ey, ez);
  if (dotp == 1) {
    ey[0] = 1;
    ey[1] = 0;
    ey[2] = 0;
    dotp = ez[0];
    if (dotp == 1) {
      ey[0] = 0;
      ey[1] = 1;
      dotp = ez[1];
    }
  }
  for (int i = 0; i < 3; i++) ey[i] -= dotp * ez[i];
  norm = NRM(ey);
  for (int i = 0; i < 3; i++) ey[i] /= norm;
  ex[0] = ey[1] * ez[2] - ey[2] * ez[1];
  ex[1] = ey[2] * ez[0] - ey[0] * ez[2];
  ex[2] = ey[0] * ez[1] - ey[1] * ez[0];
}

/* ANGLE macro (src/jurassic.h:33-34). */
static double o_angle(const double *a, const double *b) {
  double c = DOT(a, b) / NRM(a) / NRM(b);
  return acos(MIN(MAX(c, -1), 1));
}

/* Zenith angles of the secondary pencils (src/scatter.c:698-715). */
static void o_sca_alpha(double *alpha, int nalpha) {
  int n1 = 1, n2 = 2;
  double midang = 83, up = 92, down = 81, step = 1 + 2;
  alpha[0] = 0;
  for (int ir = nalpha / 2 - 4; ir < nalpha / 2 + 4; ++ir) {
    alpha[ir] = midang * M_PI / 180.;
    midang++;
  }
  for (int ir = 0; ir < nalpha / 2 - 5; ++ir) {
    alpha[nalpha / 2 + ir + 4] = up * M_PI / 180.;
    alpha[nalpha / 2 - ir - 5] = down * M_PI / 180.;
    up += step;
    down -= step;
    if (step < 13) {
      step = (double)n1 + (double)n2;
      n1 = n2;
      n2 = (int)step;
    }
  }
  alpha[nalpha - 1] = M_PI;
}

/* Secondary pencils per scattering point: the reference's 28, or an even
 * count from 10 to 28 with the same angle construction (for checking the
 * GPU path's pencil-count option). */
static int g_nalpha = 28;
static int g_nalpha_at[8];  /* per scattering order (0: g_nalpha) */

int oracle_set_nalpha(int nalpha) {
  if (nalpha < 10 || nalpha > 28 || (nalpha & 1)) return JSC_ERR_ARG;
  g_nalpha = nalpha;
  for (int i = 0; i < 8; i++) g_nalpha_at[i] = 0;
  return 0;
}

/* Pencil count of the sources of one scattering order only. */
int oracle_set_nalpha_order(int order, int nalpha) {
  if (order < 1 || order > 7 || nalpha < 10 || nalpha > 28 || (nalpha & 1)) return JSC_ERR_ARG;
  g_nalpha_at[order] = nalpha;
  return 0;
}

/* Thermal single scattering in 1-D atmospheres (src/scatter.c:666-807):
 * 28 secondary pencils at fixed zenith angles, then the phase-function
 * weighted integral over 180 x 180 directions. */
static int o_srcfunc_sca_1d(const ctl_t *ctl, const atm_t *atm, const aero_t *aero,
                            const double *x, const double *dx, int il, double *src_sca,
                            int scattering) {
  enum { NPHI = 180, NTHETA2 = 180 };
  const int NALPHA = (scattering >= 1 && scattering < 8 && g_nalpha_at[scattering])
                        ? g_nalpha_at[scattering] : g_nalpha;
  double alpha[28], dnorth[3], ek[3], lx[3], ly[3], lz[3], sx[3], sy[3], sz[3],
         theta[NTHETA], wsum[NDMAX], xv[3], mlz[3];
  obs_t *obs2 = (obs_t *)calloc(1, sizeof(obs_t));
  int st = 0;
  for (int it = 0; it < NTHETA; it++) theta[it] = (double)it * M_PI / 180.;
  dnorth[0] = -x[0];
  dnorth[1] = -x[1];
  dnorth[2] = 2 * JSC_RE - x[2];
  o_bascoord(x, dnorth, lx, ly, lz);
  o_sca_alpha(alpha, NALPHA);
  for (int ir = 0; ir < NALPHA && !st; ir++) {
    for (int i = 0; i < 3; i++)
      xv[i] = x[i] + 10. * cos(alpha[ir]) * (-1) * lz[i] + 10. * sin(alpha[ir]) * ly[i];
    obs2->nr = NALPHA;
    o_cart2geo(x, &obs2->obsz[ir], &obs2->obslon[ir], &obs2->obslat[ir]);
    o_cart2geo(xv, &obs2->vpz[ir], &obs2->vplon[ir], &obs2->vplat[ir]);
    st = o_pencil(ctl, atm, obs2, aero, scattering - 1, ir, NULL, NULL);
  }
  o_bascoord(dx, x, sx, sy, sz);
  for (int id = 0; id < ctl->nd; id++) {
    src_sca[id] = 0;
    wsum[id] = 0;
  }
  for (int i = 0; i < 3; i++) mlz[i] = -1. * lz[i];
  for (int itheta = 0; itheta < NTHETA2; itheta++) {
    double theta2 = (0.5 + itheta) * M_PI / 180.;
    for (int iphi = 0; iphi < NPHI; iphi++) {
      double phi = 2. * (0.5 + iphi) * M_PI / 180.;
      for (int i = 0; i < 3; i++)
        ek[i] = sin(theta2) * sin(phi) * sx[i] + sin(theta2) * cos(phi) * sy[i] + cos(theta2) * sz[i];
      int idp = o_locate(theta, NTHETA, theta2);
      double alpha2 = o_angle(mlz, ek);
      int idx = o_locate(alpha, NALPHA, alpha2);
      for (int id = 0; id < ctl->nd; id++) {
        double phase2 = LINV(theta[idp], aero->p[il][id][idp], theta[idp + 1],
                             aero->p[il][id][idp + 1], theta2);
        double w = sin(theta2) * phase2;
        double rad = LINV(alpha[idx], obs2->rad[id][idx], alpha[idx + 1], obs2->rad[id][idx + 1],
                          alpha2);
        src_sca[id] += w * rad;
        wsum[id] += w;
      }
    }
  }
  for (int id = 0; id < ctl->nd; id++) src_sca[id] /= wsum[id];
  free(obs2);
  return st;
}

/* Solar position (src/scatter.c:999-1041). */
static void o_suncoord(double sec, double lon, double lat, double *azi, double *sza) {
  double D = sec / 86400 - 0.5;
  double g = (357.529 + 0.98560028 * D) * M_PI / 180;
  double q = 280.459 + 0.98564736 * D;
  double L = (q + 1.915 * sin(g) + 0.020 * sin(2 * g)) * M_PI / 180;
  double e = (23.439 - 0.00000036 * D) * M_PI / 180;
  double dec = asin(sin(e) * sin(L));
  double ra = atan2(cos(e) * sin(L), cos(L));
  double GMST = 18.697374558 + 24.06570982441908 * D;
  double LST = GMST + lon / 15;
  double h = LST / 12 * M_PI - ra;
  lat *= M_PI / 180;
  *azi = atan2(-sin(h), cos(lat) * tan(dec) - sin(lat) * cos(h)) * 180 / M_PI;
  *sza = acos(sin(lat) * sin(dec) + cos(lat) * cos(dec) * cos(h)) * 180 / M_PI;
}

/* Solar single scattering (src/scatter.c:899-995). */
static int o_srcfunc_sca_sun(const ctl_t *ctl, const atm_t *atm, const aero_t *aero, double sec,
                             const double *x, const double *dx, int il, double *src_sca) {
  double azi, dnorth[3], dout[3], ek[3], lx[3], ly[3], lz[3], sza, sza_beam, sza_cor,
         theta[NTHETA], x0[3], x1[3];
  olos_t *los = los_new();
  obs_t *obs = (obs_t *)calloc(1, sizeof(obs_t));
  int st = 0;
  for (int it = 0; it < NTHETA; it++) theta[it] = M_PI * (double)it / (NTHETA - 1);
  dnorth[0] = -x[0];
  dnorth[1] = -x[1];
  dnorth[2] = 2 * JSC_RE - x[2];
  o_bascoord(x, dnorth, lx, ly, lz);
  obs->nr = 1;
  o_cart2geo(x, &obs->obsz[0], &obs->obslon[0], &obs->obslat[0]);
  o_suncoord(sec, obs->obslon[0], obs->obslat[0], &azi, &sza);
  sza_cor = sza;
  for (int i2 = 0; i2 < 10; i2++) {
    for (int i = 0; i < 3; i++) {
      ek[i] = sin(sza_cor * M_PI / 180) * sin(azi * M_PI / 180) * lx[i] +
              sin(sza_cor * M_PI / 180) * cos(azi * M_PI / 180) * ly[i] +
              cos(sza_cor * M_PI / 180) * lz[i];
      x1[i] = x[i] + 10 * ek[i];
    }
    o_cart2geo(x1, &obs->vpz[0], &obs->vplon[0], &obs->vplat[0]);
    st = o_raytrace(ctl, atm, obs, aero, los, 0);
    if (st || los->np < 2) break;
    o_geo2cart(los->z[los->np - 2], los->lon[los->np - 2], los->lat[los->np - 2], x0);
    o_geo2cart(los->z[los->np - 1], los->lon[los->np - 1], los->lat[los->np - 1], x1);
    for (int i = 0; i < 3; i++) dout[i] = x1[i] - x0[i];
    sza_beam = o_angle(x, dout) * 180 / M_PI;
    if (fabs(sza_beam - sza) < 0.01) break;
    sza_cor -= 0.61803 * (sza_beam - sza);
    sza_cor = MIN(MAX(sza_cor, 0), 180);
  }
  if (!st && los->tsurf < 0) {
    st = o_pencil(ctl, atm, obs, aero, 0, 0, NULL, NULL);
    double theta2 = o_angle(ek, dx);
    int idx = o_locate(theta, NTHETA, theta2);
    for (int id = 0; id < ctl->nd; id++) {
      double phase2 = LINV(theta[idx], aero->p[il][id][idx], theta[idx + 1],
                           aero->p[il][id][idx + 1], theta2);
      src_sca[id] += 6.764e-5 * phase2 * oracle_planck(JSC_TSUN, ctl->nu[id]) * obs->tau[id][0];
    }
  }
  los_free(los);
  free(obs);
  return st;
}

/* Pencil beam (src/forwardmodel.c:224-405): trace, then EGA, continua,
 * Planck and radiative transfer per LOS point, with the scattering source
 * at aerosol points when scattering > 0. */
static int o_pencil(const ctl_t *ctl, const atm_t *atm, obs_t *obs, const aero_t *aero,
                    int scattering, int ir, uint64_t *dig, int *nlos) {
  double beta[NDMAX], src[NDMAX], tau_seg[NDMAX], src_sca[NDMAX], x[3], x0[3], x1[3], dx[3];
  double (*tau_path)[NDMAX] = malloc(sizeof(double) * NGMAX * NDMAX);
  olos_t *los = los_new();
  /* per (channel, emitter) index digests, folded per channel at the end */
  uint64_t *gdig = dig ? (uint64_t *)calloc((size_t)NDMAX * NGMAX, sizeof(uint64_t)) : NULL;
  int st = o_raytrace(ctl, atm, obs, aero, los, ir);
  const int beta_a = strcmp(ctl->sca_ext, "beta_a") == 0;
  if (nlos) *nlos = los->np;
  for (int id = 0; id < ctl->nd; id++) {
    obs->rad[id][ir] = 0;
    obs->tau[id][ir] = 1;
  }
  for (int ip = 0; ip < los->np && !st; ip++) {
    o_intpol_tbl(ctl, los, ip, tau_path, tau_seg, gdig);
    o_continua(ctl, los, ip, beta);
    o_srcfunc_planck(ctl, los->t[ip], src);
    const double af = los->aerofac[ip];
    const int ia = los->aeroi[ip];
    if (scattering > 0 && af > 0) {
      /* the reference's neighbour index is ip+1 even at the last point
       * (src/forwardmodel.c:323); the last point stands in for itself */
      int ip0 = (ip > 0 ? ip - 1 : ip), ip1 = (ip + 1 < los->np ? ip + 1 : ip);
      o_geo2cart(los->z[ip], los->lon[ip], los->lat[ip], x);
      o_geo2cart(los->z[ip0], los->lon[ip0], los->lat[ip0], x0);
      o_geo2cart(los->z[ip1], los->lon[ip1], los->lat[ip1], x1);
      for (int i = 0; i < 3; i++) dx[i] = x1[i] - x0[i];
      st = o_srcfunc_sca_1d(ctl, atm, aero, x, dx, ia, src_sca, scattering);
      if (!st && JSC_TSUN > 0)
        st = o_srcfunc_sca_sun(ctl, atm, aero, obs->time[ir], x, dx, ia, src_sca);
      for (int id = 0; id < ctl->nd; id++)
        if (tau_seg[id] > 0) {
          double bext = (-1.) * log(tau_seg[id]) / los->ds[ip] + beta[id] + af * aero->beta_e[ia][id];
          double eps = 1 - exp(-1 * bext * los->ds[ip]);
          double src_all = ((bext - af * aero->beta_s[ia][id]) * src[id] +
                            af * aero->beta_s[ia][id] * src_sca[id]) / bext;
          obs->rad[id][ir] += obs->tau[id][ir] * eps * src_all;
          obs->tau[id][ir] *= exp(-1. * bext * los->ds[ip]);
        }
    } else {
      for (int id = 0; id < ctl->nd; id++)
        if (tau_seg[id] > 0) {
          double eps;
          if (ctl->sca_n == 0 || af == 0)
            eps = 1 - tau_seg[id] * exp(-1. * beta[id] * los->ds[ip]);
          else if (beta_a)
            eps = 1 - tau_seg[id] * exp(-1. * (beta[id] + af * aero->beta_a[ia][id]) * los->ds[ip]);
          else
            eps = 1 - tau_seg[id] * exp(-1. * (beta[id] + af * aero->beta_e[ia][id]) * los->ds[ip]);
          obs->rad[id][ir] += src[id] * eps * obs->tau[id][ir];
          obs->tau[id][ir] *= (1 - eps);
        }
    }
  }
  if (!st && los->tsurf > 0) {
    o_srcfunc_planck(ctl, los->tsurf, src);
    for (int id = 0; id < ctl->nd; id++) obs->rad[id][ir] += src[id] * obs->tau[id][ir];
  }
  if (dig) {
    for (int id = 0; id < ctl->nd; id++) {
      dig[id] = 0;
      for (int ig = 0; ig < ctl->ng; ig++) dig[id] = dig[id] * 1000003u + gdig[id * ctl->ng + ig];
    }
    free(gdig);
  }
  los_free(los);
  free(tau_path);
  return st;
}

static int run_rays(const ctl_t *ctl, atm_t *atm, obs_t *obs, const aero_t *aero, uint64_t *dig,
                    int *nlos) {
  g_err = 0;
  o_hydrostatic(ctl, atm);
  int st = load_tables(ctl);
  if (st) return st;
#pragma omp parallel for schedule(dynamic)
  for (int ir = 0; ir < obs->nr; ir++) {
    int s = o_pencil(ctl, atm, obs, aero, ctl->sca_mult, ir,
                     dig ? dig + (size_t)ir * ctl->nd : NULL, nlos ? &nlos[ir] : NULL);
    if (s) fail(s);
  }
  return g_err;
}

/* formod (src/forwardmodel.c:15-116), IP=1 without field of view. */
int oracle_formod(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero) {
  if (ctl->ip != 1 || ctl->fov[0] != '-') return JSC_ERR_UNSUPPORTED;
  int nd = ctl->nd, nr = obs->nr;
  unsigned char *mask = (unsigned char *)malloc((size_t)nd * (nr > 0 ? nr : 1));
  for (int id = 0; id < nd; id++)
    for (int ir = 0; ir < nr; ir++) mask[id * nr + ir] = !isfinite(obs->rad[id][ir]);
  int st = run_rays(ctl, atm, obs, aero, NULL, NULL);
  if (ctl->write_bbt)
    for (int ir = 0; ir < nr; ir++)
      for (int id = 0; id < nd; id++)
        obs->rad[id][ir] = oracle_brightness(obs->rad[id][ir], ctl->nu[id]);
  for (int id = 0; id < nd; id++)
    for (int ir = 0; ir < nr; ir++)
      if (mask[id * nr + ir]) obs->rad[id][ir] = NAN;
  free(mask);
  return st;
}

/* LOS point counts per ray and EGA index checksums per (ray, channel):
 * digest[ir*nd+id] = fold over emitters of D_g, where D_g folds, over the
 * LOS points with a full interpolation of emitter g, the (p, T) bracket
 * code ipr*961+it0*31+it1 followed by the eps->u and u->eps interval
 * indices of the four (p, T) nodes in the order (ipr,it0), (ipr,it0+1),
 * (ipr+1,it1), (ipr+1,it1+1); fold: d = d*1000003 + v.
 * The radiances are computed as by oracle_formod. */
int oracle_diagnostics(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero, int *nlos,
                       uint64_t *digest) {
  return run_rays(ctl, atm, obs, aero, digest, nlos);
}

/* One ray's LOS (after hydrostatic balance of atm by the caller): fills
 * z/lon/lat/p/t/ds [NLOS], q/u [NLOS][ng] and k [NLOS][nw]; returns the
 * point count (negative status on error). */
int oracle_raytrace(ctl_t *ctl, atm_t *atm, obs_t *obs, int ir, double *z, double *lon,
                    double *lat, double *p, double *t, double *ds, double *q, double *k,
                    double *u, double *tsurf) {
  olos_t *los = los_new();
  aero_t *aero = (aero_t *)calloc(1, sizeof(aero_t));
  int st = o_raytrace(ctl, atm, obs, aero, los, ir), n = los->np;
  free(aero);
  if (st) n = -st;
  for (int i = 0; i < los->np; i++) {
    z[i] = los->z[i];
    lon[i] = los->lon[i];
    lat[i] = los->lat[i];
    p[i] = los->p[i];
    t[i] = los->t[i];
    ds[i] = los->ds[i];
    for (int ig = 0; ig < ctl->ng; ig++) {
      q[i * ctl->ng + ig] = los->q[i][ig];
      u[i * ctl->ng + ig] = los->u[i][ig];
    }
    for (int iw = 0; iw < ctl->nw; iw++) k[i * ctl->nw + iw] = los->k[i][iw];
  }
  *tsurf = los->tsurf;
  los_free(los);
  return n;
}

void oracle_hydrostatic(ctl_t *ctl, atm_t *atm) { o_hydrostatic(ctl, atm); }

/* Filter-weighted Planck source of channel id at temperature t. */
double oracle_srcfunc(ctl_t *ctl, int id, double t) {
  double src[NDMAX];
  if (load_tables(ctl)) return NAN;
  o_srcfunc_planck(ctl, t, src);
  return src[id];
}
