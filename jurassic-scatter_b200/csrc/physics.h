/*
 * Geometry and atmosphere helpers shared by host C code and device code.
 * Each keeps the operation order of the reference expression it restates,
 * so that, without FMA contraction, host and device agree with the
 * reference to the last bit wherever the libm functions involved do.
 */
#ifndef JSC_PHYSICS_H
#define JSC_PHYSICS_H

#include <math.h>
#include "jsc_internal.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Geographic -> Cartesian (src/misc.c:61-72). */
JSC_HD void jsc_geo2cart(double z, double lon, double lat, double *x) {
  double radius = z + JSC_RE;
  x[0] = radius * cos(lat / 180 * M_PI) * cos(lon / 180 * M_PI);
  x[1] = radius * cos(lat / 180 * M_PI) * sin(lon / 180 * M_PI);
  x[2] = radius * sin(lat / 180 * M_PI);
}

/* Cartesian -> geographic (src/misc.c:5-16). */
JSC_HD void jsc_cart2geo(const double *x, double *z, double *lon, double *lat) {
  double radius = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  *lat = asin(x[2] / radius) * 180 / M_PI;
  *lon = atan2(x[1], x[0]) * 180 / M_PI;
  *z = radius - JSC_RE;
}

/* EXP macro (src/jurassic.h:54-57): log-linear where both ends are > 0. */
JSC_HD double jsc_exp_interp(double x0, double y0, double x1, double y1,
                             double x) {
  return ((y0) > 0 && (y1) > 0)
             ? ((y0) * exp(log((y1) / (y0)) / ((x1) - (x0)) * ((x) - (x0))))
             : jsc_lin(x0, y0, x1, y1, x);
}

/* Refractivity of air at 4-15 micron (src/lineofsight.c:376-381). */
JSC_HD double jsc_refractivity(double p, double t) {
  return 7.753e-05 * p / t;
}

/* Gravity, 1967 Geodetic Reference System (src/atmosphere.c:153-159). */
JSC_HD double jsc_gravity(double z, double lat) {
  double s1 = sin(lat / 180 * M_PI), s2 = sin(2 * lat / 180 * M_PI);
  return 9.780318 * (1 + 0.0053024 * (s1 * s1) - 0.0000058 * (s2 * s2)) -
         3.086e-3 * z;
}

/* Hydrostatic pressure for levels [ip0, ip1) of one profile
 * (src/atmosphere.c:188-243).  qh2o: water vapour VMR of the same levels or
 * NULL when H2O is not an emitter. */
JSC_HD void jsc_hydrostatic_1d(double hydz, const double *z, const double *lat,
                               const double *t, const double *qh2o, double *p,
                               int ip0, int ip1) {
  const double mmair = 28.96456e-3, mmh2o = 18.0153e-3;
  const int ipts = 20;
  double dzmin = 1e99, e = 0, mean, zz;
  int ipref = 0;
  for (int ip = ip0; ip < ip1; ip++)
    if (fabs(z[ip] - hydz) < dzmin) {
      dzmin = fabs(z[ip] - hydz);
      ipref = ip;
    }
  for (int ip = ipref + 1; ip < ip1; ip++) {
    mean = 0;
    for (int i = 0; i < ipts; i++) {
      zz = jsc_lin(0.0, z[ip - 1], ipts - 1.0, z[ip], (double)i);
      if (qh2o) e = jsc_lin(0.0, qh2o[ip - 1], ipts - 1.0, qh2o[ip], (double)i);
      mean += (e * mmh2o + (1 - e) * mmair) * jsc_gravity(zz, lat[ipref]) /
              JSC_RGAS / jsc_lin(0.0, t[ip - 1], ipts - 1.0, t[ip], (double)i) /
              ipts;
    }
    p[ip] = exp(log(p[ip - 1]) - mean * 1000 * (z[ip] - z[ip - 1]));
  }
  for (int ip = ipref - 1; ip >= ip0; ip--) {
    mean = 0;
    for (int i = 0; i < ipts; i++) {
      zz = jsc_lin(0.0, z[ip + 1], ipts - 1.0, z[ip], (double)i);
      if (qh2o) e = jsc_lin(0.0, qh2o[ip + 1], ipts - 1.0, qh2o[ip], (double)i);
      mean += (e * mmh2o + (1 - e) * mmair) * jsc_gravity(zz, lat[ipref]) /
              JSC_RGAS / jsc_lin(0.0, t[ip + 1], ipts - 1.0, t[ip], (double)i) /
              ipts;
    }
    p[ip] = exp(log(p[ip + 1]) - mean * 1000 * (z[ip] - z[ip + 1]));
  }
}

/* Hydrostatic balance over all profiles of an atmosphere, a profile being a
 * run of points with the same lon/lat (src/atmosphere.c:163-184). */
JSC_HD void jsc_hydrostatic(double hydz, int np, const double *z,
                            const double *lon, const double *lat,
                            const double *t, const double *qh2o, double *p) {
  double lat0 = -999, lon0 = -999;
  int ip0 = -999;
  if (hydz < 0) return;
  for (int ip = 0; ip < np; ip++)
    if (lon[ip] != lon0 || lat[ip] != lat0) {
      if (ip > 0) jsc_hydrostatic_1d(hydz, z, lat, t, qh2o, p, ip0, ip);
      lon0 = lon[ip];
      lat0 = lat[ip];
      ip0 = ip;
    }
  if (np > 0) jsc_hydrostatic_1d(hydz, z, lat, t, qh2o, p, ip0, np);
}

#endif /* JSC_PHYSICS_H */
