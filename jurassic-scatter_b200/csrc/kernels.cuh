// Device kernels of the clear-air forward model.
//
//   hydro_kernel      one thread per profile: hydrostatic pressure
//                     (src/atmosphere.c:163-243) and the profile's z range.
//   raytrace_kernel   one thread per ray, FP64 refracted ray march
//                     (src/lineofsight.c:5-190); a counting pass sizes the
//                     line of sight, a storing pass writes the LOS records.
//   scan_kernel       exclusive prefix sum of LOS points per ray.
//   refine_count_kernel, refine_store_kernel
//                     aerosol/cloud layer-edge refinement of the LOS.
//   (ega_rt_kernel, the EGA + continua + Planck + radiative-transfer
//   kernel, is in ega_kernel.cuh.)
//
// All arithmetic that decides a table index is FP64 in the reference's
// operation order (the library is built with --fmad=false), so the indices
// and segment counts agree with the reference.
#pragma once
#include <math.h>
#include <stdint.h>

#include "jsc_model.h"
#include "physics.h"
#include "cuda_util.cuh"
#include "device_common.cuh"

#define JSC_ZREFRAC 60.0   // refraction is evaluated up to this altitude [km]
#define JSC_FD_STEP 0.02   // finite-difference step of the refractivity gradient [km]

// ----------------------------------------------------------------- inputs --

struct AtmArgs {
  int n_atm, n_levels, ng, nw, ig_h2o;
  const int *off;
  const double *z, *lon, *lat, *p_in, *t, *q, *k;
  double *p, *zmin, *zmax;
  double hydz;
};

// Hydrostatic balance and altitude range of each profile.
static __global__ void hydro_kernel(AtmArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atm) return;
  const int lo = a.off[i], n = a.off[i + 1] - lo;
  for (int l = 0; l < n; l++) a.p[lo + l] = a.p_in[lo + l];
  if (a.hydz >= 0 && n > 0) {
    const double *qh = a.ig_h2o >= 0 ? a.q + (size_t)a.ig_h2o * a.n_levels + lo : nullptr;
    jsc_hydrostatic(a.hydz, n, a.z + lo, a.lon + lo, a.lat + lo, a.t + lo, qh,
                    a.p + lo);
  }
  // gsl_stats_min/max: first element, then strict comparisons; NaN wins.
  double mn = n > 0 ? a.z[lo] : 0.0, mx = mn;
  bool nan = false;
  for (int l = 0; l < n; l++) {
    double v = a.z[lo + l];
    if (v < mn) mn = v;
    if (v > mx) mx = v;
    if (isnan(v)) nan = true;
  }
  a.zmin[i] = nan ? NAN : mn;
  a.zmax[i] = nan ? NAN : mx;
}

// --------------------------------------------------------------- raytrace --

struct RayArgs {
  int n_rays, ng, nw, ig_h2o, n_levels;
  int refrac;
  double rayds, raydz;
  const int *ray_atm, *atm_off;
  const double *time, *obsz, *obslon, *obslat, *vpz, *vplon, *vplat;
  const double *z, *p, *t, *q, *k, *zmin, *zmax;
  int *nlos;
  const int64_t *los_off;
  int64_t max_seg;
  int W;
  double *geo, *pts, *tsurf, *tp;  // tp: [3][n_rays]
  unsigned *status;
  // (p, T) grid shared by every table, or null when there are several
  int grid_np;
  const double *grid_p, *grid_t;
  const int *grid_nt;
  int raw_q;  // store volume mixing ratios instead of column densities
  // IP 2/3 (horizontally varying atmosphere, src/atmosphere.c:324-482):
  // every profile of the batch belongs to the one atmosphere; psurf holds
  // the surface Cartesian position of each profile (IP 2) or level (IP 3)
  int ip, n_prof;
  const double *psurf, *lat;
  double cz, cx;
};

struct Profile {
  const double *z, *p, *t, *q, *k;
  int n, stride;  // levels; stride between emitter/window blocks
};

// Pressure and temperature at altitude z0 (src/atmosphere.c:298-315).
__device__ __forceinline__ void atm_pt(const Profile &a, double z0, double *p,
                                       double *t) {
  int ip = jsc_locate(a.z, a.n, z0);
  *p = jsc_exp_interp(a.z[ip], a.p[ip], a.z[ip + 1], a.p[ip + 1], z0);
  *t = jsc_lin(a.z[ip], a.t[ip], a.z[ip + 1], a.t[ip + 1], z0);
}

// Pressure and temperature at altitude z0; returns the profile level below
// z0 for the remaining LIN interpolations (src/atmosphere.c:298-320).
__device__ __forceinline__ int atm_full(const Profile &a, double z0, double *p,
                                        double *t) {
  int ip = jsc_locate(a.z, a.n, z0);
  *p = jsc_exp_interp(a.z[ip], a.p[ip], a.z[ip + 1], a.p[ip + 1], z0);
  *t = jsc_lin(a.z[ip], a.t[ip], a.z[ip + 1], a.t[ip + 1], z0);
  return ip;
}

__device__ __forceinline__ double atm_lin(const double *v, const Profile &a,
                                          int ip, double z0) {
  return jsc_lin(a.z[ip], v[ip], a.z[ip + 1], v[ip + 1], z0);
}

__device__ __forceinline__ double dist2(const double *a, const double *b) {
  return (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) +
         (a[2] - b[2]) * (a[2] - b[2]);
}

// Atmospheric state at (z0, lon0, lat0) for IP 2 and 3: p, T and, when qk
// is given, the VMRs [ng] then the extinctions [nw].
// IP 2 (intpol_atm_2d, src/atmosphere.c:324-418): the two profiles nearest
// in horizontal distance, each interpolated vertically (intpol_atm_1d),
// blended linearly by the position between them.
// IP 3 (intpol_atm_3d, :422-482): every level within cz vertically and cx
// horizontally (and in latitude), weighted (1 - dz/cz)(1 - dx/cx).
// The atmosphere as the IP 2/3 lookups see it (all profiles of the batch).
struct GeoAtm {
  int ng, nw, n_levels, n_prof;
  const int *atm_off;
  const double *z, *p, *t, *q, *k, *lat, *psurf;
  double cz, cx;
};

template <typename Args>
__device__ __forceinline__ GeoAtm geo_atm(const Args &A) {
  GeoAtm g;
  g.ng = A.ng;
  g.nw = A.nw;
  g.n_levels = A.n_levels;
  g.n_prof = A.n_prof;
  g.atm_off = A.atm_off;
  g.z = A.z;
  g.p = A.p;
  g.t = A.t;
  g.q = A.q;
  g.k = A.k;
  g.lat = A.lat;
  g.psurf = A.psurf;
  g.cz = A.cz;
  g.cx = A.cx;
  return g;
}

template <int IP>
__device__ void atm_geo(const GeoAtm &A, double z0, double lon0, double lat0, double *p,
                        double *t, double *qk) {
  double x0[3];
  jsc_geo2cart(0, lon0, lat0, x0);
  const int nq = A.ng + A.nw;
  const size_t nl = (size_t)A.n_levels;
  if (IP == 2) {
    double dmin0 = 1e99, dmin1 = 1e99;
    int ix0 = 0, ix1 = 0;
    for (int ix = 0; ix < A.n_prof; ix++) {
      const double dh = dist2(x0, A.psurf + 3 * ix);
      if (dh <= dmin0) {
        dmin1 = dmin0;
        ix1 = ix0;
        dmin0 = dh;
        ix0 = ix;
      } else if (dh <= dmin1) {
        dmin1 = dh;
        ix1 = ix;
      }
    }
    const int lo0 = A.atm_off[ix0], lo1 = A.atm_off[ix1];
    const int i0 = lo0 + jsc_locate(A.z + lo0, A.atm_off[ix0 + 1] - lo0, z0);
    const int i1 = lo1 + jsc_locate(A.z + lo1, A.atm_off[ix1 + 1] - lo1, z0);
    const double p0 = jsc_exp_interp(A.z[i0], A.p[i0], A.z[i0 + 1], A.p[i0 + 1], z0);
    const double t0 = jsc_lin(A.z[i0], A.t[i0], A.z[i0 + 1], A.t[i0 + 1], z0);
    const double p1 = jsc_exp_interp(A.z[i1], A.p[i1], A.z[i1 + 1], A.p[i1 + 1], z0);
    const double t1 = jsc_lin(A.z[i1], A.t[i1], A.z[i1 + 1], A.t[i1 + 1], z0);
    const double x2 = dist2(A.psurf + 3 * ix0, A.psurf + 3 * ix1);
    const double x = sqrt(x2);
    const double r0 = (dmin0 - dmin1 + x2) / (2 * x), r1 = x - r0;
    const double r = r0 <= 0 ? 0 : (r1 <= 0 ? 1 : r0 / (r0 + r1));
    *p = (1 - r) * p0 + r * p1;
    *t = (1 - r) * t0 + r * t1;
    if (qk)
      for (int c = 0; c < nq; c++) {
        const double *v = c < A.ng ? A.q + (size_t)c * nl : A.k + (size_t)(c - A.ng) * nl;
        const double a0 = jsc_lin(A.z[i0], v[i0], A.z[i0 + 1], v[i0 + 1], z0);
        const double a1 = jsc_lin(A.z[i1], v[i1], A.z[i1 + 1], v[i1 + 1], z0);
        qk[c] = (1 - r) * a0 + r * a1;
      }
  } else {
    double wsum = 0, sp = 0, st = 0;
    if (qk)
      for (int c = 0; c < nq; c++) qk[c] = 0;
    for (int ip = 0; ip < A.n_levels; ip++) {
      const double dz = fabs(A.z[ip] - z0);
      if (dz > A.cz) continue;
      if (fabs(A.lat[ip] - lat0) * 111.13 > A.cx) continue;
      const double dx2 = dist2(x0, A.psurf + 3 * (size_t)ip);
      if (dx2 > A.cx * A.cx) continue;
      const double w = (1 - dz / A.cz) * (1 - sqrt(dx2) / A.cx);
      wsum += w;
      sp += w * A.p[ip];
      st += w * A.t[ip];
      if (qk)
        for (int c = 0; c < nq; c++) {
          const double *v = c < A.ng ? A.q + (size_t)c * nl : A.k + (size_t)(c - A.ng) * nl;
          qk[c] += w * v[ip];
        }
    }
    *p = sp / wsum;
    *t = st / wsum;
    if (qk)
      for (int c = 0; c < nq; c++) qk[c] /= wsum;
  }
}

// Surface Cartesian positions for IP 2 (first level of each profile) and
// IP 3 (every level).
static __global__ void psurf_kernel(int n, int per_level, const int *atm_off, const double *lon,
                                    const double *lat, double *psurf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l = per_level ? i : atm_off[i];
  jsc_geo2cart(0, lon[l], lat[l], psurf + 3 * (size_t)i);
}

// One LOS point: geometry, state, raw step.  Written by the storing pass.
template <bool STORE>
__device__ __forceinline__ void emit_point(const RayArgs &A, const Profile &a,
                                           int64_t idx, double z, double lon,
                                           double lat, double p, double t,
                                           int ipz, double zq, double raw_ds,
                                           double ds) {
  if (!STORE) return;
  double *g = A.geo + idx * 4;
  g[0] = z;
  g[1] = lon;
  g[2] = lat;
  g[3] = raw_ds;
  double *r = A.pts + idx * A.W;
  r[REC_P] = p;
  r[REC_T] = t;
  r[REC_DS] = ds;
  r[REC_QH2O] = A.ig_h2o >= 0 ? atm_lin(a.q + (size_t)A.ig_h2o * a.stride, a, ipz, zq) : 0.0;
  r[REC_GRID] = A.grid_p ? (double)grid_code(A.grid_np, A.grid_p, A.grid_nt, A.grid_t, p, t) : -1.0;
  r[REC_PLK] = (double)planck_index(t);
  r[REC_AF] = 0.0;
  r[REC_AI] = -999.0;
  for (int w = 0; w < A.nw; w++) r[REC_K + w] = atm_lin(a.k + (size_t)w * a.stride, a, ipz, zq);
  // Column density (src/lineofsight.c:182-185) with the final step length.
  for (int g2 = 0; g2 < A.ng; g2++) {
    double q = atm_lin(a.q + (size_t)g2 * a.stride, a, ipz, zq);
    r[REC_K + A.nw + g2] = A.raw_q ? q : 10 * q * p / (JSC_KBOLTZ * t) * ds;
  }
}

// emit_point for IP 2/3 with the state interpolated horizontally: qk
// holds the VMRs [ng] then the extinctions [nw] at the point.
__device__ __forceinline__ void emit_point_geo(const RayArgs &A, int64_t idx, double z,
                                               double lon, double lat, double p, double t,
                                               const double *qk, double raw_ds, double ds) {
  double *g = A.geo + idx * 4;
  g[0] = z;
  g[1] = lon;
  g[2] = lat;
  g[3] = raw_ds;
  double *r = A.pts + idx * A.W;
  r[REC_P] = p;
  r[REC_T] = t;
  r[REC_DS] = ds;
  r[REC_QH2O] = A.ig_h2o >= 0 ? qk[A.ig_h2o] : 0.0;
  r[REC_GRID] = A.grid_p ? (double)grid_code(A.grid_np, A.grid_p, A.grid_nt, A.grid_t, p, t) : -1.0;
  r[REC_PLK] = (double)planck_index(t);
  r[REC_AF] = 0.0;
  r[REC_AI] = -999.0;
  for (int w = 0; w < A.nw; w++) r[REC_K + w] = qk[A.ng + w];
  for (int g2 = 0; g2 < A.ng; g2++) {
    const double q = qk[g2];
    r[REC_K + A.nw + g2] = A.raw_q ? q : 10 * q * p / (JSC_KBOLTZ * t) * ds;
  }
}

// Observer and view point of one ray.
struct RayIn {
  double obsz, obslon, obslat, vpz, vplon, vplat;
};

// What the end-tracking march reports: the surface temperature it would
// store (-999 when the ray leaves at the top), and the geometry (z, lon,
// lat) of the last two LOS points.
struct RayEnd {
  double tsurf;
  double g[2][3];
};

// Ray march of one ray (src/lineofsight.c:5-190 without the aerosol layer
// refinement) through profile ai.  MODE 0 (count): returns the number of LOS
// points.  MODE 1 (store): writes the points at los_off[r], the tangent
// point and surface temperature of ray r.  MODE 2 (ends): counts like
// MODE 0 and reports the last two points and the surface temperature in
// *end.
template <int MODE, int IP = 1>
__device__ int trace_core(const RayArgs &A, int ai, int r, const RayIn &in, RayEnd *end) {
  constexpr bool STORE = MODE == 1;
  const int lo = A.atm_off[ai];
  Profile a;
  a.n = A.atm_off[ai + 1] - lo;
  a.stride = A.n_levels;
  a.z = A.z + lo;
  a.p = A.p + lo;
  a.t = A.t + lo;
  a.q = A.q + lo;
  a.k = A.k + lo;
  double zmin = A.zmin[ai], zmax = A.zmax[ai];
  if (IP != 1) {  // the range of the whole atmosphere (src/lineofsight.c:26-27)
    zmin = A.zmin[0];
    zmax = A.zmax[0];
    for (int ix = 1; ix < A.n_prof; ix++) {
      zmin = A.zmin[ix] < zmin ? A.zmin[ix] : zmin;
      zmax = A.zmax[ix] > zmax ? A.zmax[ix] : zmax;
    }
  }
  double qk[IP == 1 ? 1 : NGMAX + NWMAX];
  const GeoAtm G = geo_atm(A);
  const double obsz = in.obsz, vpz = in.vpz;
  int64_t base = 0;
  if (STORE) {
    base = A.los_off[r];
    A.tp[r] = vpz;
    A.tp[A.n_rays + r] = in.vplon;
    A.tp[2 * A.n_rays + r] = in.vplat;
    A.tsurf[r] = -999;
  }
  if (MODE == 2) end->tsurf = -999;
  if (obsz < zmin) {
    atomicOr(A.status, JSC_DEV_ERR_OBSERVER);
    return 0;
  }
  if (vpz > zmax - 0.001) return 0;

  double xobs[3], xvp[3], ex0[3], ex1[3], x[3], xh[3], ng[3];
  jsc_geo2cart(obsz, in.obslon, in.obslat, xobs);
  jsc_geo2cart(vpz, in.vplon, in.vplat, xvp);
  for (int i = 0; i < 3; i++) ex0[i] = xvp[i] - xobs[i];
  double norm = sqrt(ex0[0] * ex0[0] + ex0[1] * ex0[1] + ex0[2] * ex0[2]);
  for (int i = 0; i < 3; i++) ex0[i] /= norm;
  for (int i = 0; i < 3; i++) x[i] = xobs[i];

  double z = 1e99, lon = 0, lat = 0, p = 0, t = 0;
  // Observer above the atmosphere: bisect for the entry point.
  if (obsz > zmax) {
    double dmin = 0, dmax = norm, d;
    while (fabs(dmin - dmax) > 0.001) {
      d = (dmax + dmin) / 2;
      for (int i = 0; i < 3; i++) x[i] = xobs[i] + d * ex0[i];
      jsc_cart2geo(x, &z, &lon, &lat);
      if (z <= zmax && z > zmax - 0.001) break;
      if (z < zmax - 0.0005) dmax = d; else dmin = d;
    }
  }

  int np = 0, stop = 0;
  double zprev = 0, lonprev = 0, latprev = 0, rprev = 0, rprev2 = 0, dprev = 0;
  double ends[3][3] = {};  // MODE 2: the last three points, newest last
  while (1) {
    double ds = A.rayds;
    if (A.raydz > 0) {
      norm = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
      for (int i = 0; i < 3; i++) xh[i] = x[i] / norm;
      double cosa = fabs(ex0[0] * xh[0] + ex0[1] * xh[1] + ex0[2] * xh[2]);
      if (cosa != 0) {
        const double dz = A.raydz / cosa;
        ds = (A.rayds < dz ? A.rayds : dz);  // GSL_MIN
      }
    }
    jsc_cart2geo(x, &z, &lon, &lat);

    double pz, plon, plat, pp, pt, raw;
    if (z < zmin + 0.001 || z > zmax + 0.001) {
      // Last point: where the segment from the previous point crosses the
      // boundary (intersection_point, src/lineofsight.c:385-407).
      stop = (z < zmin + 0.001 ? 2 : 1);
      const double zlim = (stop == 2 ? zmin : zmax);
      const double z0 = np > 0 ? zprev : z, lon0 = np > 0 ? lonprev : lon,
                   lat0 = np > 0 ? latprev : lat;
      double x1[3], x2[3];
      const double frac = (z0 - zlim) / (z0 - z);
      jsc_geo2cart(z0, lon0, lat0, x1);
      jsc_geo2cart(z, lon, lat, x2);
      for (int i = 0; i < 3; i++) x2[i] = x1[i] + frac * (x2[i] - x1[i]);
      jsc_cart2geo(x2, &pz, &plon, &plat);
      raw = 0.;
    } else {
      pz = z;
      plon = lon;
      plat = lat;
      raw = ds;
    }
    int ipz = 0;
    pp = pt = 0;
    if (IP == 1) {
      if (STORE || !stop) ipz = atm_full(a, pz, &pp, &pt);
    } else {
      if (STORE || !stop) atm_geo<IP>(G, pz, plon, plat, &pp, &pt, STORE ? qk : nullptr);
    }
    if (!stop) {
      p = pp;
      t = pt;
    }
    if (np >= NLOS) {
      atomicOr(A.status, JSC_DEV_ERR_NLOS);
      return np;
    }
    // Step lengths are smoothed in place along the ray
    // (src/lineofsight.c:177-179): d[0] = r[0]/2, d[i] = (d[i-1] + r[i])/2.
    const double dsm = (np == 0) ? 0.5 * raw : 0.5 * (dprev + raw);
    if (STORE) {
      if (base + np >= A.max_seg) {
        atomicOr(A.status, JSC_DEV_ERR_NLOS);
        return np;
      }
      if (IP == 1)
        emit_point<true>(A, a, base + np, pz, plon, plat, pp, pt, ipz, pz, raw, dsm);
      else
        emit_point_geo(A, base + np, pz, plon, plat, pp, pt, qk, raw, dsm);
    }
    np++;
    if (MODE == 2) {
      for (int j = 0; j < 2; j++)
        for (int c = 0; c < 3; c++) ends[j][c] = ends[j + 1][c];
      ends[2][0] = pz;
      ends[2][1] = plon;
      ends[2][2] = plat;
    }
    rprev2 = rprev;
    rprev = raw;
    dprev = dsm;
    zprev = pz;
    lonprev = plon;
    latprev = plat;
    if (stop) {
      if (STORE) A.tsurf[r] = (stop == 2 ? t : -999);
      if (MODE == 2) end->tsurf = (stop == 2 ? t : -999);
      break;
    }

    // Refraction (src/lineofsight.c:122-166).
    double n = (A.refrac && z <= JSC_ZREFRAC) ? 1 + jsc_refractivity(p, t) : 1;
    for (int i = 0; i < 3; i++) ex1[i] = ex0[i] * n;
    if (A.refrac && z <= JSC_ZREFRAC) {
      for (int i = 0; i < 3; i++) xh[i] = x[i] + 0.5 * ds * ex0[i];
      jsc_cart2geo(xh, &z, &lon, &lat);
      if (IP == 1) atm_pt(a, z, &p, &t);
      else atm_geo<IP>(G, z, lon, lat, &p, &t, nullptr);
      n = jsc_refractivity(p, t);
      for (int i = 0; i < 3; i++) {
        xh[i] += JSC_FD_STEP;
        jsc_cart2geo(xh, &z, &lon, &lat);
        if (IP == 1) atm_pt(a, z, &p, &t);
        else atm_geo<IP>(G, z, lon, lat, &p, &t, nullptr);
        const double naux = jsc_refractivity(p, t);
        ng[i] = (naux - n) / JSC_FD_STEP;
        xh[i] -= JSC_FD_STEP;
      }
    } else {
      for (int i = 0; i < 3; i++) ng[i] = 0;
    }
    for (int i = 0; i < 3; i++) ex1[i] += ds * ng[i];
    norm = sqrt(ex1[0] * ex1[0] + ex1[1] * ex1[1] + ex1[2] * ex1[2]);
    for (int i = 0; i < 3; i++) ex1[i] /= norm;
    for (int i = 0; i < 3; i++) x[i] += 0.5 * ds * (ex0[i] + ex1[i]);
    for (int i = 0; i < 3; i++) ex0[i] = ex1[i];
  }

  // Drop a last point that follows a too-short step (src/lineofsight.c:170-171).
  bool dropped = false;
  if (np >= 3 && rprev2 < 1e-3) {
    np--;
    dropped = true;
  }
  if (MODE == 2) {
    for (int j = 0; j < 2; j++)
      for (int c = 0; c < 3; c++) end->g[j][c] = ends[j + (dropped ? 0 : 1)][c];
  }

  if (STORE) {
    // Tangent point (src/lineofsight.c:411-452) from the stored geometry.
    const double *g = A.geo + base * 4;
    size_t m = 0;
    double mn = g[0];
    for (int i = 0; i < np; i++) {
      const double v = g[(size_t)i * 4];
      if (v < mn) {
        mn = v;
        m = (size_t)i;
      }
      if (isnan(v)) {
        m = (size_t)i;
        break;
      }
    }
    double tpz, tplon, tplat;
    if (m <= 0 || m >= (size_t)np - 1) {
      tpz = g[(size_t)(np - 1) * 4];
      tplon = g[(size_t)(np - 1) * 4 + 1];
      tplat = g[(size_t)(np - 1) * 4 + 2];
    } else {
      const double yy0 = g[(m - 1) * 4], yy1 = g[m * 4], yy2 = g[(m + 1) * 4];
      const double d1 = g[m * 4 + 3], d2 = g[(m + 1) * 4 + 3];
      const double x1 = sqrt(d1 * d1 - (yy1 - yy0) * (yy1 - yy0));
      const double x2 = x1 + sqrt(d2 * d2 - (yy2 - yy1) * (yy2 - yy1));
      const double aa = 1 / (x1 - x2) * (-(yy0 - yy1) / x1 + (yy0 - yy2) / x2);
      const double bb = -(yy0 - yy1) / x1 - aa * x1;
      const double cc = yy0;
      const double xx = -bb / (2 * aa);
      double v0[3], v2[3], v[3], dummy;
      tpz = aa * xx * xx + bb * xx + cc;
      jsc_geo2cart(g[(m - 1) * 4], g[(m - 1) * 4 + 1], g[(m - 1) * 4 + 2], v0);
      jsc_geo2cart(g[(m + 1) * 4], g[(m + 1) * 4 + 1], g[(m + 1) * 4 + 2], v2);
      for (int i = 0; i < 3; i++) v[i] = jsc_lin(0.0, v0[i], x2, v2[i], xx);
      jsc_cart2geo(v, &dummy, &tplon, &tplat);
    }
    A.tp[r] = tpz;
    A.tp[A.n_rays + r] = tplon;
    A.tp[2 * A.n_rays + r] = tplat;
  }
  return np;
}

template <bool STORE, int IP>
__device__ __forceinline__ int trace_ray(const RayArgs &A, int r) {
  const RayIn in = {A.obsz[r], A.obslon[r], A.obslat[r], A.vpz[r], A.vplon[r], A.vplat[r]};
  return trace_core<STORE ? 1 : 0, IP>(A, A.ray_atm[r], r, in, nullptr);
}

template <bool STORE, int IP = 1>
__global__ void __launch_bounds__(128, 7) raytrace_kernel(RayArgs A) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n_rays) return;
  const int np = trace_ray<STORE, IP>(A, r);
  if (!STORE) A.nlos[r] = np;
  else if (np != A.nlos[r]) atomicOr(A.status, JSC_DEV_ERR_NLOS);
}

// The pencils of one round of a fixed-capacity scattering run as a device
// work queue: a persistent grid pulls them a warp (32 pencils) at a time
// from the queue head until the round's live count, which only the device
// knows; slots past it are never traced (their nlos stays 0, cleared
// before the counting pass).  Pulling balances the uneven pencil lengths
// across the SMs.
template <bool STORE, int IP = 1>
__global__ void __launch_bounds__(128, 7) raytrace_queue_kernel(RayArgs A, unsigned *head,
                                                               const int *live) {
  const int lane = threadIdx.x & 31;
  const int n = *live < A.n_rays ? *live : A.n_rays;
  for (;;) {
    int r0 = 0;
    if (lane == 0) r0 = (int)atomicAdd(head, 32u);
    r0 = __shfl_sync(0xffffffffu, r0, 0);
    if (r0 >= n) break;
    const int r = r0 + lane;
    if (r < n) {
      const int np = trace_ray<STORE, IP>(A, r);
      if (!STORE) A.nlos[r] = np;
      else if (np != A.nlos[r]) atomicOr(A.status, JSC_DEV_ERR_NLOS);
    }
  }
}

// ------------------------------------------------------ aerosol layers --

struct RefineArgs {
  int n_rays, ng, nw, W, n_levels, ig_h2o;
  const int *ray_atm, *atm_off;
  const double *z, *p, *t, *q, *k;       // atmospheric profiles
  const int *nlos_b;                     // ray-traced LOS (raw records)
  const int64_t *off_b;
  const double *geo_b, *pts_b;
  int *nlos;                             // refined LOS
  const int64_t *off;
  double *geo, *pts;
  int64_t max_seg;
  int nl, n_alti;
  double altimax, altimin, transs;
  const double *top, *bottom, *trans, *alti;
  int grid_np;
  const double *grid_p, *grid_t;
  const int *grid_nt;
  unsigned *status;
  // IP 2/3: as in RayArgs
  int ip, n_prof;
  const double *psurf, *lat;
  double cz, cx;
};

// Point where the segment between raw points ip-1 and ip crosses znew, with
// the atmospheric state there (intersection_point, src/lineofsight.c:385-407).
template <int IP = 1>
__device__ __forceinline__ void refine_cross(const RefineArgs &A, const Profile &a,
                                             const double *gb, int ip, double znew,
                                             double *go, double *po) {
  double x1[3], x2[3], zz, lon, lat, p, t;
  const double *g0 = gb + (size_t)(ip - 1) * 4, *g1 = gb + (size_t)ip * 4;
  const double frac = (g0[0] - znew) / (g0[0] - g1[0]);
  jsc_geo2cart(g0[0], g0[1], g0[2], x1);
  jsc_geo2cart(g1[0], g1[1], g1[2], x2);
  for (int i = 0; i < 3; i++) x2[i] = x1[i] + frac * (x2[i] - x1[i]);
  jsc_cart2geo(x2, &zz, &lon, &lat);
  go[0] = zz;
  go[1] = lon;
  go[2] = lat;
  if (IP != 1) {
    double qk[NGMAX + NWMAX];
    atm_geo<IP>(geo_atm(A), zz, lon, lat, &p, &t, qk);
    po[REC_P] = p;
    po[REC_T] = t;
    po[REC_QH2O] = A.ig_h2o >= 0 ? qk[A.ig_h2o] : 0.0;
    for (int w = 0; w < A.nw; w++) po[REC_K + w] = qk[A.ng + w];
    for (int g = 0; g < A.ng; g++) po[REC_K + A.nw + g] = qk[g];
    return;
  }
  const int ipz = atm_full(a, zz, &p, &t);
  po[REC_P] = p;
  po[REC_T] = t;
  po[REC_QH2O] = A.ig_h2o >= 0 ? atm_lin(a.q + (size_t)A.ig_h2o * a.stride, a, ipz, zz) : 0.0;
  for (int w = 0; w < A.nw; w++) po[REC_K + w] = atm_lin(a.k + (size_t)w * a.stride, a, ipz, zz);
  for (int g = 0; g < A.ng; g++) po[REC_K + A.nw + g] = atm_lin(a.q + (size_t)g * a.stride, a, ipz, zz);
}

// Chord step length, column densities, (p, T) bracket, Planck index and
// aerosol layer/factor of refined point i (the per-point part of
// add_aerosol_layers, src/lineofsight.c:300-372).  xp, xc, xn: Cartesian
// positions of points i-1, i, i+1 (xp unused at i = 0, xn at i = o-1).
__device__ __forceinline__ void refine_point(const RefineArgs &A, int64_t base, int o, int i,
                                             const double *xp, const double *xc,
                                             const double *xn) {
  double ds;
  if (o == 1) {
    ds = 0;
  } else if (i == 0) {
    ds = 0.5 * sqrt((xc[0] - xn[0]) * (xc[0] - xn[0]) + (xc[1] - xn[1]) * (xc[1] - xn[1]) +
                    (xc[2] - xn[2]) * (xc[2] - xn[2]));
  } else if (i == o - 1) {
    ds = 0.5 * sqrt((xc[0] - xp[0]) * (xc[0] - xp[0]) + (xc[1] - xp[1]) * (xc[1] - xp[1]) +
                    (xc[2] - xp[2]) * (xc[2] - xp[2]));
  } else {
    ds = 0.5 * (sqrt((xp[0] - xc[0]) * (xp[0] - xc[0]) + (xp[1] - xc[1]) * (xp[1] - xc[1]) +
                     (xp[2] - xc[2]) * (xp[2] - xc[2])) +
                sqrt((xc[0] - xn[0]) * (xc[0] - xn[0]) + (xc[1] - xn[1]) * (xc[1] - xn[1]) +
                     (xc[2] - xn[2]) * (xc[2] - xn[2])));
  }
  double *go = A.geo + base * 4;
  double *rec = A.pts + (base + i) * A.W;
  const double p = rec[REC_P], t = rec[REC_T], z = go[(size_t)i * 4];
  rec[REC_DS] = ds;
  go[(size_t)i * 4 + 3] = ds;
  for (int g = 0; g < A.ng; g++) {
    const double q = rec[REC_K + A.nw + g];
    rec[REC_K + A.nw + g] = 10 * q * p / (JSC_KBOLTZ * t) * ds;
  }
  rec[REC_GRID] = A.grid_p ? (double)grid_code(A.grid_np, A.grid_p, A.grid_nt, A.grid_t, p, t) : -1.0;
  rec[REC_PLK] = (double)planck_index(t);
  // At i = 0 the reference compares z[-1]; the first point, at the top
  // of the atmosphere and outside every layer, stands in for it.
  const double zprev = go[(size_t)(i > 0 ? i - 1 : 0) * 4];
  int aeroi = -999;
  double aerofac = 0.;
  if ((zprev < A.altimax || z < A.altimax) && (zprev > A.altimin || z > A.altimin)) {
    for (int il = 0; il < A.nl; il++) {
      if (z <= A.top[il] && z >= A.bottom[il]) {
        aeroi = il;
        aerofac = 1.;
      }
      if (A.trans[il] > A.transs && z <= (A.top[il] + A.trans[il]) && z > A.top[il]) {
        aeroi = il;
        aerofac = (A.top[il] + A.trans[il] - z) / A.trans[il];
      }
      if (A.trans[il] > A.transs && z < A.bottom[il] && z >= (A.bottom[il] - A.trans[il])) {
        aeroi = il;
        aerofac = fabs(A.bottom[il] - A.trans[il] - z) / A.trans[il];
      }
    }
  }
  rec[REC_AF] = aerofac;
  rec[REC_AI] = (double)aeroi;
}

// Profile of ray r's atmosphere.
__device__ __forceinline__ Profile refine_profile(const RefineArgs &A, int r) {
  const int ai = A.ray_atm[r];
  const int lo = A.atm_off[ai];
  Profile a;
  a.n = A.atm_off[ai + 1] - lo;
  a.stride = A.n_levels;
  a.z = A.z + lo;
  a.p = A.p + lo;
  a.t = A.t + lo;
  a.q = A.q + lo;
  a.k = A.k + lo;
  return a;
}

// STORE pass of the layer-edge refinement with a warp per ray (the COUNT
// pass is refine_count_kernel): lanes take 32 raw points at a time, a
// warp scan of their output counts (crossing points of the segment before
// the point, then the point) places them in the order the serial pass
// writes them, the raw records are copied with coalesced loads, then lanes
// take 32 refined points at a time for refine_point, with the neighbours'
// Cartesian positions passed by shuffles.  Same outputs as the serial pass,
// including its overflow status.
template <int IP = 1>
__global__ void __launch_bounds__(128, 8) refine_store_kernel(RefineArgs A) {
  const int r = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  if (r >= A.n_rays) return;  // whole warps leave together
  const int nb = A.nlos_b[r];
  if (nb == 0) return;
  const Profile a = refine_profile(A, r);
  const double *gb = A.geo_b + A.off_b[r] * 4, *pb = A.pts_b + A.off_b[r] * A.W;
  const int64_t base = A.off[r];
  const int nmax = A.nlos[r];
  const int W = A.W;
  int o = 0;
  for (int c0 = 0; c0 < nb; c0 += 32) {
    const int ip = c0 + lane;
    int cnt = 0;
    double zp = 0, zc = 0;
    bool win = false;
    if (ip < nb) {
      cnt = 1;
      if (ip >= 1) {
        zp = gb[(size_t)(ip - 1) * 4];
        zc = gb[(size_t)ip * 4];
        win = (zp < A.altimax || zc < A.altimax) && (zp > A.altimin || zc > A.altimin);
        if (win)
          for (int il = 0; il < A.n_alti; il++) {
            const double z1 = A.alti[il], z2 = A.alti[A.n_alti - il - 1];
            cnt += (zp > z1 && zc < z1) + (zp < z2 && zc > z2);
          }
      }
    }
    int incl = cnt;
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(full, incl, d);
      if (lane >= d) incl += v;
    }
    const int total = __shfl_sync(full, incl, 31);
    if (o + total > nmax || base + o + total > A.max_seg) {
      if (lane == 0) atomicOr(A.status, JSC_DEV_ERR_NLOS);
      return;
    }
    int slot = o + incl - cnt;  // first output slot of this lane
    if (ip < nb) {
      if (win)
        for (int il = 0; il < A.n_alti; il++) {
          const double z1 = A.alti[il], z2 = A.alti[A.n_alti - il - 1];
          if (zp > z1 && zc < z1) {
            refine_cross<IP>(A, a, gb, ip, z1, A.geo + (base + slot) * 4, A.pts + (base + slot) * W);
            slot++;
          }
          if (zp < z2 && zc > z2) {
            refine_cross<IP>(A, a, gb, ip, z2, A.geo + (base + slot) * 4, A.pts + (base + slot) * W);
            slot++;
          }
        }
      double *go = A.geo + (base + slot) * 4;
      const double *gs = gb + (size_t)ip * 4;
      go[0] = gs[0];
      go[1] = gs[1];
      go[2] = gs[2];
    }
    // raw records of the chunk's points, copied element by element
    const int m = min(32, nb - c0);
    const int ne = m * W;
    for (int e0 = 0; e0 < ne; e0 += 32) {
      const int e = e0 + lane;
      const int pp = e < ne ? e / W : 0;
      const int sl = __shfl_sync(full, slot, pp);
      if (e < ne) A.pts[(base + sl) * W + (e - pp * W)] = pb[(size_t)c0 * W + e];
    }
    o += total;
  }
  if (o > NLOS) {
    if (lane == 0) atomicOr(A.status, JSC_DEV_ERR_NLOS);
    return;
  }
  __syncwarp();  // the points written above, for every lane
  const double *go = A.geo + base * 4;
  double carry[3] = {0, 0, 0};  // position of the point before the chunk
  for (int i0 = 0; i0 < o; i0 += 32) {
    const int i = i0 + lane;
    double xc[3] = {0, 0, 0}, xp[3], xn[3];
    if (i < o) jsc_geo2cart(go[(size_t)i * 4], go[(size_t)i * 4 + 1], go[(size_t)i * 4 + 2], xc);
    for (int c = 0; c < 3; c++) {
      const double up = __shfl_up_sync(full, xc[c], 1);
      const double dn = __shfl_down_sync(full, xc[c], 1);
      xp[c] = lane == 0 ? carry[c] : up;
      xn[c] = dn;
      carry[c] = __shfl_sync(full, xc[c], 31);
    }
    if (lane == 31 && i + 1 < o)
      jsc_geo2cart(go[(size_t)(i + 1) * 4], go[(size_t)(i + 1) * 4 + 1],
                   go[(size_t)(i + 1) * 4 + 2], xn);
    if (i < o) refine_point(A, base, o, i, xp, xc, xn);
  }
}

// COUNT pass of the layer-edge refinement (add_aerosol_layers,
// src/lineofsight.c:193-372): the number of refined LOS points of each ray,
// the raw points plus the points where a segment crosses a layer edge or a
// transition-layer level; refine_store_kernel writes them.
static __global__ void __launch_bounds__(128) refine_count_kernel(RefineArgs A) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n_rays) return;
  const int nb = A.nlos_b[r];
  if (nb == 0) {
    A.nlos[r] = 0;
    return;
  }
  const double *gb = A.geo_b + A.off_b[r] * 4;
  int o = 1;
  for (int ip = 1; ip < nb; ip++) {
    const double zp = gb[(size_t)(ip - 1) * 4], zc = gb[(size_t)ip * 4];
    if ((zp < A.altimax || zc < A.altimax) && (zp > A.altimin || zc > A.altimin))
      for (int il = 0; il < A.n_alti; il++) {
        const double z1 = A.alti[il], z2 = A.alti[A.n_alti - il - 1];
        o += (zp > z1 && zc < z1) + (zp < z2 && zc > z2);
      }
    o++;
  }
  if (o > NLOS || o > A.max_seg) {
    atomicOr(A.status, JSC_DEV_ERR_NLOS);
    A.nlos[r] = 0;
    return;
  }
  A.nlos[r] = o;
}

// Exclusive prefix sum of n counts into off[0..n] in one pass over many
// blocks (decoupled look-back, Merrill and Garland 2016).  Tiles of
// JSC_SCAN_TILE counts are claimed in order through a ticket counter; a
// tile publishes its own sum, walks back over the tiles before it adding
// published values until it meets a published inclusive prefix, then
// publishes its inclusive prefix.  Tiles are claimed only by running
// blocks, so a tile waits only on tiles that resident blocks are working
// on.  Every wait is bounded: after `budget` polls of an unpublished tile
// the waiting tile flags JSC_DEV_ERR_WATCHDOG in the status word, publishes
// a prefix anyway (no later tile waits on it for ever) and returns its
// outputs invalid.  flags[] (one word per tile: value << 2 | state, state 1
// sum, 2 inclusive prefix) and the ticket must be zero at launch.
// stall_tile >= 0 names a tile that never publishes: the diagnostic of the
// watchdog path (its successor's wait runs out).
#define JSC_SCAN_THREADS 256
#define JSC_SCAN_PER 8
#define JSC_SCAN_TILE (JSC_SCAN_THREADS * JSC_SCAN_PER)

struct ScanArgs {
  const int *in;               // [n] counts
  int n;
  int64_t *out;                // [n + 1]
  unsigned long long *flags;   // [tiles]
  unsigned *ticket;
  unsigned *status;
  unsigned budget;             // polls of an unpublished tile before giving up
  int stall_tile;
};

__device__ __forceinline__ void scan_publish(unsigned long long *f, int64_t v, unsigned st) {
  atomicExch(f, ((unsigned long long)v << 2) | st);
}

static __global__ void __launch_bounds__(JSC_SCAN_THREADS) scan_lookback_kernel(ScanArgs A) {
  __shared__ int tile_s;
  __shared__ int64_t wsum[JSC_SCAN_THREADS / 32];
  __shared__ int64_t prefix_s;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  constexpr int NW = JSC_SCAN_THREADS / 32;
  if (tid == 0) tile_s = (int)atomicAdd(A.ticket, 1u);
  __syncthreads();
  const int tile = tile_s;
  const int64_t base = (int64_t)tile * JSC_SCAN_TILE + (int64_t)tid * JSC_SCAN_PER;
  int v[JSC_SCAN_PER];
  int64_t s = 0;
#pragma unroll
  for (int q = 0; q < JSC_SCAN_PER; q++) {
    const int64_t i = base + q;
    v[q] = i < A.n ? A.in[i] : 0;
    s += v[q];
  }
  int64_t x = s;  // inclusive scan within the warp
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int64_t t = lane < NW ? wsum[lane] : 0;
#pragma unroll
    for (int d = 1; d < NW; d <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, t, d);
      if (lane >= d) t += y;
    }
    if (lane < NW) wsum[lane] = t;
  }
  __syncthreads();
  const int64_t excl = x - s + (w > 0 ? wsum[w - 1] : 0);
  const int64_t agg = wsum[NW - 1];
  if (tid == 0) {
    int64_t prefix = 0;
    if (tile == A.stall_tile) {
      // never publishes (diagnostic)
    } else if (tile == 0) {
      scan_publish(&A.flags[0], agg, 2);
    } else {
      scan_publish(&A.flags[tile], agg, 1);
      unsigned polls = 0;
      bool gave_up = false;
      for (int j = tile - 1; j >= 0;) {
        const unsigned long long f = atomicAdd(&A.flags[j], 0ull);
        const unsigned st = (unsigned)(f & 3ull);
        if (st == 0) {
          if (++polls > A.budget) {
            gave_up = true;
            break;
          }
          __nanosleep(64);
          continue;
        }
        prefix += (int64_t)(f >> 2);
        if (st == 2) break;
        j--;
      }
      if (gave_up) atomicOr(A.status, JSC_DEV_ERR_WATCHDOG);
      scan_publish(&A.flags[tile], prefix + agg, 2);
    }
    prefix_s = prefix;
  }
  __syncthreads();
  int64_t run = prefix_s + excl;
#pragma unroll
  for (int q = 0; q < JSC_SCAN_PER; q++) {
    const int64_t i = base + q;
    if (i < A.n) A.out[i] = run;
    run += v[q];
  }
  const int tiles = (A.n + JSC_SCAN_TILE - 1) / JSC_SCAN_TILE;
  if (tile == tiles - 1 && tid == JSC_SCAN_THREADS - 1) A.out[A.n] = prefix_s + agg;
}

// Exclusive scan of nlos into off[0..n] by one block.
static __global__ void scan_kernel(const int *nlos, int n, int64_t *off) {
  __shared__ int64_t part[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int chunk = (n + nt - 1) / nt;
  const int b = tid * chunk, e = min(n, b + chunk);
  int64_t s = 0;
  for (int i = b; i < e; i++) s += nlos[i];
  part[tid] = s;
  __syncthreads();
  for (int d = 1; d < nt; d <<= 1) {
    int64_t v = tid >= d ? part[tid - d] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  int64_t run = part[tid] - s;
  for (int i = b; i < e; i++) {
    off[i] = run;
    run += nlos[i];
  }
  if (tid == nt - 1) off[n] = part[nt - 1];
}

