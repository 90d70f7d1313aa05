// Device kernels of the clear-air forward model.
//
//   hydro_kernel      one thread per profile: hydrostatic pressure
//                     (src/atmosphere.c:163-243) and the profile's z range.
//   raytrace_kernel   one thread per ray, FP64 refracted ray march
//                     (src/lineofsight.c:5-190); a counting pass sizes the
//                     line of sight, a storing pass writes the LOS records.
//   scan_kernel       exclusive prefix sum of LOS points per ray.
//   ega_rt_kernel     a group of lanes per ray, lanes over channels: EGA
//                     table interpolation (src/forwardmodel.c:409-565),
//                     continua (src/forwardmodel.c:120-152, src/continua.c),
//                     Planck source (src/forwardmodel.c:743-794) and the
//                     radiative-transfer recursion
//                     (src/forwardmodel.c:302-399), fused, serial along the
//                     ray because the EGA carries the path transmittance.
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
__global__ void hydro_kernel(AtmArgs a) {
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

__device__ __forceinline__ double planck_temp(int i) {
  return jsc_lin(0.0, JSC_PLANCK_TMIN, JSC_NPLANCK - 1.0, JSC_PLANCK_TMAX, (double)i);
}

// Result of locate() on the uniform Planck temperature grid: the bracket
// from the grid spacing, corrected against the exact node values.
__device__ __forceinline__ int planck_index(double t) {
  if (!(t == t)) return JSC_NPLANCK - 2;
  const double f = floor((t - JSC_PLANCK_TMIN) * 4.0);
  int i = f < 0 ? 0 : (f > JSC_NPLANCK - 2 ? JSC_NPLANCK - 2 : (int)f);
  while (i > 0 && planck_temp(i) > t) i--;
  while (i < JSC_NPLANCK - 2 && planck_temp(i + 1) <= t) i++;
  return i;
}

__device__ __forceinline__ double planck_src(const jsc_dev_model &m, int d,
                                             int it, double t) {
  const size_t o = (size_t)d * JSC_NPLANCK + it;
  return m.planck_b[o] + m.planck_s[o] * (t - planck_temp(it));
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
};

// Packed (p, T) bracket of a point on the shared grid: ipr << 10 | it0 << 5
// | it1, plus 1 << 16 when both temperature rows have two nodes or more.
// locate() (src/misc.c:237-265) as intpol_tbl calls it (src/forwardmodel.c:447-449).
__device__ __forceinline__ int grid_code(int np, const double *gp, const int *gnt,
                                         const double *gt, double p, double t) {
  const int ipr = jsc_locate(gp, np, p);
  const int it0 = jsc_locate(gt + ipr * TBLNTMAX, gnt[ipr], t);
  const int it1 = jsc_locate(gt + (ipr + 1) * TBLNTMAX, gnt[ipr + 1], t);
  const int ok = (gnt[ipr] >= 2 && gnt[ipr + 1] >= 2) ? (1 << 16) : 0;
  return ok | (ipr << 10) | (it0 << 5) | it1;
}

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

// Ray march of one ray (src/lineofsight.c:5-190 without the aerosol layer
// refinement).  COUNT pass: returns the number of LOS points.  STORE pass:
// writes the points at los_off[r], the tangent point and surface temperature.
template <bool STORE>
__device__ int trace_ray(const RayArgs &A, int r) {
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
  const double zmin = A.zmin[ai], zmax = A.zmax[ai];
  const double obsz = A.obsz[r], vpz = A.vpz[r];
  int64_t base = 0;
  if (STORE) {
    base = A.los_off[r];
    A.tp[r] = vpz;
    A.tp[A.n_rays + r] = A.vplon[r];
    A.tp[2 * A.n_rays + r] = A.vplat[r];
    A.tsurf[r] = -999;
  }
  if (obsz < zmin) {
    atomicOr(A.status, JSC_DEV_ERR_OBSERVER);
    return 0;
  }
  if (vpz > zmax - 0.001) return 0;

  double xobs[3], xvp[3], ex0[3], ex1[3], x[3], xh[3], ng[3];
  jsc_geo2cart(obsz, A.obslon[r], A.obslat[r], xobs);
  jsc_geo2cart(vpz, A.vplon[r], A.vplat[r], xvp);
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
    if (STORE || !stop) ipz = atm_full(a, pz, &pp, &pt);
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
      emit_point<true>(A, a, base + np, pz, plon, plat, pp, pt, ipz, pz, raw, dsm);
    }
    np++;
    rprev2 = rprev;
    rprev = raw;
    dprev = dsm;
    zprev = pz;
    lonprev = plon;
    latprev = plat;
    if (stop) {
      if (STORE) A.tsurf[r] = (stop == 2 ? t : -999);
      break;
    }

    // Refraction (src/lineofsight.c:122-166).
    double n = (A.refrac && z <= JSC_ZREFRAC) ? 1 + jsc_refractivity(p, t) : 1;
    for (int i = 0; i < 3; i++) ex1[i] = ex0[i] * n;
    if (A.refrac && z <= JSC_ZREFRAC) {
      for (int i = 0; i < 3; i++) xh[i] = x[i] + 0.5 * ds * ex0[i];
      jsc_cart2geo(xh, &z, &lon, &lat);
      atm_pt(a, z, &p, &t);
      n = jsc_refractivity(p, t);
      for (int i = 0; i < 3; i++) {
        xh[i] += JSC_FD_STEP;
        jsc_cart2geo(xh, &z, &lon, &lat);
        atm_pt(a, z, &p, &t);
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
  if (np >= 3 && rprev2 < 1e-3) np--;

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

template <bool STORE>
__global__ void __launch_bounds__(128) raytrace_kernel(RayArgs A) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n_rays) return;
  const int np = trace_ray<STORE>(A, r);
  if (!STORE) A.nlos[r] = np;
  else if (np != A.nlos[r]) atomicOr(A.status, JSC_DEV_ERR_NLOS);
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
};

// Point where the segment between raw points ip-1 and ip crosses znew, with
// the atmospheric state there (intersection_point, src/lineofsight.c:385-407).
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
  const int ipz = atm_full(a, zz, &p, &t);
  go[0] = zz;
  go[1] = lon;
  go[2] = lat;
  po[REC_P] = p;
  po[REC_T] = t;
  po[REC_QH2O] = A.ig_h2o >= 0 ? atm_lin(a.q + (size_t)A.ig_h2o * a.stride, a, ipz, zz) : 0.0;
  for (int w = 0; w < A.nw; w++) po[REC_K + w] = atm_lin(a.k + (size_t)w * a.stride, a, ipz, zz);
  for (int g = 0; g < A.ng; g++) po[REC_K + A.nw + g] = atm_lin(a.q + (size_t)g * a.stride, a, ipz, zz);
}

// Extra LOS points at the layer edges and through the transition layers,
// chord step lengths, column densities, layer index and scaling factor per
// point (add_aerosol_layers, src/lineofsight.c:193-372).  COUNT pass sizes
// the refined LOS, STORE pass writes it.
template <bool STORE>
__global__ void __launch_bounds__(128) refine_kernel(RefineArgs A) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n_rays) return;
  const int nb = A.nlos_b[r];
  if (nb == 0) {
    if (!STORE) A.nlos[r] = 0;
    return;
  }
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
  const double *gb = A.geo_b + A.off_b[r] * 4, *pb = A.pts_b + A.off_b[r] * A.W;
  const int64_t base = STORE ? A.off[r] : 0;
  const int nmax = STORE ? A.nlos[r] : NLOS + 1;
  int o = 0;
  bool over = false;
#define JSC_PUT_BASE(ip)                                                     \
  do {                                                                       \
    if (o >= nmax || base + o >= A.max_seg) { over = true; break; }          \
    if (STORE) {                                                             \
      double *go = A.geo + (base + o) * 4, *po = A.pts + (base + o) * A.W;   \
      const double *gs = gb + (size_t)(ip) * 4, *ps = pb + (size_t)(ip) * A.W; \
      go[0] = gs[0]; go[1] = gs[1]; go[2] = gs[2];                           \
      for (int c = 0; c < A.W; c++) po[c] = ps[c];                           \
    }                                                                        \
    o++;                                                                     \
  } while (0)
  JSC_PUT_BASE(0);
  for (int ip = 1; ip < nb && !over; ip++) {
    const double zp = gb[(size_t)(ip - 1) * 4], zc = gb[(size_t)ip * 4];
    if ((zp < A.altimax || zc < A.altimax) && (zp > A.altimin || zc > A.altimin)) {
      for (int il = 0; il < A.n_alti && !over; il++) {
        const double z1 = A.alti[il], z2 = A.alti[A.n_alti - il - 1];
        if (zp > z1 && zc < z1) {
          if (o >= nmax || base + o >= A.max_seg) { over = true; break; }
          if (STORE) refine_cross(A, a, gb, ip, z1, A.geo + (base + o) * 4, A.pts + (base + o) * A.W);
          o++;
        }
        if (zp < z2 && zc > z2) {
          if (o >= nmax || base + o >= A.max_seg) { over = true; break; }
          if (STORE) refine_cross(A, a, gb, ip, z2, A.geo + (base + o) * 4, A.pts + (base + o) * A.W);
          o++;
        }
      }
    }
    if (!over) JSC_PUT_BASE(ip);
  }
#undef JSC_PUT_BASE
  if (over || o > NLOS) {
    atomicOr(A.status, JSC_DEV_ERR_NLOS);
    if (!STORE) A.nlos[r] = 0;
    return;
  }
  if (!STORE) {
    A.nlos[r] = o;
    return;
  }
  // Chord step lengths, column densities, layer index and factor.
  double xp[3], xc[3], xn[3];
  double *go = A.geo + base * 4;
  jsc_geo2cart(go[0], go[1], go[2], xc);
  if (o > 1) jsc_geo2cart(go[4], go[5], go[6], xn);
  for (int i = 0; i < o; i++) {
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
    for (int c = 0; c < 3; c++) {
      xp[c] = xc[c];
      xc[c] = xn[c];
    }
    if (i + 2 < o) jsc_geo2cart(go[(size_t)(i + 2) * 4], go[(size_t)(i + 2) * 4 + 1],
                                go[(size_t)(i + 2) * 4 + 2], xn);
  }
}

// Exclusive scan of nlos into off[0..n] by one block.
__global__ void scan_kernel(const int *nlos, int n, int64_t *off) {
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

// ------------------------------------------------------------- EGA + RT --


// Continuum extinction of one channel at one LOS point
// (src/forwardmodel.c:120-152 with src/continua.c:5-2049).
__device__ __forceinline__ double continua(const jsc_dev_model &m,
                                           const jsc_run_cfg &cfg,
                                           const jsc_ctm_coef &c, double nu,
                                           double kwin, double P, double T,
                                           double DS, double qh2o,
                                           const double *u) {
  double beta = kwin;
  if (cfg.ctm_co2) {
    double ctm = 0;
    if (m.ig_co2 >= 0 && c.co2_on) {
      const double dt230 = T - 230, dt260 = T - 260, dt296 = T - 296;
      const double ctw = dt260 * 5.050505e-4 * dt296 * c.co2_c230 -
                         dt230 * 9.259259e-4 * dt296 * c.co2_c260 +
                         dt230 * 4.208754e-4 * dt260 * c.co2_c296;
      ctm = u[m.ig_co2] / JSC_AVOGADRO / 1000 * P / JSC_P0 * ctw;
    }
    beta += ctm / DS;
  }
  if (cfg.ctm_h2o) {
    double ctm = 0;
    if (m.ig_h2o >= 0 && c.h2o_on) {
      const double ctwslf = c.h2o_self296 * pow(c.h2o_ratio, (296 - T) / (296 - 260));
      const double a1 = nu * u[m.ig_h2o] * tanh(.7193876 / T * nu);
      const double a2 = 296 / T;
      const double a3 = P / JSC_P0 * (qh2o * ctwslf + (1 - qh2o) * c.h2o_frn) * 1e-20;
      ctm = a1 * a2 * a3;
    }
    beta += ctm / DS;
  }
  if (cfg.ctm_n2 && c.n2_on) {
    const double t0 = 273, tr = 296, q_n2 = 0.79;
    const double pp = P / JSC_P0, tt = t0 / T;
    beta += 0.1 * (pp * pp) * (tt * tt) * q_n2 * c.n2_b *
            exp(c.n2_beta * (1 / tr - 1 / T)) *
            (q_n2 + (1 - q_n2) * (1.294 - 0.4545 * T / tr));
  }
  if (cfg.ctm_o2 && c.o2_on) {
    const double t0 = 273, tr = 296, q_o2 = 0.21;
    const double pp = P / JSC_P0, tt = t0 / T;
    beta += 0.1 * (pp * pp) * (tt * tt) * q_o2 * c.o2_b *
            exp(c.o2_beta * (1 / tr - 1 / T));
  }
  return beta;
}

// Key of node i (u or eps).
template <bool U>
__device__ __forceinline__ float nkey(const jsc_node *row, int i) {
  return U ? __ldg(&row[i].u) : __ldg(&row[i].e);
}

// locate_tbl (src/forwardmodel.c:546-565) on one table row of n >= 2
// points.  key > x is evaluated as key > RD(x) (x rounded down to float),
// which is exact for float keys.
template <bool U>
__device__ __forceinline__ int bisect_row(const jsc_node *row, int n, double x) {
  const float xf = __double2float_rd(x);
  const bool nan = !(x == x);
  int ilo = 0, ihi = n - 1;
  while (ihi > ilo + 1) {
    const int i = (ihi + ilo) >> 1;
    if (!nan && nkey<U>(row, i) > xf) ihi = i; else ilo = i;
  }
  return ilo;
}

// Same result as bisect_row for a row with strictly increasing keys,
// found by an exponential search from the guess h: the largest i <= n-2
// with key[i] <= x, or 0.
template <bool U>
__device__ __forceinline__ int search_row(const jsc_node *row, int n, double x, int h) {
  if (!(x == x)) return n - 2;
  const float xf = __double2float_rd(x);
  const int last = n - 2;
  int i = h < 0 ? 0 : (h > last ? last : h);
  const float klo = nkey<U>(row, i), khi = nkey<U>(row, i + 1);
  int lo, hi;
  if (!(klo > xf)) {
    if (khi > xf || i == last) return i;
    lo = i + 1;
    int step = 1;
    while (true) {
      const int pr = lo + step;
      if (pr > last) { hi = last + 1; break; }
      if (nkey<U>(row, pr) > xf) { hi = pr; break; }
      lo = pr;
      step <<= 1;
    }
  } else {
    if (i == 0) return 0;
    hi = i;
    int step = 1;
    while (true) {
      const int pr = hi - step;
      if (pr <= 0) { lo = 0; break; }
      if (!(nkey<U>(row, pr) > xf)) { lo = pr; break; }
      hi = pr;
      step <<= 1;
    }
  }
  while (hi > lo + 1) {
    const int mid = (lo + hi) >> 1;
    if (nkey<U>(row, mid) > xf) hi = mid; else lo = mid;
  }
  return lo;
}

// LIN on float table entries with the slope already in float, as the
// reference evaluates it: y0 + slope * (x - x0), promoted to double.
__device__ __forceinline__ double lin_node(float x0, float y0, float slope, double x) {
  return (double)y0 + (double)slope * (x - (double)x0);
}

// Emissivity of the extended path at one (p, T) node of a table
// (intpol_tbl_u then intpol_tbl_eps, src/forwardmodel.c:460-474): invert
// the path emissivity x1 to a column density on the row, add the segment's
// column, look the emissivity up again, clamp to [0, 1].
//
// Fast path: the row is strictly increasing, the interval [h, h+1] of the
// previous point still brackets x1 and the extended column stays in the
// same interval -- then the two nodes h, h+1 (one 32-byte sector) answer
// both lookups.  Otherwise the exact searches above find the intervals.
template <bool DIG>
__device__ __forceinline__ double ega_node(const jsc_node *__restrict__ nodes, jsc_row rd,
                                           double x1, double useg, int hint, int *jout,
                                           unsigned long long *dig) {
  const int n = rd.nf & 0xffff;
  const bool strict = (rd.nf >> 16) & JSC_ROW_STRICT;
  const jsc_node *row = nodes + rd.off;
  const int last = n - 2;
  int k = hint < 0 ? 0 : (hint > last ? last : hint);
  float4 a = __ldg(reinterpret_cast<const float4 *>(row + k));
  float4 b = __ldg(reinterpret_cast<const float4 *>(row + k + 1));
  const float x1f = __double2float_rd(x1);
  // bracket for x1 on eps: (e[k] <= x1 or k == 0) and (x1 < e[k+1] or k == last)
  if (!(strict && (!(a.y > x1f) || k == 0) && (b.y > x1f || k == last) && x1 == x1)) {
    k = strict ? search_row<false>(row, n, x1, k) : bisect_row<false>(row, n, x1);
    a = __ldg(reinterpret_cast<const float4 *>(row + k));
    b = __ldg(reinterpret_cast<const float4 *>(row + k + 1));
  }
  const double x2 = lin_node(a.y, a.x, a.z, x1) + useg;
  const float x2f = __double2float_rd(x2);
  int j = k;
  if (!(strict && (!(a.x > x2f) || k == 0) && (b.x > x2f || k == last) && x2 == x2)) {
    j = strict ? search_row<true>(row, n, x2, k) : bisect_row<true>(row, n, x2);
    if (j != k) a = __ldg(reinterpret_cast<const float4 *>(row + j));
  }
  if (DIG) *dig = (*dig * 1000003ull + (unsigned long long)k) * 1000003ull + (unsigned long long)j;
  *jout = j;
  return jsc_clamp01(lin_node(a.x, a.y, a.w, x2));
}

// One thread per (ray, channel).  The path state of every emitter lives in
// registers (GMAX >= ng, the emitter loop is unrolled so the lookups of
// different emitters overlap); LOS records are read by all threads of a
// ray (broadcast loads).
template <int GMAX, bool DIG, int BLK, int MINB>
__global__ void __launch_bounds__(BLK, MINB) ega_rt_kernel(EgaArgs A) {
  const jsc_dev_model &m = A.m;
  const int nd = m.nd, ng = m.ng;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = tid / A.ndp;
  const int d = tid - r * A.ndp;
  if (r >= A.n_rays || d >= nd) return;

  // per-channel constants
  const int w = m.window[d];
  const bool has_w = w < m.nw;
  const jsc_ctm_coef cc = m.ctm[d];
  const double nu = m.nu[d];
  const double *__restrict__ pb = m.planck_b + (size_t)d * JSC_NPLANCK;
  const double *__restrict__ ps = m.planck_s + (size_t)d * JSC_NPLANCK;
  const jsc_row *__restrict__ rows_d = m.rows + (size_t)d * ng * (TBLNPMAX * TBLNTMAX);
  unsigned okmask = 0;
  for (int g = 0; g < ng && g < GMAX; g++)
    if (m.tab_grid[d * ng + g] >= 0) okmask |= 1u << g;

  double tp[GMAX];
  int hint[GMAX];
#pragma unroll
  for (int g = 0; g < GMAX; g++) {
    tp[g] = 1;
    hint[g] = 0;
  }
  double rad = 0, tau = 1;
  unsigned long long dig = 0;
  unsigned n_ega = 0;
  const int np = A.nlos[r];
  const double *__restrict__ rec = A.pts + (size_t)A.los_off[r] * A.W;

  for (int ip = 0; ip < np; ip++, rec += A.W) {
    const double P = rec[REC_P], T = rec[REC_T], DS = rec[REC_DS];
    const int itp = (int)rec[REC_PLK];
    int code = (int)rec[REC_GRID];
    double tau_gas = 1;
#pragma unroll
    for (int g = 0; g < GMAX; g++) {
      if (g >= ng) break;
      double eps = 0;
      const double tpg = tp[g];
      if (!((okmask >> g) & 1u)) {
        eps = 0;
      } else if (tpg < 1e-9) {
        eps = 1;
      } else {
        const int gid = A.single_grid ? 0 : m.tab_grid[d * ng + g];
        if (!A.single_grid)
          code = grid_code(m.grid_np[gid], m.grid_p + (size_t)gid * TBLNPMAX,
                           m.grid_nt + (size_t)gid * TBLNPMAX,
                           m.grid_t + (size_t)gid * TBLNPMAX * TBLNTMAX, P, T);
        if (code & (1 << 16)) {
          const int ipr = (code >> 10) & 63, it0 = (code >> 5) & 31, it1 = code & 31;
          const jsc_row *rw = rows_d + (size_t)g * (TBLNPMAX * TBLNTMAX);
          const jsc_row r00 = rw[ipr * TBLNTMAX + it0];
          const jsc_row r01 = rw[ipr * TBLNTMAX + it0 + 1];
          const jsc_row r10 = rw[(ipr + 1) * TBLNTMAX + it1];
          const jsc_row r11 = rw[(ipr + 1) * TBLNTMAX + it1 + 1];
          if ((r00.nf & 0xffff) >= 2 && (r01.nf & 0xffff) >= 2 &&
              (r10.nf & 0xffff) >= 2 && (r11.nf & 0xffff) >= 2) {
            const double x1 = 1 - tpg, useg = rec[REC_K + m.nw + g];
            if (DIG) dig = dig * 1000003ull + (unsigned long long)(ipr * 961 + it0 * 31 + it1);
            int j00, jx;
            const double e00 = ega_node<DIG>(m.nodes, r00, x1, useg, hint[g], &j00, &dig);
            const double e01 = ega_node<DIG>(m.nodes, r01, x1, useg, hint[g], &jx, &dig);
            const double e10 = ega_node<DIG>(m.nodes, r10, x1, useg, hint[g], &jx, &dig);
            const double e11 = ega_node<DIG>(m.nodes, r11, x1, useg, hint[g], &jx, &dig);
            hint[g] = j00;
            const double *gp = m.grid_p + (size_t)gid * TBLNPMAX;
            const double *gt = m.grid_t + (size_t)gid * TBLNPMAX * TBLNTMAX;
            double ea = jsc_clamp01(jsc_lin(gt[ipr * TBLNTMAX + it0], e00,
                                            gt[ipr * TBLNTMAX + it0 + 1], e01, T));
            const double eb = jsc_clamp01(jsc_lin(gt[(ipr + 1) * TBLNTMAX + it1], e10,
                                                  gt[(ipr + 1) * TBLNTMAX + it1 + 1], e11, T));
            ea = jsc_clamp01(jsc_lin(gp[ipr], ea, gp[ipr + 1], eb, P));
            eps = 1 - (1 - ea) / tpg;
            n_ega++;
          }
        }
      }
      tp[g] = tpg * (1 - eps);
      tau_gas *= (1 - eps);
    }
    const double beta = continua(m, A.cfg, cc, nu, has_w ? rec[REC_K + w] : 0.0, P, T, DS,
                                 rec[REC_QH2O], rec + REC_K + m.nw);
    const double src = pb[itp] + ps[itp] * (T - planck_temp(itp));
    if (tau_gas > 0) {
      // clear air, or aerosol/cloud extinction without a scattering source
      // (src/forwardmodel.c:365-389)
      const double af = rec[REC_AF];
      double eps;
      if (A.cfg.sca_n == 0 || af == 0) {
        eps = 1 - tau_gas * exp(-1. * beta * DS);
      } else {
        const int ia = (int)rec[REC_AI];
        const double bx = A.beta[(A.cfg.sca_ext_beta_a ? 2 : 0) * A.aero_nl * nd + ia * nd + d];
        eps = 1 - tau_gas * exp(-1. * (beta + af * bx) * DS);
      }
      rad += src * eps * tau;
      tau *= (1 - eps);
    }
  }
  const double ts = A.tsurf[r];
  if (ts > 0) {
    const int its = planck_index(ts);
    rad += (pb[its] + ps[its] * (ts - planck_temp(its))) * tau;
  }
  A.rad[(size_t)r * nd + d] = rad;
  A.tau[(size_t)r * nd + d] = tau;
  if (DIG) A.digest[(size_t)r * nd + d] = dig;
  const unsigned mask = __activemask();
  const unsigned tot = __reduce_add_sync(mask, n_ega);
  if ((threadIdx.x & 31) == __ffs(mask) - 1) atomicAdd(&A.counters[1], (unsigned long long)tot);
}
