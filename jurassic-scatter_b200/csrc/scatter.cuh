// Device kernels of the scattering source (srcfunc_sca, src/scatter.c:643-807
// for thermal radiation in 1-D atmospheres, :899-1041 for the sun).
//
//   sp_count_kernel     scattering points per ray (LOS points with aerosol
//                       factor > 0, src/forwardmodel.c:317)
//   sp_list_kernel      one record per scattering point: position, LOS
//                       direction, layer, observation time, profile
//   sp_spawn_kernel     the secondary pencils of a chunk of points, written
//                       as the rays of a child batch (src/scatter.c:698-735)
//   sp_integral_kernel  phase-function weighted integral of the secondary
//                       radiances over 180 x 180 directions (:737-800)
//   sun_kernel          solar direction search by repeated ray tracing and
//                       the solar pencil of each point (:899-995)
//   sun_add_kernel      adds the attenuated solar term to the source
//
// A batch whose rays scatter runs, bottom up: its own ray tracing and
// layer refinement, these kernels (the secondary and solar pencils run as
// child batches of one scattering order less), then the radiative transfer
// with the scattering source at every scattering point.
#pragma once
#include "kernels.cuh"

#define JSC_SP_REC 10     // doubles per scattering point record
#define JSC_NPHI_SCA 180  // azimuth steps of the source integral
#define JSC_NTH_SCA 180   // polar steps of the source integral
#define JSC_NALPHA_MAX 32 // secondary pencils per scattering point

// Scattering point record (doubles): x[3], dx[3], layer, time, pressure,
// temperature.
enum { SP_X = 0, SP_DX = 3, SP_IL = 6, SP_TIME = 7, SP_P = 8, SP_T = 9 };

// Orthonormal basis with ez along dz and ey in the plane of dy and dz
// (bascoord, src/scatter.c:6-52).
__device__ inline void jsc_bascoord(const double *dz, const double *dy, double *ex, double *ey,
                                    double *ez) {
  double dotp, norm = sqrt(dz[0] * dz[0] + dz[1] * dz[1] + dz[2] * dz[2]);
  for (int i = 0; i < 3; i++) ez[i] = dz[i] / norm;
  norm = sqrt(dy[0] * dy[0] + dy[1] * dy[1] + dy[2] * dy[2]);
  for (int i = 0; i < 3; i++) ey[i] = dy[i] / norm;
  dotp = ey[0] * ez[0] + ey[1] * ez[1] + ey[2] * ez[2];
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
  norm = sqrt(ey[0] * ey[0] + ey[1] * ey[1] + ey[2] * ey[2]);
  for (int i = 0; i < 3; i++) ey[i] /= norm;
  ex[0] = ey[1] * ez[2] - ey[2] * ez[1];
  ex[1] = ey[2] * ez[0] - ey[0] * ez[2];
  ex[2] = ey[0] * ez[1] - ey[1] * ez[0];
}

// Angle between two vectors (the ANGLE macro, src/jurassic.h:33-34).
__device__ __forceinline__ double jsc_angle(const double *a, const double *b) {
  const double c = (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) /
                   sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) /
                   sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
  return acos(fmin(fmax(c, -1.0), 1.0));
}

// Local frame at x: lz up, ly towards north (src/scatter.c:690-693).
__device__ __forceinline__ void local_frame(const double *x, double *lx, double *ly, double *lz) {
  double dnorth[3];
  dnorth[0] = -x[0];
  dnorth[1] = -x[1];
  dnorth[2] = 2 * JSC_RE - x[2];
  jsc_bascoord(x, dnorth, lx, ly, lz);
}

// --------------------------------------------------------- point list --

// Points of a chunk [first, first + n_pts) of a point list whose total
// count is on the device (n_total; null: all n_pts are real).  Fixed-
// capacity scattering runs launch every chunk up to the list's capacity;
// slots past the real count become null pencils (observer and view point
// far above the atmosphere: no LOS point, no work) and their sources are
// never read.
__device__ __forceinline__ int live_points(const int64_t *n_total, int64_t first, int n_pts) {
  if (!n_total) return n_pts;
  const int64_t left = *n_total - first;
  return left <= 0 ? 0 : (left < n_pts ? (int)left : n_pts);
}

#define JSC_NULL_Z 1.0e4  // altitude of a null pencil's observer and view point [km]

struct SpArgs {
  int n_rays, W;
  const int *nlos;
  const int64_t *los_off;
  const double *geo, *pts;
  const double *time;       // [n_rays]
  const int *ray_atm;
  int *nsp;                 // [n_rays] scattering points per ray
  const int64_t *sp_off;    // [n_rays+1]
  double *sp;               // [n_sp][JSC_SP_REC]
  int *sp_atm;              // [n_sp] profile of the point
  int64_t max_sp;           // capacity of sp (fixed-capacity runs; 0: unbounded)
  int *nlos_mut;            // rays whose points do not fit: their LOS is emptied
  unsigned *status;
  unsigned long long *n_listed;  // points actually listed (fixed-capacity runs)
};

// Points a fixed-capacity run lists: all of them, or up to the first ray
// whose points do not fit (sp_list_kernel lowers it with atomicMin).
static __global__ void sp_listed_init_kernel(const int64_t *sp_total, int64_t max_sp,
                                             unsigned long long *n_listed) {
  const int64_t t = *sp_total;
  *n_listed = (unsigned long long)(t < max_sp ? t : max_sp);
}

static __global__ void sp_count_kernel(SpArgs A) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n_rays) return;
  const double *rec = A.pts + A.los_off[r] * A.W;
  int n = 0;
  for (int ip = 0; ip < A.nlos[r]; ip++)
    if (rec[(size_t)ip * A.W + REC_AF] > 0) n++;
  A.nsp[r] = n;
}

// x is the point, dx the chord between its neighbours
// (src/forwardmodel.c:319-327).  The reference takes ip+1 as the next
// point even at the last LOS point, which reads past the line of sight;
// the last point stands in for its missing neighbour.
static __global__ void sp_list_kernel(SpArgs A) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n_rays) return;
  const int np = A.nlos[r];
  if (A.max_sp > 0 && A.sp_off[r + 1] > A.max_sp) {
    // more scattering points than the fixed capacity: the run reports the
    // overflow and this ray keeps no LOS point, so nothing reads past sp
    atomicOr(A.status, JSC_DEV_ERR_QUEUE);
    atomicMin(A.n_listed, (unsigned long long)A.sp_off[r]);
    A.nlos_mut[r] = 0;
    return;
  }
  const double *rec = A.pts + A.los_off[r] * A.W;
  const double *geo = A.geo + A.los_off[r] * 4;
  int64_t k = A.sp_off[r];
  for (int ip = 0; ip < np; ip++) {
    const double *rc = rec + (size_t)ip * A.W;
    if (!(rc[REC_AF] > 0)) continue;
    const int ip0 = ip > 0 ? ip - 1 : ip, ip1 = ip + 1 < np ? ip + 1 : ip;
    double x[3], x0[3], x1[3];
    jsc_geo2cart(geo[(size_t)ip * 4], geo[(size_t)ip * 4 + 1], geo[(size_t)ip * 4 + 2], x);
    jsc_geo2cart(geo[(size_t)ip0 * 4], geo[(size_t)ip0 * 4 + 1], geo[(size_t)ip0 * 4 + 2], x0);
    jsc_geo2cart(geo[(size_t)ip1 * 4], geo[(size_t)ip1 * 4 + 1], geo[(size_t)ip1 * 4 + 2], x1);
    double *o = A.sp + (size_t)k * JSC_SP_REC;
    for (int i = 0; i < 3; i++) {
      o[SP_X + i] = x[i];
      o[SP_DX + i] = x1[i] - x0[i];
    }
    o[SP_IL] = rc[REC_AI];
    o[SP_TIME] = A.time[r];
    o[SP_P] = rc[REC_P];
    o[SP_T] = rc[REC_T];
    A.sp_atm[k] = A.ray_atm[r];
    k++;
  }
}

// ------------------------------------------------------- secondary rays --

struct SpawnArgs {
  int n_pts, nalpha;        // points of this chunk, pencils per point
  const int64_t *n_total;   // device count of the whole list (null: all real)
  int64_t first;            // index of the chunk's first point in the list
  const double *sp;         // first record of the chunk
  const int *sp_atm;
  double alpha[JSC_NALPHA_MAX];
  int *ray_atm;             // child batch inputs, n_pts * nalpha rays
  double *ray;              // [7][n_pts * nalpha]: time obsz obslon obslat vpz vplon vplat
};

// Secondary pencil ir of point k: from x towards the view point 10 km away
// at zenith angle alpha[ir] in the north-up plane (src/scatter.c:722-735).
static __global__ void sp_spawn_kernel(SpawnArgs A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = A.n_pts * A.nalpha;
  if (t >= n) return;
  const int k = t / A.nalpha, ir = t - k * A.nalpha;
  if (k >= live_points(A.n_total, A.first, A.n_pts)) {  // null pencil
    A.ray_atm[t] = 0;
    for (int i = 0; i < 7; i++) A.ray[(size_t)i * n + t] = (i == 1 || i == 4) ? JSC_NULL_Z : 0.0;
    return;
  }
  const double *o = A.sp + (size_t)k * JSC_SP_REC;
  const double x[3] = {o[SP_X], o[SP_X + 1], o[SP_X + 2]};
  double lx[3], ly[3], lz[3], xv[3];
  local_frame(x, lx, ly, lz);
  const double al = A.alpha[ir];
  for (int i = 0; i < 3; i++) xv[i] = x[i] + 10. * cos(al) * (-1) * lz[i] + 10. * sin(al) * ly[i];
  double oz, olon, olat, vz, vlon, vlat;
  jsc_cart2geo(x, &oz, &olon, &olat);
  jsc_cart2geo(xv, &vz, &vlon, &vlat);
  A.ray_atm[t] = A.sp_atm[k];
  A.ray[t] = 0;  // the reference leaves the secondary observation time at 0
  A.ray[(size_t)n + t] = oz;
  A.ray[2 * (size_t)n + t] = olon;
  A.ray[3 * (size_t)n + t] = olat;
  A.ray[4 * (size_t)n + t] = vz;
  A.ray[5 * (size_t)n + t] = vlon;
  A.ray[6 * (size_t)n + t] = vlat;
}

// --------------------------------------------------------- source integral --

struct IntegralArgs {
  int n_pts, nalpha, nd, nl;
  const int64_t *n_total;   // device count of the whole list (null: all real)
  int64_t first;
  const double *sp;          // first record of the chunk
  double alpha[JSC_NALPHA_MAX];
  const double *rad;         // [n_pts * nalpha][nd] secondary radiances
  const double *phase;       // [nl][nd][NTHETA]
  double *src;               // [n_pts][nd] of the chunk
};

#define JSC_INT_THREADS 256
#define JSC_INT_CH 16  // channels per pass over the directions

// One block per scattering point.  Directions (itheta, iphi) are spread
// over the threads; the polar factor sin(theta2) * phase(theta2) of each
// (itheta, channel), the secondary radiances, their slopes and the pencil
// angles sit in shared memory.  The radiance and slope rows have odd
// strides in doubles, so lanes whose directions fall in different alpha
// intervals read different banks.  Weighted sums follow
// src/scatter.c:737-805 up to the order of the sum.
static __global__ void __launch_bounds__(JSC_INT_THREADS)
sp_integral_kernel(IntegralArgs A) {
  extern __shared__ double sh[];
  const int k = blockIdx.x;
  if (k >= live_points(A.n_total, A.first, A.n_pts)) return;
  const int nd = A.nd, na = A.nalpha;
  const int ndp = nd | 1, SL = JSC_INT_CH + 1;      // odd row strides
  double *wt = sh;                                   // [JSC_NTH_SCA][nd]
  double *rd = wt + (size_t)JSC_NTH_SCA * nd;        // [na][ndp]
  double *trig = rd + (size_t)na * ndp;              // sin/cos of theta2 and phi
  double *red = trig + 4 * JSC_NTH_SCA;              // [JSC_INT_THREADS / 32][JSC_INT_CH]
  double *slp = red + (JSC_INT_THREADS / 32) * JSC_INT_CH;  // [na - 1][SL]
  double *alf = slp + (size_t)na * SL;               // [na] pencil angles
  const double *o = A.sp + (size_t)k * JSC_SP_REC;
  const int il = (int)o[SP_IL];
  for (int i = threadIdx.x; i < JSC_NTH_SCA; i += blockDim.x) {
    const double th = (0.5 + i) * M_PI / 180.;
    const double ph = 2. * (0.5 + i) * M_PI / 180.;
    trig[i] = sin(th);
    trig[JSC_NTH_SCA + i] = cos(th);
    trig[2 * JSC_NTH_SCA + i] = sin(ph);
    trig[3 * JSC_NTH_SCA + i] = cos(ph);
  }
  for (int i = threadIdx.x; i < na * nd; i += blockDim.x) {
    const int ir = i / nd, id = i - ir * nd;
    rd[(size_t)ir * ndp + id] = A.rad[((size_t)k * na + ir) * nd + id];
  }
  for (int i = threadIdx.x; i < na; i += blockDim.x) alf[i] = A.alpha[i];
  __syncthreads();
  // Polar weight sin(theta2) * phase(theta2); phase on the 1-degree grid.
  const double *ph = A.phase + (size_t)il * nd * NTHETA;
  for (int i = threadIdx.x; i < JSC_NTH_SCA * nd; i += blockDim.x) {
    const int it = i / nd, id = i - it * nd;
    const double th = (0.5 + it) * M_PI / 180.;
    // locate(theta, NTHETA, theta2) on theta[i] = i * pi / 180
    int j = 0, hi = NTHETA - 1;
    while (hi > j + 1) {
      const int mid = (hi + j) >> 1;
      if ((double)mid * M_PI / 180. > th) hi = mid; else j = mid;
    }
    const double a0 = (double)j * M_PI / 180., a1 = (double)(j + 1) * M_PI / 180.;
    const double phase2 = jsc_lin(a0, ph[(size_t)id * NTHETA + j], a1, ph[(size_t)id * NTHETA + j + 1], th);
    wt[i] = trig[it] * phase2;
  }
  __syncthreads();

  double x[3], dx[3], lx[3], ly[3], lz[3], sx[3], sy[3], sz[3], mlz[3];
  for (int i = 0; i < 3; i++) {
    x[i] = o[SP_X + i];
    dx[i] = o[SP_DX + i];
  }
  local_frame(x, lx, ly, lz);
  jsc_bascoord(dx, x, sx, sy, sz);
  for (int i = 0; i < 3; i++) mlz[i] = -1. * lz[i];
  const int ndir = JSC_NTH_SCA * JSC_NPHI_SCA;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c0 = 0; c0 < nd; c0 += JSC_INT_CH) {
    // slopes (r1 - r0) / (a1 - a0) of the pass's channels per alpha
    // interval, the quotient jsc_lin evaluates first
    for (int i = threadIdx.x; i < (na - 1) * JSC_INT_CH; i += blockDim.x) {
      const int lo = i / JSC_INT_CH, c = i - lo * JSC_INT_CH;
      if (c0 + c < nd)
        slp[lo * SL + c] = (rd[(size_t)(lo + 1) * ndp + c0 + c] - rd[(size_t)lo * ndp + c0 + c]) /
                           (alf[lo + 1] - alf[lo]);
    }
    __syncthreads();
    double acc[JSC_INT_CH];
#pragma unroll
    for (int c = 0; c < JSC_INT_CH; c++) acc[c] = 0;
    for (int dir = threadIdx.x; dir < ndir; dir += blockDim.x) {
      const int it = dir / JSC_NPHI_SCA, iq = dir - it * JSC_NPHI_SCA;
      const double st = trig[it], ct = trig[JSC_NTH_SCA + it];
      const double sp = trig[2 * JSC_NTH_SCA + iq], cp = trig[3 * JSC_NTH_SCA + iq];
      double ek[3];
      for (int i = 0; i < 3; i++) ek[i] = st * sp * sx[i] + st * cp * sy[i] + ct * sz[i];
      const double alpha2 = jsc_angle(mlz, ek);
      // locate(alpha, nalpha, alpha2): alpha increases from 0 to pi
      int lo = 0, hi = na - 1;
      while (hi > lo + 1) {
        const int mid = (hi + lo) >> 1;
        if (alf[mid] > alpha2) hi = mid; else lo = mid;
      }
      const double da = alpha2 - alf[lo];
      const double *w = wt + (size_t)it * nd + c0;
      const double *r0 = rd + (size_t)lo * ndp + c0, *s0 = slp + lo * SL;
#pragma unroll
      for (int c = 0; c < JSC_INT_CH; c++)
        if (c0 + c < nd) acc[c] += w[c] * (r0[c] + s0[c] * da);  // jsc_lin, slope precomputed
    }
    // block reduction per channel
#pragma unroll
    for (int c = 0; c < JSC_INT_CH; c++) {
      double v = acc[c];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) red[warp * JSC_INT_CH + c] = v;
    }
    __syncthreads();
    if (threadIdx.x < JSC_INT_CH && c0 + threadIdx.x < nd) {
      const int id = c0 + threadIdx.x;
      double s = 0, wsum = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w * JSC_INT_CH + threadIdx.x];
      for (int it = 0; it < JSC_NTH_SCA; it++) wsum += wt[(size_t)it * nd + id];
      wsum *= JSC_NPHI_SCA;
      A.src[(size_t)k * nd + id] = s / wsum;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ sun --

struct SunArgs {
  RayArgs ra;                // profiles, tracing switches, status word
  int n_pts;
  const int64_t *n_total;    // device count of the whole list (null: all real)
  int64_t first;
  const double *sp;          // first record of the chunk
  const int *sp_atm;
  // aerosol refinement edges (the last segment of each solar ray)
  int n_alti;
  double altimax, altimin;
  const double *alti;
  // outputs: the solar pencil of each point as a child-batch ray
  int *ray_atm;
  double *ray;               // [7][n_pts]
  double *theta2;            // [n_pts] scattering angle, or -1: no solar term
};

// Solar position (src/scatter.c:999-1041).
__device__ inline void jsc_suncoord(double sec, double lon, double lat, double *azi, double *sza) {
  const double D = sec / 86400 - 0.5;
  const double g = (357.529 + 0.98560028 * D) * M_PI / 180;
  const double q = 280.459 + 0.98564736 * D;
  const double L = (q + 1.915 * sin(g) + 0.020 * sin(2 * g)) * M_PI / 180;
  const double e = (23.439 - 0.00000036 * D) * M_PI / 180;
  const double dec = asin(sin(e) * sin(L));
  const double ra = atan2(cos(e) * sin(L), cos(L));
  const double GMST = 18.697374558 + 24.06570982441908 * D;
  const double LST = GMST + lon / 15;
  const double h = LST / 12 * M_PI - ra;
  lat *= M_PI / 180;
  *azi = atan2(-sin(h), cos(lat) * tan(dec) - sin(lat) * cos(h)) * 180 / M_PI;
  *sza = acos(sin(lat) * sin(dec) + cos(lat) * cos(dec) * cos(h)) * 180 / M_PI;
}

// The point before the last of the refined line of sight: the last layer
// edge inserted between the last two traced points (add_aerosol_layers,
// src/lineofsight.c:210-290, applied to the final segment), else the
// traced point before the last.
__device__ inline void refined_prev(const SunArgs &A, const double *g0, const double *g1,
                                    double *out) {
  const double zp = g0[0], zc = g1[0];
  out[0] = g0[0];
  out[1] = g0[1];
  out[2] = g0[2];
  if (!((zp < A.altimax || zc < A.altimax) && (zp > A.altimin || zc > A.altimin))) return;
  for (int il = 0; il < A.n_alti; il++) {
    const double z1 = A.alti[il], z2 = A.alti[A.n_alti - il - 1];
    double znew;
    if (zp > z1 && zc < z1) znew = z1;
    else if (zp < z2 && zc > z2) znew = z2;
    else continue;
    double x1[3], x2[3];
    const double frac = (zp - znew) / (zp - zc);
    jsc_geo2cart(g0[0], g0[1], g0[2], x1);
    jsc_geo2cart(g1[0], g1[1], g1[2], x2);
    for (int i = 0; i < 3; i++) x2[i] = x1[i] + frac * (x2[i] - x1[i]);
    jsc_cart2geo(x2, &out[0], &out[1], &out[2]);
  }
}

// Solar pencil of each scattering point: search the zenith angle whose
// refracted ray arrives from the sun's direction (up to 10 corrections),
// then, when that ray does not end on the ground, hand it to the solar
// child batch with the scattering angle to the LOS direction.
template <int IP = 1>
__global__ void __launch_bounds__(128) sun_kernel(SunArgs A) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= A.n_pts) return;
  if (k >= live_points(A.n_total, A.first, A.n_pts)) {  // null solar pencil, no term
    const int n = A.n_pts;
    A.ray_atm[k] = 0;
    for (int i = 0; i < 7; i++) A.ray[(size_t)i * n + k] = (i == 1 || i == 4) ? JSC_NULL_Z : 0.0;
    A.theta2[k] = -1.0;
    return;
  }
  const double *o = A.sp + (size_t)k * JSC_SP_REC;
  const double x[3] = {o[SP_X], o[SP_X + 1], o[SP_X + 2]};
  const double dx[3] = {o[SP_DX], o[SP_DX + 1], o[SP_DX + 2]};
  const int ai = A.sp_atm[k];
  double lx[3], ly[3], lz[3], ek[3] = {0, 0, 0}, x1[3], azi, sza;
  local_frame(x, lx, ly, lz);
  RayIn in;
  jsc_cart2geo(x, &in.obsz, &in.obslon, &in.obslat);
  jsc_suncoord(o[SP_TIME], in.obslon, in.obslat, &azi, &sza);
  double sza_cor = sza;
  RayEnd end;
  end.tsurf = -999;
  for (int i2 = 0; i2 < 10; i2++) {
    for (int i = 0; i < 3; i++) {
      ek[i] = sin(sza_cor * M_PI / 180) * sin(azi * M_PI / 180) * lx[i] +
              sin(sza_cor * M_PI / 180) * cos(azi * M_PI / 180) * ly[i] +
              cos(sza_cor * M_PI / 180) * lz[i];
      x1[i] = x[i] + 10 * ek[i];
    }
    jsc_cart2geo(x1, &in.vpz, &in.vplon, &in.vplat);
    const int np = trace_core<2, IP>(A.ra, ai, 0, in, &end);
    if (np < 2) break;
    double g0[3], xa[3], xb[3], dout[3];
    refined_prev(A, end.g[0], end.g[1], g0);
    jsc_geo2cart(g0[0], g0[1], g0[2], xa);
    jsc_geo2cart(end.g[1][0], end.g[1][1], end.g[1][2], xb);
    for (int i = 0; i < 3; i++) dout[i] = xb[i] - xa[i];
    const double sza_beam = jsc_angle(x, dout) * 180 / M_PI;
    if (fabs(sza_beam - sza) < 0.01) break;
    sza_cor -= 0.61803 * (sza_beam - sza);
    sza_cor = fmin(fmax(sza_cor, 0.0), 180.0);
  }
  const int n = A.n_pts;
  A.ray_atm[k] = ai;
  A.ray[k] = 0;
  A.ray[(size_t)n + k] = in.obsz;
  A.ray[2 * (size_t)n + k] = in.obslon;
  A.ray[3 * (size_t)n + k] = in.obslat;
  A.ray[4 * (size_t)n + k] = in.vpz;
  A.ray[5 * (size_t)n + k] = in.vplon;
  A.ray[6 * (size_t)n + k] = in.vplat;
  A.theta2[k] = end.tsurf < 0 ? jsc_angle(ek, dx) : -1.0;
}

struct SunAddArgs {
  int n_pts, nd;
  const double *sp;          // first record of the chunk
  const double *theta2;      // [n_pts]
  const double *tau;         // [n_pts][nd] transmittance of the solar pencils
  const double *phase;       // [nl][nd][NTHETA]
  const double *planck_sun;  // [nd] Planck radiance at the solar temperature
  double *src;               // [n_pts][nd] of the chunk
};

// src_sca += 6.764e-5 (solid angle of the sun) x phase x B(TSUN) x tau
// (src/scatter.c:980-990).
static __global__ void sun_add_kernel(SunAddArgs A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.n_pts * A.nd) return;
  const int k = t / A.nd, id = t - k * A.nd;
  const double th2 = A.theta2[k];
  if (th2 < 0) return;
  const int il = (int)A.sp[(size_t)k * JSC_SP_REC + SP_IL];
  // locate(theta, NTHETA, theta2) on theta[i] = pi * i / (NTHETA - 1)
  int lo = 0, hi = NTHETA - 1;
  while (hi > lo + 1) {
    const int mid = (hi + lo) >> 1;
    if (M_PI * (double)mid / (NTHETA - 1) > th2) hi = mid; else lo = mid;
  }
  const double *ph = A.phase + ((size_t)il * A.nd + id) * NTHETA;
  const double phase2 = jsc_lin(M_PI * (double)lo / (NTHETA - 1), ph[lo],
                                M_PI * (double)(lo + 1) / (NTHETA - 1), ph[lo + 1], th2);
  A.src[t] += 6.764e-5 * phase2 * A.planck_sun[id] * A.tau[t];
}

// ------------------------------------------------- 3-D scattering source --
// srcfunc_sca_3d (src/scatter.c:811-895), used with horizontally varying
// atmospheres (IP 2/3): a secondary pencil in every direction of the
// 180 x 180 (polar, azimuth) grid around the line of sight, cast 10 km
// towards its view point, and the phase-function weighted sum of their
// radiances.

#define JSC_NDIR3 (JSC_NTH_SCA * JSC_NPHI_SCA)

struct Spawn3Args {
  int n_pts;
  const double *sp;          // first record of the chunk
  const int *sp_atm;
  int *ray_atm;              // child batch inputs, n_pts * JSC_NDIR3 rays
  double *ray;               // [7][n_pts * JSC_NDIR3]
};

static __global__ void sp_spawn3_kernel(Spawn3Args A) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = (int64_t)A.n_pts * JSC_NDIR3;
  if (t >= n) return;
  const int k = (int)(t / JSC_NDIR3), dir = (int)(t - (int64_t)k * JSC_NDIR3);
  const int it = dir / JSC_NPHI_SCA, iq = dir - it * JSC_NPHI_SCA;
  const double *o = A.sp + (size_t)k * JSC_SP_REC;
  const double x[3] = {o[SP_X], o[SP_X + 1], o[SP_X + 2]};
  const double dx[3] = {o[SP_DX], o[SP_DX + 1], o[SP_DX + 2]};
  double sx[3], sy[3], sz[3], xv[3];
  jsc_bascoord(dx, x, sx, sy, sz);
  const double theta2 = (0.5 + it) / JSC_NTH_SCA * M_PI;
  const double phi = (0.5 + iq) / JSC_NPHI_SCA * 2 * M_PI;
  for (int i = 0; i < 3; i++)
    xv[i] = x[i] + 10 * sin(theta2) * sin(phi) * sx[i] + 10 * sin(theta2) * cos(phi) * sy[i] +
            10 * cos(theta2) * sz[i];
  double oz, olon, olat, vz, vlon, vlat;
  jsc_cart2geo(x, &oz, &olon, &olat);
  jsc_cart2geo(xv, &vz, &vlon, &vlat);
  A.ray_atm[t] = A.sp_atm[k];
  A.ray[t] = 0;  // the secondary observation time stays 0, as in the reference
  A.ray[(size_t)n + t] = oz;
  A.ray[2 * (size_t)n + t] = olon;
  A.ray[3 * (size_t)n + t] = olat;
  A.ray[4 * (size_t)n + t] = vz;
  A.ray[5 * (size_t)n + t] = vlon;
  A.ray[6 * (size_t)n + t] = vlat;
}

struct Integral3Args {
  int n_pts, nd;
  const double *sp;          // first record of the chunk
  const double *rad;         // [n_pts * JSC_NDIR3][nd] secondary radiances
  const double *phase;       // [nl][nd][NTHETA]
  double *src;               // [n_pts][nd] of the chunk
};

// One block per scattering point, channels in passes of JSC_INT_CH: the
// weight pi/180 * 2 pi sin(theta2)/180 * phase(theta2) of each (polar
// angle, channel) in shared memory, directions spread over the threads.
// The reference divides every channel by one sum of the weights over all
// directions *and* channels (src/scatter.c:872-891); so does this.
static __global__ void __launch_bounds__(JSC_INT_THREADS) sp_integral3_kernel(Integral3Args A) {
  __shared__ double wt[JSC_NTH_SCA][JSC_INT_CH];
  __shared__ double red[JSC_INT_THREADS / 32][JSC_INT_CH + 1];
  __shared__ double total;
  const int k = blockIdx.x;
  if (k >= A.n_pts) return;
  const int nd = A.nd;
  const double *o = A.sp + (size_t)k * JSC_SP_REC;
  const int il = (int)o[SP_IL];
  const double *ph = A.phase + (size_t)il * nd * NTHETA;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) total = 0;
  for (int c0 = 0; c0 < nd; c0 += JSC_INT_CH) {
    __syncthreads();
    for (int i = threadIdx.x; i < JSC_NTH_SCA * JSC_INT_CH; i += blockDim.x) {
      const int it = i / JSC_INT_CH, c = i - it * JSC_INT_CH, id = c0 + c;
      double w = 0;
      if (id < nd) {
        const double theta2 = (0.5 + it) / JSC_NTH_SCA * M_PI;
        // locate(theta, NTHETA, theta2) on theta[i] = pi i / (NTHETA - 1)
        int j = 0, hi = NTHETA - 1;
        while (hi > j + 1) {
          const int mid = (hi + j) >> 1;
          if (M_PI * (double)mid / (NTHETA - 1) > theta2) hi = mid; else j = mid;
        }
        const double a0 = M_PI * (double)j / (NTHETA - 1), a1 = M_PI * (double)(j + 1) / (NTHETA - 1);
        const double phase2 = jsc_lin(a0, ph[(size_t)id * NTHETA + j], a1,
                                      ph[(size_t)id * NTHETA + j + 1], theta2);
        w = M_PI / JSC_NTH_SCA * 2 * M_PI * sin(theta2) / JSC_NPHI_SCA * phase2;
      }
      wt[it][c] = w;
    }
    __syncthreads();
    double acc[JSC_INT_CH], ws = 0;
#pragma unroll
    for (int c = 0; c < JSC_INT_CH; c++) acc[c] = 0;
    for (int dir = threadIdx.x; dir < JSC_NDIR3; dir += blockDim.x) {
      const int it = dir / JSC_NPHI_SCA;
      const double *r = A.rad + ((size_t)k * JSC_NDIR3 + dir) * nd + c0;
#pragma unroll
      for (int c = 0; c < JSC_INT_CH; c++)
        if (c0 + c < nd) {
          acc[c] += wt[it][c] * r[c];
          ws += wt[it][c];
        }
    }
#pragma unroll
    for (int c = 0; c <= JSC_INT_CH; c++) {
      double v = c < JSC_INT_CH ? acc[c] : ws;
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x <= JSC_INT_CH) {
      double v = 0;
      for (int w = 0; w < JSC_INT_THREADS / 32; w++) v += red[w][threadIdx.x];
      if (threadIdx.x == JSC_INT_CH) total += v;
      else if (c0 + (int)threadIdx.x < nd) A.src[(size_t)k * nd + c0 + threadIdx.x] = v;
    }
  }
  __syncthreads();
  for (int id = threadIdx.x; id < nd; id += blockDim.x) A.src[(size_t)k * nd + id] /= total;
}
