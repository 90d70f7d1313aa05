// Device functions shared by the ray-tracing and radiative-transfer
// kernels: Planck source lookup, (p, T) table brackets, continua and the
// EGA table lookups.
#pragma once
#include <math.h>
#include <stdint.h>

#include "jsc_model.h"
#include "physics.h"
#include "cuda_util.cuh"

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

// ------------------------------------------------------------- EGA + RT --


// Continuum extinction of one channel at one LOS point
// (src/forwardmodel.c:120-152 with src/continua.c:5-2049): jsc_continuum
// with the model's emitter indices and the run's switches.
__device__ __forceinline__ double continua(const jsc_dev_model &m,
                                           const jsc_run_cfg &cfg,
                                           const jsc_ctm_coef &c, double nu,
                                           double kwin, double P, double T,
                                           double DS, double qh2o,
                                           const double *u) {
  return jsc_continuum(&c, m.ig_co2, m.ig_h2o, cfg.ctm_co2, cfg.ctm_h2o, cfg.ctm_n2,
                       cfg.ctm_o2, nu, kwin, P, T, DS, qh2o, u);
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

// The exact interval search of ega_node's slow path, kept out of line: the
// fast path is inlined for every (emitter, node) of the unrolled EGA loop,
// the searches are called rarely and would otherwise multiply the code size
// (instruction-fetch stalls).
template <bool U>
__device__ __noinline__ int find_interval(const jsc_node *row, int n, bool strict, double x, int h) {
  return strict ? search_row<U>(row, n, x, h) : bisect_row<U>(row, n, x);
}

// Interval hints of the four (p, T) corner rows, packed 16 bits each in
// the order (ipr, it0), (ipr, it0+1), (ipr+1, it1), (ipr+1, it1+1) of a
// packed bracket code; remap_hints moves them from the corners of code
// `from` to those of code `to`, taking for every new row the old row of the
// same pressure level (else the nearest level) and the nearest temperature.
__device__ __forceinline__ unsigned long long remap_hints(unsigned long long h, int from, int to) {
  const int pi = (from >> 10) & 63, p0 = (from >> 5) & 31, p1 = from & 31;
  const int ni = (to >> 10) & 63, n0 = (to >> 5) & 31, n1 = to & 31;
  unsigned long long out = 0;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const int L = ni + (c >> 1), t = (c >> 1 ? n1 : n0) + (c & 1);
    int src;
    if (L <= pi) src = t <= p0 ? 0 : 1;
    else src = t <= p1 ? 2 : 3;
    out |= ((h >> (16 * src)) & 0xffffull) << (16 * c);
  }
  return out;
}

// Slope of the interval from (x0, y0) to (x1, y1) as LIN evaluates it on
// float table entries: (y1 - y0) / (x1 - x0) in IEEE single precision.
__device__ __forceinline__ float float_slope(float y0, float x0, float y1, float x1) {
  return __fdiv_rn(__fsub_rn(y1, y0), __fsub_rn(x1, x0));
}

// LIN on float table entries with the slope already in float, as the
// reference evaluates it: y0 + slope * (x - x0), promoted to double.
__device__ __forceinline__ double lin_node(float x0, float y0, float slope, double x) {
  return (double)y0 + (double)slope * (x - (double)x0);
}

// Key of a node read as float2 (u, eps).
template <bool U>
__device__ __forceinline__ float key2(float2 v) { return U ? v.x : v.y; }

// Near miss of an interval guess on a strictly increasing row: the guess i
// (nodes *a = i, *b = i+1) failed the bracket test for xf = RD(x), x not
// NaN.  Tries the two intervals on the side where x lies with independent
// loads (one round of latency); on success moves *k, *a, *b there and
// returns true.  The accepted interval passes the same bracket test as the
// exact search's result, so it is that result (the bracket is unique on a
// strictly increasing row).
template <bool U>
__device__ __forceinline__ bool near_interval(const jsc_node *row, int last, float xf, int *k,
                                              float2 *a, float2 *b) {
  const int i = *k;
  if (key2<U>(*a) > xf) {  // below the interval (then i > 0)
    const float2 m1 = __ldg(reinterpret_cast<const float2 *>(row + i - 1));
    const float2 m2 = i >= 2 ? __ldg(reinterpret_cast<const float2 *>(row + i - 2)) : m1;
    if (!(key2<U>(m1) > xf) || i == 1) {
      *b = *a;
      *a = m1;
      *k = i - 1;
      return true;
    }
    if (!(key2<U>(m2) > xf) || i == 2) {  // i >= 2 here
      *b = m1;
      *a = m2;
      *k = i - 2;
      return true;
    }
    return false;
  }
  // at or above the upper key (then i < last)
  const float2 p2 = __ldg(reinterpret_cast<const float2 *>(row + i + 2));
  const float2 p3 = i + 2 <= last ? __ldg(reinterpret_cast<const float2 *>(row + i + 3)) : p2;
  if (key2<U>(p2) > xf || i + 1 == last) {
    *a = *b;
    *b = p2;
    *k = i + 1;
    return true;
  }
  if (key2<U>(p3) > xf || i + 2 == last) {  // i + 2 <= last here
    *a = p2;
    *b = p3;
    *k = i + 2;
    return true;
  }
  return false;
}

// Emissivity of the extended path at one (p, T) node of a table
// (intpol_tbl_u then intpol_tbl_eps, src/forwardmodel.c:460-474): invert
// the path emissivity x1 to a column density on the row, add the segment's
// column, look the emissivity up again, clamp to [0, 1].
//
// Fast path: the row is strictly increasing, the interval [h, h+1] of the
// hint still brackets x1 and the extended column falls in the interval
// k + dj guessed from the previous point's distance -- then one or two
// node pairs (8 bytes a node) answer both lookups.  A guess off by one or
// two intervals is corrected by near_interval (NEAR; kernels that inline
// many ega_node copies leave it out for code size); otherwise the exact
// searches above find the intervals, starting from the guesses.  *kout and
// *jout receive the intervals (they do not depend on the guesses).
template <bool DIG, bool NEAR = true>
__device__ __forceinline__ double ega_node(const jsc_node *__restrict__ nodes, jsc_row rd,
                                           double x1, double useg, int hint, int dj, int *kout,
                                           int *jout, unsigned long long *dig) {
  const int n = rd.nf & 0xffff;
  const bool strict = (rd.nf >> 16) & JSC_ROW_STRICT;
  const jsc_node *row = nodes + rd.off;
  const int last = n - 2;
  int k = hint < 0 ? 0 : (hint > last ? last : hint);
  float2 a = __ldg(reinterpret_cast<const float2 *>(row + k));      // (u, eps)[k]
  float2 b = __ldg(reinterpret_cast<const float2 *>(row + k + 1));  // (u, eps)[k+1]
  const float x1f = __double2float_rd(x1);
  // bracket for x1 on eps: (e[k] <= x1 or k == 0) and (x1 < e[k+1] or k == last)
  if (!(strict && (!(a.y > x1f) || k == 0) && (b.y > x1f || k == last) && x1 == x1) &&
      !(NEAR && strict && x1 == x1 && near_interval<false>(row, last, x1f, &k, &a, &b))) {
    k = find_interval<false>(row, n, strict, x1, k);
    a = __ldg(reinterpret_cast<const float2 *>(row + k));
    b = __ldg(reinterpret_cast<const float2 *>(row + k + 1));
  }
  const double x2 = lin_node(a.y, a.x, float_slope(a.x, a.y, b.x, b.y), x1) + useg;
  const float x2f = __double2float_rd(x2);
  int j = k + (dj > 0 ? dj : 0);
  if (j > last) j = last;
  if (j != k) {
    a = __ldg(reinterpret_cast<const float2 *>(row + j));
    b = __ldg(reinterpret_cast<const float2 *>(row + j + 1));
  }
  if (!(strict && (!(a.x > x2f) || j == 0) && (b.x > x2f || j == last) && x2 == x2) &&
      !(NEAR && strict && x2 == x2 && near_interval<true>(row, last, x2f, &j, &a, &b))) {
    const int j0 = j;
    j = find_interval<true>(row, n, strict, x2, j0);
    if (j != j0) {
      a = __ldg(reinterpret_cast<const float2 *>(row + j));
      b = __ldg(reinterpret_cast<const float2 *>(row + j + 1));
    }
  }
  if (DIG) *dig = (*dig * 1000003ull + (unsigned long long)k) * 1000003ull + (unsigned long long)j;
  *kout = k;
  *jout = j;
  return jsc_clamp01(lin_node(a.x, a.y, float_slope(a.y, a.x, b.y, b.x), x2));
}

