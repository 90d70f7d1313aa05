// Mie scattering of homogeneous spheres on the GPU, for the aerosol/cloud
// optical properties of get_opt_prop (src/scatter.c:330-512).
//
// The series is the Bohren-Huffman one (C. F. Bohren and D. R. Huffman,
// "Absorption and Scattering of Light by Small Particles", 1983, appendix
// A), which the reference evaluates in bhmie (src/scatter.c:56-234):
// logarithmic derivative D_n(mx) by downward recurrence from D_nmx = 0,
// Riccati-Bessel functions psi_n(x), chi_n(x) by upward recurrence, the
// coefficients a_n, b_n, and the amplitudes S1, S2 at (NTHETA+1)/2 angles
// in [0, 90] degrees plus their mirror images in (90, 180], with
// nstop = x + 4 x^0.3333 + 2 terms and nmx = max(nstop, |mx|) + 15.
//
// mie_kernel: one warp per task (a size parameter and a refractive
// index; opt_prop_mie_log has one per Gauss-Hermite radius node and
// channel).  Lane 0 runs the downward recurrence into the task's slot of a
// global scratch array (it is inherently serial); then every lane runs the
// upward recurrence (the coefficients are the same in all lanes) and sums
// the series for its own angles (lane, lane + 32, lane + 64).  Output per
// task: Q_ext, Q_sca and the normalised phase function at NTHETA angles.
#include <math.h>
#include <stdint.h>

#include <vector>

#include "cuda_util.cuh"
#include "jsc_internal.h"

namespace {

struct cplx {
  double re, im;
};

__device__ __forceinline__ cplx cmake(double r, double i) { return cplx{r, i}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return cplx{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return cplx{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx cscale(cplx a, double s) { return cplx{a.re * s, a.im * s}; }
__device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }
// a / b with b scaled by its modulus first (no overflow for large |b|).
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  const double s = 1.0 / cabs_(b);
  const double br = s * b.re, bi = s * b.im;
  return cplx{(a.re * br + a.im * bi) * s, (a.im * br - a.re * bi) * s};
}

constexpr int kHalf = (NTHETA + 1) / 2;   // angles 0..90 degrees
constexpr int kPerLane = (kHalf + 31) / 32;

struct MieArgs {
  int n;
  const double *x, *nr, *ni;  // [n] size parameter, refractive index
  const int64_t *doff;        // [n + 1] slots of the D_n scratch
  cplx *dbuf;
  double *out;                // [n][2 + NTHETA]: Q_ext, Q_sca, phase
  unsigned *status;
};

__global__ void __launch_bounds__(128) mie_kernel(MieArgs A) {
  const int task = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (task >= A.n) return;  // whole warps leave together
  const double x = A.x[task];
  const cplx m = cmake(A.nr[task], A.ni[task]);
  const cplx y = cmul(cmake(x, 0.0), m);
  const double xstop = x + 4.0 * pow(x, 0.3333) + 2.0;
  const int nstop = (int)xstop;
  const double ymod = cabs_(y);
  const int nmx = (int)((xstop > ymod ? xstop : ymod) + 15);
  cplx *D = A.dbuf + A.doff[task];
  if (nmx + 1 > A.doff[task + 1] - A.doff[task] || nstop >= nmx) {
    if (lane == 0) atomicOr(A.status, 1u);  // the host sized the scratch otherwise
    return;
  }
  if (lane == 0) {
    D[nmx] = cmake(0.0, 0.0);
    for (int k = nmx; k >= 2; k--) {
      const cplx q = cdiv(cmake((double)k, 0.0), y);
      D[k - 1] = csub(q, cdiv(cmake(1.0, 0.0), cadd(D[k], q)));
    }
  }
  __syncwarp();  // D_n visible to every lane

  const double dang = 0.5 * M_PI / (double)(kHalf - 1);
  double mu[kPerLane], pprev[kPerLane], pcur[kPerLane];
  cplx s1[kPerLane], s2[kPerLane], s1m[kPerLane], s2m[kPerLane];
#pragma unroll
  for (int a = 0; a < kPerLane; a++) {
    const int j = lane + 32 * a;
    mu[a] = j < kHalf ? cos((double)j * dang) : 0.0;
    pprev[a] = 0.0;
    pcur[a] = 1.0;
    s1[a] = s2[a] = s1m[a] = s2m[a] = cmake(0.0, 0.0);
  }
  double psi0 = cos(x), psi1 = sin(x), chi0 = -sin(x), chi1 = cos(x);
  cplx xi1 = cmake(psi1, -chi1);
  double qsca = 0.0;
  for (int n = 1; n <= nstop; n++) {
    const double rn = (double)n;
    const double fn = (2.0 * rn + 1.0) / (rn * (rn + 1.0));
    const double psi = (2.0 * rn - 1.0) * psi1 / x - psi0;
    const double chi = (2.0 * rn - 1.0) * chi1 / x - chi0;
    const cplx xi = cmake(psi, -chi);
    const cplx dn = D[n];
    const cplx ga = cadd(cdiv(dn, m), cmake(rn / x, 0.0));
    const cplx an = cdiv(csub(cscale(ga, psi), cmake(psi1, 0.0)), csub(cmul(ga, xi), xi1));
    const cplx gb = cadd(cmul(m, dn), cmake(rn / x, 0.0));
    const cplx bn = cdiv(csub(cscale(gb, psi), cmake(psi1, 0.0)), csub(cmul(gb, xi), xi1));
    const double aa = cabs_(an), bb = cabs_(bn);
    qsca += (2.0 * rn + 1.0) * (aa * aa + bb * bb);
    const double sodd = (n & 1) ? 1.0 : -1.0;  // (-1)^(n-1); (-1)^n = -sodd
#pragma unroll
    for (int a = 0; a < kPerLane; a++) {
      const int j = lane + 32 * a;
      if (j < kHalf) {
        const double p = pcur[a];
        const double t = rn * mu[a] * p - (rn + 1.0) * pprev[a];
        s1[a] = cadd(s1[a], cscale(cadd(cscale(an, p), cscale(bn, t)), fn));
        s2[a] = cadd(s2[a], cscale(cadd(cscale(an, t), cscale(bn, p)), fn));
        if (j != kHalf - 1) {  // the mirror angle 180 - theta
          s1m[a] = cadd(s1m[a], cscale(cadd(cscale(an, p * sodd), cscale(bn, t * -sodd)), fn));
          s2m[a] = cadd(s2m[a], cscale(cadd(cscale(an, t * -sodd), cscale(bn, p * sodd)), fn));
        }
        pcur[a] = ((2.0 * rn + 1.0) * mu[a] * p - (rn + 1.0) * pprev[a]) / rn;
        pprev[a] = p;
      }
    }
    psi0 = psi1;
    psi1 = psi;
    chi0 = chi1;
    chi1 = chi;
    xi1 = cmake(psi1, -chi1);
  }
  const double qs = (2.0 / (x * x)) * qsca;
  double *o = A.out + (size_t)task * (2 + NTHETA);
  if (lane == 0) {
    o[0] = (4.0 / (x * x)) * s1[0].re;  // forward amplitude: extinction theorem
    o[1] = qs;
  }
  const double f = 2.0 / (x * x * qs);
#pragma unroll
  for (int a = 0; a < kPerLane; a++) {
    const int j = lane + 32 * a;
    if (j < kHalf) {
      o[2 + j] = f * (s1[a].re * s1[a].re + s1[a].im * s1[a].im + s2[a].re * s2[a].re +
                      s2[a].im * s2[a].im);
      if (j != kHalf - 1)
        o[2 + (NTHETA - 1 - j)] = f * (s1m[a].re * s1m[a].re + s1m[a].im * s1m[a].im +
                                       s2m[a].re * s2m[a].re + s2m[a].im * s2m[a].im);
    }
  }
}

}  // namespace

// Terms of the D_n recurrence of size parameter x and refractive index
// (nr, ni), as mie_kernel counts them, plus slack for a last-bit difference
// of pow between host and device.
static int64_t mie_slots(double x, double nr, double ni) {
  const double xstop = x + 4.0 * pow(x, 0.3333) + 2.0;
  const double ymod = hypot(x * nr, x * ni);
  return (int64_t)((xstop > ymod ? xstop : ymod) + 15) + 3;
}

extern "C" int jsc_mie_eval(int device, int n, const double *x, const double *nr,
                            const double *ni, double *out) {
  if (n <= 0) return JSC_OK;
  {
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
      jsc_set_error(JSC_ERR_CUDA, "Mie: cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
      return JSC_ERR_CUDA;
    }
  }
  std::vector<int64_t> off((size_t)n + 1, 0);
  for (int i = 0; i < n; i++) {
    const int64_t s = mie_slots(x[i], nr[i], ni[i]);
    if (!(x[i] > 0) || s > 10000 + 3) {
      jsc_set_error(JSC_ERR_ARG, "Mie: size parameter %g needs more than 10000 terms", x[i]);
      return JSC_ERR_ARG;
    }
    off[i + 1] = off[i] + s;
  }
  double *dx = nullptr, *dnr = nullptr, *dni = nullptr, *dout = nullptr;
  int64_t *doff = nullptr;
  cplx *dbuf = nullptr;
  unsigned *dst = nullptr;
  int st = JSC_OK;
  auto fail = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && !st) {
      jsc_set_error(JSC_ERR_CUDA, "Mie: %s: %s", what, cudaGetErrorString(e));
      st = JSC_ERR_CUDA;
    }
  };
  fail(cudaMalloc(&dx, 3 * (size_t)n * sizeof(double)), "cudaMalloc");
  fail(cudaMalloc(&dout, (size_t)n * (2 + NTHETA) * sizeof(double)), "cudaMalloc");
  fail(cudaMalloc(&doff, ((size_t)n + 1) * sizeof(int64_t)), "cudaMalloc");
  fail(cudaMalloc(&dbuf, (size_t)off[n] * sizeof(cplx)), "cudaMalloc");
  fail(cudaMalloc(&dst, sizeof(unsigned)), "cudaMalloc");
  if (!st) {
    dnr = dx + n;
    dni = dx + 2 * (size_t)n;
    fail(cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice), "copy");
    fail(cudaMemcpy(dnr, nr, n * sizeof(double), cudaMemcpyHostToDevice), "copy");
    fail(cudaMemcpy(dni, ni, n * sizeof(double), cudaMemcpyHostToDevice), "copy");
    fail(cudaMemcpy(doff, off.data(), ((size_t)n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice),
         "copy");
    fail(cudaMemset(dst, 0, sizeof(unsigned)), "memset");
  }
  if (!st) {
    MieArgs a;
    a.n = n;
    a.x = dx;
    a.nr = dnr;
    a.ni = dni;
    a.doff = doff;
    a.dbuf = dbuf;
    a.out = dout;
    a.status = dst;
    mie_kernel<<<(unsigned)(((int64_t)n * 32 + 127) / 128), 128>>>(a);
    jsc_count_launch();
    fail(cudaGetLastError(), "mie_kernel launch");
    unsigned hs = 0;
    fail(cudaMemcpy(&hs, dst, sizeof(unsigned), cudaMemcpyDeviceToHost), "mie_kernel");
    if (!st && hs) {
      jsc_set_error(JSC_ERR_ARG, "Mie: recurrence scratch too small");
      st = JSC_ERR_ARG;
    }
    fail(cudaMemcpy(out, dout, (size_t)n * (2 + NTHETA) * sizeof(double), cudaMemcpyDeviceToHost),
         "copy back");
  }
  cudaFree(dx);
  cudaFree(dout);
  cudaFree(doff);
  cudaFree(dbuf);
  cudaFree(dst);
  return st;
}
