// Scattering-source surrogate: a small MLP that maps features of a
// scattering point to the log of its scattering source per channel, in
// place of the secondary pencils, source integral and solar search of
// srcfunc_sca (src/scatter.c:643-1041).
//
// Network: x[SUR_NF] -> tanh(W0 x + b0) -> tanh(W1 . + b1) -> tanh(W2 . + b2)
// -> W3 . + b3 = y[nout], width SUR_W; W_l stored [out][in].
//
// Training (FP32, this file): tiled SGEMM forward/backward, tanh, MSE loss
// on standardised targets, Adam.  Inference: BF16 weights on the tensor
// cores (mma.sync m16n8k16, FP32 accumulation), tanh in FP32.
//
// Features of a scattering point (sur_features_kernel): altitude, cosine
// of the LOS chord's zenith angle, temperature, log pressure, cosine of the
// solar zenith angle, cosine of the angle between the (unrefracted) solar
// direction and the chord, layer index, and the sun's elevation above the
// point's geometric horizon [deg] (where the solar term switches off).  They are standardised with the
// training set's mean and spread; a point whose raw features leave the
// training set's range (widened by 2 % of it) is outside the envelope and
// takes the plain path.
#include <cuda_bf16.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "scatter.cuh"
#include "surrogate.h"
#include "surrogate_tc.h"

// ------------------------------------------------------------ features --

static __global__ void sur_features_kernel(int n, const double *sp, float *feat) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double *o = sp + (size_t)k * JSC_SP_REC;
  const double x[3] = {o[SP_X], o[SP_X + 1], o[SP_X + 2]};
  const double dx[3] = {o[SP_DX], o[SP_DX + 1], o[SP_DX + 2]};
  const double rx = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  const double rd = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
  const double mu = rd > 0 ? (x[0] * dx[0] + x[1] * dx[1] + x[2] * dx[2]) / (rx * rd) : 0.0;
  double lx[3], ly[3], lz[3], z, lon, lat, azi, sza;
  local_frame(x, lx, ly, lz);
  jsc_cart2geo(x, &z, &lon, &lat);
  jsc_suncoord(o[SP_TIME], lon, lat, &azi, &sza);
  const double sz = sin(sza * M_PI / 180), cz = cos(sza * M_PI / 180);
  const double sa = sin(azi * M_PI / 180), ca = cos(azi * M_PI / 180);
  double cth = 0;
  for (int i = 0; i < 3; i++) cth += (sz * sa * lx[i] + sz * ca * ly[i] + cz * lz[i]) * dx[i];
  cth = rd > 0 ? cth / rd : 0.0;
  float *f = feat + (size_t)k * SUR_NF;
  f[0] = (float)z;
  f[1] = (float)mu;
  f[2] = (float)o[SP_T];
  f[3] = (float)log(o[SP_P]);
  f[4] = (float)cz;
  f[5] = (float)cth;
  f[6] = (float)o[SP_IL];
  // elevation above the geometric horizon: 90 - sza + dip, dip = acos(RE / (RE + z))
  const double zz = z > 0 ? z : 0.0;
  f[7] = (float)(90.0 - sza + acos(JSC_RE / (JSC_RE + zz)) * 180 / M_PI);
}

// ------------------------------------------------------- FP32 training --

#define TG_M 64
#define TG_N 64
#define TG_K 16

// C[M][N] (ldc) = op(A) op(B) (+ bias[n]) with op(A)(m,k) = TA ? A[k*lda+m]
// : A[m*lda+k] and op(B)(k,n) = TB ? B[n*ldb+k] : B[k*ldb+n].  256 threads,
// a 64 x 64 tile per block, 4 x 4 outputs per thread.  With gridDim.z > 1
// the K range is split over blockIdx.z and block z writes its partial
// product to the slice C + z M ldc (no bias); ksum_kernel adds the slices
// in order, so training is deterministic.
template <bool TA, bool TB>
static __global__ void __launch_bounds__(256)
sgemm_kernel(int M, int N, int K, const float *A, int lda, const float *B, int ldb, float *C,
             int ldc, const float *bias) {
  __shared__ float As[TG_K][TG_M + 4];
  __shared__ float Bs[TG_K][TG_N + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * TG_M, n0 = blockIdx.x * TG_N;
  const int kchunk = (K + (int)gridDim.z - 1) / (int)gridDim.z;
  const int kb = (int)blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  float acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += TG_K) {
    for (int i = threadIdx.x; i < TG_K * TG_M; i += 256) {
      const int kk = i / TG_M, mm = i - kk * TG_M;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < ke) ? (TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k]) : 0.f;
    }
    for (int i = threadIdx.x; i < TG_K * TG_N; i += 256) {
      const int kk = i / TG_N, nn = i - kk * TG_N;
      const int n = n0 + nn, k = k0 + kk;
      Bs[kk][nn] = (n < N && k < ke) ? (TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TG_K; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        a[i] = As[kk][ty * 4 + i];
        b[i] = Bs[kk][tx * 4 + i];
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
      if (m < M && n < N) {
        if (gridDim.z > 1) C[((size_t)blockIdx.z * M + m) * ldc + n] = acc[i][j];
        else C[(size_t)m * ldc + n] = acc[i][j] + (bias ? bias[n] : 0.f);
      }
    }
}

// C[i] = sum over z = 0 .. nz-1, in that order, of ws[z mn + i].
static __global__ void ksum_kernel(int64_t mn, int nz, const float *ws, float *c) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mn) return;
  float t = 0;
  for (int z = 0; z < nz; z++) t += ws[(size_t)z * mn + i];
  c[i] = t;
}

// Most K slices of a split product (sizes the workspace).
#define SUR_KSPLIT_MAX 64

// ksplit > 1: split-K for products with a long K and a small output (the
// weight gradients: K = batch), partial products in ws (ksplit M ldc
// floats, ksplit <= SUR_KSPLIT_MAX), bias ignored.
template <bool TA, bool TB>
static void sgemm(int M, int N, int K, const float *A, int lda, const float *B, int ldb, float *C,
                  int ldc, const float *bias, cudaStream_t s, int ksplit = 1,
                  float *ws = nullptr) {
  if (ksplit > 1 && ws) {
    dim3 grid((N + TG_N - 1) / TG_N, (M + TG_M - 1) / TG_M, ksplit);
    sgemm_kernel<TA, TB><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, ws, ldc, nullptr);
    const int64_t mn = (int64_t)M * ldc;
    ksum_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, s>>>(mn, ksplit, ws, C);
    return;
  }
  dim3 grid((N + TG_N - 1) / TG_N, (M + TG_M - 1) / TG_M, 1);
  sgemm_kernel<TA, TB><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias);
}

static __global__ void tanh_kernel(int64_t n, float *h) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) h[i] = tanhf(h[i]);
}

// dZ = dH * (1 - H^2) in place
static __global__ void tanh_bwd_kernel(int64_t n, const float *h, float *dh) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dh[i] *= 1.f - h[i] * h[i];
}

// dY = 2 (Y - T) / n, and the per-block partial sums of (Y - T)^2.
static __global__ void mse_kernel(int64_t cnt, int n, const float *y, const float *t, float *dy,
                                  float *part) {
  __shared__ float red[256];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float e2 = 0;
  if (i < cnt) {
    const float e = y[i] - t[i];
    dy[i] = 2.f * e / (float)n;
    e2 = e * e;
  }
  red[threadIdx.x] = e2;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// db[o] = sum over the batch of dZ[:, o]: block (32 columns) x (8 row
// lanes), coalesced over the columns.
static __global__ void colsum_kernel(int n, int cols, const float *dz, float *db) {
  const int o = blockIdx.x * 32 + (threadIdx.x & 31), r0 = threadIdx.x >> 5;
  float sacc = 0;
  if (o < cols)
    for (int i = r0; i < n; i += 8) sacc += dz[(size_t)i * cols + o];
  __shared__ float red[8][32];
  red[r0][threadIdx.x & 31] = sacc;
  __syncthreads();
  if (r0 == 0 && o < cols) {
    float t = 0;
    for (int j = 0; j < 8; j++) t += red[j][threadIdx.x];
    db[o] = t;
  }
}

static __global__ void adam_kernel(int64_t n, float *p, const float *g, float *m, float *v,
                                   float lr, float b1, float b2, float c1, float c2, float eps) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1 - b1) * gi;
  const float vi = b2 * v[i] + (1 - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Gather a minibatch: rows idx[i] of X (standardised here) and T.
static __global__ void gather_kernel(int n, int nout, const int *idx, const float *X,
                                     const float *T, const float *xm, const float *xs, float *xb,
                                     float *tb) {
  const int i = blockIdx.x;
  if (i >= n) return;
  const int64_t r = idx[i];
  for (int c = threadIdx.x; c < SUR_NF; c += blockDim.x)
    xb[(size_t)i * SUR_NF + c] = (X[r * SUR_NF + c] - xm[c]) / xs[c];
  for (int c = threadIdx.x; c < nout; c += blockDim.x) tb[(size_t)i * nout + c] = T[r * nout + c];
}

// ------------------------------------------------------ BF16 inference --

#define SUR_KP 136  // padded row (bf16) of a 128-wide layer
#define SUR_K0 16   // first-layer K: SUR_NF padded to one k-step
#define SUR_K0P 24  // padded row of the first layer
#define SUR_INF_WARPS 4

// Shared-memory image of the network (bf16 weights, rows padded against
// bank conflicts) followed by the biases; the same layout in global memory
// is copied in with 16-byte loads.
struct SurImage {
  size_t w0, w1, w2, w3, bias, bytes;  // byte offsets
};

static __host__ __device__ SurImage sur_image(int noutp) {
  SurImage im;
  im.w0 = 0;
  im.w1 = im.w0 + (size_t)SUR_W * SUR_K0P * 2;
  im.w2 = im.w1 + (size_t)SUR_W * SUR_KP * 2;
  im.w3 = im.w2 + (size_t)SUR_W * SUR_KP * 2;
  im.bias = im.w3 + (size_t)noutp * SUR_KP * 2;
  im.bytes = im.bias + (size_t)(3 * SUR_W + noutp) * 4;
  im.bytes = (im.bytes + 15) & ~(size_t)15;
  return im;
}

__device__ __forceinline__ void mma_bf16(float *c, uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// One layer for the 16 rows of a warp: acc[nt][4] = act[16][K] W^T over NT
// n-tiles of 8 outputs.
template <int NT, int KSTEPS, int KP>
__device__ __forceinline__ void warp_layer(const __nv_bfloat16 *act, const __nv_bfloat16 *w,
                                           float (*acc)[4], int g, int t) {
#pragma unroll
  for (int nt = 0; nt < NT; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
  for (int ks = 0; ks < KSTEPS; ks++) {
    const int k0 = ks * 16;
    const uint32_t a0 = *reinterpret_cast<const uint32_t *>(act + g * KP + k0 + 2 * t);
    const uint32_t a1 = *reinterpret_cast<const uint32_t *>(act + (g + 8) * KP + k0 + 2 * t);
    const uint32_t a2 = *reinterpret_cast<const uint32_t *>(act + g * KP + k0 + 2 * t + 8);
    const uint32_t a3 = *reinterpret_cast<const uint32_t *>(act + (g + 8) * KP + k0 + 2 * t + 8);
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      const __nv_bfloat16 *wr = w + (nt * 8 + g) * KP + k0 + 2 * t;
      const uint32_t b0 = *reinterpret_cast<const uint32_t *>(wr);
      const uint32_t b1 = *reinterpret_cast<const uint32_t *>(wr + 8);
      mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
    }
  }
}

// bias + tanh, written back as the next layer's bf16 input rows
template <int NT>
__device__ __forceinline__ void warp_act(float (*acc)[4], const float *bias, __nv_bfloat16 *act,
                                         int g, int t) {
#pragma unroll
  for (int nt = 0; nt < NT; nt++) {
    const int c = nt * 8 + 2 * t;
    const float v0 = tanhf(acc[nt][0] + bias[c]), v1 = tanhf(acc[nt][1] + bias[c + 1]);
    const float v2 = tanhf(acc[nt][2] + bias[c]), v3 = tanhf(acc[nt][3] + bias[c + 1]);
    *reinterpret_cast<__nv_bfloat162 *>(act + g * SUR_KP + c) = __floats2bfloat162_rn(v0, v1);
    *reinterpret_cast<__nv_bfloat162 *>(act + (g + 8) * SUR_KP + c) = __floats2bfloat162_rn(v2, v3);
  }
}

struct SurInferArgs {
  int n, nout, noutp;
  const float *feat;                 // [n][SUR_NF] raw features
  const unsigned char *image;        // global copy of the shared-memory image
  float xm[SUR_NF], xs[SUR_NF];      // feature standardisation
  const float *ym, *ys;              // [nout] target standardisation (log source)
  double *src;                       // [n][nd] output
  int nd;
};

// Persistent blocks of 4 warps; each warp runs 16 points through the four
// layers with its activations in a private shared-memory tile.
template <int NTOUT>
static __global__ void __launch_bounds__(SUR_INF_WARPS * 32)
sur_infer_kernel(SurInferArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SurImage im = sur_image(NTOUT * 8);
  for (size_t i = threadIdx.x * 16; i < im.bytes; i += blockDim.x * 16)
    *reinterpret_cast<uint4 *>(smem + i) = *reinterpret_cast<const uint4 *>(A.image + i);
  __syncthreads();
  const __nv_bfloat16 *w0 = reinterpret_cast<const __nv_bfloat16 *>(smem + im.w0);
  const __nv_bfloat16 *w1 = reinterpret_cast<const __nv_bfloat16 *>(smem + im.w1);
  const __nv_bfloat16 *w2 = reinterpret_cast<const __nv_bfloat16 *>(smem + im.w2);
  const __nv_bfloat16 *w3 = reinterpret_cast<const __nv_bfloat16 *>(smem + im.w3);
  const float *bias = reinterpret_cast<const float *>(smem + im.bias);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  __nv_bfloat16 *act = reinterpret_cast<__nv_bfloat16 *>(smem + im.bytes) + warp * 16 * SUR_KP;
  float acc[16][4];
  const int ntiles = (A.n + 15) / 16;
  for (int tile = blockIdx.x * SUR_INF_WARPS + warp; tile < ntiles;
       tile += gridDim.x * SUR_INF_WARPS) {
    const int p0 = tile * 16;
    // standardised features as bf16 rows of SUR_K0P (zero past SUR_NF)
    for (int i = lane; i < 16 * SUR_K0; i += 32) {
      const int rr = i / SUR_K0, c = i - rr * SUR_K0;
      float v = 0.f;
      if (c < SUR_NF && p0 + rr < A.n) v = (A.feat[(size_t)(p0 + rr) * SUR_NF + c] - A.xm[c]) / A.xs[c];
      act[rr * SUR_K0P + c] = __float2bfloat16_rn(v);
    }
    __syncwarp();
    warp_layer<16, 1, SUR_K0P>(act, w0, acc, g, t);
    __syncwarp();
    warp_act<16>(acc, bias, act, g, t);
    __syncwarp();
    warp_layer<16, 8, SUR_KP>(act, w1, acc, g, t);
    __syncwarp();
    warp_act<16>(acc, bias + SUR_W, act, g, t);
    __syncwarp();
    warp_layer<16, 8, SUR_KP>(act, w2, acc, g, t);
    __syncwarp();
    warp_act<16>(acc, bias + 2 * SUR_W, act, g, t);
    __syncwarp();
    warp_layer<NTOUT, 8, SUR_KP>(act, w3, acc, g, t);
    const float *b3 = bias + 3 * SUR_W;
#pragma unroll
    for (int nt = 0; nt < NTOUT; nt++) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int rr = g + (q >= 2 ? 8 : 0), c = nt * 8 + 2 * t + (q & 1);
        const int p = p0 + rr;
        if (p < A.n && c < A.nout) {
          const float y = acc[nt][q] + b3[c];
          A.src[(size_t)p * A.nd + c] = exp((double)(y * A.ys[c] + A.ym[c]));
        }
      }
    }
    __syncwarp();
  }
}

// FP32 master weights -> the padded bf16 image (+ FP32 biases).
static __global__ void sur_pack_kernel(int nout, int noutp, const float *w0, const float *w1,
                                       const float *w2, const float *w3, const float *b0,
                                       const float *b1, const float *b2, const float *b3,
                                       unsigned char *image) {
  const SurImage im = sur_image(noutp);
  __nv_bfloat16 *q0 = reinterpret_cast<__nv_bfloat16 *>(image + im.w0);
  __nv_bfloat16 *q1 = reinterpret_cast<__nv_bfloat16 *>(image + im.w1);
  __nv_bfloat16 *q2 = reinterpret_cast<__nv_bfloat16 *>(image + im.w2);
  __nv_bfloat16 *q3 = reinterpret_cast<__nv_bfloat16 *>(image + im.w3);
  float *bb = reinterpret_cast<float *>(image + im.bias);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (int i = tid; i < SUR_W * SUR_K0P; i += nt) {
    const int o = i / SUR_K0P, k = i - o * SUR_K0P;
    q0[i] = __float2bfloat16_rn(k < SUR_NF ? w0[o * SUR_NF + k] : 0.f);
  }
  for (int i = tid; i < SUR_W * SUR_KP; i += nt) {
    const int o = i / SUR_KP, k = i - o * SUR_KP;
    q1[i] = __float2bfloat16_rn(k < SUR_W ? w1[o * SUR_W + k] : 0.f);
    q2[i] = __float2bfloat16_rn(k < SUR_W ? w2[o * SUR_W + k] : 0.f);
  }
  for (int i = tid; i < noutp * SUR_KP; i += nt) {
    const int o = i / SUR_KP, k = i - o * SUR_KP;
    q3[i] = __float2bfloat16_rn((o < nout && k < SUR_W) ? w3[o * SUR_W + k] : 0.f);
  }
  for (int i = tid; i < 3 * SUR_W + noutp; i += nt) {
    float v;
    if (i < SUR_W) v = b0[i];
    else if (i < 2 * SUR_W) v = b1[i - SUR_W];
    else if (i < 3 * SUR_W) v = b2[i - 2 * SUR_W];
    else v = (i - 3 * SUR_W < nout) ? b3[i - 3 * SUR_W] : 0.f;
    bb[i] = v;
  }
}

// ------------------------------------------------------------ the object --

struct jsc_surrogate {
  int device, nout, noutp;
  int in[4], out[4];
  float *d_p[4][2];         // W, b per layer (FP32 master)
  float *d_g[4][2];         // gradients
  float *d_m[4][2], *d_v[4][2];  // Adam moments
  int64_t adam_t;
  unsigned char *d_image;   // bf16 inference image (mma.sync path)
  int tc;                   // 1: tcgen05 inference path
  unsigned char *d_tc_image;
  int tc_packed;
  unsigned *d_tc_status;    // the tcgen05 kernel's wait status
  float xm[SUR_NF], xs[SUR_NF];
  float lo[SUR_NF], hi[SUR_NF];  // envelope of raw features
  float *d_ym, *d_ys;       // [nout] target standardisation
  float h_ym[NDMAX], h_ys[NDMAX];
  int trained, packed;
  // training scratch
  int max_batch;
  float *d_h[5];            // activations per layer, [max_batch][width]
  float *d_dh[2];           // two ping-pong gradient buffers [max_batch][SUR_W]
  float *d_xb, *d_tb, *d_part;
  float *d_ksum;            // split-K partial products of the weight gradients
  int *d_idx;               // [max_batch] (gradient checks)
  int *d_perm;              // [n_train] per-epoch permutation
  float *d_X, *d_T;         // device copy of the training set
  int64_t n_train;
};

extern "C" int jsc_surrogate_param_count(const jsc_surrogate *s) {
  if (!s) return -1;
  int n = 0;
  for (int l = 0; l < 4; l++) n += s->out[l] * s->in[l] + s->out[l];
  return n;
}

static void free_train(jsc_surrogate *s) {
  for (int i = 0; i < 5; i++) cudaFree(s->d_h[i]), s->d_h[i] = nullptr;
  for (int i = 0; i < 2; i++) cudaFree(s->d_dh[i]), s->d_dh[i] = nullptr;
  // d_xb is the first activation buffer d_h[0], freed above
  cudaFree(s->d_tb);
  cudaFree(s->d_part);
  cudaFree(s->d_ksum);
  cudaFree(s->d_idx);
  s->d_xb = s->d_tb = s->d_part = s->d_ksum = nullptr;
  s->d_idx = nullptr;
  s->max_batch = 0;
}

extern "C" void jsc_surrogate_destroy(jsc_surrogate *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  for (int l = 0; l < 4; l++)
    for (int j = 0; j < 2; j++) {
      cudaFree(s->d_p[l][j]);
      cudaFree(s->d_g[l][j]);
      cudaFree(s->d_m[l][j]);
      cudaFree(s->d_v[l][j]);
    }
  cudaFree(s->d_image);
  cudaFree(s->d_tc_image);
  cudaFree(s->d_tc_status);
  cudaFree(s->d_ym);
  cudaFree(s->d_ys);
  cudaFree(s->d_X);
  cudaFree(s->d_T);
  cudaFree(s->d_perm);
  free_train(s);
  free(s);
}

// splitmix64: seeded initial weights
static uint64_t mix64(uint64_t *st) {
  uint64_t z = (*st += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

extern "C" int jsc_surrogate_create(int nd, int device, uint64_t seed, jsc_surrogate **out) {
  if (!out || nd < 1 || nd > SUR_NOUT_MAX) {
    jsc_set_error(JSC_ERR_ARG, "jsc_surrogate_create: nd=%d outside 1..%d", nd, SUR_NOUT_MAX);
    return JSC_ERR_ARG;
  }
  *out = nullptr;
  JSC_CUDA_TRY(cudaSetDevice(device));
  jsc_surrogate *s = (jsc_surrogate *)calloc(1, sizeof(jsc_surrogate));
  if (!s) return JSC_ERR_NOMEM;
  s->device = device;
  s->nout = nd;
  s->noutp = (nd + 7) / 8 * 8;
  s->tc = 1;  // tcgen05 inference by default
  const int in[4] = {SUR_NF, SUR_W, SUR_W, SUR_W}, outw[4] = {SUR_W, SUR_W, SUR_W, nd};
  int st = JSC_OK;
  uint64_t rs = seed;
  for (int l = 0; l < 4 && !st; l++) {
    s->in[l] = in[l];
    s->out[l] = outw[l];
    const size_t nw = (size_t)in[l] * outw[l], nb = outw[l];
    const size_t sz[2] = {nw, nb};
    for (int j = 0; j < 2 && !st; j++) {
      st = st ? st : jsc_dmalloc(&s->d_p[l][j], sz[j]);
      st = st ? st : jsc_dmalloc(&s->d_g[l][j], sz[j]);
      st = st ? st : jsc_dmalloc(&s->d_m[l][j], sz[j]);
      st = st ? st : jsc_dmalloc(&s->d_v[l][j], sz[j]);
      if (!st) {
        cudaMemset(s->d_m[l][j], 0, sz[j] * sizeof(float));
        cudaMemset(s->d_v[l][j], 0, sz[j] * sizeof(float));
      }
    }
    if (!st) {
      // uniform(-a, a) with a = sqrt(6 / (in + out)) (Glorot), zero biases
      float *h = (float *)malloc(nw * sizeof(float));
      if (!h) {
        st = JSC_ERR_NOMEM;
        break;
      }
      const double a = sqrt(6.0 / (in[l] + outw[l]));
      for (size_t i = 0; i < nw; i++) h[i] = (float)(a * (2.0 * ((mix64(&rs) >> 11) * 0x1.0p-53) - 1.0));
      if (cudaMemcpy(s->d_p[l][0], h, nw * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        st = JSC_ERR_CUDA;
      free(h);
      if (!st) cudaMemset(s->d_p[l][1], 0, nb * sizeof(float));
    }
  }
  st = st ? st : jsc_dmalloc(&s->d_image, sur_image(s->noutp).bytes);
  st = st ? st : jsc_dmalloc(&s->d_ym, (size_t)nd);
  st = st ? st : jsc_dmalloc(&s->d_ys, (size_t)nd);
  for (int c = 0; c < SUR_NF; c++) {
    s->xm[c] = 0.f;
    s->xs[c] = 1.f;
    s->lo[c] = -INFINITY;
    s->hi[c] = INFINITY;
  }
  for (int c = 0; c < nd; c++) {
    s->h_ym[c] = 0.f;
    s->h_ys[c] = 1.f;
  }
  if (!st && (cudaMemcpy(s->d_ym, s->h_ym, nd * sizeof(float), cudaMemcpyHostToDevice) ||
              cudaMemcpy(s->d_ys, s->h_ys, nd * sizeof(float), cudaMemcpyHostToDevice)))
    st = JSC_ERR_CUDA;
  if (st) {
    jsc_surrogate_destroy(s);
    return st;
  }
  *out = s;
  return JSC_OK;
}

extern "C" int jsc_surrogate_get_scaling(const jsc_surrogate *s, float *xm, float *xs, float *ym,
                                         float *ys) {
  if (!s) return JSC_ERR_ARG;
  for (int c = 0; c < SUR_NF; c++) {
    if (xm) xm[c] = s->xm[c];
    if (xs) xs[c] = s->xs[c];
  }
  for (int d = 0; d < s->nout; d++) {
    if (ym) ym[d] = s->h_ym[d];
    if (ys) ys[d] = s->h_ys[d];
  }
  return JSC_OK;
}

extern "C" int jsc_surrogate_get_params(const jsc_surrogate *s, float *out) {
  if (!s || !out) return JSC_ERR_ARG;
  JSC_CUDA_TRY(cudaSetDevice(s->device));
  size_t o = 0;
  for (int l = 0; l < 4; l++) {
    const size_t nw = (size_t)s->in[l] * s->out[l], nb = s->out[l];
    JSC_CUDA_TRY(cudaMemcpy(out + o, s->d_p[l][0], nw * sizeof(float), cudaMemcpyDeviceToHost));
    o += nw;
    JSC_CUDA_TRY(cudaMemcpy(out + o, s->d_p[l][1], nb * sizeof(float), cudaMemcpyDeviceToHost));
    o += nb;
  }
  return JSC_OK;
}

extern "C" int jsc_surrogate_set_params(jsc_surrogate *s, const float *in) {
  if (!s || !in) return JSC_ERR_ARG;
  JSC_CUDA_TRY(cudaSetDevice(s->device));
  size_t o = 0;
  for (int l = 0; l < 4; l++) {
    const size_t nw = (size_t)s->in[l] * s->out[l], nb = s->out[l];
    JSC_CUDA_TRY(cudaMemcpy(s->d_p[l][0], in + o, nw * sizeof(float), cudaMemcpyHostToDevice));
    o += nw;
    JSC_CUDA_TRY(cudaMemcpy(s->d_p[l][1], in + o, nb * sizeof(float), cudaMemcpyHostToDevice));
    o += nb;
  }
  s->packed = 0;
  s->tc_packed = 0;
  return JSC_OK;
}

static int ensure_train(jsc_surrogate *s, int batch) {
  if (s->max_batch >= batch) return JSC_OK;
  free_train(s);
  int st = JSC_OK;
  const int width[5] = {SUR_NF, SUR_W, SUR_W, SUR_W, s->nout};
  for (int i = 0; i < 5 && !st; i++) st = jsc_dmalloc(&s->d_h[i], (size_t)batch * width[i]);
  for (int i = 0; i < 2 && !st; i++) st = jsc_dmalloc(&s->d_dh[i], (size_t)batch * SUR_W);
  st = st ? st : jsc_dmalloc(&s->d_tb, (size_t)batch * s->nout);
  st = st ? st : jsc_dmalloc(&s->d_part, (size_t)(batch * SUR_NOUT_MAX + 255) / 256 + 1);
  st = st ? st : jsc_dmalloc(&s->d_idx, (size_t)batch);
  st = st ? st : jsc_dmalloc(&s->d_ksum, (size_t)SUR_KSPLIT_MAX * SUR_W *
                                             (SUR_NOUT_MAX > SUR_W ? SUR_NOUT_MAX : SUR_W));
  if (st) {
    free_train(s);
    return st;
  }
  s->d_xb = s->d_h[0];
  s->max_batch = batch;
  return JSC_OK;
}

// Forward and backward over one standardised minibatch already in d_h[0] /
// d_tb; gradients into d_g, returns the loss (mean over the batch of the
// squared error summed over outputs).
static int forward_backward(jsc_surrogate *s, int n, cudaStream_t st, float *loss) {
  for (int l = 0; l < 4; l++) {
    sgemm<false, true>(n, s->out[l], s->in[l], s->d_h[l], s->in[l], s->d_p[l][0], s->in[l],
                       s->d_h[l + 1], s->out[l], s->d_p[l][1], st);
    if (l < 3) {
      const int64_t cnt = (int64_t)n * s->out[l];
      tanh_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(cnt, s->d_h[l + 1]);
    }
  }
  const int64_t cnt = (int64_t)n * s->nout;
  const int nblk = (int)((cnt + 255) / 256);
  float *dy = s->d_dh[0];
  mse_kernel<<<nblk, 256, 0, st>>>(cnt, n, s->d_h[4], s->d_tb, dy, s->d_part);
  float *dcur = dy, *dnext = s->d_dh[1];
  for (int l = 3; l >= 0; l--) {
    // dW = dZ^T H_l, db = colsum(dZ)
    const int tiles = ((s->out[l] + TG_M - 1) / TG_M) * ((s->in[l] + TG_N - 1) / TG_N);
    int ksplit = 296 / tiles;  // about two blocks per SM
    if (ksplit > n / 64) ksplit = n / 64 > 0 ? n / 64 : 1;
    if (ksplit > SUR_KSPLIT_MAX) ksplit = SUR_KSPLIT_MAX;
    sgemm<true, false>(s->out[l], s->in[l], n, dcur, s->out[l], s->d_h[l], s->in[l],
                       s->d_g[l][0], s->in[l], nullptr, st, ksplit > 1 ? ksplit : 1, s->d_ksum);
    colsum_kernel<<<(s->out[l] + 31) / 32, 256, 0, st>>>(n, s->out[l], dcur, s->d_g[l][1]);
    if (l > 0) {
      // dH_l = dZ W_l, then dZ_{l-1} = dH_l (1 - H_l^2)
      sgemm<false, false>(n, s->in[l], s->out[l], dcur, s->out[l], s->d_p[l][0], s->in[l], dnext,
                          s->in[l], nullptr, st);
      const int64_t c2 = (int64_t)n * s->in[l];
      tanh_bwd_kernel<<<(unsigned)((c2 + 255) / 256), 256, 0, st>>>(c2, s->d_h[l], dnext);
      float *tmp = dcur;
      dcur = dnext;
      dnext = tmp;
    }
  }
  JSC_LAUNCH_CHECK();
  if (loss) {
    float *h = (float *)malloc(nblk * sizeof(float));
    if (!h) return JSC_ERR_NOMEM;
    JSC_CUDA_TRY(cudaMemcpyAsync(h, s->d_part, nblk * sizeof(float), cudaMemcpyDeviceToHost, st));
    JSC_CUDA_TRY(cudaStreamSynchronize(st));
    double acc = 0;
    for (int i = 0; i < nblk; i++) acc += h[i];
    free(h);
    *loss = (float)(acc / n);
  }
  return JSC_OK;
}

extern "C" int jsc_surrogate_loss_grad(jsc_surrogate *s, const float *x, const float *t, int n,
                                       float *loss, float *grads) {
  if (!s || !x || !t || n < 1) return JSC_ERR_ARG;
  JSC_CUDA_TRY(cudaSetDevice(s->device));
  int st = ensure_train(s, n);
  if (st) return st;
  JSC_CUDA_TRY(cudaMemcpy(s->d_h[0], x, (size_t)n * SUR_NF * sizeof(float), cudaMemcpyHostToDevice));
  JSC_CUDA_TRY(cudaMemcpy(s->d_tb, t, (size_t)n * s->nout * sizeof(float), cudaMemcpyHostToDevice));
  if ((st = forward_backward(s, n, 0, loss))) return st;
  JSC_CUDA_TRY(cudaDeviceSynchronize());
  if (grads) {
    size_t o = 0;
    for (int l = 0; l < 4; l++) {
      const size_t nw = (size_t)s->in[l] * s->out[l], nb = s->out[l];
      JSC_CUDA_TRY(cudaMemcpy(grads + o, s->d_g[l][0], nw * sizeof(float), cudaMemcpyDeviceToHost));
      o += nw;
      JSC_CUDA_TRY(cudaMemcpy(grads + o, s->d_g[l][1], nb * sizeof(float), cudaMemcpyDeviceToHost));
      o += nb;
    }
  }
  return JSC_OK;
}

extern "C" int jsc_surrogate_train(jsc_surrogate *s, const float *X, const double *src,
                                   int64_t n, int epochs, int batch, float lr, uint64_t seed,
                                   float *loss_per_epoch) {
  if (!s || !X || !src || n < 16 || epochs < 1 || batch < 16 || batch > (1 << 16)) {
    jsc_set_error(JSC_ERR_ARG, "jsc_surrogate_train: invalid arguments");
    return JSC_ERR_ARG;
  }
  JSC_CUDA_TRY(cudaSetDevice(s->device));
  const int nd = s->nout;
  // Standardisation and envelope from the training set.
  double sum[SUR_NF] = {0}, sum2[SUR_NF] = {0};
  float lo[SUR_NF], hi[SUR_NF];
  for (int c = 0; c < SUR_NF; c++) {
    lo[c] = INFINITY;
    hi[c] = -INFINITY;
  }
  for (int64_t i = 0; i < n; i++)
    for (int c = 0; c < SUR_NF; c++) {
      const float v = X[i * SUR_NF + c];
      sum[c] += v;
      sum2[c] += (double)v * v;
      if (v < lo[c]) lo[c] = v;
      if (v > hi[c]) hi[c] = v;
    }
  for (int c = 0; c < SUR_NF; c++) {
    const double m = sum[c] / n, var = sum2[c] / n - m * m;
    s->xm[c] = (float)m;
    s->xs[c] = var > 1e-12 ? (float)sqrt(var) : 1.f;
    const float w = 0.02f * (hi[c] - lo[c]);
    s->lo[c] = lo[c] - w;
    s->hi[c] = hi[c] + w;
  }
  float *T = (float *)malloc((size_t)n * nd * sizeof(float));
  if (!T) return JSC_ERR_NOMEM;
  for (int d = 0; d < nd; d++) {
    double m = 0, m2 = 0;
    for (int64_t i = 0; i < n; i++) {
      const double y = log(fmax(src[i * nd + d], 1e-300));
      m += y;
      m2 += y * y;
    }
    m /= n;
    const double var = m2 / n - m * m;
    s->h_ym[d] = (float)m;
    s->h_ys[d] = var > 1e-12 ? (float)sqrt(var) : 1.f;
    for (int64_t i = 0; i < n; i++)
      T[i * nd + d] = (float)((log(fmax(src[i * nd + d], 1e-300)) - m) / s->h_ys[d]);
  }
  int st = JSC_OK;
  cudaFree(s->d_X);
  cudaFree(s->d_T);
  cudaFree(s->d_perm);
  s->d_X = s->d_T = nullptr;
  s->d_perm = nullptr;
  st = st ? st : jsc_dmalloc(&s->d_X, (size_t)n * SUR_NF);
  st = st ? st : jsc_dmalloc(&s->d_T, (size_t)n * nd);
  st = st ? st : jsc_dmalloc(&s->d_perm, (size_t)n);
  if (!st && (cudaMemcpy(s->d_X, X, (size_t)n * SUR_NF * sizeof(float), cudaMemcpyHostToDevice) ||
              cudaMemcpy(s->d_T, T, (size_t)n * nd * sizeof(float), cudaMemcpyHostToDevice) ||
              cudaMemcpy(s->d_ym, s->h_ym, nd * sizeof(float), cudaMemcpyHostToDevice) ||
              cudaMemcpy(s->d_ys, s->h_ys, nd * sizeof(float), cudaMemcpyHostToDevice)))
    st = JSC_ERR_CUDA;
  free(T);
  if (st) return st;
  s->n_train = n;
  if ((st = ensure_train(s, batch))) return st;
  float *d_xm = nullptr, *d_xs = nullptr;
  st = jsc_dmalloc(&d_xm, SUR_NF);
  st = st ? st : jsc_dmalloc(&d_xs, SUR_NF);
  if (!st && (cudaMemcpy(d_xm, s->xm, sizeof(s->xm), cudaMemcpyHostToDevice) ||
              cudaMemcpy(d_xs, s->xs, sizeof(s->xs), cudaMemcpyHostToDevice)))
    st = JSC_ERR_CUDA;
  int *perm = (int *)malloc((size_t)n * sizeof(int));
  if (!perm) st = st ? st : JSC_ERR_NOMEM;
  uint64_t rs = seed;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int ep = 0; ep < epochs && !st; ep++) {
    for (int64_t i = 0; i < n; i++) perm[i] = (int)i;
    for (int64_t i = n - 1; i > 0; i--) {
      const int64_t j = (int64_t)(mix64(&rs) % (uint64_t)(i + 1));
      const int tmp = perm[i];
      perm[i] = perm[j];
      perm[j] = tmp;
    }
    double ep_loss = 0;
    int64_t ep_n = 0;
    const float lr_ep = lr * (float)(0.5 * (1 + cos(M_PI * ep / epochs)));  // cosine decay
    // one upload of the epoch's permutation; the minibatch steps then run
    // back to back on the stream without host synchronisation
    if (cudaMemcpy(s->d_perm, perm, (size_t)n * sizeof(int), cudaMemcpyHostToDevice)) {
      st = JSC_ERR_CUDA;
      break;
    }
    for (int64_t b0 = 0; b0 + batch <= n && !st; b0 += batch) {
      gather_kernel<<<batch, 32>>>(batch, nd, s->d_perm + b0, s->d_X, s->d_T, d_xm, d_xs,
                                   s->d_h[0], s->d_tb);
      const bool last = b0 + 2 * batch > n;
      float l = 0;
      st = forward_backward(s, batch, 0, last ? &l : nullptr);
      if (last) {
        ep_loss += l;
        ep_n++;
      }
      s->adam_t++;
      const float c1 = 1 - powf(b1, (float)s->adam_t), c2 = 1 - powf(b2, (float)s->adam_t);
      for (int l2 = 0; l2 < 4 && !st; l2++)
        for (int j = 0; j < 2; j++) {
          const int64_t cnt = j ? s->out[l2] : (int64_t)s->out[l2] * s->in[l2];
          adam_kernel<<<(unsigned)((cnt + 255) / 256), 256>>>(cnt, s->d_p[l2][j], s->d_g[l2][j],
                                                              s->d_m[l2][j], s->d_v[l2][j], lr_ep,
                                                              b1, b2, c1, c2, 1e-8f);
        }
    }
    if (!st) {
      cudaError_t e = cudaDeviceSynchronize();
      if (e != cudaSuccess) {
        jsc_set_error(JSC_ERR_CUDA, "surrogate training: %s", cudaGetErrorString(e));
        st = JSC_ERR_CUDA;
      }
    }
    if (loss_per_epoch && !st) loss_per_epoch[ep] = ep_n ? (float)(ep_loss / ep_n) : NAN;
  }
  free(perm);
  cudaFree(d_xm);
  cudaFree(d_xs);
  if (st) return st;
  s->trained = 1;
  s->packed = 0;
  s->tc_packed = 0;
  return JSC_OK;
}

static int pack(jsc_surrogate *s, cudaStream_t st) {
  if (s->packed) return JSC_OK;
  sur_pack_kernel<<<64, 256, 0, st>>>(s->nout, s->noutp, s->d_p[0][0], s->d_p[1][0], s->d_p[2][0],
                                      s->d_p[3][0], s->d_p[0][1], s->d_p[1][1], s->d_p[2][1],
                                      s->d_p[3][1], s->d_image);
  JSC_LAUNCH_CHECK();
  s->packed = 1;
  return JSC_OK;
}

// ------------------------------------------------- use inside a batch --

int jsc_sur_features(int n, const double *sp, float *feat, cudaStream_t st) {
  if (n <= 0) return JSC_OK;
  sur_features_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, sp, feat);
  JSC_LAUNCH_CHECK();
  return JSC_OK;
}

static int infer_tc(jsc_surrogate *s, int n, const float *feat, double *src, int nd,
                    cudaStream_t st) {
  int e;
  if (!s->d_tc_image) {
    if ((e = jsc_dmalloc(&s->d_tc_image, (size_t)jsc_sur_tc_image_bytes(s->nout)))) return e;
    if ((e = jsc_dmalloc(&s->d_tc_status, 1))) return e;
  }
  if (!s->tc_packed) {
    const float *w[4] = {s->d_p[0][0], s->d_p[1][0], s->d_p[2][0], s->d_p[3][0]};
    const float *b[4] = {s->d_p[0][1], s->d_p[1][1], s->d_p[2][1], s->d_p[3][1]};
    jsc_count_launch();
    if ((e = jsc_sur_tc_pack(s->nout, w, b, s->d_tc_image, st))) {
      jsc_set_error(JSC_ERR_CUDA, "tcgen05 weight packing: %s", cudaGetErrorString((cudaError_t)e));
      return JSC_ERR_CUDA;
    }
    s->tc_packed = 1;
  }
  TcInferArgs a;
  a.n = n;
  a.nout = s->nout;
  a.nd = nd;
  a.feat = feat;
  a.image = s->d_tc_image;
  for (int c = 0; c < SUR_NF; c++) {
    a.xm[c] = s->xm[c];
    a.xs[c] = s->xs[c];
  }
  a.ym = s->d_ym;
  a.ys = s->d_ys;
  a.src = src;
  a.status = s->d_tc_status;
  JSC_CUDA_TRY(cudaMemsetAsync(s->d_tc_status, 0, sizeof(unsigned), st));
  jsc_count_launch();
  if ((e = jsc_sur_tc_infer(a, st))) {
    jsc_set_error(JSC_ERR_CUDA, "tcgen05 inference launch: %s", cudaGetErrorString((cudaError_t)e));
    return JSC_ERR_CUDA;
  }
  unsigned hs = 0;
  JSC_CUDA_TRY(cudaMemcpyAsync(&hs, s->d_tc_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  JSC_CUDA_TRY(cudaStreamSynchronize(st));
  if (hs) {
    jsc_set_error(JSC_ERR_WATCHDOG, "tcgen05 inference: an MMA completion wait gave up");
    return JSC_ERR_WATCHDOG;
  }
  return JSC_OK;
}

extern "C" int jsc_surrogate_set_tensor_path(jsc_surrogate *s, int tcgen05) {
  if (!s) return JSC_ERR_ARG;
  s->tc = tcgen05 != 0;
  return JSC_OK;
}

int jsc_sur_infer(jsc_surrogate *s, int n, const float *feat, double *src, int nd,
                  cudaStream_t st) {
  if (n <= 0) return JSC_OK;
  if (s->tc) return infer_tc(s, n, feat, src, nd, st);
  int e = pack(s, st);
  if (e) return e;
  SurInferArgs a;
  a.n = n;
  a.nout = s->nout;
  a.noutp = s->noutp;
  a.feat = feat;
  a.image = s->d_image;
  for (int c = 0; c < SUR_NF; c++) {
    a.xm[c] = s->xm[c];
    a.xs[c] = s->xs[c];
  }
  a.ym = s->d_ym;
  a.ys = s->d_ys;
  a.src = src;
  a.nd = nd;
  const size_t smem = sur_image(s->noutp).bytes + (size_t)SUR_INF_WARPS * 16 * SUR_KP * 2;
  const int tiles = (n + 15) / 16;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  int blocks = (tiles + SUR_INF_WARPS - 1) / SUR_INF_WARPS;
  if (blocks > 2 * nsm) blocks = 2 * nsm;
#define SUR_LAUNCH(NT)                                                                       \
  do {                                                                                       \
    JSC_CUDA_TRY(cudaFuncSetAttribute(sur_infer_kernel<NT>,                                  \
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    sur_infer_kernel<NT><<<blocks, SUR_INF_WARPS * 32, smem, st>>>(a);                       \
  } while (0)
  switch (s->noutp / 8) {
    case 1: SUR_LAUNCH(1); break;
    case 2: SUR_LAUNCH(2); break;
    case 3: SUR_LAUNCH(3); break;
    case 4: SUR_LAUNCH(4); break;
    case 5: SUR_LAUNCH(5); break;
    case 6: SUR_LAUNCH(6); break;
    case 7: SUR_LAUNCH(7); break;
    default: SUR_LAUNCH(8); break;
  }
#undef SUR_LAUNCH
  JSC_LAUNCH_CHECK();
  return JSC_OK;
}

int jsc_sur_nout(const jsc_surrogate *s) { return s->nout; }
int jsc_sur_trained(const jsc_surrogate *s) { return s->trained; }

void jsc_sur_envelope(const jsc_surrogate *s, float *lo, float *hi) {
  for (int c = 0; c < SUR_NF; c++) {
    lo[c] = s->lo[c];
    hi[c] = s->hi[c];
  }
}

// Run the surrogate on host features (tests and tools).
extern "C" int jsc_surrogate_predict(jsc_surrogate *s, const float *feat, int n, double *src) {
  if (!s || !feat || !src || n < 0) return JSC_ERR_ARG;
  if (n == 0) return JSC_OK;
  JSC_CUDA_TRY(cudaSetDevice(s->device));
  float *d_f = nullptr;
  double *d_s = nullptr;
  int st = jsc_dmalloc(&d_f, (size_t)n * SUR_NF);
  st = st ? st : jsc_dmalloc(&d_s, (size_t)n * s->nout);
  if (!st && cudaMemcpy(d_f, feat, (size_t)n * SUR_NF * sizeof(float), cudaMemcpyHostToDevice))
    st = JSC_ERR_CUDA;
  if (!st) st = jsc_sur_infer(s, n, d_f, d_s, s->nout, 0);
  if (!st && cudaMemcpy(src, d_s, (size_t)n * s->nout * sizeof(double), cudaMemcpyDeviceToHost))
    st = JSC_ERR_CUDA;
  cudaFree(d_f);
  cudaFree(d_s);
  return st;
}
