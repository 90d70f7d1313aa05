// Surrogate inference on the 5th-generation tensor cores (tcgen05, sm_100a):
// 128 scattering points per tile, two threads per point (each half of the
// columns of the point's accumulator row), the four layers as
// tcgen05.mma (kind::f16, BF16 operands from shared memory, FP32
// accumulator in tensor memory), bias + tanh in registers between layers.
//
// Per block: one 128-column TMEM accumulator (M = 128 rows = points, N <= 128
// columns), the four weight matrices and the activation tile in shared
// memory in the canonical no-swizzle K-major layout (8-row x 16-byte core
// matrices; LBO = 128 B between core matrices along K, SBO = K/8 * 128 B
// between 8-row groups).  Thread 0 issues the MMAs and commits them to an
// mbarrier; every thread polls it with an iteration limit, after which the
// block records an error, releases its tensor memory and returns.
#include <cuda_bf16.h>
#include <stdint.h>

#include "surrogate_tc.h"

#define TC_M 128
#define TC_T 256          // threads per block: two warps per TMEM lane quadrant
#define TC_K0 16          // first-layer K: the 8 features padded to one k-step
#define TC_W 128          // hidden width
#define TC_SPIN (1 << 21) // polls with 64 ns sleeps: a wait gives up after ~0.2 s

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start, leading and stride byte offsets
// (16-byte units), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (r, k) of a K-major tile with K columns.
__host__ __device__ __forceinline__ uint32_t tc_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
      : "memory");
}

// Non-blocking polls of the mbarrier phase with short sleeps, a bounded number.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (int i = 0; i < TC_SPIN; i++) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Image layout (bytes): W0 [128 x 16], W1, W2 [128 x 128], W3 [noutp16 x 128]
// (bf16, K-major core matrices), biases FP32 [3*128 + noutp16].
__host__ __device__ inline size_t tc_image_bytes(int noutp16) {
  return (size_t)TC_W * TC_K0 * 2 + 2 * (size_t)TC_W * TC_W * 2 + (size_t)noutp16 * TC_W * 2 +
         (size_t)(3 * TC_W + noutp16) * 4;
}

// Pack FP32 master weights into the image.
static __global__ void tc_pack_kernel(int nout, int noutp16, const float *w0, const float *w1,
                                      const float *w2, const float *w3, const float *b0,
                                      const float *b1, const float *b2, const float *b3,
                                      unsigned char *image) {
  unsigned char *q0 = image;
  unsigned char *q1 = q0 + TC_W * TC_K0 * 2;
  unsigned char *q2 = q1 + TC_W * TC_W * 2;
  unsigned char *q3 = q2 + TC_W * TC_W * 2;
  float *bb = reinterpret_cast<float *>(q3 + (size_t)noutp16 * TC_W * 2);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (int i = tid; i < TC_W * TC_K0; i += nt) {
    const int o = i / TC_K0, k = i - o * TC_K0;
    *reinterpret_cast<__nv_bfloat16 *>(q0 + tc_off(o, k, TC_K0)) =
        __float2bfloat16_rn(k < 8 ? w0[o * 8 + k] : 0.f);
  }
  for (int i = tid; i < TC_W * TC_W; i += nt) {
    const int o = i / TC_W, k = i - o * TC_W;
    *reinterpret_cast<__nv_bfloat16 *>(q1 + tc_off(o, k, TC_W)) = __float2bfloat16_rn(w1[i]);
    *reinterpret_cast<__nv_bfloat16 *>(q2 + tc_off(o, k, TC_W)) = __float2bfloat16_rn(w2[i]);
  }
  for (int i = tid; i < noutp16 * TC_W; i += nt) {
    const int o = i / TC_W, k = i - o * TC_W;
    *reinterpret_cast<__nv_bfloat16 *>(q3 + tc_off(o, k, TC_W)) =
        __float2bfloat16_rn(o < nout ? w3[o * TC_W + k] : 0.f);
  }
  for (int i = tid; i < 3 * TC_W + noutp16; i += nt) {
    float v;
    if (i < TC_W) v = b0[i];
    else if (i < 2 * TC_W) v = b1[i - TC_W];
    else if (i < 3 * TC_W) v = b2[i - 2 * TC_W];
    else v = (i - 3 * TC_W < nout) ? b3[i - 3 * TC_W] : 0.f;
    bb[i] = v;
  }
}

// Hardware tanh (one MUFU operation, relative error about 2^-11): its result
// is rounded to BF16 (relative step 2^-8) right away.
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// bias + tanh of columns [c0, c0 + 64) of this thread's row of the
// accumulator, written as the next layer's K-major BF16 activation row.
__device__ __forceinline__ void tc_act(uint32_t tmem_row, const float *bias, unsigned char *act,
                                       int row, int c0) {
#pragma unroll 1
  for (int c = c0; c < c0 + TC_W / 2; c += 16) {
    float v[16];
    tmem_ld16(tmem_row + (uint32_t)c, v);
    __align__(16) __nv_bfloat16 h[16];
#pragma unroll
    for (int i = 0; i < 16; i++) h[i] = __float2bfloat16_rn(tanh_fast(v[i] + bias[c + i]));
    *reinterpret_cast<uint4 *>(act + tc_off(row, c, TC_W)) = *reinterpret_cast<uint4 *>(&h[0]);
    *reinterpret_cast<uint4 *>(act + tc_off(row, c + 8, TC_W)) = *reinterpret_cast<uint4 *>(&h[8]);
  }
}

template <int NOUT16>
static __global__ void __launch_bounds__(TC_T, 2) sur_infer_tc_kernel(TcInferArgs A) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const size_t ib = tc_image_bytes(NOUT16 * 16);
  unsigned char *w0 = sm;
  unsigned char *w1 = w0 + TC_W * TC_K0 * 2;
  unsigned char *w2 = w1 + TC_W * TC_W * 2;
  unsigned char *w3 = w2 + TC_W * TC_W * 2;
  const float *bias = reinterpret_cast<const float *>(w3 + (size_t)NOUT16 * 16 * TC_W * 2);
  unsigned char *act = sm + ((ib + 1023) & ~(size_t)1023);  // [128 x 128] bf16, K-major
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  // warp w reads TMEM lanes (rows) 32 (w % 4) .. +31, columns of half w / 4
  const int quad = warp & 3, half = warp >> 2;
  const int row = quad * 32 + (tid & 31);

  for (size_t i = (size_t)tid * 16; i < ib; i += TC_T * 16)
    *reinterpret_cast<uint4 *>(sm + i) = *reinterpret_cast<const uint4 *>(A.image + i);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(
                     smem_addr(&tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t tmem_row = tmem + ((uint32_t)(quad * 32) << 16);  // this warp's 32 lanes
  const uint32_t mb = smem_addr(&mbar);
  uint32_t phase = 0;
  const uint32_t a_base = smem_addr(act), w0a = smem_addr(w0), w1a = smem_addr(w1),
                 w2a = smem_addr(w2), w3a = smem_addr(w3);

  const int ntiles = (A.n + TC_M - 1) / TC_M;
  bool aborted = false;  // block-uniform
  for (int tile = blockIdx.x; tile < ntiles && !aborted; tile += gridDim.x) {
    const int p = tile * TC_M + row;
    if (half == 0) {
      // layer 0 input: standardised features as a 128 x 16 K-major tile
      __align__(16) __nv_bfloat16 h[16];
#pragma unroll
      for (int c = 0; c < 16; c++) {
        float v = 0.f;
        if (c < 8 && p < A.n) v = (A.feat[(size_t)p * 8 + c] - A.xm[c]) / A.xs[c];
        h[c] = __float2bfloat16_rn(v);
      }
      *reinterpret_cast<uint4 *>(act + tc_off(row, 0, TC_K0)) = *reinterpret_cast<uint4 *>(&h[0]);
      *reinterpret_cast<uint4 *>(act + tc_off(row, 8, TC_K0)) = *reinterpret_cast<uint4 *>(&h[8]);
    }
#pragma unroll 1
    for (int layer = 0; layer < 4; layer++) {
      fence_async_smem();
      tc_before_sync();
      __syncthreads();
      tc_after_sync();
      if (tid == 0) {
        const int K = layer == 0 ? TC_K0 : TC_W;
        const int N = layer == 3 ? NOUT16 * 16 : TC_W;
        const uint32_t wa = layer == 0 ? w0a : (layer == 1 ? w1a : (layer == 2 ? w2a : w3a));
        const uint32_t sbo = (uint32_t)(K / 8) * 128;
        const uint32_t idesc = tc_idesc(TC_M, N);
        for (int s = 0; s < K / 16; s++)
          tc_mma(tmem, tc_desc(a_base + (uint32_t)s * 256, 128, sbo),
                 tc_desc(wa + (uint32_t)s * 256, 128, sbo), idesc, s > 0 ? 1u : 0u);
        tc_commit(mb);
      }
      const bool ok = mbar_wait(mb, phase);
      phase ^= 1;
      if (__syncthreads_or(!ok)) {  // every thread takes the same branch
        if (tid == 0) atomicOr(A.status, 1u);
        aborted = true;
        break;
      }
      tc_after_sync();
      if (layer < 3) {
        tc_act(tmem_row, bias + layer * TC_W, act, row, half * (TC_W / 2));
      } else {
        const float *b3 = bias + 3 * TC_W;
#pragma unroll 1
        for (int c = half * 16; c < NOUT16 * 16; c += 32) {
          float v[16];
          tmem_ld16(tmem_row + (uint32_t)c, v);
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int o = c + i;
            if (p < A.n && o < A.nout)
              A.src[(size_t)p * A.nd + o] = exp((double)((v[i] + b3[o]) * A.ys[o] + A.ym[o]));
          }
        }
      }
      tc_before_sync();
    }
    __syncthreads();
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem) : "memory");
}

int jsc_sur_tc_image_bytes(int nout) { return (int)tc_image_bytes((nout + 15) / 16 * 16); }

int jsc_sur_tc_pack(int nout, const float *const *w, const float *const *b, unsigned char *image,
                    cudaStream_t st) {
  tc_pack_kernel<<<64, 256, 0, st>>>(nout, (nout + 15) / 16 * 16, w[0], w[1], w[2], w[3], b[0],
                                     b[1], b[2], b[3], image);
  return (int)cudaGetLastError();
}

int jsc_sur_tc_infer(const TcInferArgs &a, cudaStream_t st) {
  const int n16 = (a.nout + 15) / 16;
  const size_t ib = tc_image_bytes(n16 * 16);
  const size_t smem = ((ib + 1023) & ~(size_t)1023) + (size_t)TC_M * TC_W * 2 + 1024;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // two resident blocks per SM where the shared memory allows it: one
  // block's epilogue (tanh, BF16 stores) overlaps the other's MMAs
  const int tiles = (a.n + TC_M - 1) / TC_M;
  int per_sm = 1;
  {
    int smem_sm = 0;
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (2 * (smem + 2048) <= (size_t)smem_sm) per_sm = 2;
  }
  const int blocks = tiles < per_sm * nsm ? tiles : per_sm * nsm;
  if (blocks < 1) return 0;
  cudaError_t e = cudaSuccess;
#define TC_LAUNCH(N)                                                                        \
  do {                                                                                      \
    e = cudaFuncSetAttribute(sur_infer_tc_kernel<N>,                                        \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);       \
    if (e != cudaSuccess) return (int)e;                                                    \
    sur_infer_tc_kernel<N><<<blocks, TC_T, smem, st>>>(a);                                  \
  } while (0)
  switch (n16) {
    case 1: TC_LAUNCH(1); break;
    case 2: TC_LAUNCH(2); break;
    case 3: TC_LAUNCH(3); break;
    default: TC_LAUNCH(4); break;
  }
#undef TC_LAUNCH
  return (int)cudaGetLastError();
}
