// Ray-tile EGA kernel instantiations (up to 16 emitters) and the ray order
// its tiles follow.
#include <cub/device/device_radix_sort.cuh>

#include "ega_lane.cuh"

void jsc_ega_ray_launch(const EgaArgs &ea, int v, bool dig, cudaStream_t s) {
  if (ea.m.ng <= 2) ega_ray_variant<2>(ea, v, dig, s);
  else if (ea.m.ng <= 4) ega_ray_variant<4>(ea, v, dig, s);
  else if (ea.m.ng <= 8) ega_ray_variant<8>(ea, v, dig, s);
  else ega_ray_variant<16>(ea, v, dig, s);
}

// Sort key of ray r: rays that hit the surface after the others, then LOS
// point count, tangent altitude (metres, 23 bits) and profile, so that the
// 32 rays of a tile pass the same altitudes at the same LOS point index.
static __global__ void ray_key_kernel(int n, const int *ray_atm, const int *nlos,
                                      const double *tsurf, const double *tpz,
                                      unsigned long long *key, int *idx) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const unsigned long long hit = tsurf[r] > 0 ? 1ull : 0ull;
  const unsigned long long np = (unsigned long long)min(max(nlos[r], 0), 65535);
  const double zm = fmin(fmax(tpz[r] * 1000.0, 0.0), 8388607.0);
  const unsigned long long zq = (unsigned long long)zm;
  const unsigned long long atm = (unsigned long long)(ray_atm[r] & 0xffffff);
  key[r] = (hit << 63) | (np << 47) | (zq << 24) | atm;
  idx[r] = r;
}

size_t jsc_ray_order_tmp_bytes(int max_rays) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long *)nullptr,
                                  (unsigned long long *)nullptr, (const int *)nullptr,
                                  (int *)nullptr, max_rays);
  return bytes;
}

// order[0, n): ray indices by key; keys and order each hold 2 n_max
// entries (input and output halves), tmp the sort's scratch.
int jsc_ray_order(int n_rays, const int *ray_atm, const int *nlos, const double *tsurf,
                  const double *tpz, unsigned long long *keys, int *order, void *tmp,
                  size_t tmp_bytes, cudaStream_t s) {
  if (n_rays <= 0) return 0;
  unsigned long long *k_in = keys + n_rays;
  int *i_in = order + n_rays;
  ray_key_kernel<<<(n_rays + 255) / 256, 256, 0, s>>>(n_rays, ray_atm, nlos, tsurf, tpz, k_in,
                                                      i_in);
  jsc_count_launch();  // the CUB sort's own launches are not counted
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  size_t bytes = tmp_bytes;
  e = cub::DeviceRadixSort::SortPairs(tmp, bytes, k_in, keys, i_in, order, n_rays, 0, 64, s);
  return (int)e;
}
