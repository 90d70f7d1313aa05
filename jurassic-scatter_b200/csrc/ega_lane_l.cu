// EGA lane-kernel instantiations for 5 to NGMAX emitters, and the
// continuum/Planck kernel.
#include "ega_lane.cuh"

void jsc_ega_lane_launch_l(const EgaArgs &ea, int v, bool dig, cudaStream_t s) {
  if (ea.m.ng <= 8) ega_lane_variant<8>(ea, v, dig, s);
  else if (ea.m.ng <= 16) ega_lane_variant<16>(ea, v, dig, s);
  else ega_lane_variant<32>(ea, v, dig, s);
}

void jsc_ctm_src_launch(const CtmArgs &ca, cudaStream_t s) {
  const int64_t n = ca.n_points * ca.m.nd;
  if (n <= 0) return;
  int64_t blocks = (n + 255) / 256;
  // a count known only on the device: a grid of a few blocks per SM walks it
  if (ca.n_live && blocks > 148 * 16) blocks = 148 * 16;
  ctm_src_kernel<<<(unsigned)blocks, 256, 0, s>>>(ca);
}
