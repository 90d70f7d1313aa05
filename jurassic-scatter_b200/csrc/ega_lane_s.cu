// EGA lane-kernel instantiations for up to 4 emitters.
#include "ega_lane.cuh"

void jsc_ega_lane_launch_s(const EgaArgs &ea, int v, bool dig, cudaStream_t s) {
  if (ea.m.ng <= 1) ega_lane_variant<1>(ea, v, dig, s);
  else if (ea.m.ng <= 2) ega_lane_variant<2>(ea, v, dig, s);
  else ega_lane_variant<4>(ea, v, dig, s);
}
