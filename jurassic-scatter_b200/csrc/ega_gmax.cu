// EGA kernel instantiations for 9 to NGMAX emitters (default variant).
#include "ega_kernel.cuh"

void jsc_ega_launch_gmax(const EgaArgs &ea, unsigned g128, unsigned g256, int v, bool dig,
                         cudaStream_t s) {
  (void)v;
  if (ea.m.ng <= 16) {
    if (dig) ega_launch_variant<16, true>(ea, g128, g256, JSC_EGA_DEFAULT_VARIANT, s);
    else ega_launch_variant<16, false>(ea, g128, g256, JSC_EGA_DEFAULT_VARIANT, s);
  } else {
    if (dig) ega_launch_variant<NGMAX, true>(ea, g128, g256, JSC_EGA_DEFAULT_VARIANT, s);
    else ega_launch_variant<NGMAX, false>(ea, g128, g256, JSC_EGA_DEFAULT_VARIANT, s);
  }
}
