// EGA kernel instantiations for up to 8 emitters.
#include "ega_kernel.cuh"

JSC_EGA_LAUNCHER(jsc_ega_launch_g8, 8)
