// EGA kernel instantiations for up to 2 emitters.
#include "ega_kernel.cuh"

JSC_EGA_LAUNCHER(jsc_ega_launch_g2, 2)
