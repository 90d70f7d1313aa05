// tcgen05 inference of the scattering-source surrogate (surrogate_tc.cu).
#pragma once
#include <cuda_runtime.h>

struct TcInferArgs {
  int n, nout, nd;
  const float *feat;            // [n][8] raw features
  const unsigned char *image;   // packed weights (jsc_sur_tc_pack)
  float xm[8], xs[8];           // feature standardisation
  const float *ym, *ys;         // [nout] target standardisation
  double *src;                  // [n][nd]
  unsigned *status;             // bit 0: an MMA wait gave up
};

// Bytes of the packed weight image for nout outputs.
int jsc_sur_tc_image_bytes(int nout);
// Pack the FP32 master weights w[l] [out][in] and biases b[l] into the image.
int jsc_sur_tc_pack(int nout, const float *const *w, const float *const *b, unsigned char *image,
                    cudaStream_t st);
// Launch the inference; 0 on success, else the CUDA error of the launch.
int jsc_sur_tc_infer(const TcInferArgs &a, cudaStream_t st);
