// Internal interface of the scattering-source surrogate (surrogate.cu) for
// the batch driver.
#pragma once
#include <cuda_runtime.h>

#include "jsc_internal.h"

#define SUR_NF 8           // input features per scattering point
#define SUR_W 128          // hidden width
#define SUR_NOUT_MAX 64    // channels the output layer can hold

struct jsc_surrogate;

struct SurEnvelope {
  float lo[SUR_NF], hi[SUR_NF];
};

// Features [n][SUR_NF] (raw, FP32) of n scattering-point records.
int jsc_sur_features(int n, const double *sp, float *feat, cudaStream_t st);
// Scattering source [n][nd] of n points from their features (BF16 tensor
// cores, FP32 accumulation).
int jsc_sur_infer(jsc_surrogate *s, int n, const float *feat, double *src, int nd,
                  cudaStream_t st);
int jsc_sur_nout(const jsc_surrogate *s);
int jsc_sur_trained(const jsc_surrogate *s);
// Raw-feature envelope of the training set (widened by 2 % of its range).
void jsc_sur_envelope(const jsc_surrogate *s, float *lo, float *hi);
