// Learned SGS coefficient network (alfa_mlp.cu): sizes, feature inputs and
// the host launchers of its kernels.
#pragma once
#include <cuda_bf16.h>

#include "alfa_internal.cuh"

namespace alfa {

constexpr int MLP_IN = 10;
constexpr int MLP_H = 64;
constexpr int MLP_NPARAM = MLP_H * MLP_IN + MLP_H + MLP_H * MLP_H + MLP_H + 2 * MLP_H + 2;

struct MlpFeatIn {
  const double* g[9];      // velocity gradients (velocityGradients order)
  const double* dTHdz;     // w nodes
  double L, dz, g_over_T0;
  int nz;
};

// norm: 24 floats, means of the 10 features and 2 targets, then their
// standard deviations
void mlp_sample(cudaStream_t st, const MlpFeatIn& a, const double* Cs2, const double* beta,
                size_t N, unsigned long long seed, int k, float* X, float* T, int offset,
                int cap);
void mlp_norm(cudaStream_t st, const float* X, const float* T, int n, float* norm);
void mlp_grad(cudaStream_t st, const float* P, const float* X, const float* T, const int* idx,
              int s0, int n, int total, const float* norm, float* grad, float* loss);
void mlp_adam(cudaStream_t st, float* P, float* G, float* M, float* V, __nv_bfloat16* Pb,
              float lr, int t);
void mlp_to_bf16(cudaStream_t st, const float* P, __nv_bfloat16* Pb);
// level_scale: nz per-level factors of the Cs^2 output, or null
void mlp_infer(cudaStream_t st, int sms, const MlpFeatIn& a, const __nv_bfloat16* Pb,
               const float* norm, size_t N, const double* level_scale, double* Cs2,
               double* beta);
// Cs^2 only, the hidden layer on the tensor cores (BF16 activations); a
// tensor-core wait that gives up leaves NaN in the affected points
void mlp_infer_tc(cudaStream_t st, int sms, const MlpFeatIn& a, const __nv_bfloat16* Pb,
                  const float* norm, size_t N, const double* level_scale, double* Cs2);
void mlp_features_all(cudaStream_t st, const MlpFeatIn& a, size_t N, float* X);

}  // namespace alfa
