// Internal declarations of the cost-model kernels (emd_sched.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace emdb {

constexpr int kNFeat = 32;
constexpr int kHidden = 128;
constexpr int kNOut = 2;
constexpr int kNBands = 8;
constexpr int kNSeg = 8;
constexpr int kNParams = kNFeat * kHidden + kHidden + kHidden * kHidden + kHidden + kHidden * kNOut + kNOut;

struct FeatParams {
  const double* values;
  const int64_t* offsets;  // NULL = dense [batch, dense_n]
  int dense_n;
  int batch;
  float* feat;             // [batch, 32]
};

struct MlpFwdParams {
  const float* params;     // kNParams floats
  const float* X;          // [B, 32] raw features
  const float* mu;         // [32]
  const float* sd;         // [32]
  int B;
  float* Z1; float* H1; float* Z2; float* H2;  // [B, 128]
  float* Y;                // [B, 2]
};

struct MlpBwdParams {
  const float* params;
  const float* X; const float* mu; const float* sd;
  const float* Z1; const float* H1; const float* Z2; const float* H2;
  const float* Y; const float* T;  // [B, 2]
  int B;
  float* dY; float* dZ2; float* dZ1;
  float* loss;             // accumulates mean squared error
};

struct MlpInferParams {
  const __nv_bfloat16* params_bf16;  // kNParams
  const float* X; const float* mu; const float* sd;
  int B;
  float* Y;
};

cudaError_t launch_features(const FeatParams& p, int grid, cudaStream_t st);
cudaError_t launch_mlp_forward(const MlpFwdParams& p, cudaStream_t st);
cudaError_t launch_mlp_backward(const MlpBwdParams& p, float* grads, cudaStream_t st);
cudaError_t launch_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                        float eps, int t, __nv_bfloat16* wbf, cudaStream_t st);
cudaError_t launch_mlp_infer(const MlpInferParams& p, int grid, cudaStream_t st);

}  // namespace emdb
