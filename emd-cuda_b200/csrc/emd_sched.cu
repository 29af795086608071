// Learned queue-order cost model: per-trace features, an MLP 32->128->128->2
// (GELU, tanh form) trained on the GPU with FP32 master weights (forward,
// backward, Adam) and served by a BF16-weight / FP32-accumulate inference
// kernel.  The model only orders the sift work queue; it never touches the
// decomposition arithmetic.  The network is tiny (21k parameters, ~42k FLOP
// per trace): every kernel here is latency-bound, so it runs on the FP32
// pipes with weights staged in shared memory rather than on tensor cores.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "emdb_sched.cuh"

namespace emdb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kFT = 128;        // threads per CTA
constexpr int kRows = 32;       // batch rows per CTA tile
constexpr float kGeluC = 0.7978845608028654f;

__device__ inline float gelu(float z) {
  return 0.5f * z * (1.0f + tanhf(kGeluC * (z + 0.044715f * z * z * z)));
}
__device__ inline float gelu_grad(float z) {
  float u = kGeluC * (z + 0.044715f * z * z * z);
  float t = tanhf(u);
  float du = kGeluC * (1.0f + 3.0f * 0.044715f * z * z);
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * du;
}

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(kFull, v, s);
  return v;
}
__device__ inline double warp_max(double v) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, s));
  return v;
}

// ---------------------------------------------------------------------------
// Features: 32 per trace (definitions restated in oracle/sched_oracle.py).
// One 128-thread CTA per trace, persistent over the batch.
// ---------------------------------------------------------------------------
enum { A_E0, A_E1, A_E2, A_SUM, A_X4, A_ZC, A_NMAX, A_NMIN, A_INFL, A_Z0, A_ZD1, A_Q0, A_Q3,
       A_B0, A_S0 = A_B0 + kNBands, A_MAXABS = A_S0 + kNSeg, A_COUNT };

__global__ void __launch_bounds__(kFT) features_kernel(FeatParams p) {
  __shared__ double red[A_COUNT][kFT / 32];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int b = blockIdx.x; b < p.batch; b += gridDim.x) {
    const int64_t off = p.offsets ? p.offsets[b] : (int64_t)b * p.dense_n;
    const int N = p.offsets ? (int)(p.offsets[b + 1] - off) : p.dense_n;
    const double* x = p.values + off;
    double acc[A_COUNT];
#pragma unroll
    for (int k = 0; k < A_COUNT; ++k) acc[k] = 0.0;
    const int q = N / 4 > 0 ? N / 4 : 1;
    for (int i = tid; i < N; i += kFT) {
      double v = x[i];
      acc[A_E0] += v * v;
      acc[A_SUM] += v;
      acc[A_X4] += v * v * v * v;
      acc[A_MAXABS] = fmax(acc[A_MAXABS], fabs(v));
      if (v == 0.0) acc[A_Z0] += 1.0;
      if (i < q) acc[A_Q0] += v;
      if (i >= N - q) acc[A_Q3] += v;
      if (i + 1 < N) {
        double vn = x[i + 1];
        double d = vn - v;
        acc[A_E1] += d * d;
        if (d == 0.0) acc[A_ZD1] += 1.0;
        if (v * vn < 0.0) acc[A_ZC] += 1.0;
        if (i + 2 < N) {
          double d2n = x[i + 2] - vn;
          double dd = d2n - d;
          acc[A_E2] += dd * dd;
          double p1 = d * d2n;             // extremum at i+1
          if (p1 < 0.0) {
            if (d > 0.0) acc[A_NMAX] += 1.0; else acc[A_NMIN] += 1.0;
            int seg = (int)(((int64_t)(i + 1) * kNSeg) / N);
            seg = seg < kNSeg - 1 ? seg : kNSeg - 1;
            acc[A_S0 + seg] += 1.0;
          }
          if (i + 3 < N) {
            double d3n = x[i + 3] - x[i + 2];
            double dd2 = d3n - d2n;
            if (dd * dd2 < 0.0) acc[A_INFL] += 1.0;
          }
        }
      }
    }
    // dyadic detail energies: thread t streams 256-sample chunks t, t+128, ...
    for (int c = tid; c * 256 < N; c += kFT) {
      int base = c * 256;
      int lim = min(256, N - base);
      double first[kNBands];
#pragma unroll
      for (int k = 0; k < kNBands; ++k) first[k] = 0.0;
      for (int j = 0; j < lim; ++j) {
        double s = x[base + j];
        // block of size 1 at index j completes; merge upwards
        int pos = j;
        int k = 0;
        double cur = s;
        while (k < kNBands) {
          if ((pos & 1) == 0) { first[k] = cur; break; }
          double A = first[k];
          double dd = A - cur;
          acc[A_B0 + k] += dd * dd / (double)(2 << k);
          cur = A + cur;
          pos >>= 1;
          ++k;
        }
      }
    }
    // block reduce (sums; MAXABS by max)
#pragma unroll
    for (int k = 0; k < A_COUNT; ++k) {
      double v = k == A_MAXABS ? warp_max(acc[k]) : warp_sum(acc[k]);
      if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (tid < 32) {
      float* f = p.feat + (int64_t)b * kNFeat;
      double t[A_COUNT];
#pragma unroll
      for (int k = 0; k < A_COUNT; ++k) {
        double v = red[k][0];
        for (int w = 1; w < kFT / 32; ++w) v = k == A_MAXABS ? fmax(v, red[k][w]) : v + red[k][w];
        t[k] = v;
      }
      if (tid == 0) {
        double Nd = N > 0 ? (double)N : 1.0;
        double e0 = t[A_E0], p0 = e0 / Nd, rms = sqrt(p0);
        double o[kNFeat];
        for (int k = 0; k < kNFeat; ++k) o[k] = 0.0;
        if (N > 0) {
          o[0] = log2(Nd) / 14.0;
          o[1] = Nd / 16384.0;
          o[2] = t[A_ZC] / Nd;
          o[3] = (t[A_NMAX] + t[A_NMIN]) / Nd;
          o[4] = t[A_NMAX] / Nd;
          o[5] = t[A_NMIN] / Nd;
          o[6] = log10((t[A_E1] + 1e-300) / (e0 + 1e-300)) / 4.0;
          o[7] = log10((t[A_E2] + 1e-300) / (e0 + 1e-300)) / 4.0;
          o[8] = t[A_INFL] / Nd;
          for (int k = 0; k < kNBands; ++k) o[9 + k] = t[A_B0 + k] / (e0 + 1e-300);
          for (int k = 0; k < kNSeg; ++k) o[17 + k] = t[A_S0 + k] * kNSeg / Nd;
          o[25] = fabs(t[A_SUM] / Nd) / (rms + 1e-300);
          o[26] = (t[A_Q3] - t[A_Q0]) / (double)q / (rms + 1e-300);
          o[27] = t[A_MAXABS] / (rms + 1e-300) / 10.0;
          o[28] = t[A_X4] / Nd / (p0 * p0 + 1e-300) / 10.0;
          o[29] = t[A_Z0] / Nd;
          o[30] = N > 1 ? t[A_ZD1] / Nd : 0.0;
          o[31] = log10(rms + 1e-300) / 4.0;
        }
        for (int k = 0; k < kNFeat; ++k) f[k] = (float)o[k];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// MLP.  Parameter block layout (float): W1[32][128] b1[128] W2[128][128] b2[128]
// W3[128][2] b3[2].
// ---------------------------------------------------------------------------
struct PView {
  const float *W1, *b1, *W2, *b2, *W3, *b3;
};
__device__ inline PView pview(const float* P) {
  PView v;
  v.W1 = P;
  v.b1 = v.W1 + kNFeat * kHidden;
  v.W2 = v.b1 + kHidden;
  v.b2 = v.W2 + kHidden * kHidden;
  v.W3 = v.b2 + kHidden;
  v.b3 = v.W3 + kHidden * kNOut;
  return v;
}

// Training forward: stores Z1, H1, Z2, H2 (per row) and Y.  Features are
// standardised on the fly with (x - mu) / sd.
__global__ void __launch_bounds__(kFT) mlp_forward_kernel(MlpFwdParams p) {
  extern __shared__ float sm[];
  float* W1 = sm;                              // 32*128
  float* W2 = W1 + kNFeat * kHidden;           // 128*128
  float* W3 = W2 + kHidden * kHidden;          // 128*2
  float* b = W3 + kHidden * kNOut;             // 128 + 128 + 2 (+pad)
  float* X = b + 2 * kHidden + 4;              // kRows*32
  float* H = X + kRows * kNFeat;               // kRows*128
  const int tid = threadIdx.x;
  PView P = pview(p.params);
  for (int i = tid; i < kNFeat * kHidden; i += kFT) W1[i] = P.W1[i];
  for (int i = tid; i < kHidden * kHidden; i += kFT) W2[i] = P.W2[i];
  for (int i = tid; i < kHidden * kNOut; i += kFT) W3[i] = P.W3[i];
  for (int i = tid; i < kHidden; i += kFT) { b[i] = P.b1[i]; b[kHidden + i] = P.b2[i]; }
  if (tid < kNOut) b[2 * kHidden + tid] = P.b3[tid];
  const int r0 = blockIdx.x * kRows;
  for (int i = tid; i < kRows * kNFeat; i += kFT) {
    int r = r0 + i / kNFeat, c = i % kNFeat;
    float v = r < p.B ? p.X[(int64_t)r * kNFeat + c] : 0.0f;
    X[i] = (v - p.mu[c]) / p.sd[c];
  }
  __syncthreads();
  const int j = tid;  // hidden unit
  for (int r = 0; r < kRows; ++r) {
    float z = b[j];
    for (int i = 0; i < kNFeat; ++i) z += X[r * kNFeat + i] * W1[i * kHidden + j];
    float h = gelu(z);
    H[r * kHidden + j] = h;
    int row = r0 + r;
    if (row < p.B) { p.Z1[(int64_t)row * kHidden + j] = z; p.H1[(int64_t)row * kHidden + j] = h; }
  }
  __syncthreads();
  float h2[kRows];
  for (int r = 0; r < kRows; ++r) {
    float z = b[kHidden + j];
    for (int i = 0; i < kHidden; ++i) z += H[r * kHidden + i] * W2[i * kHidden + j];
    h2[r] = gelu(z);
    int row = r0 + r;
    if (row < p.B) { p.Z2[(int64_t)row * kHidden + j] = z; p.H2[(int64_t)row * kHidden + j] = h2[r]; }
  }
  __syncthreads();
  for (int r = 0; r < kRows; ++r) H[r * kHidden + j] = h2[r];
  __syncthreads();
  if (tid < kRows * kNOut) {
    int r = tid / kNOut, o = tid % kNOut;
    float y = b[2 * kHidden + o];
    for (int i = 0; i < kHidden; ++i) y += H[r * kHidden + i] * W3[i * kNOut + o];
    int row = r0 + r;
    if (row < p.B) p.Y[(int64_t)row * kNOut + o] = y;
  }
}

// Backward through the rows: dY = 2(Y - T)/(B*2), dZ2, dZ1 (and the loss sum).
__global__ void __launch_bounds__(kFT) mlp_backward_rows_kernel(MlpBwdParams p) {
  extern __shared__ float sm[];
  float* W2T = sm;                             // [j][i] = W2[i][j]
  float* W3 = W2T + kHidden * kHidden;         // 128*2
  float* D = W3 + kHidden * kNOut;             // kRows*128 (dZ2 tile)
  float* dY = D + kRows * kHidden;             // kRows*2
  __shared__ float lred[kFT / 32];
  const int tid = threadIdx.x;
  PView P = pview(p.params);
  for (int i = tid; i < kHidden * kHidden; i += kFT) {
    int r = i / kHidden, c = i % kHidden;
    W2T[c * kHidden + r] = P.W2[i];
  }
  for (int i = tid; i < kHidden * kNOut; i += kFT) W3[i] = P.W3[i];
  const int r0 = blockIdx.x * kRows;
  float lsum = 0.0f;
  if (tid < kRows * kNOut) {
    int r = tid / kNOut, o = tid % kNOut, row = r0 + r;
    float d = 0.0f;
    if (row < p.B) {
      float e = p.Y[(int64_t)row * kNOut + o] - p.T[(int64_t)row * kNOut + o];
      lsum = e * e;
      d = 2.0f * e / (float)(p.B * kNOut);
      p.dY[(int64_t)row * kNOut + o] = d;
    }
    dY[tid] = d;
  }
  __syncthreads();
  const int i = tid;  // hidden unit
  for (int r = 0; r < kRows; ++r) {
    int row = r0 + r;
    float dh = 0.0f;
#pragma unroll
    for (int o = 0; o < kNOut; ++o) dh += dY[r * kNOut + o] * W3[i * kNOut + o];
    float dz = row < p.B ? dh * gelu_grad(p.Z2[(int64_t)row * kHidden + i]) : 0.0f;
    D[r * kHidden + i] = dz;
    if (row < p.B) p.dZ2[(int64_t)row * kHidden + i] = dz;
  }
  __syncthreads();
  for (int r = 0; r < kRows; ++r) {
    int row = r0 + r;
    float dh = 0.0f;
    for (int j = 0; j < kHidden; ++j) dh += D[r * kHidden + j] * W2T[j * kHidden + i];
    if (row < p.B) p.dZ1[(int64_t)row * kHidden + i] = dh * gelu_grad(p.Z1[(int64_t)row * kHidden + i]);
  }
  // loss partial
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) lsum += __shfl_xor_sync(kFull, lsum, s);
  if ((tid & 31) == 0) lred[tid >> 5] = lsum;
  __syncthreads();
  if (tid == 0) {
    float t = 0.0f;
    for (int w = 0; w < kFT / 32; ++w) t += lred[w];
    atomicAdd(p.loss, t / (float)(p.B * kNOut));
  }
}

// Weight gradients: G[in][out] = sum_r A[r][in] * D[r][out]; bias = sum_r D[r][out].
// One thread per output element, rows streamed.
__global__ void mlp_weight_grad_kernel(const float* __restrict__ A, const float* __restrict__ mu,
                                       const float* __restrict__ sd, const float* __restrict__ Dm,
                                       int B, int nin, int nout, float* __restrict__ G,
                                       float* __restrict__ gb) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  int total = nin * nout + nout;
  if (e >= total) return;
  if (e < nin * nout) {
    int i = e / nout, o = e % nout;
    float acc = 0.0f;
    float m = mu ? mu[i] : 0.0f, s = sd ? sd[i] : 1.0f;
    for (int r = 0; r < B; ++r) {
      float a = A[(int64_t)r * nin + i];
      if (mu) a = (a - m) / s;
      acc += a * Dm[(int64_t)r * nout + o];
    }
    G[e] = acc;
  } else {
    int o = e - nin * nout;
    float acc = 0.0f;
    for (int r = 0; r < B; ++r) acc += Dm[(int64_t)r * nout + o];
    gb[o] = acc;
  }
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                            float bc1, float bc2, __nv_bfloat16* __restrict__ wbf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  float mi = b1 * m[i] + (1.0f - b1) * gi;
  float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  w[i] = wi;
  if (wbf) wbf[i] = __float2bfloat16(wi);
}

// BF16-weight inference: same tiling as the training forward, weights staged
// as bf16 in shared memory, FP32 accumulation.  Output Y [B, 2].
__global__ void __launch_bounds__(kFT) mlp_infer_bf16_kernel(MlpInferParams p) {
  extern __shared__ __align__(16) unsigned char smb[];
  __nv_bfloat16* W1 = reinterpret_cast<__nv_bfloat16*>(smb);
  __nv_bfloat16* W2 = W1 + kNFeat * kHidden;
  __nv_bfloat16* W3 = W2 + kHidden * kHidden;
  __nv_bfloat16* bb = W3 + kHidden * kNOut;                 // 258 (+pad to 260)
  float* X = reinterpret_cast<float*>(bb + 2 * kHidden + 4);
  float* H = X + kRows * kNFeat;
  const int tid = threadIdx.x;
  const __nv_bfloat16* P = p.params_bf16;
  const int nW1 = kNFeat * kHidden, nW2 = kHidden * kHidden, nW3 = kHidden * kNOut;
  for (int i = tid; i < nW1; i += kFT) W1[i] = P[i];
  for (int i = tid; i < kHidden; i += kFT) { bb[i] = P[nW1 + i]; bb[kHidden + i] = P[nW1 + kHidden + nW2 + i]; }
  for (int i = tid; i < nW2; i += kFT) W2[i] = P[nW1 + kHidden + i];
  for (int i = tid; i < nW3; i += kFT) W3[i] = P[nW1 + kHidden + nW2 + kHidden + i];
  if (tid < kNOut) bb[2 * kHidden + tid] = P[nW1 + kHidden + nW2 + kHidden + nW3 + tid];
  for (int tile = blockIdx.x; tile * kRows < p.B; tile += gridDim.x) {
    const int r0 = tile * kRows;
    __syncthreads();
    for (int i = tid; i < kRows * kNFeat; i += kFT) {
      int r = r0 + i / kNFeat, c = i % kNFeat;
      float v = r < p.B ? p.X[(int64_t)r * kNFeat + c] : 0.0f;
      X[i] = (v - p.mu[c]) / p.sd[c];
    }
    __syncthreads();
    const int j = tid;
    for (int r = 0; r < kRows; ++r) {
      float z = __bfloat162float(bb[j]);
      for (int i = 0; i < kNFeat; ++i) z += X[r * kNFeat + i] * __bfloat162float(W1[i * kHidden + j]);
      H[r * kHidden + j] = gelu(z);
    }
    __syncthreads();
    float h2[kRows];
    for (int r = 0; r < kRows; ++r) {
      float z = __bfloat162float(bb[kHidden + j]);
      for (int i = 0; i < kHidden; ++i) z += H[r * kHidden + i] * __bfloat162float(W2[i * kHidden + j]);
      h2[r] = gelu(z);
    }
    __syncthreads();
    for (int r = 0; r < kRows; ++r) H[r * kHidden + j] = h2[r];
    __syncthreads();
    if (tid < kRows * kNOut) {
      int r = tid / kNOut, o = tid % kNOut;
      float y = __bfloat162float(bb[2 * kHidden + o]);
      for (int i = 0; i < kHidden; ++i) y += H[r * kHidden + i] * __bfloat162float(W3[i * kNOut + o]);
      int row = r0 + r;
      if (row < p.B) p.Y[(int64_t)row * kNOut + o] = y;
    }
  }
}

}  // namespace

size_t mlp_fwd_smem() {
  return sizeof(float) * (kNFeat * kHidden + kHidden * kHidden + kHidden * kNOut + 2 * kHidden + 4 +
                          kRows * kNFeat + kRows * kHidden);
}
size_t mlp_bwd_smem() {
  return sizeof(float) * (kHidden * kHidden + kHidden * kNOut + kRows * kHidden + kRows * kNOut);
}
size_t mlp_infer_smem() {
  return sizeof(__nv_bfloat16) * (kNFeat * kHidden + kHidden * kHidden + kHidden * kNOut + 2 * kHidden + 4) +
         sizeof(float) * (kRows * kNFeat + kRows * kHidden);
}

cudaError_t launch_features(const FeatParams& p, int grid, cudaStream_t st) {
  features_kernel<<<grid, kFT, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const MlpFwdParams& p, cudaStream_t st) {
  size_t sm = mlp_fwd_smem();
  cudaError_t e = cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int grid = (p.B + kRows - 1) / kRows;
  if (grid > 0) mlp_forward_kernel<<<grid, kFT, sm, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_mlp_backward(const MlpBwdParams& p, float* grads, cudaStream_t st) {
  size_t sm = mlp_bwd_smem();
  cudaError_t e = cudaFuncSetAttribute(mlp_backward_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int grid = (p.B + kRows - 1) / kRows;
  if (grid > 0) mlp_backward_rows_kernel<<<grid, kFT, sm, st>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  float* gW1 = grads;
  float* gb1 = gW1 + kNFeat * kHidden;
  float* gW2 = gb1 + kHidden;
  float* gb2 = gW2 + kHidden * kHidden;
  float* gW3 = gb2 + kHidden;
  float* gb3 = gW3 + kHidden * kNOut;
  auto launch = [&](const float* A, const float* mu, const float* sd, const float* Dm, int nin, int nout,
                    float* G, float* gb) {
    int total = nin * nout + nout;
    mlp_weight_grad_kernel<<<(total + 255) / 256, 256, 0, st>>>(A, mu, sd, Dm, p.B, nin, nout, G, gb);
  };
  launch(p.X, p.mu, p.sd, p.dZ1, kNFeat, kHidden, gW1, gb1);
  launch(p.H1, nullptr, nullptr, p.dZ2, kHidden, kHidden, gW2, gb2);
  launch(p.H2, nullptr, nullptr, p.dY, kHidden, kNOut, gW3, gb3);
  return cudaGetLastError();
}

cudaError_t launch_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                        float eps, int t, __nv_bfloat16* wbf, cudaStream_t st) {
  float bc1 = 1.0f - powf(b1, (float)t), bc2 = 1.0f - powf(b2, (float)t);
  adam_kernel<<<(n + 255) / 256, 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, eps, bc1, bc2, wbf);
  return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const MlpInferParams& p, int grid, cudaStream_t st) {
  size_t sm = mlp_infer_smem();
  cudaError_t e = cudaFuncSetAttribute(mlp_infer_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  if (p.B > 0) mlp_infer_bf16_kernel<<<grid, kFT, sm, st>>>(p);
  return cudaGetLastError();
}

}  // namespace emdb
