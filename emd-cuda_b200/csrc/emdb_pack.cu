// Packing of ragged (CSR) results for the copy back to host memory.
//
// A ragged launch writes trace b's max_imfs rows of N_b samples at
// imfs + max_imfs*offsets[b]; rows past the trace's data are zeros.  Before
// the device->host copy only the leading rows that may hold data are worth
// moving, so this kernel gathers rows [0, n_rows[b]) of every trace into one
// dense buffer (trace b at packed + row_off[b]) and the copy moves that
// buffer alone.  A straight gather, HBM-bound: one CTA walks one trace at a
// time (grid-stride over traces), its threads copying consecutive doubles.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/emdb200.h"

namespace {

__global__ void __launch_bounds__(256) pack_rows_kernel(const double* __restrict__ imfs,
                                                        const int64_t* __restrict__ offsets,
                                                        const int* __restrict__ n_rows,
                                                        const int64_t* __restrict__ row_off,
                                                        int batch, int max_imfs,
                                                        double* __restrict__ packed) {
  for (int b = blockIdx.x; b < batch; b += gridDim.x) {
    const int64_t off = offsets[b];
    const int64_t n = offsets[b + 1] - off;
    int k = n_rows[b];
    k = k < 0 ? 0 : (k > max_imfs ? max_imfs : k);
    const double* src = imfs + (int64_t)max_imfs * off;
    double* dst = packed + row_off[b];
    const int64_t len = (int64_t)k * n;
    for (int64_t i = threadIdx.x; i < len; i += blockDim.x) dst[i] = src[i];
  }
}

}  // namespace

// sets the thread's last-error message (emdb_api.cu, not exported)
extern "C" __attribute__((visibility("hidden"))) int emdb_internal_fail(int code, const char* msg);

extern "C" int emdb_pack_rows(const double* imfs, const int64_t* offsets, const int* n_rows,
                              const int64_t* row_off, int batch, int max_imfs, double* packed,
                              void* stream) {
  if (batch < 0 || max_imfs < 1) return emdb_internal_fail(EMDB_ERR_INVALID, "bad pack arguments");
  if (batch == 0) return EMDB_OK;
  if (!imfs || !offsets || !n_rows || !row_off || !packed)
    return emdb_internal_fail(EMDB_ERR_INVALID, "NULL buffer");
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return emdb_internal_fail(EMDB_ERR_CUDA, cudaGetErrorString(e));
  const int grid = batch < 8 * sms ? batch : 8 * sms;
  pack_rows_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(imfs, offsets, n_rows, row_off, batch,
                                                           max_imfs, packed);
  e = cudaGetLastError();
  if (e != cudaSuccess) return emdb_internal_fail(EMDB_ERR_CUDA, cudaGetErrorString(e));
  return EMDB_OK;
}
