// emdb_run_noalloc: the dense sift entry point for callers that cannot
// allocate device memory.
//
// Who needs it: services that reserve all device memory up front and forbid
// allocations on their request path, hosts whose own allocator owns the
// device (allocating behind its back breaks its accounting), and latency-
// critical paths that cannot afford cudaMalloc/cudaFree (which may
// synchronise the device).  emdb_run needs a plan, and creating a plan
// allocates its work-queue ticket, status word and spill slab; this entry
// point instead uses one file-scope device array as that scratch.
//
// The array is kNoAllocScratchBytes (32 MiB) and lives on every GPU that
// loads the library until the process exits.  Its first 256 bytes hold the
// queue ticket, the status word and the pass counters; the ticket and
// counters are cleared before every launch, the status word only by
// emdb_noalloc_status (so a flag raised by any call stays visible until it is
// read).  The rest is the per-CTA spill slab, which bounds how many CTAs one
// call runs: a config whose per-CTA slab does not fit even once is rejected.
// Every call shares the array, so calls that overlap on the GPU (different
// streams, or another thread) race on it: serialise them.  The array's device
// address is looked up once per device, on that device's first call, so make
// the first call before any stream capture; a cudaDeviceReset between calls
// is not supported (the module, and with it the array, may move).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/emdb200.h"
#include "emdb_internal.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr size_t kCtlBytes = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

}  // namespace

// defined in emdb_api.cu, not exported: set the thread's last-error message;
// the planned path's config check; its automatic arena rule
extern "C" __attribute__((visibility("hidden"))) int emdb_noalloc_fail(int code, const char* msg);
extern "C" __attribute__((visibility("hidden"))) int emdb_noalloc_check_config(const emdb_config* c);
extern "C" __attribute__((visibility("hidden"))) int emdb_noalloc_auto_arena(int smem_optin, int nbsym,
                                                                             int max_n);

namespace {

// The array's device address on the current device, looked up on the
// device's first use (nullptr and an error message on failure).
void* scratch_base(int* dev_out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    emdb_noalloc_fail(EMDB_ERR_CUDA, "no usable current device");
    return nullptr;
  }
  *dev_out = dev;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* a = nullptr;
    if (cudaGetSymbolAddress(&a, g_noalloc_scratch) != cudaSuccess || !a) {
      emdb_noalloc_fail(EMDB_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
      return nullptr;
    }
    g_addr[dev] = a;
  }
  return g_addr[dev];
}

}  // namespace

extern "C" int emdb_run_noalloc(const emdb_config* cfg, const double* signals, const double* T,
                                int batch, int N, double* imfs, int* n_imfs, int* overflow,
                                int* dbg_n, int* dbg_extno, int* dbg_nzm, void* stream) {
  // the same config rules as a plan (max_extrema in [4, 2^20], nbsym, ...)
  int rc = emdb_noalloc_check_config(cfg);
  if (rc) return rc;
  if (batch < 0 || N < 0) return emdb_noalloc_fail(EMDB_ERR_INVALID, "batch and N must be >= 0");
  if (batch == 0) return EMDB_OK;
  if ((N > 0 && (!signals || !imfs)) || !n_imfs || !overflow || !dbg_n || !dbg_extno || !dbg_nzm)
    return emdb_noalloc_fail(EMDB_ERR_INVALID, "NULL buffer");

  const size_t stride = (emdb::sift_slab_bytes(cfg->max_extrema, cfg->nbsym) + 255) & ~size_t(255);
  if (kCtlBytes + stride > kNoAllocScratchBytes)
    return emdb_noalloc_fail(EMDB_ERR_UNSUPPORTED,
                             ("max_extrema " + std::to_string(cfg->max_extrema) + " needs " +
                              std::to_string(stride) + " bytes of spill scratch per CTA; the "
                              "no-allocation entry point has " +
                              std::to_string(kNoAllocScratchBytes - kCtlBytes) + " bytes").c_str());
  int dev = 0;
  void* base = scratch_base(&dev);
  if (!base) return EMDB_ERR_CUDA;
  int sms = 0, optin = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess || sms < 1 || optin < 1)
    return emdb_noalloc_fail(EMDB_ERR_CUDA, "device attribute query failed");
  // shared-memory arena: the planned path's automatic rule (most resident
  // CTAs whose arena holds the trace plus room for knots, at least 3 per SM
  // when the trace fits, 128-byte rounded)
  const int arena = emdb_noalloc_auto_arena(optin, cfg->nbsym, N);
  if (arena <= 0 || emdb::sift_fixed_smem(std::max(N, 1)) + 64 > (size_t)arena)
    return emdb_noalloc_fail(EMDB_ERR_UNSUPPORTED,
                             ("trace length " + std::to_string(N) +
                              " does not fit this device's shared memory").c_str());
  int per_sm = 0;
  e = emdb::sift_occupancy(arena, 4, &per_sm);
  if (e != cudaSuccess || per_sm < 1) return emdb_noalloc_fail(EMDB_ERR_CUDA, "occupancy query failed");
  const int by_scratch = (int)((kNoAllocScratchBytes - kCtlBytes) / stride);
  const int grid = std::min(std::min(batch, per_sm * sms), by_scratch);

  unsigned char* ctl = static_cast<unsigned char*>(base);
  cudaStream_t st = (cudaStream_t)stream;
  // queue ticket (bytes 0-3) and pass counters (8-23) start at zero; the
  // status word (4-7) keeps earlier flags until emdb_noalloc_status reads it
  e = cudaMemsetAsync(ctl, 0, 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctl + 8, 0, 16, st);
  if (e != cudaSuccess) return emdb_noalloc_fail(EMDB_ERR_CUDA, "clearing the scratch control words failed");

  emdb::SiftParams sp{};
  sp.values = signals;
  sp.offsets = nullptr;
  sp.dense_n = N;
  sp.T = T;
  sp.t_mode = T ? emdb::kTShared : emdb::kTArange;
  sp.batch = batch;
  sp.order = nullptr;
  sp.imfs = imfs;
  sp.n_imfs = n_imfs;
  sp.overflow = overflow;
  sp.dbg_n = dbg_n;
  sp.dbg_ext = dbg_extno;
  sp.dbg_nzm = dbg_nzm;
  sp.queue = reinterpret_cast<int*>(ctl);
  sp.status = reinterpret_cast<int*>(ctl + 4);
  sp.counters = reinterpret_cast<unsigned long long*>(ctl + 8);
  sp.slab = reinterpret_cast<char*>(ctl + kCtlBytes);
  sp.slab_stride = stride;
  sp.arena_bytes = arena;
  sp.max_extrema = cfg->max_extrema;
  sp.nbsym = cfg->nbsym;
  sp.max_iteration = cfg->max_iteration;
  sp.max_imfs = cfg->max_imfs;
  sp.variant = 4;
  e = emdb::launch_sift(sp, grid, st);
  if (e != cudaSuccess) return emdb_noalloc_fail(EMDB_ERR_CUDA, cudaGetErrorString(e));
  return EMDB_OK;
}

extern "C" int emdb_noalloc_status(int* status, void* stream) {
  if (!status) return emdb_noalloc_fail(EMDB_ERR_INVALID, "status is NULL");
  *status = 0;
  int dev = 0;
  void* base = scratch_base(&dev);
  if (!base) return EMDB_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  int* word = reinterpret_cast<int*>(static_cast<unsigned char*>(base) + 4);
  int h = 0;
  // read into host memory, then clear; both on `stream`, after the calls on it
  cudaError_t e = cudaMemcpyAsync(&h, word, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(word, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return emdb_noalloc_fail(EMDB_ERR_CUDA, cudaGetErrorString(e));
  *status = h;
  return EMDB_OK;
}
