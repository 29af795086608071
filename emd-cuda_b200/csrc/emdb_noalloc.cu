// emdb_run_noalloc: the dense sift entry point for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs while a CUDA stream is being captured into a
// graph (device allocation is not allowed there), services that reserve all
// device memory up front and forbid allocations on their request path, and
// hosts whose allocator owns the device (allocating behind its back breaks
// its accounting).  emdb_run needs a plan, and creating a plan allocates its
// work-queue ticket, status word and spill slab; this entry point instead
// uses one file-scope device array as that scratch.
//
// The array is kNoAllocScratchBytes (32 MiB) and lives on every GPU that
// loads the library until the process exits.  Its first 256 bytes hold the
// queue ticket and status word (cleared before every launch); the rest is the
// per-CTA spill slab, which bounds how many CTAs one call runs: a config
// whose per-CTA slab does not fit even once is rejected.  Every call shares
// the array, so calls that overlap on the GPU (different streams, or another
// thread) race on it: serialise them.  The array's device address is looked
// up once per device, on that device's first call, so make the first call
// outside any stream capture.
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

// sets the thread's last-error message (defined in emdb_api.cu, not exported)
extern "C" __attribute__((visibility("hidden"))) int emdb_noalloc_fail(int code, const char* msg);

extern "C" int emdb_run_noalloc(const emdb_config* cfg, const double* signals, const double* T,
                                int batch, int N, double* imfs, int* n_imfs, int* overflow,
                                int* dbg_n, int* dbg_extno, int* dbg_nzm, void* stream) {
  if (!cfg) return emdb_noalloc_fail(EMDB_ERR_INVALID, "config is NULL");
  if (cfg->nbsym < 1 || cfg->nbsym > emdb::kMaxNbsym || cfg->max_extrema < 4 ||
      cfg->max_iteration < 1 || cfg->max_imfs < 2 || cfg->max_imfs > emdb::kMaxImfsCap)
    return emdb_noalloc_fail(EMDB_ERR_INVALID, "invalid config");
  if (cfg->threads_per_block != emdb::kThreads)
    return emdb_noalloc_fail(EMDB_ERR_UNSUPPORTED, "threads_per_block must be 128");
  if (batch < 0 || N < 0) return emdb_noalloc_fail(EMDB_ERR_INVALID, "batch and N must be >= 0");
  if (batch == 0) return EMDB_OK;
  if ((N > 0 && (!signals || !imfs)) || !n_imfs || !overflow || !dbg_n || !dbg_extno || !dbg_nzm)
    return emdb_noalloc_fail(EMDB_ERR_INVALID, "NULL buffer");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return emdb_noalloc_fail(EMDB_ERR_CUDA, "no usable current device");
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      e = cudaGetSymbolAddress(&g_addr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_addr[dev] = nullptr;
        return emdb_noalloc_fail(EMDB_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
      }
    }
    base = g_addr[dev];
  }

  const size_t stride = (emdb::sift_slab_bytes(cfg->max_extrema, cfg->nbsym) + 255) & ~size_t(255);
  if (kCtlBytes + stride > kNoAllocScratchBytes)
    return emdb_noalloc_fail(EMDB_ERR_UNSUPPORTED,
                             ("max_extrema " + std::to_string(cfg->max_extrema) + " needs " +
                              std::to_string(stride) + " bytes of spill scratch per CTA; the "
                              "no-allocation entry point has " +
                              std::to_string(kNoAllocScratchBytes - kCtlBytes) + " bytes").c_str());
  int sms = 0, optin = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  // shared-memory arena: the largest that keeps 4 CTAs resident, else the
  // smallest that holds the trace
  const size_t fixed = emdb::sift_fixed_smem(std::max(N, 1));
  int arena = 0;
  for (int want = 4; want >= 1 && !arena; --want) {
    int a = std::min(233472 / want - 1024, optin) & ~15;
    if ((size_t)a >= fixed + 64) arena = a;
  }
  if (!arena) return emdb_noalloc_fail(EMDB_ERR_UNSUPPORTED, "trace length does not fit shared memory");
  int per_sm = 0;
  e = emdb::sift_occupancy(arena, 4, &per_sm);
  if (e != cudaSuccess || per_sm < 1) return emdb_noalloc_fail(EMDB_ERR_CUDA, "occupancy query failed");
  const int by_scratch = (int)((kNoAllocScratchBytes - kCtlBytes) / stride);
  const int grid = std::min(std::min(batch, per_sm * sms), by_scratch);

  unsigned char* ctl = static_cast<unsigned char*>(base);
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemsetAsync(ctl, 0, kCtlBytes, st);   // queue ticket, status word, counters start at zero
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
