// C ABI of libemdb200.so (declared in include/emdb200.h): plans, launches,
// status read-back and error strings.  Host code only; kernels live in
// emd_sift.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>   // header-only NVTX v3: ranges cost nothing without a profiler

#include "../../include/emdb200.h"
#include "emdb_internal.cuh"

struct emdb_plan {
  emdb_config cfg;
  int device = 0;
  int num_sms = 0;
  int smem_optin = 0;
  int arena_override = 0;
  int variant = 0;            // kernel instance (register variant); 0 = by trace length
  int max_ctas = 0;           // cap on a launch's persistent grid (0 = resident CTAs)
  int tail = -1;              // tail migration: 0 off, -1 below the SM count, > 0 that many
  int* d_tail = nullptr;      // [0] traces in flight, [1] resume tickets
  int* d_cont_valid = nullptr;
  int cont_valid_cap = 0;
  char* d_cont = nullptr;     // continuation records
  size_t cont_bytes = 0;
  int* d_ctl = nullptr;       // [0] sift queue, [1] status, [2] envelope queue
  unsigned long long* d_cnt = nullptr;  // [0] sift passes, [1] spilled passes, [2] / [3]
                                        // load / trace cycles, [4..13] phase cycles
                                        // (instrumented build)
  char* d_slab = nullptr;
  size_t slab_stride = 0;     // knot slab per CTA (the wide instance adds trace arrays)
  size_t slab_bytes = 0;      // allocated
  // host-memory pipeline (emdb_run_host): device staging grown on demand, a
  // non-blocking copy stream, chunk counters and their mapped host flags
  char* d_stage = nullptr;
  size_t stage_bytes = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_kernel = nullptr;
  unsigned* d_chunk_count = nullptr;
  unsigned* d_chunk_rows = nullptr;   // per chunk: rows that may hold data
  unsigned* h_chunk_flag = nullptr;   // pinned, mapped
  unsigned* d_chunk_flag = nullptr;   // its device alias
  // input groups: each group of traces is its own launch on its own stream,
  // with its own queue ticket and slab region, started once its input is in
  static constexpr int kGroups = 4;
  cudaStream_t group_stream[kGroups] = {};
  cudaEvent_t ev_in[kGroups] = {};
  cudaEvent_t ev_group[kGroups] = {};
  int* d_group_queue = nullptr;
  char* d_group_slab = nullptr;
  size_t group_slab_bytes = 0;
  unsigned long long host_h2d = 0, host_d2h = 0;   // bytes the last emdb_run_host moved
  std::mutex mu;
};

// Per-trace completion flags for ragged launches (emdb_run_ragged_notify):
// device counters and row maxima, and flags in mapped host memory.
struct emdb_notify {
  int device = 0;
  int capacity = 0;
  unsigned* d_count = nullptr;
  unsigned* d_rows = nullptr;
  unsigned* h_flag = nullptr;   // pinned, mapped
  unsigned* d_flag = nullptr;   // its device alias
};

namespace {

constexpr int kCounters = 14;   // see emdb_plan::d_cnt

thread_local std::string g_last_error;

// NVTX range for the span of a scope (plan, launch and copy steps show up by
// name on an Nsight timeline; without a tool attached the calls are no-ops)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return fail(e == cudaErrorMemoryAllocation ? EMDB_ERR_NOMEM : EMDB_ERR_CUDA, m);
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Per-SM shared memory is 228 KB on B200 with 1 KB reserved per CTA.  The
// arena for `want` resident CTAs is the largest share that keeps them all.
// Choice: the most CTAs (up to the plan's register variant) whose arena holds
// the trace plus room for ~2 x 96 knots; failing that, still 3 CTAs/SM if
// that arena holds the trace at all, before fewer.  Measured on B200 with
// seismic traces: N = 8192 (4,096 traces) 1,121 ms at 3 CTAs/SM vs 1,435 ms
// at 2 -- below 12 warps per SM latency hiding collapses; N = 2048 (8,192
// traces) 38.4 ms at 4 vs 42.2 ms at 3; N = 4096 within a few percent either
// way, depending on the batch (81 vs 99 ms at 3 vs 4 CTAs/SM for 2,048
// traces, 223 vs 218 ms for 8,192).
// The sift kernels per value type: the FP64 build (the reference's REAL_T)
// and the FP32 build of the same source.
template <typename R> struct SiftKernels;
template <> struct SiftKernels<double> {
  using Params = emdb::SiftParams;
  static size_t fixed_smem(int N, int variant, bool g = false) {
    return emdb::sift_fixed_smem(N, variant, g);
  }
  static cudaError_t occupancy(int arena, int variant, int* per_sm, bool g = false) {
    return emdb::sift_occupancy(arena, variant, per_sm, g);
  }
  static cudaError_t launch(const Params& sp, int grid, cudaStream_t st) {
    return emdb::launch_sift(sp, grid, st);
  }
};
template <> struct SiftKernels<float> {
  using Params = emdb::f32::SiftParams;
  static size_t fixed_smem(int N, int variant, bool g = false) {
    return emdb::f32::sift_fixed_smem(N, variant, g);
  }
  static cudaError_t occupancy(int arena, int variant, int* per_sm, bool g = false) {
    return emdb::f32::sift_occupancy(arena, variant, per_sm, g);
  }
  static cudaError_t launch(const Params& sp, int grid, cudaStream_t st) {
    return emdb::f32::launch_sift(sp, grid, st);
  }
};

template <typename R = double>
int auto_arena_for(int smem_optin, int variant, int nbsym, int max_n) {
  const int per_sm = 233472;
  const size_t fixed = SiftKernels<R>::fixed_smem(std::max(max_n, 1), variant);
  auto share = [&](int want) {
    int arena = std::min(per_sm / want - 1024, smem_optin);
    // shared memory is allocated in 128-byte units: a 16-byte-rounded share
    // can round up past the SM's capacity and lose a CTA (e.g. 5 per SM)
    return arena & ~127;
  };
  const size_t knot_room = (size_t)(11 * 2 * (96 + 2 * nbsym + 2)) * sizeof(R);
  for (int want = variant; want >= 1; --want)
    if ((size_t)share(want) >= fixed + knot_room) {
      if (want >= 3) return share(want);
      break;                                   // would drop below 3 CTAs/SM
    }
  for (int want = std::min(variant, 3); want >= 1; --want)
    if ((size_t)share(want) >= fixed + 64) return share(want);
  const size_t need = fixed + 64;
  return need <= (size_t)smem_optin ? (int)((need + 15) & ~size_t(15)) : 0;
}

// The plan's kernel instance for traces up to max_n.  Unless one was set
// (or an arena, which is sized for the 128-thread instance): four 128-thread
// CTAs per SM up to 2048 samples, two 256-thread CTAs per SM up to 4096, one
// 512-thread CTA per SM beyond.  Measured on B200, dense seismic batches,
// 128 / 256 / 512 threads: 16,384 x 2048 68 / 80 / 110 ms; 2,048 x 4096 72.1
// / 46.3 / 51.6 ms; 1,024 x 8192 491.6 / 360.4 / 292.4 ms (three-tone and
// chirp traces of 4096-8192 samples gain 1.6-2.9x on the wide instance).
int effective_variant(const emdb_plan* p, int max_n) {
  if (p->variant != 0) return p->variant;
  if (p->arena_override > 0) return 4;
  return max_n > 4096 ? 1 : max_n > 2048 ? 2 : 4;
}

template <typename R = double>
int auto_arena(const emdb_plan* p, int max_n) {
  return auto_arena_for<R>(p->smem_optin, effective_variant(p, max_n), p->cfg.nbsym, max_n);
}

template <typename R = double>
int arena_for(const emdb_plan* p, int max_n) {
  if (p->arena_override > 0) return p->arena_override;
  return auto_arena<R>(p, max_n);
}

int ensure_slab(emdb_plan* p, size_t bytes) {
  if (bytes <= p->slab_bytes) return EMDB_OK;
  if (p->d_slab) cudaFree(p->d_slab);
  p->d_slab = nullptr;
  p->slab_bytes = 0;
  cudaError_t e = cudaMalloc(&p->d_slab, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "allocating the spill slab");
  p->slab_bytes = bytes;
  return EMDB_OK;
}

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

int check_config(const emdb_config* c) {
  if (!c) return fail(EMDB_ERR_INVALID, "config is NULL");
  if (c->max_extrema < 4 || c->max_extrema > (1 << 20))
    return fail(EMDB_ERR_INVALID, "max_extrema must be in [4, 2^20]");
  if (c->nbsym < 1 || c->nbsym > emdb::kMaxNbsym)
    return fail(EMDB_ERR_INVALID, "nbsym must be in [1, 8]");
  if (c->max_iteration < 1) return fail(EMDB_ERR_INVALID, "max_iteration must be >= 1");
  if (c->max_imfs < 2 || c->max_imfs > emdb::kMaxImfsCap)
    return fail(EMDB_ERR_INVALID, "max_imfs must be in [2, 64]");
  if (c->threads_per_block != emdb::kThreads)
    return fail(EMDB_ERR_UNSUPPORTED,
                "threads_per_block must be 128: the reduction order of the stop tests is defined "
                "over 128 lanes");
  return EMDB_OK;
}

// Host threads that write the zero rows of the host pipeline's IMF output
// (rows past each chunk's copied ones) while the GPU sifts: `count` blocks of
// `len` bytes, `stride` apart, per job.
class ZeroRows {
 public:
  explicit ZeroRows(bool on) {
    if (!on) return;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = (int)std::max(1u, std::min(8u, hw > 2 ? hw / 2 : 1u));
    for (int k = 0; k < nt; ++k) workers_.emplace_back([this] { run(); });
  }
  ~ZeroRows() { finish(); }
  void add(char* base, size_t count, size_t stride, size_t len) {
    if (workers_.empty()) {
      for (size_t t = 0; t < count; ++t) std::memset(base + t * stride, 0, len);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      jobs_.push_back({base, count, stride, len});
    }
    cv_.notify_one();
  }
  void finish() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      closing_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
    workers_.clear();
  }

 private:
  struct Job { char* base; size_t count, stride, len; };
  void run() {
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return closing_ || !jobs_.empty(); });
        if (jobs_.empty()) return;
        j = jobs_.back();
        jobs_.pop_back();
      }
      for (size_t t = 0; t < j.count; ++t) std::memset(j.base + t * j.stride, 0, j.len);
    }
  }
  std::vector<std::thread> workers_;
  std::vector<Job> jobs_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool closing_ = false;
};

// Arena, occupancy and the launch-independent SiftParams fields; *grid = the
// persistent grid for sp.batch traces.
// Longest trace a launch takes: the per-warp extrema prefixes of the scan
// masks are 16-bit, so at most 2^17 samples (< 2^16 extrema of a kind).
constexpr int kMaxTraceLen = 1 << 17;

template <typename R>
int prepare_sift(emdb_plan* p, typename SiftKernels<R>::Params& sp, int max_n, int* grid,
                 int force_variant = 0) {
  using K = SiftKernels<R>;
  if (max_n > kMaxTraceLen)
    return fail(EMDB_ERR_UNSUPPORTED, "trace length " + std::to_string(max_n) +
                " exceeds the longest supported trace (131072 samples)");
  // force_variant: that instance at its automatic arena (the tail's resume launch)
  int variant = force_variant ? force_variant : effective_variant(p, max_n);
  int arena = force_variant ? auto_arena_for<R>(p->smem_optin, force_variant, p->cfg.nbsym, max_n)
                            : arena_for<R>(p, max_n);
  bool gimf = false;
  if ((arena <= 0 || K::fixed_smem(max_n, variant) + 64 > (size_t)arena) &&
      p->arena_override == 0) {
    // Too long for the plan's instance (at its automatic arena; an explicit
    // arena that cannot hold the trace is the caller's error, below): the
    // wide instance at the full arena
    // (the reference keeps whole traces in global memory, kernels.py:869-878,
    // so it has no length limit; neither does this fallback): the proto-IMF in
    // shared memory while it fits, else in the CTA's global slab.
    variant = 1;
    arena = p->smem_optin & ~127;
    gimf = K::fixed_smem(max_n, 1) + 64 > (size_t)arena;
  }
  if (arena <= 0 || K::fixed_smem(max_n, variant, gimf) + 64 > (size_t)arena)
    return fail(EMDB_ERR_UNSUPPORTED, "trace length " + std::to_string(max_n) +
                " does not fit this device's shared memory");
  int per_sm = 0;
  cudaError_t e = K::occupancy(arena, variant, &per_sm, gimf);
  if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
  if (per_sm < 1) return fail(EMDB_ERR_UNSUPPORTED, "kernel cannot be resident with this arena");
  *grid = std::min(sp.batch, per_sm * p->num_sms);
  if (p->max_ctas > 0) *grid = std::min(*grid, p->max_ctas);
  sp.variant = variant;
  sp.status = p->d_ctl + 1;
  sp.counters = p->d_cnt;
  sp.slab_stride = p->slab_stride;
  sp.park_off = sp.q_off = sp.imf_off = 0;
  if (emdb::variant_threads(variant) > emdb::kThreads) {
    // the wide instance parks the proto-IMF and keeps the stop-test
    // quotients in two trace-length arrays after the knot slab (and, for a
    // trace longer than shared memory holds, the proto-IMF itself after them)
    const size_t trace = al256((size_t)std::max(max_n, 1) * sizeof(R));
    sp.park_off = al256(p->slab_stride);
    sp.q_off = sp.park_off + trace;
    sp.slab_stride = sp.q_off + trace;
    if (gimf) {
      sp.imf_off = sp.slab_stride;
      sp.slab_stride += trace;
    }
  }
  sp.arena_bytes = arena;
  sp.max_extrema = p->cfg.max_extrema;
  sp.nbsym = p->cfg.nbsym;
  sp.max_iteration = p->cfg.max_iteration;
  sp.max_imfs = p->cfg.max_imfs;
  return EMDB_OK;
}

// Device buffers of tail migration for `grid` CTAs and traces up to max_n.
template <typename R>
int ensure_tail(emdb_plan* p, int grid, int max_n, size_t* stride) {
  *stride = al256(emdb::cont_data_off() + (size_t)std::max(max_n, 1) * sizeof(R));
  cudaError_t e = cudaSuccess;
  if (!p->d_tail) e = cudaMalloc(&p->d_tail, 2 * sizeof(int));
  if (e == cudaSuccess && grid > p->cont_valid_cap) {
    if (p->d_cont_valid) cudaFree(p->d_cont_valid);
    p->d_cont_valid = nullptr;
    p->cont_valid_cap = 0;
    e = cudaMalloc(&p->d_cont_valid, (size_t)grid * sizeof(int));
    if (e == cudaSuccess) p->cont_valid_cap = grid;
  }
  const size_t bytes = *stride * (size_t)grid;
  if (e == cudaSuccess && bytes > p->cont_bytes) {
    if (p->d_cont) cudaFree(p->d_cont);
    p->d_cont = nullptr;
    p->cont_bytes = 0;
    e = cudaMalloc(&p->d_cont, bytes);
    if (e == cudaSuccess) p->cont_bytes = bytes;
  }
  if (e != cudaSuccess) return cuda_fail(e, "allocating the tail-migration records");
  return EMDB_OK;
}

template <typename R = double>
int launch_common(emdb_plan* p, typename SiftKernels<R>::Params& sp, int max_n, cudaStream_t st) {
  int grid = 0;
  int rc = prepare_sift<R>(p, sp, max_n, &grid);
  if (rc) return rc;
  // tail migration: the traces still in flight when the queue runs dry move
  // to a second launch of the 512-thread instance (not for launches of that
  // instance already)
  // (the 256-thread instance gains nothing from it: 2,048 x 4096 seismic
  // 46.1 ms without, 47.4-47.9 ms with thresholds of 74-444 traces)
  const bool tail = p->tail != 0 && sp.variant == 4;
  typename SiftKernels<R>::Params rp{};
  int rgrid = 0;
  size_t cont_stride = 0;
  if (tail) {
    rp = sp;
    rc = prepare_sift<R>(p, rp, max_n, &rgrid, 1);
    if (rc) return rc;
    rgrid = std::min(rgrid, grid);
    rc = ensure_tail<R>(p, grid, max_n, &cont_stride);
    if (rc) return rc;
  }
  rc = ensure_slab(p, std::max(sp.slab_stride * (size_t)grid,
                               tail ? rp.slab_stride * (size_t)rgrid : 0));
  if (rc) return rc;
  sp.queue = p->d_ctl;
  sp.slab = p->d_slab;
  cudaError_t e = cudaMemsetAsync(p->d_ctl, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(e, "queue reset");
  if (tail) {
    e = cudaMemsetAsync(p->d_tail, 0, 2 * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->d_cont_valid, 0, (size_t)grid * sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "tail reset");
    sp.active = p->d_tail;
    sp.cont_ticket = p->d_tail + 1;
    // automatic: three traces per SM -- the resume launch runs a trace
    // ~2.5x faster on a whole SM than a 128-thread CTA does, so handing
    // over pays once fewer than that remain (B200, cfg1 shape: 16,384
    // traces 67.1 ms at 1 per SM, 66.7-66.9 at 3, 67.2 at 4; 4,096 traces
    // 22.4 / 21.9 / 21.9 ms)
    sp.yield_below = p->tail < 0 ? 3 * p->num_sms : p->tail;
    sp.cont_buf = p->d_cont;
    sp.cont_stride = cont_stride;
    sp.cont_valid = p->d_cont_valid;
    sp.cont_cap = grid;
    sp.resume = 0;
  }
  e = SiftKernels<R>::launch(sp, grid, st);
  if (e != cudaSuccess) return cuda_fail(e, "sift launch");
  if (tail) {
    rp.queue = p->d_ctl;
    rp.slab = p->d_slab;
    rp.active = nullptr;
    rp.cont_ticket = p->d_tail + 1;
    rp.cont_buf = p->d_cont;
    rp.cont_stride = cont_stride;
    rp.cont_valid = p->d_cont_valid;
    rp.cont_cap = grid;
    rp.resume = 1;
    e = SiftKernels<R>::launch(rp, rgrid, st);
    if (e != cudaSuccess) return cuda_fail(e, "tail launch");
  }
  return EMDB_OK;
}

}  // namespace

extern "C" {

int emdb_version(void) { return 10000; }

int emdb_last_error(char* buf, size_t len) {
  if (buf && len) {
    std::strncpy(buf, g_last_error.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  return EMDB_OK;
}

int emdb_plan_create(const emdb_config* cfg, int device, emdb_plan** out) {
  NvtxRange nvtx_range("emdb_plan_create");
  if (!out) return fail(EMDB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int rc = check_config(cfg);
  if (rc) return rc;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) return fail(EMDB_ERR_INVALID, "device out of range");
  DeviceGuard g(device);
  emdb_plan* p = new emdb_plan();
  p->cfg = *cfg;
  p->device = device;
  cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&p->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  p->slab_stride = emdb::sift_slab_bytes(cfg->max_extrema, cfg->nbsym);
  e = cudaMalloc(&p->d_ctl, 4 * sizeof(int));
  if (e != cudaSuccess) {
    delete p;
    return cuda_fail(e, "allocating plan control words");
  }
  cudaMemset(p->d_ctl, 0, 4 * sizeof(int));
  e = cudaMalloc(&p->d_cnt, kCounters * sizeof(unsigned long long));
  if (e != cudaSuccess) {
    cudaFree(p->d_ctl);
    delete p;
    return cuda_fail(e, "allocating plan counters");
  }
  cudaMemset(p->d_cnt, 0, kCounters * sizeof(unsigned long long));
  *out = p;
  return EMDB_OK;
}

int emdb_plan_destroy(emdb_plan* p) {
  if (!p) return EMDB_OK;
  {
    DeviceGuard g(p->device);
    if (p->d_slab) cudaFree(p->d_slab);
    if (p->d_tail) cudaFree(p->d_tail);
    if (p->d_cont_valid) cudaFree(p->d_cont_valid);
    if (p->d_cont) cudaFree(p->d_cont);
    if (p->d_ctl) cudaFree(p->d_ctl);
    if (p->d_cnt) cudaFree(p->d_cnt);
    if (p->d_stage) cudaFree(p->d_stage);
    if (p->d_chunk_count) cudaFree(p->d_chunk_count);
    if (p->d_chunk_rows) cudaFree(p->d_chunk_rows);
    if (p->h_chunk_flag) cudaFreeHost(p->h_chunk_flag);
    if (p->ev_kernel) cudaEventDestroy(p->ev_kernel);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    for (int g = 0; g < emdb_plan::kGroups; ++g) {
      if (p->group_stream[g]) cudaStreamDestroy(p->group_stream[g]);
      if (p->ev_in[g]) cudaEventDestroy(p->ev_in[g]);
      if (p->ev_group[g]) cudaEventDestroy(p->ev_group[g]);
    }
    if (p->d_group_queue) cudaFree(p->d_group_queue);
    if (p->d_group_slab) cudaFree(p->d_group_slab);
  }
  delete p;
  return EMDB_OK;
}

int emdb_plan_set_arena(emdb_plan* p, int arena_bytes) {
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  if (arena_bytes < 0 || arena_bytes > p->smem_optin)
    return fail(EMDB_ERR_INVALID, "arena exceeds the device's per-block shared memory");
  std::lock_guard<std::mutex> lk(p->mu);
  p->arena_override = arena_bytes & ~15;
  return EMDB_OK;
}

int emdb_plan_set_variant(emdb_plan* p, int min_ctas_per_sm) {
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  if (min_ctas_per_sm != 0 && !emdb::sift_variant_ok(min_ctas_per_sm))
    return fail(EMDB_ERR_INVALID,
                "variant must be 4, 5 or 6 (128-thread CTAs), 2 (256-thread CTAs), 1 "
                "(512-thread wide CTAs) or 0 (by trace length)");
  std::lock_guard<std::mutex> lk(p->mu);
  p->variant = min_ctas_per_sm;
  return EMDB_OK;
}

int emdb_plan_set_tail(emdb_plan* p, int yield_below) {
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  if (yield_below < -1) return fail(EMDB_ERR_INVALID, "yield_below must be >= -1");
  std::lock_guard<std::mutex> lk(p->mu);
  p->tail = yield_below;
  return EMDB_OK;
}

int emdb_plan_set_max_ctas(emdb_plan* p, int max_ctas) {
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  if (max_ctas < 0) return fail(EMDB_ERR_INVALID, "max_ctas must be >= 0");
  std::lock_guard<std::mutex> lk(p->mu);
  p->max_ctas = max_ctas;
  return EMDB_OK;
}

}  // extern "C"

template <typename R>
static int plan_query(emdb_plan* p, int max_n, int* arena_bytes, int* ctas_per_sm,
                      int* grid_max) {
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  DeviceGuard g(p->device);
  int arena = arena_for<R>(p, max_n);
  int per_sm = 0;
  if (arena > 0) {
    cudaError_t e = SiftKernels<R>::occupancy(arena, effective_variant(p, max_n), &per_sm);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
  }
  if (arena_bytes) *arena_bytes = arena;
  if (ctas_per_sm) *ctas_per_sm = per_sm;
  if (grid_max) *grid_max = per_sm * p->num_sms;
  return EMDB_OK;
}

extern "C" {

int emdb_plan_query(emdb_plan* p, int max_n, int* arena_bytes, int* ctas_per_sm, int* grid_max) {
  return plan_query<double>(p, max_n, arena_bytes, ctas_per_sm, grid_max);
}

int emdb_plan_query_f32(emdb_plan* p, int max_n, int* arena_bytes, int* ctas_per_sm,
                        int* grid_max) {
  return plan_query<float>(p, max_n, arena_bytes, ctas_per_sm, grid_max);
}

int emdb_host_bytes(emdb_plan* p, unsigned long long* h2d, unsigned long long* d2h) {
  if (!p || !h2d || !d2h) return fail(EMDB_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(p->mu);
  *h2d = p->host_h2d;
  *d2h = p->host_d2h;
  return EMDB_OK;
}

int emdb_min_arena(int max_n, int* arena_bytes) {
  if (max_n < 0 || !arena_bytes) return fail(EMDB_ERR_INVALID, "bad arguments");
  *arena_bytes = (int)((emdb::sift_fixed_smem(std::max(max_n, 1)) + 64 + 15) & ~size_t(15));
  return EMDB_OK;
}

int emdb_pass_placement(const emdb_config* cfg, int N, int arena_bytes, int n_max, int n_min,
                        int* placement) {
  int rc = check_config(cfg);
  if (rc) return rc;
  if (N < 1 || arena_bytes < 0 || n_max < 0 || n_min < 0 || n_max > cfg->max_extrema ||
      n_min > cfg->max_extrema || !placement)
    return fail(EMDB_ERR_INVALID, "bad arguments");
  const int kc0 = n_max + 2 * cfg->nbsym + 2, kc1 = n_min + 2 * cfg->nbsym + 2;
  *placement = emdb::sift_pass_placement(N, arena_bytes & ~15,
                                         emdb::sift_slab_bytes(cfg->max_extrema, cfg->nbsym),
                                         kc0, kc1);
  return EMDB_OK;
}

}  // extern "C"

namespace {
template <typename R>
int run_dense(emdb_plan* p, const R* signals, const R* T, int batch, int N, R* imfs, int* n_imfs,
              int* overflow, int* dbg_n, int* dbg_extno, int* dbg_nzm, void* stream) {
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  if (batch < 0 || N < 0) return fail(EMDB_ERR_INVALID, "batch and N must be >= 0");
  if (batch == 0) return EMDB_OK;
  if ((N > 0 && (!signals || !imfs)) || !n_imfs || !overflow || !dbg_n || !dbg_extno || !dbg_nzm)
    return fail(EMDB_ERR_INVALID, "NULL buffer");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  typename SiftKernels<R>::Params sp{};
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
  return launch_common<R>(p, sp, N, (cudaStream_t)stream);
}
}  // namespace

extern "C" {

int emdb_run(emdb_plan* p, const double* signals, const double* T, int batch, int N,
             double* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno, int* dbg_nzm,
             void* stream) {
  NvtxRange nvtx_range("emdb_run");
  return run_dense<double>(p, signals, T, batch, N, imfs, n_imfs, overflow, dbg_n, dbg_extno,
                           dbg_nzm, stream);
}

int emdb_run_f32(emdb_plan* p, const float* signals, const float* T, int batch, int N,
                 float* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                 int* dbg_nzm, void* stream) {
  NvtxRange nvtx_range("emdb_run_f32");
  return run_dense<float>(p, signals, T, batch, N, imfs, n_imfs, overflow, dbg_n, dbg_extno,
                          dbg_nzm, stream);
}

int emdb_run_host(emdb_plan* p, const double* signals, const double* T, int batch, int N,
                  double* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                  int* dbg_nzm, void* stream) {
  NvtxRange nvtx_range("emdb_run_host");
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  if (batch < 0 || N < 0) return fail(EMDB_ERR_INVALID, "batch and N must be >= 0");
  if (batch == 0) return EMDB_OK;
  if ((N > 0 && (!signals || !imfs)) || !n_imfs || !overflow || !dbg_n || !dbg_extno || !dbg_nzm)
    return fail(EMDB_ERR_INVALID, "NULL buffer");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int mi = p->cfg.max_imfs;
  const size_t B = (size_t)batch, n = (size_t)N;
  // staging layout: signals | T | imfs | n_imfs | overflow | dbg x3, 256-byte aligned
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_sig = 0, o_T = al(o_sig + B * n * 8), o_imf = al(o_T + (T ? n * 8 : 0));
  const size_t o_n = al(o_imf + B * mi * n * 8), o_ov = al(o_n + B * 4), o_dbg = al(o_ov + B * 4);
  const size_t dbg_bytes = B * mi * 4, total = o_dbg + 3 * al(dbg_bytes);
  cudaError_t e;
  if (total > p->stage_bytes) {
    if (p->d_stage) cudaFree(p->d_stage);
    p->d_stage = nullptr;
    p->stage_bytes = 0;
    e = cudaMalloc(&p->d_stage, total);
    if (e != cudaSuccess) return cuda_fail(e, "allocating host-pipeline staging");
    p->stage_bytes = total;
  }
  constexpr int kMaxChunks = 256;
  constexpr int kG = emdb_plan::kGroups;
  if (!p->copy_stream) {
    e = cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_kernel, cudaEventDisableTiming);
    for (int k = 0; k < kG && e == cudaSuccess; ++k) {
      e = cudaStreamCreateWithFlags(&p->group_stream[k], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_in[k], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_group[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMalloc(&p->d_group_queue, kG * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_chunk_count, kMaxChunks * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_chunk_rows, kMaxChunks * sizeof(unsigned));
    if (e == cudaSuccess)
      e = cudaHostAlloc(&p->h_chunk_flag, kMaxChunks * sizeof(unsigned), cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&p->d_chunk_flag, p->h_chunk_flag, 0);
    if (e != cudaSuccess) return cuda_fail(e, "setting up the host pipeline");
  }
  // chunks of >= 64 traces, at most kMaxChunks of them; groups are whole
  // chunks (4 groups for large batches, so the first launch starts after a
  // quarter of the input copy)
  const int chunk = std::max(64, (batch + kMaxChunks - 1) / kMaxChunks);
  const int nchunk = (batch + chunk - 1) / chunk;
  const int ngroup = nchunk >= 4 * kG ? kG : 1;
  volatile unsigned* flag = p->h_chunk_flag;
  // the previous call on this plan has returned, so no kernel writes the flags now
  for (int c = 0; c < nchunk; ++c) flag[c] = 0u;

  char* d = p->d_stage;
  double* d_sig = reinterpret_cast<double*>(d + o_sig);
  double* d_T = T ? reinterpret_cast<double*>(d + o_T) : nullptr;
  double* d_imf = reinterpret_cast<double*>(d + o_imf);
  int* d_n = reinterpret_cast<int*>(d + o_n);
  int* d_ov = reinterpret_cast<int*>(d + o_ov);
  int* d_dn = reinterpret_cast<int*>(d + o_dbg);
  int* d_de = reinterpret_cast<int*>(d + o_dbg + al(dbg_bytes));
  int* d_dz = reinterpret_cast<int*>(d + o_dbg + 2 * al(dbg_bytes));

  // launch-independent parameters and the per-group grid
  emdb::SiftParams base{};
  base.offsets = nullptr;
  base.dense_n = N;
  base.T = d_T;
  base.t_mode = T ? emdb::kTShared : emdb::kTArange;
  base.order = nullptr;
  base.chunk_flag = p->d_chunk_flag;
  base.chunk_traces = chunk;
  int gchunks[kG], gstart[kG], gcount[kG], grid[kG];
  for (int k = 0, c = 0; k < ngroup; ++k) {
    gchunks[k] = nchunk / ngroup + (k < nchunk % ngroup ? 1 : 0);
    gstart[k] = c * chunk;
    gcount[k] = std::min(batch, (c + gchunks[k]) * chunk) - gstart[k];
    c += gchunks[k];
    emdb::SiftParams sp = base;
    sp.batch = gcount[k];
    int rc = prepare_sift<double>(p, sp, N, &grid[k]);
    if (rc) return rc;
    if (k == 0) base = sp;                     // arena and config fields are shared
  }
  size_t slab_need = 0;
  for (int k = 0; k < ngroup; ++k) slab_need += (size_t)grid[k] * base.slab_stride;
  if (slab_need > p->group_slab_bytes) {
    if (p->d_group_slab) cudaFree(p->d_group_slab);
    p->d_group_slab = nullptr;
    p->group_slab_bytes = 0;
    e = cudaMalloc(&p->d_group_slab, slab_need);
    if (e != cudaSuccess) return cuda_fail(e, "allocating host-pipeline spill slabs");
    p->group_slab_bytes = slab_need;
  }

  // inputs group by group on the caller's stream; each group launches on its
  // own stream once its traces are in
  e = cudaMemsetAsync(p->d_chunk_count, 0, nchunk * sizeof(unsigned), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(p->d_chunk_rows, 0, nchunk * sizeof(unsigned), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(p->d_group_queue, 0, kG * sizeof(int), st);
  if (e == cudaSuccess && T) e = cudaMemcpyAsync(d_T, T, n * 8, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "host-pipeline set-up");
  unsigned long long h2d = (unsigned long long)(B * n * 8 + (T ? n * 8 : 0)), d2h = 0;
  // on a failure after the first launch, let what was issued finish before
  // returning: the staging and slabs are reused by the next call
  auto drain = [&](cudaError_t err, const char* what) {
    for (int k = 0; k < ngroup; ++k) cudaStreamSynchronize(p->group_stream[k]);
    cudaStreamSynchronize(st);
    return cuda_fail(err, what);
  };
  size_t slab_off = 0;
  for (int k = 0; k < ngroup; ++k) {
    const size_t t0 = (size_t)gstart[k], cnt = (size_t)gcount[k];
    if (N > 0)
      e = cudaMemcpyAsync(d_sig + t0 * n, signals + t0 * n, cnt * n * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_in[k], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->group_stream[k], p->ev_in[k], 0);
    if (e != cudaSuccess) return drain(e, "host-pipeline input copy");
    emdb::SiftParams sp = base;
    sp.values = d_sig + t0 * n;
    sp.batch = (int)cnt;
    sp.imfs = d_imf + t0 * (size_t)mi * n;
    sp.n_imfs = d_n + t0;
    sp.overflow = d_ov + t0;
    sp.dbg_n = d_dn + t0 * mi;
    sp.dbg_ext = d_de + t0 * mi;
    sp.dbg_nzm = d_dz + t0 * mi;
    sp.queue = p->d_group_queue + k;
    sp.slab = p->d_group_slab + slab_off;
    sp.chunk_span = (int)cnt;
    sp.chunk_count = p->d_chunk_count + gstart[k] / chunk;
    sp.chunk_rows = p->d_chunk_rows + gstart[k] / chunk;
    sp.chunk_flag = p->d_chunk_flag + gstart[k] / chunk;
    slab_off += (size_t)grid[k] * base.slab_stride;
    e = emdb::launch_sift(sp, grid[k], p->group_stream[k]);
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_group[k], p->group_stream[k]);
    if (e != cudaSuccess) return drain(e, "sift launch");
  }
  // only now does the caller's stream wait for the kernels: waiting inside the
  // loop would hold the next group's input copy behind this group's kernel
  for (int k = 0; k < ngroup && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(st, p->ev_group[k], 0);
  if (e == cudaSuccess) e = cudaEventRecord(p->ev_kernel, st);     // after every group's kernel
  if (e != cudaSuccess) return drain(e, "host-pipeline event");

  NvtxRange nvtx_copyback("emdb_run_host copy-back");
  // Copy each chunk back as soon as its flag is up: only its first `rows`
  // rows per trace (the flag holds 1 + the largest count of rows that may
  // hold data); host threads write the zero rows after them meanwhile.  Once
  // the kernels have finished every remaining chunk is copied in full, so
  // this loop ends with them whatever the flags say.
  const size_t trace_bytes = (size_t)mi * n * 8, row_bytes = n * 8;
  std::string err;
  std::vector<char> done(nchunk, 0);
  ZeroRows zero(imfs != nullptr && trace_bytes > 0);
  int left = nchunk;
  bool kernel_done = false;
  while (left > 0) {
    bool moved = false;
    for (int c = 0; c < nchunk; ++c) {
      if (done[c]) continue;
      const unsigned f = flag[c];
      if (!(kernel_done || f != 0u)) continue;
      const size_t t0 = (size_t)c * chunk, cnt = std::min((size_t)chunk, B - t0);
      const size_t rows = f != 0u ? std::min((size_t)(f - 1u), (size_t)mi) : (size_t)mi;
      char* dst = reinterpret_cast<char*>(imfs) + t0 * trace_bytes;
      const char* src = reinterpret_cast<const char*>(d_imf) + t0 * trace_bytes;
      if (trace_bytes > 0 && rows > 0) {
        d2h += (unsigned long long)(cnt * rows * row_bytes);
        e = rows == (size_t)mi
                ? cudaMemcpyAsync(dst, src, cnt * trace_bytes, cudaMemcpyDeviceToHost, p->copy_stream)
                : cudaMemcpy2DAsync(dst, trace_bytes, src, trace_bytes, rows * row_bytes, cnt,
                                    cudaMemcpyDeviceToHost, p->copy_stream);
        if (e != cudaSuccess && err.empty()) err = "IMF copy-back";
      }
      if (trace_bytes > 0 && rows < (size_t)mi)
        zero.add(dst + rows * row_bytes, cnt, trace_bytes, ((size_t)mi - rows) * row_bytes);
      done[c] = 1;
      --left;
      moved = true;
    }
    if (left == 0) break;
    if (!kernel_done) {
      e = cudaEventQuery(p->ev_kernel);
      if (e == cudaSuccess) {
        kernel_done = true;
        continue;
      }
      if (e != cudaErrorNotReady) {
        cudaStreamSynchronize(p->copy_stream);
        return drain(e, "sift kernel");
      }
    }
    if (!moved) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  // per-trace counts and debug rows after every kernel
  e = cudaStreamWaitEvent(p->copy_stream, p->ev_kernel, 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(n_imfs, d_n, B * 4, cudaMemcpyDeviceToHost, p->copy_stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(overflow, d_ov, B * 4, cudaMemcpyDeviceToHost, p->copy_stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dbg_n, d_dn, dbg_bytes, cudaMemcpyDeviceToHost, p->copy_stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dbg_extno, d_de, dbg_bytes, cudaMemcpyDeviceToHost, p->copy_stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dbg_nzm, d_dz, dbg_bytes, cudaMemcpyDeviceToHost, p->copy_stream);
  cudaError_t e2 = cudaStreamSynchronize(p->copy_stream);
  zero.finish();
  p->host_h2d = h2d;
  p->host_d2h = d2h + (unsigned long long)(2 * B * 4 + 3 * dbg_bytes);
  if (e != cudaSuccess) return cuda_fail(e, "host-pipeline result copy");
  if (e2 != cudaSuccess) return cuda_fail(e2, "host-pipeline copy stream");
  if (!err.empty()) return fail(EMDB_ERR_CUDA, err);
  return EMDB_OK;
}

}  // extern "C"

template <typename R>
static int run_ragged_impl(emdb_plan* p, const R* values, const int64_t* offsets, int batch,
                           int max_n, const R* T, int t_per_trace, const int* order,
                           R* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                           int* dbg_nzm, emdb_notify* nt, int n_traces, void* stream) {
  NvtxRange nvtx_range(sizeof(R) == 4 ? "emdb_run_ragged_f32" : "emdb_run_ragged");
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  if (batch < 0 || max_n < 0) return fail(EMDB_ERR_INVALID, "batch and max_n must be >= 0");
  if (batch == 0) return EMDB_OK;
  if (!values || !offsets || !imfs || !n_imfs || !overflow || !dbg_n || !dbg_extno || !dbg_nzm)
    return fail(EMDB_ERR_INVALID, "NULL buffer");
  if (nt && (n_traces < batch || n_traces > nt->capacity || nt->device != p->device))
    return fail(EMDB_ERR_INVALID, "notify object too small or on another device");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  typename SiftKernels<R>::Params sp{};
  sp.values = values;
  sp.offsets = offsets;
  sp.dense_n = 0;
  sp.T = T;
  sp.t_mode = T ? (t_per_trace ? emdb::kTPerTrace : emdb::kTShared) : emdb::kTArange;
  sp.batch = batch;
  sp.order = order;
  sp.imfs = imfs;
  sp.n_imfs = n_imfs;
  sp.overflow = overflow;
  sp.dbg_n = dbg_n;
  sp.dbg_ext = dbg_extno;
  sp.dbg_nzm = dbg_nzm;
  if (nt) {
    sp.chunk_count = nt->d_count;
    sp.chunk_rows = nt->d_rows;
    sp.chunk_flag = nt->d_flag;
    sp.chunk_traces = 1;
    sp.chunk_span = n_traces;
  }
  return launch_common<R>(p, sp, max_n, (cudaStream_t)stream);
}

extern "C" {

int emdb_run_ragged(emdb_plan* p, const double* values, const int64_t* offsets, int batch,
                    int max_n, const double* T, int t_per_trace, const int* order, double* imfs,
                    int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno, int* dbg_nzm,
                    void* stream) {
  return run_ragged_impl<double>(p, values, offsets, batch, max_n, T, t_per_trace, order, imfs,
                                 n_imfs, overflow, dbg_n, dbg_extno, dbg_nzm, nullptr, 0, stream);
}

int emdb_run_ragged_f32(emdb_plan* p, const float* values, const int64_t* offsets, int batch,
                        int max_n, const float* T, int t_per_trace, const int* order, float* imfs,
                        int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno, int* dbg_nzm,
                        void* stream) {
  return run_ragged_impl<float>(p, values, offsets, batch, max_n, T, t_per_trace, order, imfs,
                                n_imfs, overflow, dbg_n, dbg_extno, dbg_nzm, nullptr, 0, stream);
}

int emdb_run_ragged_notify(emdb_plan* p, const double* values, const int64_t* offsets, int batch,
                           int max_n, const double* T, int t_per_trace, const int* order,
                           double* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                           int* dbg_nzm, emdb_notify* notify, int n_traces, void* stream) {
  if (!notify) return fail(EMDB_ERR_INVALID, "notify is NULL");
  return run_ragged_impl<double>(p, values, offsets, batch, max_n, T, t_per_trace, order, imfs,
                                 n_imfs, overflow, dbg_n, dbg_extno, dbg_nzm, notify, n_traces,
                                 stream);
}

int emdb_notify_create(int capacity, int device, emdb_notify** out, unsigned** host_flags) {
  if (!out || !host_flags || capacity < 1) return fail(EMDB_ERR_INVALID, "bad arguments");
  *out = nullptr;
  *host_flags = nullptr;
  DeviceGuard g(device);
  emdb_notify* nt = new emdb_notify();
  nt->device = device;
  nt->capacity = capacity;
  cudaError_t e = cudaMalloc(&nt->d_count, capacity * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc(&nt->d_rows, capacity * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaHostAlloc(&nt->h_flag, capacity * sizeof(unsigned), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer(&nt->d_flag, nt->h_flag, 0);
  if (e == cudaSuccess) e = cudaMemset(nt->d_count, 0, capacity * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(nt->d_rows, 0, capacity * sizeof(unsigned));
  if (e != cudaSuccess) {
    emdb_notify_destroy(nt);
    return cuda_fail(e, "allocating completion flags");
  }
  std::memset(nt->h_flag, 0, capacity * sizeof(unsigned));
  *out = nt;
  *host_flags = nt->h_flag;
  return EMDB_OK;
}

int emdb_notify_reset(emdb_notify* nt, int n, void* stream) {
  if (!nt || n < 0 || n > nt->capacity) return fail(EMDB_ERR_INVALID, "bad arguments");
  DeviceGuard g(nt->device);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(nt->d_count, 0, n * sizeof(unsigned), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(nt->d_rows, 0, n * sizeof(unsigned), st);
  if (e != cudaSuccess) return cuda_fail(e, "resetting completion counters");
  // no launch that writes these flags is in flight (the caller's contract)
  volatile unsigned* f = nt->h_flag;
  for (int k = 0; k < n; ++k) f[k] = 0u;
  return EMDB_OK;
}

int emdb_notify_destroy(emdb_notify* nt) {
  if (!nt) return EMDB_OK;
  {
    DeviceGuard g(nt->device);
    if (nt->d_count) cudaFree(nt->d_count);
    if (nt->d_rows) cudaFree(nt->d_rows);
    if (nt->h_flag) cudaFreeHost(nt->h_flag);
  }
  delete nt;
  return EMDB_OK;
}

}  // extern "C"

namespace {
template <typename R> struct EnvKernels;
template <> struct EnvKernels<double> {
  using Params = emdb::EnvParams;
  static size_t fixed_smem(int N) { return emdb::sift_fixed_smem(N); }
  static cudaError_t occupancy(int arena, int* per_sm) {
    return emdb::envelope_occupancy(arena, per_sm);
  }
  static cudaError_t launch(const Params& ep, int grid, cudaStream_t st) {
    return emdb::launch_envelope(ep, grid, st);
  }
};
template <> struct EnvKernels<float> {
  using Params = emdb::f32::EnvParams;
  static size_t fixed_smem(int N) { return emdb::f32::sift_fixed_smem(N); }
  static cudaError_t occupancy(int arena, int* per_sm) {
    return emdb::f32::envelope_occupancy(arena, per_sm);
  }
  static cudaError_t launch(const Params& ep, int grid, cudaStream_t st) {
    return emdb::f32::launch_envelope(ep, grid, st);
  }
};

template <typename R>
int run_envelope(emdb_plan* p, const R* signals, const R* T, int batch, int N, R* max_env,
                 R* min_env, int* n_extrema, int* degenerate, R* max_kpos, R* max_kval,
                 R* min_kpos, R* min_kval, int* n_mirrored, void* stream) {
  using K = EnvKernels<R>;
  if (!p) return fail(EMDB_ERR_INVALID, "plan is NULL");
  if (batch < 0 || N < 0) return fail(EMDB_ERR_INVALID, "batch and N must be >= 0");
  if (batch == 0) return EMDB_OK;
  if (!signals || !max_env || !min_env || !n_extrema || !degenerate || !max_kpos || !max_kval ||
      !min_kpos || !min_kval || !n_mirrored)
    return fail(EMDB_ERR_INVALID, "NULL buffer");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  // the envelope kernel has 128-thread CTAs: the arena rule of that instance
  // unless the plan names another
  int arena = p->arena_override > 0 ? p->arena_override
                                    : auto_arena_for<R>(p->smem_optin,
                                                        p->variant ? p->variant : 4,
                                                        p->cfg.nbsym, N);
  if (arena <= 0 || K::fixed_smem(N) + 64 > (size_t)arena)
    return fail(EMDB_ERR_UNSUPPORTED, "trace length does not fit this device's shared memory");
  int per_sm = 0;
  cudaError_t e = K::occupancy(arena, &per_sm);
  if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
  if (per_sm < 1) return fail(EMDB_ERR_UNSUPPORTED, "kernel cannot be resident with this arena");
  int grid = std::min(batch, per_sm * p->num_sms);
  int rc = ensure_slab(p, p->slab_stride * (size_t)grid);
  if (rc) return rc;
  typename K::Params ep{};
  ep.values = signals;
  ep.offsets = nullptr;
  ep.dense_n = N;
  ep.T = T;
  ep.t_mode = T ? emdb::kTShared : emdb::kTArange;
  ep.batch = batch;
  ep.max_env = max_env;
  ep.min_env = min_env;
  ep.n_extrema = n_extrema;
  ep.degenerate = degenerate;
  ep.max_kpos = max_kpos;
  ep.max_kval = max_kval;
  ep.min_kpos = min_kpos;
  ep.min_kval = min_kval;
  ep.n_mirrored = n_mirrored;
  ep.mbuf = p->cfg.max_extrema + 2 * p->cfg.nbsym;
  ep.queue = p->d_ctl + 2;
  ep.status = p->d_ctl + 1;
  ep.slab = p->d_slab;
  ep.slab_stride = p->slab_stride;
  ep.arena_bytes = arena;
  ep.max_extrema = p->cfg.max_extrema;
  ep.nbsym = p->cfg.nbsym;
  e = cudaMemsetAsync(p->d_ctl + 2, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(e, "queue reset");
  e = K::launch(ep, grid, st);
  if (e != cudaSuccess) return cuda_fail(e, "envelope launch");
  return EMDB_OK;
}
}  // namespace

extern "C" {

int emdb_envelope(emdb_plan* p, const double* signals, const double* T, int batch, int N,
                  double* max_env, double* min_env, int* n_extrema, int* degenerate,
                  double* max_kpos, double* max_kval, double* min_kpos, double* min_kval,
                  int* n_mirrored, void* stream) {
  NvtxRange nvtx_range("emdb_envelope");
  return run_envelope<double>(p, signals, T, batch, N, max_env, min_env, n_extrema, degenerate,
                              max_kpos, max_kval, min_kpos, min_kval, n_mirrored, stream);
}

int emdb_envelope_f32(emdb_plan* p, const float* signals, const float* T, int batch, int N,
                      float* max_env, float* min_env, int* n_extrema, int* degenerate,
                      float* max_kpos, float* max_kval, float* min_kpos, float* min_kval,
                      int* n_mirrored, void* stream) {
  NvtxRange nvtx_range("emdb_envelope_f32");
  return run_envelope<float>(p, signals, T, batch, N, max_env, min_env, n_extrema, degenerate,
                             max_kpos, max_kval, min_kpos, min_kval, n_mirrored, stream);
}

int emdb_plan_counters(emdb_plan* p, unsigned long long* passes, unsigned long long* spilled,
                       int reset) {
  if (!p || !passes || !spilled) return fail(EMDB_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  unsigned long long h[2] = {0, 0};
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(h, p->d_cnt, sizeof(h), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && reset) e = cudaMemset(p->d_cnt, 0, sizeof(h));
  if (e != cudaSuccess) return cuda_fail(e, "counter read-back");
  *passes = h[0];
  *spilled = h[1];
  return EMDB_OK;
}

int emdb_plan_phase_clocks(emdb_plan* p, unsigned long long* cycles, int n, int reset) {
  if (!p || !cycles || n < 0) return fail(EMDB_ERR_INVALID, "bad arguments");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  unsigned long long h[kCounters - 2] = {};
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(h, p->d_cnt + 2, sizeof(h), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && reset) e = cudaMemset(p->d_cnt + 2, 0, sizeof(h));
  if (e != cudaSuccess) return cuda_fail(e, "phase clock read-back");
  for (int k = 0; k < n; ++k) cycles[k] = k < kCounters - 2 ? h[k] : 0ull;
  return EMDB_OK;
}

// Hooks for the other translation units (emdb_noalloc.cu, emdb_pack.cu), not
// exported: error reporting, the planned path's config check, its arena rule.
__attribute__((visibility("hidden"))) int emdb_noalloc_fail(int code, const char* msg) {
  return fail(code, msg);
}
__attribute__((visibility("hidden"))) int emdb_internal_fail(int code, const char* msg) {
  return fail(code, msg);
}
__attribute__((visibility("hidden"))) int emdb_noalloc_check_config(const emdb_config* c) {
  return check_config(c);
}
__attribute__((visibility("hidden"))) int emdb_noalloc_auto_arena(int smem_optin, int nbsym,
                                                                  int max_n) {
  return auto_arena_for(smem_optin, 4, nbsym, max_n);
}

int emdb_check_division(int mode, long long n, unsigned long long seed,
                        unsigned long long* mismatches) {
  if (!mismatches || mode < 0 || mode > 4 || n < 0)
    return fail(EMDB_ERR_INVALID, "bad self-test arguments");
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 3 * sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_fail(e, "self-test counter");
  e = cudaMemset(d, 0, 3 * sizeof(unsigned long long));
  if (e == cudaSuccess)
    e = mode >= 3 ? emdb::f32::launch_div_check(mode - 3, n, seed, d, 0)
                  : emdb::launch_div_check(mode, n, seed, d, 0);
  if (e == cudaSuccess)
    e = cudaMemcpy(mismatches, d, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "division self-test");
  return EMDB_OK;
}

int emdb_host_register(void* ptr, size_t bytes, int read_only) {
  if (!ptr || bytes == 0) return fail(EMDB_ERR_INVALID, "empty host range");
  unsigned flags = cudaHostRegisterPortable | (read_only ? cudaHostRegisterReadOnly : 0u);
  cudaError_t e = cudaHostRegister(ptr, bytes, flags);
  if (e != cudaSuccess) return cuda_fail(e, "page-locking the host range");
  return EMDB_OK;
}

int emdb_host_unregister(void* ptr) {
  if (!ptr) return fail(EMDB_ERR_INVALID, "NULL pointer");
  cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) return cuda_fail(e, "releasing the host range");
  return EMDB_OK;
}

int emdb_status(emdb_plan* p, int* status, void* stream) {
  if (!p || !status) return fail(EMDB_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, p->d_ctl + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(p->d_ctl + 1, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "status read-back");
  *status = v;
  return EMDB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Cost-model entry points (kernels in emd_sched.cu).
// ---------------------------------------------------------------------------
#include "emdb_sched.cuh"

extern "C" {

int emdb_features(const double* values, const int64_t* offsets, int batch, int N, float* feat,
                  void* stream) {
  if (batch < 0 || N < 0) return fail(EMDB_ERR_INVALID, "batch and N must be >= 0");
  if (batch == 0) return EMDB_OK;
  if (!values || !feat) return fail(EMDB_ERR_INVALID, "NULL buffer");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  emdb::FeatParams p{values, offsets, N, batch, feat};
  cudaError_t e = emdb::launch_features(p, std::min(batch, sms * 8), (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "features launch");
  return EMDB_OK;
}

int emdb_mlp_num_params(void) { return emdb::kNParams; }

int emdb_mlp_forward(const float* params, const float* X, const float* mu, const float* sd, int B,
                     float* Z1, float* H1, float* Z2, float* H2, float* Y, void* stream) {
  if (B < 0) return fail(EMDB_ERR_INVALID, "B must be >= 0");
  if (B == 0) return EMDB_OK;
  if (!params || !X || !mu || !sd || !Z1 || !H1 || !Z2 || !H2 || !Y)
    return fail(EMDB_ERR_INVALID, "NULL buffer");
  emdb::MlpFwdParams p{params, X, mu, sd, B, Z1, H1, Z2, H2, Y};
  cudaError_t e = emdb::launch_mlp_forward(p, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "mlp forward launch");
  return EMDB_OK;
}

int emdb_mlp_backward(const float* params, const float* X, const float* mu, const float* sd,
                      const float* Z1, const float* H1, const float* Z2, const float* H2,
                      const float* Y, const float* T, int B, float* dY, float* dZ2, float* dZ1,
                      float* grads, float* loss, void* stream) {
  if (B <= 0) return fail(EMDB_ERR_INVALID, "B must be > 0");
  if (!params || !X || !mu || !sd || !Z1 || !H1 || !Z2 || !H2 || !Y || !T || !dY || !dZ2 || !dZ1 ||
      !grads || !loss)
    return fail(EMDB_ERR_INVALID, "NULL buffer");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(float), st);
  if (e != cudaSuccess) return cuda_fail(e, "loss reset");
  emdb::MlpBwdParams p{params, X, mu, sd, Z1, H1, Z2, H2, Y, T, B, dY, dZ2, dZ1, loss};
  e = emdb::launch_mlp_backward(p, grads, st);
  if (e != cudaSuccess) return cuda_fail(e, "mlp backward launch");
  return EMDB_OK;
}

int emdb_mlp_adam(float* params, const float* grads, float* m, float* v, int n, float lr,
                  float beta1, float beta2, float eps, int step, uint16_t* params_bf16,
                  void* stream) {
  if (n <= 0 || step < 1) return fail(EMDB_ERR_INVALID, "n must be > 0 and step >= 1");
  if (!params || !grads || !m || !v) return fail(EMDB_ERR_INVALID, "NULL buffer");
  cudaError_t e = emdb::launch_adam(params, grads, m, v, n, lr, beta1, beta2, eps, step,
                                    reinterpret_cast<__nv_bfloat16*>(params_bf16),
                                    (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "adam launch");
  return EMDB_OK;
}

int emdb_mlp_infer_bf16(const uint16_t* params_bf16, const float* X, const float* mu,
                        const float* sd, int B, float* Y, void* stream) {
  if (B < 0) return fail(EMDB_ERR_INVALID, "B must be >= 0");
  if (B == 0) return EMDB_OK;
  if (!params_bf16 || !X || !mu || !sd || !Y) return fail(EMDB_ERR_INVALID, "NULL buffer");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  emdb::MlpInferParams p{reinterpret_cast<const __nv_bfloat16*>(params_bf16), X, mu, sd, B, Y};
  int tiles = (B + 31) / 32;
  cudaError_t e = emdb::launch_mlp_infer(p, std::min(tiles, sms * 2), (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "mlp inference launch");
  return EMDB_OK;
}

}  // extern "C"
