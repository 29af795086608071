// Internal declarations shared by the sift kernels and the C-ABI host code.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace emdb {

constexpr int kThreads = 128;   // one CTA = 128 threads = the reference's 128 reduction lanes
constexpr int kWarps = kThreads / 32;
// the wide instance: one long trace per SM, 16 warps; its reductions keep the
// 128 lanes above
constexpr int kWideThreads = 512;
// half-wide: two 256-thread CTAs per SM, each on one trace
constexpr int kHalfWideThreads = 256;
constexpr int kMaxNbsym = 8;
constexpr int kMaxImfsCap = 64;

// Status bits a kernel may raise (device-side error word, never a trap).
enum : int {
  kStatusStaleEnvelope = 1,   // a sample fell outside the knot span (needs non-monotone T)
  kStatusTooLong = 2,         // a trace does not fit the launch's shared-memory arena
};

// Time axis modes.
enum : int { kTArange = 0, kTShared = 1, kTPerTrace = 2 };

// R: the type the sift computes in -- double (the reference's REAL_T), or
// float for the FP32 build of the same kernel source (namespace emdb::f32).
template <typename R>
struct SiftParamsT {
  // input: CSR traces (dense [B,N] is offsets b*N)
  const R* values;
  const int64_t* offsets;     // [batch+1], or NULL for a dense [batch, dense_n] batch
  int dense_n;
  const R* T;                 // per t_mode
  int t_mode;
  int batch;
  const int* order;           // queue order (NULL = FIFO)
  // outputs: trace b's rows start at imfs + max_imfs*offsets[b], row r at +r*N_b
  R* imfs;
  int* n_imfs;
  int* overflow;
  int* dbg_n;
  int* dbg_ext;
  int* dbg_nzm;
  // scratch
  int* queue;                 // work-queue ticket counter (zeroed before launch)
  int* status;                // error word (OR of kStatus*)
  unsigned long long* counters;  // [0] sift passes, [1] passes on the global slab (may be NULL)
  char* slab;                 // per-CTA global spill area
  size_t slab_stride;         // bytes per CTA
  size_t park_off;            // wide instance: parked proto-IMF at slab + park_off (bytes)
  size_t q_off;               // wide instance: stop-test quotients at slab + q_off
  size_t imf_off;             // wide instance, traces longer than shared memory holds: the
                              // proto-IMF at slab + imf_off (0 = in shared memory)
  int arena_bytes;            // dynamic shared memory per CTA
  // chunk completion for copying finished traces back early (NULL = off):
  // traces [c*chunk_traces, (c+1)*chunk_traces) form chunk c
  unsigned* chunk_count;      // device counters, zeroed before launch
  unsigned* chunk_rows;       // device: the chunk's largest n_imfs, zeroed before launch
  unsigned* chunk_flag;       // mapped host flags: 1 + rows to copy once chunk c is complete
  int chunk_traces;
  int chunk_span;             // traces the chunk indices cover (the last chunk may be short)
  // config (EMDKernelConfig fields)
  int max_extrema;
  int nbsym;
  int max_iteration;
  int max_imfs;
  int variant;                // 4, 5, 6: 128-thread CTAs, register budget for that many per
                              // SM; 1: the 512-thread wide instance, one CTA per SM;
                              // 2: 256-thread CTAs, two per SM
  // Tail migration (cont_buf NULL = off).  Once every trace of the launch
  // has started and at most yield_below are still in flight, each of them
  // stops at its next sift-pass boundary and leaves a continuation record
  // (its proto-IMF and loop state) in the record of its CTA; a second launch
  // of the 512-thread instance with resume = 1 finishes them, one per SM.
  int* active;                // traces in flight in this launch (zeroed before it)
  int yield_below;
  char* cont_buf;             // cont_cap records of cont_stride bytes, one per CTA
  size_t cont_stride;
  int* cont_valid;            // [cont_cap]: 1 = record holds a trace (zeroed before it)
  int cont_cap;
  int* cont_ticket;           // the resume launch's ticket counter (zeroed before it)
  int resume;
};

// Header of a continuation record; the proto-IMF follows at cont_data_off().
struct ContHead {
  int b;                      // trace index
  int n;                      // sift passes done on the current IMF
  int imf_count;
  int extNo_last;
  int ovf;
  int stale;
  int dbg[3][kMaxImfsCap];    // debug_n / debug_extno / debug_nzm so far
};
__host__ __device__ constexpr size_t cont_data_off() {
  return (sizeof(ContHead) + 255) & ~size_t(255);
}

template <typename R>
struct EnvParamsT {
  const R* values;
  const int64_t* offsets;     // NULL = dense [batch, dense_n]
  int dense_n;
  const R* T;
  int t_mode;
  int batch;
  R* max_env;                 // CSR like values
  R* min_env;
  int* n_extrema;             // [batch,2]
  int* degenerate;            // [batch]
  R* max_kpos;                // [batch, mbuf]
  R* max_kval;
  R* min_kpos;
  R* min_kval;
  int* n_mirrored;            // [batch,2]
  int mbuf;
  int* queue;
  int* status;
  char* slab;
  size_t slab_stride;
  int arena_bytes;
  int max_extrema;
  int nbsym;
};

using SiftParams = SiftParamsT<double>;
using EnvParams = EnvParamsT<double>;

// Shared-memory bytes a CTA of the given variant needs beyond the knot arena
// for a trace of length N (imf_global: the wide instance with the proto-IMF in
// the global slab).
size_t sift_fixed_smem(int N, int variant = 4, bool imf_global = false);
// Threads per CTA of a kernel variant.
int variant_threads(int variant);
// Worst-case global spill bytes per CTA for a given extrema cap / nbsym.
size_t sift_slab_bytes(int max_extrema, int nbsym);
// Knot placement a sift pass takes for a trace of N samples in a CTA arena of
// arena_total bytes with kc0 / kc1 knot slots per envelope (-1: the trace does
// not fit the arena).  Values: 0 shared, 1 split, 2 slab, 3 borrow, 4 park,
// 5 compact borrow.
int sift_pass_placement(int N, int arena_total, size_t slab_stride, int kc0, int kc1);

cudaError_t launch_sift(const SiftParams& p, int grid, cudaStream_t stream);
cudaError_t launch_envelope(const EnvParams& p, int grid, cudaStream_t stream);
bool sift_variant_ok(int variant);
cudaError_t sift_occupancy(int arena_bytes, int variant, int* ctas_per_sm,
                           bool imf_global = false);
cudaError_t envelope_occupancy(int arena_bytes, int* ctas_per_sm);
cudaError_t launch_div_check(int mode, long long n, unsigned long long seed,
                             unsigned long long* mismatches, cudaStream_t stream);

// The FP32 build of the sift and envelope kernels (emd_sift.cu compiled with
// EMDB_F32=1): the same algorithm in float, with the reference kernel's mixed
// float / double expressions (its source compiled with REAL_T = float).  Sizes
// count 4-byte values.
namespace f32 {
using SiftParams = SiftParamsT<float>;
using EnvParams = EnvParamsT<float>;
size_t sift_fixed_smem(int N, int variant = 4, bool imf_global = false);
size_t sift_slab_bytes(int max_extrema, int nbsym);
int sift_pass_placement(int N, int arena_total, size_t slab_stride, int kc0, int kc1);
cudaError_t launch_sift(const SiftParams& p, int grid, cudaStream_t stream);
cudaError_t launch_envelope(const EnvParams& p, int grid, cudaStream_t stream);
cudaError_t sift_occupancy(int arena_bytes, int variant, int* ctas_per_sm,
                           bool imf_global = false);
cudaError_t envelope_occupancy(int arena_bytes, int* ctas_per_sm);
cudaError_t launch_div_check(int mode, long long n, unsigned long long seed,
                             unsigned long long* mismatches, cudaStream_t stream);
}  // namespace f32

}  // namespace emdb
