/*
 * emdb200.h -- C ABI of the B200-native batched EMD (libemdb200.so).
 *
 * Plain pointers and sizes only.  Device pointers are CUDA device memory on
 * the plan's device; `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).  Every function returns EMDB_OK (0) or an error
 * code; emdb_last_error() gives the message for the calling thread.  Calls
 * are asynchronous on `stream` unless stated.  One plan owns scratch (work
 * queue ticket, status word, per-CTA spill slab); calls on the same plan are
 * serialised by the plan, calls on distinct plans are independent.
 *
 * Reference interface each entry point replaces (SeismicFlow/emd-cuda):
 *   emdb_plan_create   EMDKernelConfig.build() + EMDBatchLauncher.__init__
 *                      (kernels.py:1277-1286, 1294-1341): config check,
 *                      shared-memory opt-in, occupancy sizing
 *   emdb_run           EMDBatchLauncher.run (kernels.py:1343-1372) launching
 *                      emd_batch_kernel (kernels.py:834-1080)
 *   emdb_run_ragged    no reference counterpart for mixed lengths: the
 *                      reference only takes [batch, N]; this is run() over
 *                      CSR traces with an optional queue order
 *   emdb_envelope      EMDBatchLauncher.run_envelope_only (kernels.py:1374-1407)
 *                      launching envelope_batch_kernel (kernels.py:1100-1166)
 *   emdb_status        the overflow / error read-back GPUBatchEMD.__call__
 *                      does after the launch (emd.py:95-105)
 */
#ifndef EMDB200_H
#define EMDB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMDB_OK 0
#define EMDB_ERR_INVALID 1      /* bad argument (maps to ValueError) */
#define EMDB_ERR_CUDA 2         /* CUDA runtime error (RuntimeError) */
#define EMDB_ERR_NOMEM 3        /* device allocation failed (MemoryError) */
#define EMDB_ERR_UNSUPPORTED 4  /* config does not fit this device (ValueError) */
#define EMDB_ERR_DEVICE 5       /* kernel raised a status bit (RuntimeError) */

/* Device status bits returned by emdb_status. */
#define EMDB_STATUS_STALE_ENVELOPE 1 /* a sample fell outside the knot span */
#define EMDB_STATUS_TOO_LONG 2       /* a trace did not fit the shared-memory arena */

/* Field-for-field the reference's EMDKernelConfig (kernels.py:1170-1176). */
typedef struct emdb_config {
  int max_extrema;       /* per-side extrema cap; >= cap sets overflow (default 1024) */
  int nbsym;             /* mirrored boundary points per side, 1..8 (default 2) */
  int max_iteration;     /* sift cap per IMF; reaching it sets overflow (default 1000) */
  int max_imfs;          /* output rows per trace, 2..64 (default 16) */
  int threads_per_block; /* reference block size; only 128 is accepted (reduction order) */
} emdb_config;

typedef struct emdb_plan emdb_plan;

int emdb_version(void);

/* Create a plan for `device`.  Validates the config, opts the kernels into
 * dynamic shared memory and allocates the plan's scratch. */
int emdb_plan_create(const emdb_config* cfg, int device, emdb_plan** out);
int emdb_plan_destroy(emdb_plan* plan);

/* Shared-memory arena per CTA for the next launches (0 = automatic).  The
 * autotuner sets this; larger arenas spill fewer knots but fit fewer CTAs
 * per SM.  Fails if the arena cannot hold a trace of length max_n. */
int emdb_plan_set_arena(emdb_plan* plan, int arena_bytes);
/* Kernel instance of the sift: 4, 5 or 6 = 128-thread CTAs compiled for at
 * least that many resident per SM (register budget), the automatic arena
 * then targets that many CTAs; 1 = the wide instance, one 512-thread CTA per
 * SM working on one trace (long traces: 16 warps and the knots on-chip);
 * 2 = two 256-thread CTAs per SM; same results bit for bit; 0 (the default)
 * = by trace length: 4 up to 2048 samples, 2 up to 4096, 1 beyond (4 when
 * an arena was set).  The ragged autotuner sets one per tier.  A launch whose traces
 * do not fit the plan's instance runs on the wide instance at the full
 * shared-memory arena, with the proto-IMF in global memory when shared
 * memory cannot hold it, so any trace length runs. */
int emdb_plan_set_variant(emdb_plan* plan, int min_ctas_per_sm);
/* Cap on the persistent grid of the plan's launches (0 = as many CTAs as
 * can be resident).  A capped launch leaves the other SMs to launches that
 * run beside it -- the learned scheduler gives the heavy traces of a tier a
 * wide launch on a share of the SMs this way.  No reference counterpart (its
 * grid is one CTA per signal, kernels.py:1366-1367). */
int emdb_plan_set_max_ctas(emdb_plan* plan, int max_ctas);
/* Tail migration for the plan's dense and ragged launches of the 128-thread
 * instance (4 per SM; no reference counterpart: its launch is one CTA per
 * signal, kernels.py:1366-1367).  Once every trace of a launch has started
 * and at most yield_below of them are still in flight, each stops at its
 * next sift-pass boundary, parks its proto-IMF and loop state in a
 * plan-owned record, and a second launch of the 512-thread instance finishes
 * them, one trace per SM -- the last traces of a batch then run on a whole
 * SM instead of a quarter of one.  Same results bit for bit.  yield_below:
 * -1 = three per SM of the device (the default), 0 = off, > 0 that many.
 * Measured on B200 (dense seismic, 2048 samples): 4,096 traces 25.9 -> 21.9
 * ms, 16,384 traces 68.0 -> 66.7 ms; in FP32, where a few traces sift to
 * the iteration cap, 16,384 traces 114.0 -> 77.0 ms. */
int emdb_plan_set_tail(emdb_plan* plan, int yield_below);
/* Arena and CTAs/SM the plan would use for traces up to max_n. */
int emdb_plan_query(emdb_plan* plan, int max_n, int* arena_bytes, int* ctas_per_sm,
                    int* grid_max);
/* Smallest arena (bytes) that holds a trace of max_n samples: its proto-IMF,
 * control block and scan masks; every knot then lives in the global slab.
 * No reference counterpart (the reference sizes one fixed knot buffer per
 * block, EMDKernelConfig.shared_mem_bytes, kernels.py:1273-1275); the
 * autotuner uses it as the floor of its candidates. */
int emdb_min_arena(int max_n, int* arena_bytes);
/* Where a sift pass keeps its knots and PCR buffers, for a trace of N samples
 * in a CTA arena of arena_bytes (as emdb_plan_set_arena takes it) whose
 * current proto-IMF has n_max maxima and n_min minima (after the max_extrema
 * cap).  *placement: 0 shared memory; 3 borrow (proto-IMF parked in the
 * global per-CTA slab, both PCR buffers on-chip); 5 compact borrow (the same
 * with the moments beside the knots); 1 split (PCR buffer 1 in the slab);
 * 4 park (PCR buffer 1 in the parked proto-IMF's space, knots and buffer 0
 * in the slab); 2 slab; -1 the trace does not fit the arena.  Host-only, no
 * device needed.  No reference counterpart (the reference keeps every knot
 * in one fixed shared buffer, kernels.py:1273-1275). */
int emdb_pass_placement(const emdb_config* cfg, int N, int arena_bytes, int n_max, int n_min,
                        int* placement);

/* Dense batch, the reference's run(): signals [batch, N], T [N] or NULL
 * (= arange(N), already normalised as emd.py:83-88 does), outputs
 * imfs [batch, max_imfs, N], n_imfs [batch], overflow [batch],
 * dbg_n / dbg_extno / dbg_nzm [batch, max_imfs] (-1 = slot not reached).
 * Every output element is written (no pre-zeroing needed). */
int emdb_run(emdb_plan* plan, const double* signals, const double* T, int batch, int N,
             double* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
             int* dbg_nzm, void* stream);

/* emdb_run with every pointer in HOST memory (the reference's GPUBatchEMD
 * called on NumPy input, emd.py:71-107, which copies in, runs and leaves the
 * copy-back to the caller).  Inputs go up on `stream`, one sift launch covers
 * the batch, and the IMF rows of each finished chunk of traces come back on
 * the plan's own copy stream while the rest still sifts; counts and debug
 * rows follow the kernel; of the IMF rows only those that may hold data are
 * copied, the zero rows after them are written by host threads meanwhile.
 * Returns once every output is in host memory.
 * Page-locked host buffers make the copies asynchronous; pageable ones work
 * but serialise them.  Device staging (inputs + outputs) is plan-owned and
 * grows to the largest batch seen. */
int emdb_run_host(emdb_plan* plan, const double* signals, const double* T, int batch, int N,
                  double* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                  int* dbg_nzm, void* stream);
/* Bytes the plan's last emdb_run_host copied host->device and device->host.
 * Of each finished chunk of traces only the rows that may hold data cross
 * the link (the kernel reports the chunk's largest count); the zero rows
 * after them are written on the host.  No reference counterpart. */
int emdb_host_bytes(emdb_plan* plan, unsigned long long* h2d, unsigned long long* d2h);

/* CSR batch of mixed lengths in one launch: trace b is
 * values[offsets[b] .. offsets[b+1]), offsets is a DEVICE int64 [batch+1]
 * array, max_n = max trace length (host value, sizes the arena).
 * T: NULL = arange per trace; else CSR-aligned per-trace time axes
 * (t_per_trace = 1) or one shared axis of length max_n (t_per_trace = 0).
 * order: DEVICE int32 [batch] permutation giving the queue order, or NULL
 * for FIFO; it changes only which CTA runs a trace when, never a result.
 * Outputs: trace b's rows at imfs + max_imfs*offsets[b], row r at +r*N_b. */
int emdb_run_ragged(emdb_plan* plan, const double* values, const int64_t* offsets, int batch,
                    int max_n, const double* T, int t_per_trace, const int* order,
                    double* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                    int* dbg_nzm, void* stream);

/* Per-trace completion flags for ragged launches, so a caller can take each
 * trace's results as soon as that trace is done instead of at the end of the
 * launch (the serving loop delivers each request this way).  No reference
 * counterpart.  create: capacity traces; *host_flags is page-locked host
 * memory the kernel writes: host_flags[b] becomes 1 + the number of rows of
 * trace b that may hold data once all of trace b's outputs are written.
 * reset: zero the first n counters (asynchronously on `stream`) and host
 * flags (immediately) -- only while no launch that uses the object runs. */
typedef struct emdb_notify emdb_notify;
int emdb_notify_create(int capacity, int device, emdb_notify** out, unsigned** host_flags);
int emdb_notify_reset(emdb_notify* notify, int n, void* stream);
int emdb_notify_destroy(emdb_notify* notify);
/* emdb_run_ragged that also raises trace b's completion flag (b is the
 * trace's index in offsets; n_traces = the number of traces offsets holds,
 * <= the notify object's capacity). */
int emdb_run_ragged_notify(emdb_plan* plan, const double* values, const int64_t* offsets,
                           int batch, int max_n, const double* T, int t_per_trace,
                           const int* order, double* imfs, int* n_imfs, int* overflow,
                           int* dbg_n, int* dbg_extno, int* dbg_nzm, emdb_notify* notify,
                           int n_traces, void* stream);

/* Gather the rows of a ragged launch's output that may hold data into one
 * dense buffer for the copy back to the host: rows [0, n_rows[b]) of trace b
 * (imfs + max_imfs*offsets[b], rows of N_b samples) go to packed + row_off[b].
 * All pointers DEVICE memory; n_rows [batch] (clamped to [0, max_imfs]),
 * row_off int64 [batch] element offsets.  Rows past n_imfs[b] + 1 are zero,
 * so n_rows = min(n_imfs + 1, max_imfs) keeps everything.  No reference
 * counterpart (the reference returns dense [batch, MAX_IMFS, N] only). */
int emdb_pack_rows(const double* imfs, const int64_t* offsets, const int* n_rows,
                   const int64_t* row_off, int batch, int max_imfs, double* packed, void* stream);

/* Extrema + mirroring + both envelopes on raw traces, no sift loop
 * (run_envelope_only): max_env/min_env [batch, N], n_extrema [batch, 2],
 * degenerate [batch], knot positions/values [batch, mbuf] each with
 * mbuf = max_extrema + 2*nbsym, n_mirrored [batch, 2].  Knot slots past
 * n_mirrored and envelopes of degenerate traces are written as zero. */
int emdb_envelope(emdb_plan* plan, const double* signals, const double* T, int batch, int N,
                  double* max_env, double* min_env, int* n_extrema, int* degenerate,
                  double* max_kpos, double* max_kval, double* min_kpos, double* min_kval,
                  int* n_mirrored, void* stream);

/* FP32 path: the same entry points computing in float.  The reference's
 * kernel source is written over REAL_T (kernels.py:78), substituted from
 * EMDKernelConfig.real_t_name when it is built (kernels.py:1277-1285); its
 * Python layer fixes that to double.  These run the reference algorithm with
 * REAL_T = float: every array and REAL_T variable is float, and the
 * source's double literals keep their C++ meaning (an expression such as
 * the envelope's "... * (h * h) / 6.0" is evaluated in double and rounded
 * once to float; "sum < 1e-10" compares in double), bit for bit like that
 * source built with REAL_T = float and -fmad=false.  Discrete outcomes
 * (extrema counts, sift counts, IMF counts) can differ from the FP64 path.
 * Arguments as for the FP64 entries, with float buffers; T must stay
 * strictly increasing in float after normalisation. */
int emdb_run_f32(emdb_plan* plan, const float* signals, const float* T, int batch, int N,
                 float* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                 int* dbg_nzm, void* stream);
int emdb_run_ragged_f32(emdb_plan* plan, const float* values, const int64_t* offsets, int batch,
                        int max_n, const float* T, int t_per_trace, const int* order,
                        float* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                        int* dbg_nzm, void* stream);
int emdb_envelope_f32(emdb_plan* plan, const float* signals, const float* T, int batch, int N,
                      float* max_env, float* min_env, int* n_extrema, int* degenerate,
                      float* max_kpos, float* max_kval, float* min_kpos, float* min_kval,
                      int* n_mirrored, void* stream);
/* emdb_plan_query for the FP32 kernels (4-byte values: more knots on-chip,
 * longer traces per CTA). */
int emdb_plan_query_f32(emdb_plan* plan, int max_n, int* arena_bytes, int* ctas_per_sm,
                        int* grid_max);

/* Sift passes the plan's launches have run so far, and how many of them kept
 * their knots in the global spill slab instead of shared memory (tuning
 * diagnostics).  Synchronises the device; reset != 0 clears the counters. */
int emdb_plan_counters(emdb_plan* plan, unsigned long long* passes,
                       unsigned long long* spilled, int reset);

/* Dense batch like emdb_run, for callers that cannot allocate device memory:
 * services that reserve all device memory up front and forbid allocations on
 * the request path, hosts whose own allocator owns the device, and paths that
 * cannot afford cudaMalloc/cudaFree (which may synchronise the device).  No
 * plan is needed: the scratch (work-queue ticket, status word, per-CTA spill
 * slab) is one 32 MiB file-scope device array, held by every GPU that loads
 * the library until the process exits.  The slab bounds how many CTAs a call
 * runs; a config whose per-CTA slab does not fit the array even once is
 * rejected with EMDB_ERR_UNSUPPORTED.  The config is checked by the same rules
 * as emdb_plan_create, and the arena follows the planned path's automatic
 * rule.  Runs on the current device, asynchronously on `stream`.  Kernel
 * status flags (EMDB_STATUS_*: a trace too long for the arena, a sample
 * outside the knot span as a non-monotone T gives) collect in the array's
 * status word until emdb_noalloc_status reads them.  Every call shares the
 * array: calls that overlap on the GPU race, so serialise them.  A device's
 * first call looks up the array's address; make it before any stream capture.
 * A cudaDeviceReset between calls is not supported.
 * No counterpart in the reference (its run() always allocates, kernels.py:1353-1363). */
int emdb_run_noalloc(const emdb_config* cfg, const double* signals, const double* T, int batch,
                     int N, double* imfs, int* n_imfs, int* overflow, int* dbg_n, int* dbg_extno,
                     int* dbg_nzm, void* stream);
/* Synchronise `stream`, then read and clear the no-allocation entry point's
 * status word on the current device (EMDB_STATUS_* bits of every call since
 * the last read) into *status.  Allocates nothing.  No counterpart in the
 * reference (its flags come back with each call's own buffers, emd.py:95-105). */
int emdb_noalloc_status(int* status, void* stream);

/* Cycle counts (clock64, summed over traces) recorded only by a library
 * built with EMDB_LOAD_CLOCKS=1 (zeros otherwise): cycles[0] loading each
 * trace into shared memory, [1] whole traces, [2..11] the sift-pass phases
 * (knot fill, mirroring, spline rows, PCR levels, diagonal solve,
 * evaluation / update, lane sums, reduction trees + extrema scan, per-IMF
 * rows, the rest), thread 0's view taken at the barriers that end them.
 * Writes n values.  Synchronises the device; reset != 0 clears them.  No
 * reference counterpart (a measurement aid). */
int emdb_plan_phase_clocks(emdb_plan* plan, unsigned long long* cycles, int n, int reset);

/* Synchronise `stream`, read and clear the plan's device status word
 * (EMDB_STATUS_* bits) into *status. */
int emdb_status(emdb_plan* plan, int* status, void* stream);

/* Page-lock an existing host range (e.g. a memory-mapped trace file) so the
 * host pipeline's copies read it by DMA in place, and release it again.
 * read_only != 0 for ranges the device only reads (file mappings opened
 * read-only).  No reference counterpart: the trace-file ingest step. */
int emdb_host_register(void* ptr, size_t bytes, int read_only);
int emdb_host_unregister(void* ptr);

/* ---- learned queue order (no reference counterpart: the reference launches
 * one CTA per signal in index order, kernels.py:1366-1371).  All on the
 * current CUDA device, asynchronous on `stream`. ---- */

/* 32 float32 features per trace (length, zero-crossing and extrema rates,
 * dyadic band energies, extrema density per eighth, moments):
 * feat [batch, 32].  offsets = DEVICE int64 [batch+1], or NULL for a dense
 * [batch, N] batch. */
int emdb_features(const double* values, const int64_t* offsets, int batch, int N, float* feat,
                  void* stream);

/* MLP 32->128->128->2 (GELU).  Parameter block (float32, emdb_mlp_num_params()
 * values): W1[32][128] b1[128] W2[128][128] b2[128] W3[128][2] b3[2].
 * Inputs are raw features, standardised inside with mu/sd [32]. */
int emdb_mlp_num_params(void);
/* Training forward (FP32): keeps Z1/H1/Z2/H2 [B,128] for the backward, Y [B,2]. */
int emdb_mlp_forward(const float* params, const float* X, const float* mu, const float* sd, int B,
                     float* Z1, float* H1, float* Z2, float* H2, float* Y, void* stream);
/* Backward of the mean squared error vs targets T [B,2]: grads (same layout
 * as params), dY/dZ2/dZ1 scratch [B,2]/[B,128]/[B,128], *loss (device float)
 * set to the batch MSE. */
int emdb_mlp_backward(const float* params, const float* X, const float* mu, const float* sd,
                      const float* Z1, const float* H1, const float* Z2, const float* H2,
                      const float* Y, const float* T, int B, float* dY, float* dZ2, float* dZ1,
                      float* grads, float* loss, void* stream);
/* One Adam step (bias-corrected, step >= 1) on n parameters; if params_bf16
 * is not NULL the updated weights are also written there as bfloat16. */
int emdb_mlp_adam(float* params, const float* grads, float* m, float* v, int n, float lr,
                  float beta1, float beta2, float eps, int step, uint16_t* params_bf16,
                  void* stream);
/* Inference with bfloat16 weights and FP32 accumulation: Y [B,2]. */
int emdb_mlp_infer_bf16(const uint16_t* params_bf16, const float* X, const float* mu,
                        const float* sd, int B, float* Y, void* stream);

/* Self-test of the division the kernels use where a reciprocal is at hand
 * (no reference counterpart): counts results that differ in any bit from the
 * hardware IEEE division, in mismatches[3] (host array).  mode 0: every
 * integer pair 0 <= a <= b <= n (count in [0]); mode 1: n seeded random
 * cases each of [0] a/b over [2^-300, 2^300], [1] a/6, [2] a/b with
 * 0 <= a <= b, b in [1, 65537).  mode 2: the branch-free division the PCR
 * rows use (no reciprocal at hand), n seeded cases each of [0] a/b over
 * [2^-1100, 2^1100] (zeros, subnormals and infinities through its fallback),
 * [1] denominators with all-ones or power-of-two significands, [2] |a| <= |b|
 * within 2^+-40 of 1.  Modes 3 and 4: the FP32 kernels' float quotients
 * against the float division -- mode 3 every integer pair 0 <= a <= b <= n
 * through the reciprocal-based quotient; mode 4 n seeded cases each of [0]
 * the reciprocal-based quotient over [2^-40, 2^40], [1] the branch-free
 * quotient over [2^-140, 2^140] (zeros, subnormals, range edges through its
 * fallback), [2] PCR-like |a| <= |b| within 2^+-40 of 1.  Synchronous on the
 * current device. */
int emdb_check_division(int mode, long long n, unsigned long long seed,
                        unsigned long long* mismatches);

/* Message of the calling thread's last error ("" if none). */
int emdb_last_error(char* buf, size_t len);

#ifdef __cplusplus
}
#endif

#endif /* EMDB200_H */
