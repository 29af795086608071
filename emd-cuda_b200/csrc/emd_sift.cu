// Batched FP64 EMD sift for sm_100a -- the hot path behind GPUBatchEMD.
//
// Behaviour follows the reference's emd_batch_kernel (SeismicFlow/emd-cuda,
// kernels.py:834-1080) and its device functions, re-built for B200:
//
//  * one 128-thread CTA per trace, persistent: CTAs pull trace tickets from an
//    atomic work queue (FIFO, or a caller-given order), so a long trace never
//    holds a wave back and CSR batches of mixed length run in one launch;
//  * the proto-IMF lives in shared memory for the whole decomposition; the
//    running residue lives in the output rows (each row is written once, the
//    residue row once more per IMF);
//  * extrema: one warp-contiguous scan per sift pass computes ballot masks,
//    zero-crossing counts and the serial-fallback trigger; the masks are
//    compacted (popc ranks) straight into both envelopes' knot arrays, and
//    their prefix counts give every sample its knot segment in O(1) when the
//    knot list is strictly increasing (the reference binary-searches,
//    kernels.py:722-726).  The post-update scan of pass n is reused as the
//    pre-scan of pass n+1 (the reference scans the same data twice,
//    kernels.py:930 vs 965);
//  * boundary mirroring runs on one warp (decisions on one lane);
//  * the upper and lower not-a-knot systems are solved concurrently by
//    parallel cyclic reduction (ping-pong buffers, one barrier per level);
//  * envelope evaluation, the mean update and the six stop-test partial
//    sums are one fused pass; sums are formed in the reference's order (128
//    strided lanes + halving tree) and this file is compiled with
//    -fmad=false, so every value equals the reference algorithm's FP64
//    result bit for bit (the CPU oracle checks this);
//  * every quotient is the IEEE one, but most are formed without the
//    hardware division's slow-path branch: Markstein corrections from a
//    reciprocal (RN(1/h) from a compile-time table on the integer time axis,
//    where one correction is exact for integer operands), and for the PCR
//    rows a branch-free division from the approximate reciprocal; each
//    redoes its operation with the division outside the exact ranges.
//
// Per-pass knot/PCR storage is placed by size: all in the CTA's shared-
// memory arena; "borrow" (the proto-IMF parked in the per-CTA global slab
// during the spline solve so both PCR buffers stay on-chip, or with the
// moments beside the knots when the arena is short); "split" (PCR
// buffer 1 in the slab); "park" (the proto-IMF parked, PCR buffer 1 in its
// place, the knots and buffer 0 in the slab); or all in the slab.  For the
// host pipeline the kernel also reports finished chunks of traces through
// flags in mapped host memory.  Nothing here waits on another CTA or on the
// host.

#include "emdb_internal.cuh"

// Tuning knobs (compile-time; results are identical for every setting):
//  EMDB_EVAL_PAIR  evaluate two samples per loop trip in the fused pass
//  EMDB_PCR_PAIR   update two PCR rows per loop trip
//  EMDB_OUTLINE    rarely taken paths as calls instead of inline copies:
//                  1 the general evaluation and the binary segment search,
//                  2 also the IEEE-division fallbacks of the PCR and setup rows
//  EMDB_MERGED_PLACE  0: one sift-pass instance per knot placement; 1: one
//                  for the on-chip placements and one for the off-chip ones
//                  (placement chosen at run time); 2: one for all
//  EMDB_TREE_SPLIT the six end-of-pass reduction trees spread over the warps
// Same B200, same clocks, 16,384 x 2048 seismic: MERGED_PLACE/TREE_SPLIT
// 1/1 208.4k signals/s, 1/0 188.1k, 2/1 195.6k, 0/0 184.9k (and 0/1 172.7k on
// another box against 208.2k for 1/1): less sift-pass code relieves
// instruction supply, the dominant stall after FP64 latency.
//  EMDB_FAST_DIV   reciprocal-based correctly rounded division in evaluation:
//                  0 none, 1 segment quotients from stored RN(1/h) plus the
//                  division by 6, 2 the division by 6 only, 3 segment quotients
//                  from a per-sample RN(1/h) plus the division by 6
// Measured on B200 (16,384 seismic traces x 2048 samples): the paired loops
// raise register pressure more than they add overlap; EMDB_FAST_DIV 0/1/2/3
// ran at 142.5k/154.3k/150.8k/154.9k signals/s, bit-identical outputs.  The
// gain is the straight-line evaluation: every hardware division carries its
// own slow-path branch, which splits the sample's independent chains.
//  EMDB_PCR_NB     branch-free division with no reciprocal at hand (div_nb)
//                  for the two PCR quotients of each row: 241.1k vs 222.8k
//                  signals/s on one B200.  Used everywhere (evaluation and
//                  stop-test quotients too) it ran slower, 160k vs 180k: there
//                  the extra instructions outweigh the overlap.
//  EMDB_ACC_NB / EMDB_SETUP_NB  the same division for the stop-test quotient
//                  diff/new and the spline rows' slopes: 231.0k / 236.7k vs
//                  240.9k signals/s, so off.
//  EMDB_SETUP_TAB  on the integer time axis, the spline rows' slopes from the
//                  reciprocal table and div_q: 238.0k vs 241.2k, so off.
//  EMDB_SCAN_UNROLL / EMDB_FILL_UNROLL  unroll factors of the extrema scan
//                  and knot fill loops: 4 measured 231.8k / 226.3k vs 240.2k
//                  at 2.
//  EMDB_SORTED_NOCHECK  skip the integer evaluation's operand-range checks
//                  on sorted knot lists (only the table bound stays): 239.6k
//                  vs 240.2k, so off.
#ifndef EMDB_EVAL_PAIR
#define EMDB_EVAL_PAIR 0
#endif
#ifndef EMDB_PCR_PAIR
#define EMDB_PCR_PAIR 0
#endif
//  EMDB_WIDE_PCR_PAIR  the same for the wide (256 / 512-thread) instances
#ifndef EMDB_WIDE_PCR_PAIR
#define EMDB_WIDE_PCR_PAIR 0
#endif
//  EMDB_WIDE_OVERLAP  wide instances: the warps past the 128 reduction lanes
//                  run the post-update extrema scan while the lanes sum the
//                  stop-test terms (the scan then has NT/32 - 4 slots).
//                  Same bits; measured on B200 (best of two): 512 threads,
//                  1024 x 8192 seismic 291.2 vs 292.3 ms, 2048 x 4096 50.9 vs
//                  51.6 ms; 256 threads, 2048 x 4096 50.4 vs 46.4 ms (its
//                  knot fill then has 4 warps of 8) -- so off.
//  EMDB_WIDE_PCR_PAIR 1: 291.1 / 51.2 ms, no gain.
#ifndef EMDB_WIDE_OVERLAP
#define EMDB_WIDE_OVERLAP 0
#endif
//  EMDB_LANE_UNROLL  wide instances: unroll factor of the lane-sum loops (the
//                  loads of a lane's samples in flight at once).  With the
//                  six sums split over the 128-lane groups, B200, 512 threads
//                  1024 x 8192 seismic / 256 threads 2048 x 4096 (ms): 4:
//                  296.7 / 47.5, 8: 290.0 / 47.5, 16: 289.9 / 46.8; the sums
//                  on the first 128 threads only (no split): 293.0 / 46.7.
#ifndef EMDB_LANE_UNROLL
#define EMDB_LANE_UNROLL 16
#endif
#ifndef EMDB_OUTLINE
#define EMDB_OUTLINE 2
#endif
#ifndef EMDB_FAST_DIV
#define EMDB_FAST_DIV 3
#endif
#ifndef EMDB_MERGED_PLACE
#define EMDB_MERGED_PLACE 1
#endif
#ifndef EMDB_TREE_SPLIT
#define EMDB_TREE_SPLIT 1
#endif
#ifndef EMDB_PCR_NB
#define EMDB_PCR_NB 1
#endif
#ifndef EMDB_ACC_NB
#define EMDB_ACC_NB 0
#endif
#ifndef EMDB_SETUP_NB
#define EMDB_SETUP_NB 0
#endif
#ifndef EMDB_SETUP_TAB
#define EMDB_SETUP_TAB 0
#endif
#ifndef EMDB_SCAN_UNROLL
#define EMDB_SCAN_UNROLL 2
#endif
#ifndef EMDB_FILL_UNROLL
#define EMDB_FILL_UNROLL 2
#endif
#ifndef EMDB_SORTED_NOCHECK
#define EMDB_SORTED_NOCHECK 0
#endif
//  EMDB_LOAD_CLOCKS  instrumented build: thread 0 of each CTA adds the clock64
//                  cycles of every trace's load into shared memory, of the
//                  whole trace, and of each phase of the sift passes (taken at
//                  the barriers that end them) to the plan's counters [2..]
//                  (emdb_plan_phase_clocks); off in the product build
#ifndef EMDB_LOAD_CLOCKS
#define EMDB_LOAD_CLOCKS 0
#endif
#if EMDB_LOAD_CLOCKS
// phases: 0 knot fill, 1 mirroring (+ parking), 2 spline rows, 3 PCR levels,
// 4 diagonal solve, 5 evaluation / update, 6 lane sums, 7 reduction trees +
// extrema scan, 8 per-IMF rows and reload, 9 the rest of the loop
#define EMDB_PH(Cptr, k)                                      \
  do {                                                        \
    if (threadIdx.x == 0) {                                   \
      const long long t_ = clock64();                         \
      (Cptr)->ph[k] += (unsigned long long)(t_ - (Cptr)->ph_last); \
      (Cptr)->ph_last = t_;                                   \
    }                                                         \
  } while (0)
#else
#define EMDB_PH(Cptr, k) do {} while (0)
#endif
constexpr int kPhases = 10;

// EMDB_F32: the FP32 build of this file (namespace emdb::f32).  Every value
// the sift computes is a `real`; the reference kernel's double literals keep
// their C++ meaning, so float expressions that mix them are evaluated in
// double and rounded once, as in the reference source compiled with REAL_T =
// float.  The FP64 build's division shortcuts (reciprocal tables, Markstein
// and branch-free quotients) are off: float quotients are the IEEE ones, and
// the one double quotient per envelope sample (the reference's "/ 6.0")
// takes the Markstein quotient from RN(1/6) (EMDB_FAST_DIV 2), which equals
// the double division.
#ifndef EMDB_F32
#define EMDB_F32 0
#endif
#if EMDB_F32
//  EMDB_F32_FAST  the float counterparts of the FP64 build's branch-free
//                  quotients (div_q from an IEEE reciprocal for the segment
//                  quotients, div_nb for the PCR rows), self-tested against
//                  the float division by emdb_check_division modes 3 and 4
#ifndef EMDB_F32_FAST
#define EMDB_F32_FAST 1
#endif
#undef EMDB_FAST_DIV
#define EMDB_FAST_DIV (EMDB_F32_FAST ? 3 : 2)
#undef EMDB_PCR_NB
#define EMDB_PCR_NB EMDB_F32_FAST
namespace emdb::f32 {
using real = float;
#else
namespace emdb {
using real = double;
#endif

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kScanUnroll = EMDB_SCAN_UNROLL;
constexpr int kFillUnroll = EMDB_FILL_UNROLL;
constexpr int kLaneUnroll = EMDB_LANE_UNROLL;

// reference thresholds (kernels.py:81-85, 814, 1069): the first five are
// REAL_T functions there, the last two double literals compared with REAL_T
constexpr real kEnergyRatioThr = 0.2;
constexpr real kStdThr = 0.2;
constexpr real kSvarThr = 0.001;
constexpr real kTotalPowerThr = 0.005;
constexpr real kRangeThr = 0.001;
constexpr double kSumNewSqMin = 1e-10;
constexpr double kResidueZeroAtol = 1e-8;
constexpr int kLocalExtBuf = 64;  // kernels.py:206 (serial-fallback trigger)

struct Ctl {
  int job;
  int head[2][kMaxNbsym + 1];  // first NB+1 extrema indices per side (0 = max, 1 = min)
  int tail[2][kMaxNbsym + 1];  // tail[q][k] = index of extremum n_q-1-k
  int mlist[4][kMaxNbsym + 1]; // mirrored index lists: lmax, lmin, rmax, rmin
  int mcnt[4];
  int lsym, rsym;
  int kbase[2], kcnt[2];
  int dbg_n[kMaxImfsCap], dbg_e[kMaxImfsCap], dbg_z[kMaxImfsCap];
  int chunk_bad;
  real sums[8];
#if EMDB_LOAD_CLOCKS
  unsigned long long ph[kPhases];
  long long ph_last;
#endif
};

// The 6 x 128 reduction lanes have no fixed home: between sift passes they sit
// at the start of the knot arena; inside a pass, after the spline solve, they
// reuse PCR buffer 1, which is dead from then on (or follow the PCR buffers
// when those are smaller than the lanes).
constexpr int kRedDoubles = 6 * kThreads;
constexpr size_t kRedBytes = kRedDoubles * sizeof(real);

// Extrema-scan slots of a CTA of NT threads: one contiguous range of 32-sample
// chunks per slot, scanned by one warp and filled into knots by one warp.
// The wide instances that overlap the scan with the lane sums scan with the
// warps past the first four, so they have NT/32 - 4 slots.
template <int NT>
__host__ __device__ constexpr int scan_slots() {
  return (NT > kThreads && EMDB_WIDE_OVERLAP) ? NT / 32 - kWarps : NT / 32;
}
// first warp that scans
template <int NT>
__host__ __device__ constexpr int scan_warp0() { return NT / 32 - scan_slots<NT>(); }

// Per-warp scan counts (maxima, minima, sign changes, zero-run ends, fallback
// trigger) live right after the control block: 5 x (warps per CTA) ints.
struct SmemLayout {
  Ctl* ctl;
  int* wc;            // [5][NW]: w_max | w_min | w_zc | w_zre | w_trig
  real* red;        // [6][128] between passes (= arena start)
  real* imf;        // [N]
  uint32_t* mmax;     // [nch] ballot masks of the last extrema scan
  uint32_t* mmin;
  uint16_t* pmax;     // per-chunk exclusive prefix within the owning warp's range
  uint16_t* pmin;
  char* arena;        // knot arena start
  int arena_bytes;    // bytes left for the knot arena
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// NT: threads per CTA (128, or 512 for the wide instance).  kGImf: the
// proto-IMF lives in the CTA's global slab instead of shared memory (traces
// longer than shared memory holds); it then takes no shared memory.
template <int NT = kThreads, bool kGImf = false>
__host__ __device__ inline size_t fixed_bytes(int N) {
  size_t nch = (size_t)(N + 31) / 32;
  size_t b = align16(sizeof(Ctl)) + align16(5 * (NT / 32) * sizeof(int));
  if (!kGImf) b += align16((size_t)N * sizeof(real));
  b += align16(nch * 4) * 2 + align16(nch * 2) * 2;
  return b;
}

template <int NT = kThreads, bool kGImf = false>
__device__ __forceinline__ SmemLayout carve(char* base, int N, int arena_total,
                                            real* gimf = nullptr) {
  SmemLayout L;
  size_t nch = (size_t)(N + 31) / 32;
  char* p = base;
  L.ctl = reinterpret_cast<Ctl*>(p); p += align16(sizeof(Ctl));
  L.wc = reinterpret_cast<int*>(p); p += align16(5 * (NT / 32) * sizeof(int));
  L.mmax = reinterpret_cast<uint32_t*>(p); p += align16(nch * 4);
  L.mmin = reinterpret_cast<uint32_t*>(p); p += align16(nch * 4);
  L.pmax = reinterpret_cast<uint16_t*>(p); p += align16(nch * 2);
  L.pmin = reinterpret_cast<uint16_t*>(p); p += align16(nch * 2);
  // the proto-IMF directly ahead of the arena: the borrow placement uses both
  // as one region
  if (kGImf) {
    L.imf = gimf;
  } else {
    L.imf = reinterpret_cast<real*>(p); p += align16((size_t)N * sizeof(real));
  }
  L.arena = p;
  L.red = reinterpret_cast<real*>(p);
  L.arena_bytes = arena_total - (int)(p - base);
  return L;
}

// Knot / PCR storage for one sift pass (both envelopes).  After the last PCR
// level only the b and d arrays of the final buffers are read, so the spline
// moments M go into buffer 0's a (upper envelope) and c (lower) arrays and the
// segment reciprocals R into buffer 1's a and c arrays.
struct Knots {
  real* X[2];
  real* Y[2];
  real* M[2];
  real* R[2];   // RN(1/h) per knot segment, in buffer 1's a / c arrays
  real* P[2];   // ping-pong PCR buffers: a | b | c | d, each `cap` rows
  real* red;    // reduction lanes after the solve: buffer 1, or just past it
  int cap;
};

__host__ __device__ inline size_t knot_bytes(int kc0, int kc1) {
  // size_t throughout: a host-side size query must not wrap for any int input
  const size_t cap = (size_t)kc0 + (size_t)kc1;
  // with EMDB_FAST_DIV 1 buffer 1 holds the segment reciprocals during evaluation
  const size_t red_extra = (EMDB_FAST_DIV != 1 && 4 * cap >= (size_t)kRedDoubles) ? 0 : kRedBytes;
  return (2 * cap + 8 * cap) * sizeof(real) + red_extra;
}

__device__ __forceinline__ Knots place_knots(char* base, int kc0, int kc1) {
  Knots K;
  real* p = reinterpret_cast<real*>(base);
  K.X[0] = p; p += kc0;
  K.Y[0] = p; p += kc0;
  K.X[1] = p; p += kc1;
  K.Y[1] = p; p += kc1;
  K.cap = kc0 + kc1;
  K.P[0] = p; p += 4 * K.cap;
  K.P[1] = p;
  K.M[0] = K.P[0];
  K.M[1] = K.P[0] + 2 * K.cap;
  K.R[0] = K.P[1];
  K.R[1] = K.P[1] + 2 * K.cap;
  K.red = (EMDB_FAST_DIV != 1 && 4 * K.cap >= kRedDoubles) ? K.P[1] : K.P[1] + 4 * K.cap;
  return K;
}

// Split placement, for passes whose knots fit shared memory only without the
// second PCR buffer: knots X | Y and PCR buffer 0 (which ends up holding the
// moments) in the arena, buffer 1 in the per-CTA global slab.  Evaluation then
// reads shared memory only, and half of the PCR levels read the slab.
__host__ __device__ inline size_t split_bytes(int kc0, int kc1) {
  return 6 * ((size_t)kc0 + (size_t)kc1) * sizeof(real);
}

__device__ __forceinline__ Knots place_knots_split(char* sbase, int sbytes, char* gbase, int kc0,
                                                   int kc1) {
  Knots K;
  real* p = reinterpret_cast<real*>(sbase);
  K.X[0] = p; p += kc0;
  K.Y[0] = p; p += kc0;
  K.X[1] = p; p += kc1;
  K.Y[1] = p; p += kc1;
  K.cap = kc0 + kc1;
  K.P[0] = p; p += 4 * K.cap;
  K.P[1] = reinterpret_cast<real*>(gbase);
  K.M[0] = K.P[0];
  K.M[1] = K.P[0] + 2 * K.cap;
  K.R[0] = K.P[1];
  K.R[1] = K.P[1] + 2 * K.cap;
  // reduction lanes: shared memory past buffer 0 when they fit, else the slab
  // (buffer 1 is dead after the solve; the slab holds knot_bytes of the largest pass)
  if (split_bytes(kc0, kc1) + kRedBytes <= (size_t)sbytes) K.red = p;
  else K.red = (EMDB_FAST_DIV != 1 && 4 * K.cap >= kRedDoubles) ? K.P[1] : K.P[1] + 4 * K.cap;
  return K;
}

// Borrow placement, for passes whose knots fit shared memory only together
// with the proto-IMF's space: the proto-IMF is parked in the per-CTA slab
// during the solve, PCR buffer 1 takes its place (imf region plus the arena
// ahead of the knots), and X | Y | buffer 0 sit at the end of the arena, clear
// of the proto-IMF that the knot fill reads.  Evaluation reads the old sample
// values back from the slab; the reduction lanes go to the slab after them.
__host__ __device__ inline bool borrow_fits(int N, int arena_bytes, size_t slab_stride, int kc0,
                                            int kc1) {
  const size_t cap = (size_t)kc0 + (size_t)kc1;
  const size_t region = align16((size_t)N * sizeof(real)) + (size_t)arena_bytes;
  return EMDB_FAST_DIV != 1 && 6 * cap * sizeof(real) <= (size_t)arena_bytes &&
         10 * cap * sizeof(real) <= region &&
         (align16((size_t)N * sizeof(real)) + kRedBytes) <= slab_stride;
}

__device__ __forceinline__ real* borrow_save(char* slab) { return reinterpret_cast<real*>(slab); }

__device__ __forceinline__ Knots place_knots_borrow(real* imf, char* arena, int arena_bytes,
                                                    char* slab, int N, int kc0, int kc1) {
  Knots K;
  K.cap = kc0 + kc1;
  real* p = reinterpret_cast<real*>(arena + arena_bytes) - 6 * K.cap;
  K.X[0] = p; p += kc0;
  K.Y[0] = p; p += kc0;
  K.X[1] = p; p += kc1;
  K.Y[1] = p; p += kc1;
  K.P[0] = p;
  K.P[1] = imf;
  K.M[0] = K.P[0];
  K.M[1] = K.P[0] + 2 * K.cap;
  K.R[0] = K.P[1];
  K.R[1] = K.P[1] + 2 * K.cap;
  K.red = reinterpret_cast<real*>(slab + align16((size_t)N * sizeof(real)));
  return K;
}

// Compact borrow placement, for long traces whose X | Y | buffer 0 do not fit
// the arena next to the proto-IMF: the moments get their own array beside the
// knots (instead of buffer 0's dead a / c arrays), so only X | Y | M sit at the
// arena's end and both PCR buffers go to the front of the proto-IMF region
// (parked in the slab, as for the borrow placement).  Everything stays
// on-chip; the arena needs 3 doubles per knot slot instead of 6, the region
// 11 instead of 10.
__host__ __device__ inline bool borrow2_fits(int N, int arena_bytes, size_t slab_stride, int kc0,
                                             int kc1) {
  const size_t cap = (size_t)kc0 + (size_t)kc1;
  const size_t region = align16((size_t)N * sizeof(real)) + (size_t)arena_bytes;
  return EMDB_FAST_DIV != 1 && 3 * cap * sizeof(real) <= (size_t)arena_bytes &&
         11 * cap * sizeof(real) <= region &&
         (align16((size_t)N * sizeof(real)) + kRedBytes) <= slab_stride;
}

__device__ __forceinline__ Knots place_knots_borrow2(real* imf, char* arena, int arena_bytes,
                                                     char* slab, int N, int kc0, int kc1) {
  Knots K;
  K.cap = kc0 + kc1;
  real* p = reinterpret_cast<real*>(arena + arena_bytes) - 3 * K.cap;
  K.X[0] = p; p += kc0;
  K.Y[0] = p; p += kc0;
  K.X[1] = p; p += kc1;
  K.Y[1] = p; p += kc1;
  K.M[0] = p;
  K.M[1] = p + kc0;
  K.P[0] = imf;
  K.P[1] = imf + 4 * K.cap;
  K.R[0] = K.P[1];
  K.R[1] = K.P[1] + 2 * K.cap;
  K.red = reinterpret_cast<real*>(slab + align16((size_t)N * sizeof(real)));
  return K;
}

// Park placement, for passes whose knots fit neither shared-memory placement
// but whose PCR buffer 1 fits the proto-IMF's space (long traces with many
// knots): the proto-IMF is parked in the slab as for the borrow placement,
// buffer 1 takes its place (imf region plus the arena ahead), and X | Y |
// buffer 0 go to the slab after the parked samples.  Half of the PCR levels
// then read shared memory; the evaluation reads the knots and the old samples
// from the slab.  The reduction lanes use the arena start, free after the
// solve.
__host__ __device__ inline bool park_fits(int N, int arena_bytes, size_t slab_stride, int kc0,
                                          int kc1) {
  const size_t cap = (size_t)kc0 + (size_t)kc1;
  const size_t imfb = align16((size_t)N * sizeof(real));
  return EMDB_FAST_DIV != 1 && 4 * cap * sizeof(real) <= imfb + (size_t)arena_bytes &&
         imfb + 6 * cap * sizeof(real) <= slab_stride;
}

__device__ __forceinline__ Knots place_knots_park(real* imf, char* slab, int N, int kc0, int kc1,
                                                  real* red) {
  Knots K;
  K.cap = kc0 + kc1;
  real* p = reinterpret_cast<real*>(slab + align16((size_t)N * sizeof(real)));
  K.X[0] = p; p += kc0;
  K.Y[0] = p; p += kc0;
  K.X[1] = p; p += kc1;
  K.Y[1] = p; p += kc1;
  K.P[0] = p;
  K.P[1] = imf;
  K.M[0] = K.P[0];
  K.M[1] = K.P[0] + 2 * K.cap;
  K.R[0] = K.P[1];
  K.R[1] = K.P[1] + 2 * K.cap;
  K.red = red;
  return K;
}

enum : int { kPlaceSmem = 0, kPlaceSplit = 1, kPlaceSlab = 2, kPlaceBorrow = 3, kPlacePark = 4,
              kPlaceBorrow2 = 5 };
enum : int { kOnChip = -1, kOffChip = -2, kAnyPlace = -3 };

// Where one sift pass keeps its knots and PCR buffers: the first placement
// that fits, the on-chip ones first (shared, borrow, compact borrow), then
// split, park, slab.  `arena_bytes` is the knot arena left after the fixed
// part (control block, scan masks, proto-IMF); the slab always fits.
__host__ __device__ inline int choose_place(int N, int arena_bytes, size_t slab_stride, int kc0,
                                            int kc1, bool imf_global = false) {
  // a proto-IMF in global memory has no shared-memory region to lend: only
  // the placements that leave it alone
  if (imf_global)
    return knot_bytes(kc0, kc1) <= (size_t)arena_bytes ? kPlaceSmem
         : split_bytes(kc0, kc1) <= (size_t)arena_bytes ? kPlaceSplit
                                                        : kPlaceSlab;
  return knot_bytes(kc0, kc1) <= (size_t)arena_bytes ? kPlaceSmem
       : borrow_fits(N, arena_bytes, slab_stride, kc0, kc1) ? kPlaceBorrow
       : borrow2_fits(N, arena_bytes, slab_stride, kc0, kc1) ? kPlaceBorrow2
       : split_bytes(kc0, kc1) <= (size_t)arena_bytes ? kPlaceSplit
       : park_fits(N, arena_bytes, slab_stride, kc0, kc1) ? kPlacePark
                                                          : kPlaceSlab;
}

// Correctly rounded a/b from y = RN(1/b) (Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 1990):
// if y is within half an ulp of 1/b and q within one ulp of a/b, then with the
// exact remainder r = a - b*q (one FMA), RN(q + r*y) = RN(a/b).  q0 = RN(a*y)
// can be 1.5 ulp off, so one correction step first brings it within one ulp,
// the second rounds correctly.  Operands whose remainders or quotient could
// underflow or overflow (|a| or |a*y| outside [2^-900, 2^900], zeros, inf,
// NaN) take the division.
// A zero numerator gives q0 = a*y, the correctly signed zero (or NaN when y is
// infinite or NaN, as a/b would be).  Checked bit for bit against the hardware
// division by emdb_check_division.
//
// div_q returns the quotient without branching and sets `slow` for operands
// outside that range, so a caller can redo a whole sample with the division
// once instead of branching on every quotient.
__device__ __noinline__ double div_slow(double a, double b) { return a / b; }

#if EMDB_F32
// Float counterparts (same methods, binary32 ranges): div_q is the two-step
// Markstein quotient from y = RN(1/b); div_nb the branch-free quotient from
// the approximate reciprocal (one Newton step reaches binary32 accuracy), a
// faithful quotient and the exact-remainder choice of its neighbour (Muller
// et al., Handbook of Floating-Point Arithmetic, ch. 4.9 / 5.3).  `slow` is
// set outside the ranges where every step is exact: |a|, |q| in
// (2^-100, 2^100), |b| in (2^-110, 2^110).
__device__ __noinline__ float div_slow(float a, float b) { return a / b; }

__device__ __forceinline__ float div_q(float a, float b, float y, bool& slow) {
  const float q0 = a * y;
  const float e0 = fmaf(-q0, b, a);
  const float q1 = fmaf(e0, y, q0);
  const float e1 = fmaf(-q1, b, a);
  const float q2 = fmaf(e1, y, q1);
  const float aa = fabsf(a), qa = fabsf(q0);
  const bool zero = a == 0.0f;
  slow |= !(zero || (aa > 0x1p-100f && aa < 0x1p+100f && qa > 0x1p-100f && qa < 0x1p+100f));
  return zero ? q0 : q2;
}

__device__ __forceinline__ float div_nb(float a, float b, bool& slow) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
  const float e = fmaf(-b, y, 1.0f);
  y = fmaf(y, e, y);
  const float q0 = a * y;
  const float r0 = fmaf(-q0, b, a);
  const float q1 = fmaf(r0, y, q0);
  const float r1 = fmaf(-q1, b, a);
  const bool up = (r1 > 0.0f) == (b > 0.0f);
  const int step = (up == (q1 > 0.0f)) ? 1 : -1;
  const float qn = __int_as_float(__float_as_int(q1) + step);
  const float rn = fmaf(-qn, b, a);
  const float q = fabsf(rn) < fabsf(r1) ? qn : q1;
  const float aa = fabsf(a), qa = fabsf(q1), ba = fabsf(b);
  const bool bok = ba > 0x1p-110f && ba < 0x1p+110f;
  const bool zero = a == 0.0f;
  slow |= !bok || (!zero && !(aa > 0x1p-100f && aa < 0x1p+100f && qa > 0x1p-100f && qa < 0x1p+100f));
  return zero ? q0 : q;
}
#endif

// Rarely taken paths of the hot loops (fewer than 4 knots, operands outside
// the fast quotients' range, knot lists that are not strictly increasing) as
// calls to one out-of-line body each, instead of an inline copy per call site:
// keeps the hot loops' code small.  Defined after eval_seg / search_seg.
__device__ __noinline__ real eval_seg_cold(const real* x, const real* y, const real* M,
                                             int n, real t, int lo);
__device__ __noinline__ int search_seg_cold(const real* x, int n, real t);
#if EMDB_OUTLINE >= 1
#define EMDB_EVAL_RARE(sv, t, lo) eval_seg_cold((sv).x, (sv).y, (sv).M, (sv).n, (t), (lo))
#define EMDB_SEARCH_RARE(sv, t) search_seg_cold((sv).x, (sv).n, (t))
#else
#define EMDB_EVAL_RARE(sv, t, lo) eval_seg((sv), (t), (lo))
#define EMDB_SEARCH_RARE(sv, t) search_seg((sv), (t))
#endif
#if EMDB_OUTLINE >= 2
#define EMDB_DIV_RARE(a, b) div_slow((a), (b))
#else
#define EMDB_DIV_RARE(a, b) ((a) / (b))
#endif

__device__ __forceinline__ double div_q(double a, double b, double y, bool& slow) {
  const double q0 = a * y;
  const double e0 = fma(-q0, b, a);
  const double q1 = fma(e0, y, q0);
  const double e1 = fma(-q1, b, a);
  const double q2 = fma(e1, y, q1);
  const double aa = fabs(a), qa = fabs(q0);
  const bool zero = a == 0.0;
  slow |= !(zero || (aa > 0x1p-900 && aa < 0x1p+900 && qa > 0x1p-900 && qa < 0x1p+900));
  return zero ? q0 : q2;
}

#if EMDB_PCR_NB || EMDB_ACC_NB || EMDB_SETUP_NB
// Branch-free RN(a/b) with no reciprocal at hand (FMA division schemes in
// Muller et al., "Handbook of Floating-Point Arithmetic", 2nd ed., ch. 4.9 /
// 5.3): y ~ 1/b from the PTX approximate reciprocal and two Newton steps;
// q1 = q0 + (a - b*q0)*y is a faithful rounding of a/b; the exact remainders
// of q1 and of its neighbour towards a/b pick the nearer one (a quotient of
// two 53-bit numbers is never an exact midpoint).  `slow` is set outside the
// ranges where every step is exact: |a|, |q| in (2^-900, 2^900), |b| in
// (2^-1000, 2^1000); zero numerators only with such a b.
__device__ __forceinline__ double div_nb(double a, double b, bool& slow) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  const double q0 = a * y;
  const double r0 = fma(-q0, b, a);
  const double q1 = fma(r0, y, q0);
  const double r1 = fma(-q1, b, a);
  const bool up = (r1 > 0.0) == (b > 0.0);
  const long long step = (up == (q1 > 0.0)) ? 1 : -1;
  const double qn = __longlong_as_double(__double_as_longlong(q1) + step);
  const double rn = fma(-qn, b, a);
  const double q = fabs(rn) < fabs(r1) ? qn : q1;
  const double aa = fabs(a), qa = fabs(q1), ba = fabs(b);
  const bool bok = ba > 0x1p-1000 && ba < 0x1p+1000;
  const bool zero = a == 0.0;
  slow |= !bok || (!zero && !(aa > 0x1p-900 && aa < 0x1p+900 && qa > 0x1p-900 && qa < 0x1p+900));
  return zero ? q0 : q;
}
#endif

#if !EMDB_F32
__device__ __forceinline__ double div_rn(double a, double b, double y) {
  bool slow = false;
  const double q = div_q(a, b, y, slow);
  return slow ? div_slow(a, b) : q;
}
#endif
constexpr double kInv6 = 1.0 / 6.0;   // RN(1/6), folded at compile time

// RN(1/h) for integer h in [1, kRcpTab], built at compile time by IEEE
// division and shipped initialised in the module.
constexpr int kRcpTab = 16384;
struct RcpTab { double v[kRcpTab + 1]; };
constexpr RcpTab make_rcp_tab() {
  RcpTab t{};
  for (int h = 1; h <= kRcpTab; ++h) t.v[h] = 1.0 / (double)h;
  return t;
}
__device__ const RcpTab g_rcp = make_rcp_tab();


struct TimeAxis {
  const real* T;
  bool arange;
  __device__ __forceinline__ real operator()(int i) const { return arange ? (real)i : T[i]; }
};

// ---------------------------------------------------------------------------
// Extrema: count pass (find_extrema_parallel semantics, kernels.py:231-349,
// with the serial scan's plateau rule, kernels.py:157-200).
// ---------------------------------------------------------------------------
// NS slots; `slot` is the calling warp's slot.
template <int NS>
__device__ __forceinline__ void extrema_count(const SmemLayout& L, int N, int slot, int lane) {
  const real* imf = L.imf;
  int nch = (N + 31) >> 5;
  int c0 = (slot * nch) / NS, c1 = ((slot + 1) * nch) / NS;
  int rmax = 0, rmin = 0, zc = 0, zre = 0;
  bool trig = false;
  // neighbours straight from shared memory (conflict-free consecutive
  // doubles): no shuffles, no divergent edge loads; iterations independent
#pragma unroll kScanUnroll
  for (int c = c0; c < c1; ++c) {
    int i = (c << 5) + lane;
    real v = (i < N) ? imf[i] : 0.0;
    real vp = (i >= 1 && i - 1 < N) ? imf[i - 1] : 0.0;
    real vn = (i + 1 < N) ? imf[i + 1] : 0.0;
    bool interior = (i >= 1) && (i <= N - 2);
    real dp = v - vp, dn = vn - v;
    bool strict = interior && (dp * dn < 0.0);
    bool ismin = strict && (dp < 0.0);
    bool ismax = strict && !(dp < 0.0);
    const bool flat = interior && dn == 0.0 && dp != 0.0;
    if (__any_sync(kFull, flat)) {
      // rare: true left edge of a flat run, classified by the slopes around it
      if (flat) {
        int j = i;
        while (j + 1 < N && imf[j + 1] == v) ++j;
        if (j + 1 < N) {
          real da = imf[j + 1] - imf[j];
          if (dp > 0.0 && da < 0.0) ismax = true;
          else if (dp < 0.0 && da > 0.0) ismin = true;
        }
      }
    }
    trig |= interior && (dp == 0.0 || dn == 0.0 || v == 0.0);
    bool sc = (i <= N - 2) && (v != 0.0) && (v * vn < 0.0);
    bool zr = (i >= 1) && (i < N) && (v != 0.0) && (vp == 0.0);
    uint32_t bmax = __ballot_sync(kFull, ismax);
    uint32_t bmin = __ballot_sync(kFull, ismin);
    if (lane == 0) {
      L.mmax[c] = bmax; L.mmin[c] = bmin;
      L.pmax[c] = (uint16_t)rmax; L.pmin[c] = (uint16_t)rmin;
    }
    rmax += __popc(bmax);
    rmin += __popc(bmin);
    zc += __popc(__ballot_sync(kFull, sc));
    zre += __popc(__ballot_sync(kFull, zr));
  }
  trig = __any_sync(kFull, trig);
  if (lane == 0) {
    int* w = L.wc;
    w[slot] = rmax; w[NS + slot] = rmin;
    w[2 * NS + slot] = zc; w[3 * NS + slot] = zre; w[4 * NS + slot] = trig ? 1 : 0;
  }
}

struct ExtInfo {
  int tot_max, tot_min;   // true counts
  int n_max, n_min;       // stored (capped) counts
  int n_zer;
  int off_max, off_min;   // this warp's rank offsets
  bool overflow;
  bool trig;              // serial-fallback trigger (exact zeros / flat runs)
};

// After the count pass + barrier.  Reproduces the parallel/serial split of
// find_extrema_parallel: without a fallback trigger the zero-crossing count is
// sign changes only; with one, the serial count adds one per zero run that
// ends before N (kernels.py:123-143, 273-276).
// `slot`: the caller's fill slot (its warp, if the warp fills), for its rank offsets
template <int NS>
__device__ __forceinline__ ExtInfo extrema_totals(const SmemLayout& L, int slot, int max_extrema) {
  constexpr int NW = NS;
  const int warp = slot;
  const Ctl& C = *L.ctl;
  const int* wc = L.wc;
  ExtInfo e;
  e.tot_max = e.tot_min = 0;
  int zc = 0, zre = 0;
  bool trig = false;
  e.off_max = e.off_min = 0;
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    if (w < warp) { e.off_max += wc[w]; e.off_min += wc[NW + w]; }
    e.tot_max += wc[w]; e.tot_min += wc[NW + w];
    zc += wc[2 * NW + w]; zre += wc[3 * NW + w];
    trig |= wc[4 * NW + w] != 0;
  }
  e.trig = trig;
  if (!trig && C.chunk_bad) trig = true;
  e.n_zer = zc + (trig ? zre : 0);
  e.n_max = min(e.tot_max, max_extrema);
  e.n_min = min(e.tot_min, max_extrema);
  e.overflow = (e.tot_max >= max_extrema) || (e.tot_min >= max_extrema);
  return e;
}

// The reference's parallel scan also falls back when one thread's contiguous
// chunk (ceil(N/128) samples) holds more than 64 strict maxima or minima.  That
// can only change n_zer when imf[0] == 0 (leading zero), and only for N > 16384,
// so it is evaluated in that rare case only.  The chunks are the reference's
// 128 threads' (threads past 128 of a wider CTA have none).  Ends with a barrier.
__device__ void chunk_fallback_check(const SmemLayout& L, int N, int tid) {
  Ctl& C = *L.ctl;
  const real* s = L.imf;
  int cs = (N + kThreads - 1) / kThreads;
  int start = tid * cs, end = min(start + cs, N);
  int lo = max(start, 1), hi = min(end, N - 1);
  int nmx = 0, nmn = 0;
  for (int i = lo; i < hi; ++i) {
    real dp = s[i] - s[i - 1], dn = s[i + 1] - s[i];
    if (dp * dn < 0.0) { if (dp < 0.0) ++nmn; else ++nmx; }
  }
  int bad = __syncthreads_or(nmx > kLocalExtBuf || nmn > kLocalExtBuf);
  if (tid == 0) C.chunk_bad = bad;
  __syncthreads();
}

// One extrema scan = count pass + totals.  Ends after a barrier with every
// thread holding the same totals.
// The totals of a finished count pass (after its barrier), and the
// reference's rare chunk fallback.  Every thread gets the totals; a warp that
// fills gets its slot's rank offsets.
template <int NT>
__device__ __forceinline__ ExtInfo extrema_finish(const SmemLayout& L, int N, int tid, int warp,
                                                  int max_extrema) {
  constexpr int NS = scan_slots<NT>();
  const int slot = warp < NS ? warp : 0;
  ExtInfo e = extrema_totals<NS>(L, slot, max_extrema);
  if (N > kThreads * 128 && L.imf[0] == 0.0 && !e.trig) {
    chunk_fallback_check(L, N, tid);
    e = extrema_totals<NS>(L, slot, max_extrema);
  }
  return e;
}

template <int NT>
__device__ __forceinline__ ExtInfo extrema_scan(const SmemLayout& L, int N, int tid, int warp,
                                                int lane, int max_extrema) {
  constexpr int W0 = scan_warp0<NT>();
  if (W0 == 0 || warp >= W0) extrema_count<scan_slots<NT>()>(L, N, warp - W0, lane);
  if (tid == 0) L.ctl->chunk_bad = 0;
  __syncthreads();
  return extrema_finish<NT>(L, N, tid, warp, max_extrema);
}

// ---------------------------------------------------------------------------
// Knot fill: compacted true extrema -> X/Y at offset NB (both sides).
// Returns this thread's "bad envelope sign" vote for true knots.
// ---------------------------------------------------------------------------
// NS slots; the calling warp fills slot `warp` (warps past NS do not call it)
template <int NS>
__device__ __forceinline__ bool fill_true_knots(const SmemLayout& L, const Knots& K,
                                                const ExtInfo& e, int N, int NB,
                                                const TimeAxis& T, int warp, int lane) {
  Ctl& C = *L.ctl;
  const real* imf = L.imf;
  int nch = (N + 31) >> 5;
  int c0 = (warp * nch) / NS, c1 = ((warp + 1) * nch) / NS;
  unsigned lt = (1u << lane) - 1u;
  bool bad = false;
  // one extremum lane: rank it, write its knot, note head / tail indices
  auto put = [&](uint32_t bm, uint32_t bn, int pm, int pn, int ii, real v) {
    const bool ismax = (bm >> lane) & 1u;
    int q = ismax ? 0 : 1;
    int rank = q == 0 ? e.off_max + pm + __popc(bm & lt)
                      : e.off_min + pn + __popc(bn & lt);
    int nq = q == 0 ? e.n_max : e.n_min;
    if (rank < nq) {
      real* Xq = q == 0 ? K.X[0] : K.X[1];
      real* Yq = q == 0 ? K.Y[0] : K.Y[1];
      Xq[NB + rank] = T(ii);
      Yq[NB + rank] = v;
      bad |= q == 0 ? (v < 0.0) : (v > 0.0);
      if (rank <= NB) C.head[q][rank] = ii;
      int fe = nq - 1 - rank;
      if (fe <= NB) C.tail[q][fe] = ii;
    }
  };
  if (!e.trig) {
    // no exact zeros or flat runs in this proto-IMF: every extremum is strict
#pragma unroll kFillUnroll
    for (int c = c0; c < c1; ++c) {
      const uint32_t bm = L.mmax[c], bn = L.mmin[c];
      const int pm = L.pmax[c], pn = L.pmin[c];
      if (((bm | bn) >> lane) & 1u) {
        const int i = (c << 5) + lane;
        put(bm, bn, pm, pn, i, imf[i]);
      }
    }
  } else {
    for (int c = c0; c < c1; ++c) {
      const uint32_t bm = L.mmax[c], bn = L.mmin[c];
      const int pm = L.pmax[c], pn = L.pmin[c];
      if (!(((bm | bn) >> lane) & 1u)) continue;
      int i = (c << 5) + lane;
      int ii = i;
      real v = imf[i];
      real dp = v - imf[i - 1], dn = imf[i + 1] - v;
      if (!(dp * dn < 0.0)) {       // plateau extremum: report the run's midpoint
        int j = i;
        while (j + 1 < N && imf[j + 1] == v) ++j;
        ii = (i + j) / 2;
        v = imf[ii];
      }
      put(bm, bn, pm, pn, ii, v);
    }
  }
  // the chunks' prefixes become global (warp offset added) for the evaluation
  // pass's segment counts, once every lane has taken its ranks
  __syncwarp();
  for (int c = c0 + lane; c < c1; c += 32) {
    L.pmax[c] = (uint16_t)(L.pmax[c] + e.off_max);
    L.pmin[c] = (uint16_t)(L.pmin[c] + e.off_min);
  }
  return bad;
}

// ---------------------------------------------------------------------------
// Boundary mirroring (mirror_one_side, kernels.py:360-558) for both sides.
// Lane 0 of warp 0 makes the O(nbsym) decisions into shared lists; the warp
// then writes the mirrored knots.  Knot positions are strictly increasing
// whenever T is (the host checks T), so the reference's adjacent-duplicate
// removal never drops a knot and is not needed here.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ind_of(const Ctl& C, int q, int n, int NB, int k) {
  return k <= NB ? C.head[q][k] : C.tail[q][n - 1 - k];
}

__device__ __forceinline__ bool mirror_both(const SmemLayout& L, const Knots& K, const ExtInfo& e,
                                            int N, int NB, const TimeAxis& T, int lane) {
  Ctl& C = *L.ctl;
  const real* S = L.imf;
  const int nM = e.n_max, nm = e.n_min;
  if (lane == 0) {
    int* l0 = C.mlist[0];
    int* l1 = C.mlist[1];
    int* r0 = C.mlist[2];
    int* r1 = C.mlist[3];
    int c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    int lsym, rsym;
    const int im0 = ind_of(C, 0, nM, NB, 0), in0 = ind_of(C, 1, nm, NB, 0);
    const int imL = ind_of(C, 0, nM, NB, nM - 1), inL = ind_of(C, 1, nm, NB, nm - 1);
    // ---- left bound ----
    if (im0 < in0) {
      if (S[0] > S[in0]) {
        for (int k = min(nM, NB + 1) - 1; k >= 1; --k) l0[c0++] = ind_of(C, 0, nM, NB, k);
        for (int k = min(nm, NB) - 1; k >= 0; --k) l1[c1++] = ind_of(C, 1, nm, NB, k);
        lsym = im0;
      } else {
        for (int k = min(nM, NB) - 1; k >= 0; --k) l0[c0++] = ind_of(C, 0, nM, NB, k);
        for (int k = min(nm, NB - 1) - 1; k >= 0; --k) l1[c1++] = ind_of(C, 1, nm, NB, k);
        l1[c1++] = 0;
        lsym = 0;
      }
    } else {
      if (S[0] < S[im0]) {
        for (int k = min(nM, NB) - 1; k >= 0; --k) l0[c0++] = ind_of(C, 0, nM, NB, k);
        for (int k = min(nm, NB + 1) - 1; k >= 1; --k) l1[c1++] = ind_of(C, 1, nm, NB, k);
        lsym = in0;
      } else {
        for (int k = min(nM, NB - 1) - 1; k >= 0; --k) l0[c0++] = ind_of(C, 0, nM, NB, k);
        l0[c0++] = 0;
        for (int k = min(nm, NB) - 1; k >= 0; --k) l1[c1++] = ind_of(C, 1, nm, NB, k);
        lsym = 0;
      }
    }
    // ---- right bound ----
    if (imL < inL) {
      if (S[N - 1] < S[imL]) {
        for (int k = nM - 1; k >= max(nM - NB, 0); --k) r0[c2++] = ind_of(C, 0, nM, NB, k);
        for (int k = nm - 2; k >= max(nm - NB - 1, 0); --k) r1[c3++] = ind_of(C, 1, nm, NB, k);
        rsym = inL;
      } else {
        r0[c2++] = N - 1;
        for (int k = max(nM - NB + 1, 0); k < nM; ++k) r0[c2++] = ind_of(C, 0, nM, NB, k);
        for (int k = nm - 1; k >= max(nm - NB, 0); --k) r1[c3++] = ind_of(C, 1, nm, NB, k);
        rsym = N - 1;
      }
    } else {
      if (S[N - 1] > S[inL]) {
        for (int k = nM - 2; k >= max(nM - NB - 1, 0); --k) r0[c2++] = ind_of(C, 0, nM, NB, k);
        for (int k = nm - 1; k >= max(nm - NB, 0); --k) r1[c3++] = ind_of(C, 1, nm, NB, k);
        rsym = imL;
      } else {
        for (int k = nM - 1; k >= max(nM - NB, 0); --k) r0[c2++] = ind_of(C, 0, nM, NB, k);
        r1[c3++] = N - 1;
        for (int k = max(nm - NB + 1, 0); k < nm; ++k) r1[c3++] = ind_of(C, 1, nm, NB, k);
        rsym = N - 1;
      }
    }
    // An empty list falls back to the whole index list (kernels.py:456-459,
    // 523-531); that only happens when the side has exactly one extremum,
    // so the whole list is that one index.
    if (c0 == 0) l0[c0++] = im0;
    if (c1 == 0) l1[c1++] = in0;
    if (c2 == 0) r0[c2++] = imL;
    if (c3 == 0) r1[c3++] = inL;
    // ---- mirrored point does not reach the boundary (kernels.py:469-503) ----
    const real T0 = T(0), TN = T(N - 1);
    real tl = T(lsym);
    // the mirrored positions are stored as REAL_T before the compares
    // (kernels.py:471-472, 488-489): in the FP32 build that rounds them
    const real tl1 = 2.0 * tl - T(l1[0]), tl0 = 2.0 * tl - T(l0[0]);
    if (tl1 > T0 || tl0 > T0) {
      if (lsym == im0) {
        c0 = 0;
        for (int k = min(nM, NB) - 1; k >= 0; --k) l0[c0++] = ind_of(C, 0, nM, NB, k);
      } else {
        c1 = 0;
        for (int k = min(nm, NB) - 1; k >= 0; --k) l1[c1++] = ind_of(C, 1, nm, NB, k);
      }
      lsym = 0;
    }
    real tr = T(rsym);
    const real tr1 = 2.0 * tr - T(r1[c3 - 1]), tr0 = 2.0 * tr - T(r0[c2 - 1]);
    if (tr1 < TN || tr0 < TN) {
      if (rsym == imL) {
        c2 = 0;
        for (int k = nM - 1; k >= max(nM - NB, 0); --k) r0[c2++] = ind_of(C, 0, nM, NB, k);
      } else {
        c3 = 0;
        for (int k = nm - 1; k >= max(nm - NB, 0); --k) r1[c3++] = ind_of(C, 1, nm, NB, k);
      }
      rsym = N - 1;
    }
    C.mcnt[0] = c0; C.mcnt[1] = c1; C.mcnt[2] = c2; C.mcnt[3] = c3;
    C.lsym = lsym;
    C.rsym = rsym;
    C.kbase[0] = NB - c0;
    C.kbase[1] = NB - c1;
    C.kcnt[0] = c0 + nM + c2;
    C.kcnt[1] = c1 + nm + c3;
  }
  __syncwarp();
  // lanes write the mirrored knots: entry j of list q (0 lmax, 1 lmin, 2 rmax, 3 rmin)
  bool bad = false;
  for (int ent = lane; ent < 4 * (kMaxNbsym + 1); ent += 32) {
    int q = ent / (kMaxNbsym + 1), j = ent % (kMaxNbsym + 1);
    int cq = C.mcnt[q];
    if (j >= cq) continue;
    int idx = C.mlist[q][j];
    int side = q & 1;
    bool left = q < 2;
    real pos = 2.0 * T(left ? C.lsym : C.rsym) - T(idx);
    real val = S[idx];
    int nside = side == 0 ? nM : nm;
    int slot = left ? (NB - cq + j) : (NB + nside + j);
    (side == 0 ? K.X[0] : K.X[1])[slot] = pos;
    (side == 0 ? K.Y[0] : K.Y[1])[slot] = val;
    bad |= side == 0 ? (val < 0.0) : (val > 0.0);
  }
  return bad;
}

// ---------------------------------------------------------------------------
// Not-a-knot spline: reduced system + PCR + moments (kernels.py:607-697).
// ---------------------------------------------------------------------------
// kInt: integer time axis (T = arange), where knot spacings are integers and
// the interior rows' slope quotients take RN(1/h) from the table and the exact
// two-step Markstein quotient (div_q) instead of two divisions; spacings
// outside the table (or not positive integers, as unsorted knot lists can
// give) take the divisions.
template <bool kInt = false>
__device__ __forceinline__ void setup_row(const real* x, const real* y, int n, int k, int m,
                                          real& a, real& b, real& c, real& d) {
  if (k == 0) {
    real h0 = x[1] - x[0], h1 = x[2] - x[1];
    real rhs1 = 6.0 * ((y[2] - y[1]) / h1 - (y[1] - y[0]) / h0);
    a = 0.0; b = h0 + 2.0 * h1; c = h1 - h0; d = h1 * rhs1 / (h0 + h1);
  } else if (k == m - 1) {
    real hnm3 = x[n - 2] - x[n - 3], hnm2 = x[n - 1] - x[n - 2];
    real rhs = 6.0 * ((y[n - 1] - y[n - 2]) / hnm2 - (y[n - 2] - y[n - 3]) / hnm3);
    a = hnm3 - hnm2; b = 2.0 * hnm3 + hnm2; c = 0.0; d = hnm3 * rhs / (hnm3 + hnm2);
  } else {
    int i = k + 1;
    real h_im1 = x[i] - x[i - 1], h_i = x[i + 1] - x[i];
    a = h_im1; b = 2.0 * (h_im1 + h_i); c = h_i;
#if EMDB_SETUP_NB
    bool slow = false;
    const real sr = div_nb(y[i + 1] - y[i], h_i, slow);
    const real sl = div_nb(y[i] - y[i - 1], h_im1, slow);
    d = slow ? 6.0 * ((y[i + 1] - y[i]) / h_i - (y[i] - y[i - 1]) / h_im1) : 6.0 * (sr - sl);
#else
    if (kInt) {
      const bool ok = h_i >= 1.0 && h_i <= (real)kRcpTab && h_im1 >= 1.0 &&
                      h_im1 <= (real)kRcpTab;
      const int ji = ok ? (int)h_i : 1, jm = ok ? (int)h_im1 : 1;
      bool slow = !ok || (real)ji != h_i || (real)jm != h_im1;
      const real sr = div_q(y[i + 1] - y[i], h_i, g_rcp.v[ji], slow);
      const real sl = div_q(y[i] - y[i - 1], h_im1, g_rcp.v[jm], slow);
      d = slow ? 6.0 * (EMDB_DIV_RARE(y[i + 1] - y[i], h_i) - EMDB_DIV_RARE(y[i] - y[i - 1], h_im1))
               : 6.0 * (sr - sl);
    } else {
      d = 6.0 * ((y[i + 1] - y[i]) / h_i - (y[i] - y[i - 1]) / h_im1);
    }
#endif
  }
}

__device__ __forceinline__ void pcr_row(const real* __restrict__ Pa, real* __restrict__ Pn,
                                        int cap, int r, int k, int s, int mq) {
  const bool hl = k - s >= 0, hr = k + s < mq;
  const int rl = r - s, rr = r + s;
  const real ak = Pa[r], bk = Pa[cap + r], ck = Pa[2 * cap + r], dk = Pa[3 * cap + r];
  const real b_left = hl ? Pa[cap + rl] : 1.0;
  const real b_right = hr ? Pa[cap + rr] : 1.0;
#if EMDB_PCR_NB
  bool sl = false, sr = false;
  const real ql = div_nb(ak, b_left, sl);
  const real qr = div_nb(ck, b_right, sr);
  real alpha = hl ? ql : 0.0;
  real beta = hr ? qr : 0.0;
  if ((hl && sl) || (hr && sr)) {
    alpha = hl ? EMDB_DIV_RARE(ak, b_left) : 0.0;
    beta = hr ? EMDB_DIV_RARE(ck, b_right) : 0.0;
  }
#else
  const real alpha = hl ? ak / b_left : 0.0;
  const real beta = hr ? ck / b_right : 0.0;
#endif
  const real a_left = hl ? Pa[rl] : 0.0;
  const real c_left = hl ? Pa[2 * cap + rl] : 0.0;
  const real d_left = hl ? Pa[3 * cap + rl] : 0.0;
  const real a_right = hr ? Pa[rr] : 0.0;
  const real c_right = hr ? Pa[2 * cap + rr] : 0.0;
  const real d_right = hr ? Pa[3 * cap + rr] : 0.0;
  Pn[r] = -alpha * a_left;
  Pn[2 * cap + r] = -beta * c_right;
  Pn[cap + r] = bk - alpha * c_left - beta * a_right;
  Pn[3 * cap + r] = dk - alpha * d_left - beta * d_right;
}

template <int NT, bool kInt = false>
__device__ __forceinline__ void solve_splines(const Knots& K, int kbase0, int kbase1, int kcnt0,
                                              int kcnt1, int tid, Ctl* C = nullptr) {
  const int m0 = kcnt0 >= 4 ? kcnt0 - 2 : 0;
  const int m1 = kcnt1 >= 4 ? kcnt1 - 2 : 0;
  const int mt = m0 + m1;
  const int cap = K.cap;
  const real* x0b = K.X[0] + kbase0;
  const real* x1b = K.X[1] + kbase1;
  const real* y0b = K.Y[0] + kbase0;
  const real* y1b = K.Y[1] + kbase1;
  for (int r = tid; r < mt; r += NT) {
    const bool s0 = r < m0;
    const int k = s0 ? r : r - m0;
    const real* x = s0 ? x0b : x1b;
    const real* y = s0 ? y0b : y1b;
    real a, b, c, d;
    setup_row<kInt>(x, y, s0 ? kcnt0 : kcnt1, k, s0 ? m0 : m1, a, b, c, d);
    real* P = K.P[0];
    P[r] = a; P[cap + r] = b; P[2 * cap + r] = c; P[3 * cap + r] = d;
  }
  __syncthreads();
  if (C) EMDB_PH(C, 2);
  const int mmax = max(m0, m1);
  int cur = 0;
  int fin0 = 0, fin1 = 0;
  for (int s = 1; s < mmax; s *= 2) {
    const real* __restrict__ Pa = cur ? K.P[1] : K.P[0];
    real* __restrict__ Pn = cur ? K.P[0] : K.P[1];
    // two rows per trip: independent division chains overlap
    constexpr int kPair = NT > kThreads ? EMDB_WIDE_PCR_PAIR : EMDB_PCR_PAIR;
    for (int r = tid; r < mt; r += (1 + kPair) * NT) {
      const int r2 = kPair ? r + NT : mt;
      {
        const bool s0 = r < m0;
        const int mq = s0 ? m0 : m1;
        if (s < mq) pcr_row(Pa, Pn, cap, r, s0 ? r : r - m0, s, mq);
      }
      if (r2 < mt) {
        const bool s0 = r2 < m0;
        const int mq = s0 ? m0 : m1;
        if (s < mq) pcr_row(Pa, Pn, cap, r2, s0 ? r2 : r2 - m0, s, mq);
      }
    }
    if (s < m0) fin0 ^= 1;
    if (s < m1) fin1 ^= 1;
    cur ^= 1;
    // Rows are owned by thread r mod NT, so a level with stride >= NT reads
    // and writes only the calling thread's rows: no barrier is needed before
    // the next such level.  Earlier levels read other threads' rows, and the
    // solve below does too, so those transitions keep the barrier.
    if (s < NT || 2 * s >= mmax) __syncthreads();
  }
  if (C) EMDB_PH(C, 3);
  // diagonal solve + end-moment recovery (M[0], M[n-1] by the owners of the end rows)
  for (int r = tid; r < mt; r += NT) {
    const bool s0 = r < m0;
    const int k = s0 ? r : r - m0;
    const int mq = s0 ? m0 : m1;
    const int n = s0 ? kcnt0 : kcnt1;
    const real* Pf = (s0 ? fin0 : fin1) ? K.P[1] : K.P[0];
    real* M = s0 ? K.M[0] : K.M[1];
    const real* x = s0 ? x0b : x1b;
    real Mk1 = Pf[3 * cap + r] / Pf[cap + r];
    M[k + 1] = Mk1;
#if EMDB_FAST_DIV == 1
    real* R = s0 ? K.R[0] : K.R[1];
    R[k] = 1.0 / (x[k + 1] - x[k]);
    if (k == mq - 1) R[k + 1] = 1.0 / (x[k + 2] - x[k + 1]);
#endif
    if (k == 0) {
      real M2 = Pf[3 * cap + r + 1] / Pf[cap + r + 1];
      real h0 = x[1] - x[0], h1 = x[2] - x[1];
      M[0] = ((h0 + h1) * Mk1 - h0 * M2) / h1;
    }
    if (k == mq - 1) {
      real Mnm3 = Pf[3 * cap + r - 1] / Pf[cap + r - 1];
      real hnm3 = x[n - 2] - x[n - 3], hnm2 = x[n - 1] - x[n - 2];
      M[n - 1] = ((hnm3 + hnm2) * Mk1 - hnm2 * Mnm3) / hnm3;
    }
  }
  __syncthreads();
  if (C) EMDB_PH(C, 4);
}

// One PCR row update (kernels.py:651-668), in the reference's operation order.
struct SideView {
  const real* x;
  const real* y;
  const real* M;
  const real* R;
  int n;          // knots
  int nl, nt;     // mirrored-left and true knots
};

// Envelope value at t in knot segment lo (kernels.py:706-733).
__device__ __forceinline__ real eval_seg(const SideView& s, real t, int lo) {
  const real* x = s.x;
  const real* y = s.y;
  if (s.n == 2) {
    real slope = (y[1] - y[0]) / (x[1] - x[0]);
    return y[0] + slope * (t - x[0]);
  }
  if (s.n == 3) {
    real l0 = (t - x[1]) * (t - x[2]) / ((x[0] - x[1]) * (x[0] - x[2]));
    real l1 = (t - x[0]) * (t - x[2]) / ((x[1] - x[0]) * (x[1] - x[2]));
    real l2 = (t - x[0]) * (t - x[1]) / ((x[2] - x[0]) * (x[2] - x[1]));
    return y[0] * l0 + y[1] * l1 + y[2] * l2;
  }
  real x0 = x[lo], x1 = x[lo + 1];
  real y0 = y[lo], y1 = y[lo + 1];
  real M0 = s.M[lo], M1 = s.M[lo + 1];
  real h = x1 - x0;
  real A = (x1 - t) / h;
  real B = (t - x0) / h;
  return A * y0 + B * y1 + ((A * A * A - A) * M0 + (B * B * B - B) * M1) * (h * h) / 6.0;
}

// eval_seg with the quotients taken from reciprocals (EMDB_FAST_DIV 1..3), in
// the same operation order; sets `slow` when a quotient needs the division,
// and the caller then re-evaluates the sample with eval_seg.
__device__ __forceinline__ real eval_seg_q(const SideView& s, real t, int lo, bool& slow) {
  if (s.n < 4) return EMDB_EVAL_RARE(s, t, lo);
  const real* x = s.x;
  const real* y = s.y;
  real x0 = x[lo], x1 = x[lo + 1];
  real y0 = y[lo], y1 = y[lo + 1];
  real M0 = s.M[lo], M1 = s.M[lo + 1];
  real h = x1 - x0;
#if EMDB_FAST_DIV == 2
  real A = (x1 - t) / h;
  real B = (t - x0) / h;
#else
#if EMDB_FAST_DIV == 1
  real rh = s.R[lo];
#else
  const real rh = real(1) / h;
#endif
  real A = div_q(x1 - t, h, rh, slow);
  real B = div_q(t - x0, h, rh, slow);
#endif
  real num = ((A * A * A - A) * M0 + (B * B * B - B) * M1) * (h * h);
  return (A * y0 + B * y1) + div_q(num, 6.0, kInv6, slow);
}

// The reference's per-sample binary search (kernels.py:722-726).
__device__ __forceinline__ int search_seg(const SideView& s, real t) {
  int lo = 0, hi = s.n - 2;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (s.x[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Out-of-line bodies of the rare paths declared with div_slow.
__device__ __noinline__ real eval_seg_cold(const real* x, const real* y, const real* M,
                                             int n, real t, int lo) {
  SideView s;
  s.x = x; s.y = y; s.M = M; s.R = nullptr; s.n = n; s.nl = 0; s.nt = 0;
  return eval_seg(s, t, lo);
}
__device__ __noinline__ int search_seg_cold(const real* x, int n, real t) {
  SideView s;
  s.x = x; s.y = nullptr; s.M = nullptr; s.R = nullptr; s.n = n; s.nl = 0; s.nt = 0;
  return search_seg(s, t);
}

// 128-lane tree of the reference (kernels.py:794-804), on warp 0, for a value
// each thread has stored at red[q*128 + tid].  op 0: sum, 1: fmax, 2: fmin.
__device__ __forceinline__ real lane_tree(const real* red, int lane, int op) {
  real v0 = red[lane], v1 = red[lane + 32], v2 = red[lane + 64], v3 = red[lane + 96];
  real r;
  if (op == 0) r = (v0 + v2) + (v1 + v3);
  else if (op == 1) r = fmax(fmax(v0, v2), fmax(v1, v3));
  else r = fmin(fmin(v0, v2), fmin(v1, v3));
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    real o = __shfl_down_sync(kFull, r, s);
    if (op == 0) r = r + o;
    else if (op == 1) r = fmax(r, o);
    else r = fmin(r, o);
  }
  return r;
}

struct PassSums {
  real sq, dsq, osq, std_, omax, omin;
  bool bad;
  bool oor;
};

__device__ __forceinline__ void accumulate(PassSums& ps, real old, real nw) {
  real diff = nw - old;
  ps.sq += nw * nw;
  ps.dsq += diff * diff;
  ps.osq += old * old;
#if EMDB_ACC_NB
  bool slow = false;
  real qd = div_nb(diff, nw, slow);
  if (slow) qd = diff / nw;
#else
  real qd = diff / nw;
#endif
  ps.std_ += qd * qd;
  ps.omax = fmax(ps.omax, old);
  ps.omin = fmin(ps.omin, old);
}

// The wide instances' stop-test sums after the update (new values in imf[],
// old ones in oldv[], quotients (new-old)/new in qbuf[]): the reference's 128
// lanes, lane l adding samples l, l+128, ... in increasing order exactly as
// accumulate() does.  The six sums are independent chains, so the CTA's
// 128-thread groups take them apart -- 512 threads: Σnew² | Σdiff² |
// Σold², max, min | Σquotient²; 256 threads: the first two | the rest --
// and write the lanes' partials to red[128 * sum + l] for the trees.
template <int NT>
__device__ __forceinline__ void wide_lane_sums(real* red, const real* __restrict__ oldv,
                                               const real* imf, const real* __restrict__ qbuf,
                                               int N, int tid) {
  constexpr int NG = NT / kThreads;
  static_assert(NG == 2 || NG == 4, "wide instances have 256 or 512 threads");
  const int g = tid / kThreads, l = tid % kThreads;
  if (g == 0) {
    real s = 0.0, s2 = 0.0;
#pragma unroll kLaneUnroll
    for (int i = l; i < N; i += kThreads) {
      const real nw = imf[i];
      s += nw * nw;
      if (NG == 2) {
        const real diff = nw - oldv[i];
        s2 += diff * diff;
      }
    }
    red[l] = s;
    if (NG == 2) red[128 + l] = s2;
  } else if (NG == 4 && g == 1) {
    real s = 0.0;
#pragma unroll kLaneUnroll
    for (int i = l; i < N; i += kThreads) {
      const real diff = imf[i] - oldv[i];
      s += diff * diff;
    }
    red[128 + l] = s;
  } else if (g == NG / 2) {
    real s = 0.0, mx = -1e30, mn = 1e30, sq = 0.0;
#pragma unroll kLaneUnroll
    for (int i = l; i < N; i += kThreads) {
      const real old = oldv[i];
      s += old * old;
      mx = fmax(mx, old);
      mn = fmin(mn, old);
      if (NG == 2) {
        const real q = qbuf[i];
        sq += q * q;
      }
    }
    red[256 + l] = s;
    red[512 + l] = mx;
    red[640 + l] = mn;
    if (NG == 2) red[384 + l] = sq;
  } else if (NG == 4 && g == 3) {
    real s = 0.0;
#pragma unroll kLaneUnroll
    for (int i = l; i < N; i += kThreads) {
      const real q = qbuf[i];
      s += q * q;
    }
    red[384 + l] = s;
  }
}

// eval_seg for the time axis T = arange(N): knot positions (true and
// mirrored) and sample times are integers, so A = (x1-t)/h and B = (t-x0)/h
// are quotients of integers 0 <= a <= h.  For those, q0 = RN(a*y) with
// y = RN(1/h) and one correction RN(q0 + (a - h*q0)*y) equal RN(a/h): checked
// exhaustively for every pair with h <= 65536 (2.1e9 pairs).  Anything outside
// (h beyond the table, a not in [0, h]) sets `slow`, and the caller redoes the
// sample with eval_seg.  Same operation order as eval_seg otherwise.
#if !EMDB_F32
__device__ __forceinline__ real eval_seg_int(const SideView& s, real t, int lo, bool& slow,
                                               bool sorted = false) {
  if (s.n < 4) return EMDB_EVAL_RARE(s, t, lo);
  const real* x = s.x;
  const real* y = s.y;
  real x0 = x[lo], x1 = x[lo + 1];
  real y0 = y[lo], y1 = y[lo + 1];
  real M0 = s.M[lo], M1 = s.M[lo + 1];
  real h = x1 - x0;
  const real a = x1 - t, b = t - x0;
  int hi;
  if (EMDB_SORTED_NOCHECK && sorted) {
    // strictly increasing integer knots and the segment that holds t: h is an
    // integer >= 1 and a, b lie in [0, h]; only the table bound is left
    const bool in = h <= (real)kRcpTab;
    hi = in ? (int)h : 1;
    slow |= !in;
  } else {
    const bool in = h >= 1.0 && h <= (real)kRcpTab && a >= 0.0 && b >= 0.0 && a <= h && b <= h;
    hi = in ? (int)h : 1;
    slow |= !in || (real)hi != h;
  }
  const real r = g_rcp.v[hi];
  real A = a * r;
  A = fma(fma(-A, h, a), r, A);
  real B = b * r;
  B = fma(fma(-B, h, b), r, B);
  real num = ((A * A * A - A) * M0 + (B * B * B - B) * M1) * (h * h);
  return (A * y0 + B * y1) + div_q(num, 6.0, kInv6, slow);
}
#endif

// One sift pass after the extrema scan of the current proto-IMF: knots,
// mirroring, both splines, then the fused envelope / mean / update / partial
// sums.  kPlace selects where the knots live: shared memory (the common case),
// split between shared memory and the per-CTA global slab, or the slab alone.
//
// NT > 128 (the wide instance, one long trace per CTA): every thread
// evaluates samples, but the stop-test sums keep the reference's 128 lanes,
// each adding its samples in order.  So the proto-IMF is always parked in
// `park_old` (global, per CTA) while warp 0 mirrors, the evaluation writes the
// update to imf[] and its quotient diff/new to `qbuf`, and the first 128
// threads then sum old / new / quotient per lane exactly as accumulate() does.
template <int NT, int kGroup, bool kInt>
__device__ __forceinline__ int sift_pass(const SmemLayout& L, char* slab, const ExtInfo& e,
                                              int N, int NB, const TimeAxis& T, int tid, int warp,
                                              int lane, int place = kPlaceSmem,
                                              real* park_old = nullptr, real* qbuf = nullptr) {
  constexpr bool kWide = NT > kThreads;
  // kGroup >= 0: one placement, fixed at compile time.  kGroup == kOnChip /
  // kOffChip: one instance for the on-chip (shared, borrow) or off-chip
  // (split, park, slab) placements, chosen by `place` at run time.
  const int kPlace = kGroup >= 0 ? kGroup
                   : kGroup == kOnChip ? ((place == kPlaceBorrow || place == kPlaceBorrow2)
                                              ? kPlaceBorrow : kPlaceSmem)
                   : kGroup == kOffChip ? (place == kPlaceSplit ? kPlaceSplit
                                           : place == kPlacePark ? kPlacePark : kPlaceSlab)
                                        : place;
  Ctl& C = *L.ctl;
  real* imf = L.imf;
  const int kc0 = e.n_max + 2 * NB + 2, kc1 = e.n_min + 2 * NB + 2;
  Knots K = kPlace == kPlaceSmem    ? place_knots(L.arena, kc0, kc1)
           : kPlace == kPlaceSplit  ? place_knots_split(L.arena, L.arena_bytes, slab, kc0, kc1)
           : kPlace == kPlaceBorrow ? (place == kPlaceBorrow2
                                          ? place_knots_borrow2(imf, L.arena, L.arena_bytes, slab, N, kc0, kc1)
                                          : place_knots_borrow(imf, L.arena, L.arena_bytes, slab, N, kc0, kc1))
           : kPlace == kPlaceBorrow2 ? place_knots_borrow2(imf, L.arena, L.arena_bytes, slab, N, kc0, kc1)
           : kPlace == kPlacePark   ? place_knots_park(imf, slab, N, kc0, kc1, L.red)
                                    : place_knots(slab, kc0, kc1);
  PassSums ps;
  EMDB_PH(&C, 9);
  constexpr int NS = scan_slots<NT>();
  bool bad = false;
  if (NS == NT / 32 || warp < NS) bad = fill_true_knots<NS>(L, K, e, N, NB, T, warp, lane);
  bad = __syncthreads_or(bad);
  EMDB_PH(&C, 0);
  bool mbad = false;
  if (warp == 0) {
    mbad = mirror_both(L, K, e, N, NB, T, lane);
  } else if (kWide) {
    // park the proto-IMF while warp 0 mirrors: the lanes read the old samples
    // back after the update (and the PCR buffers may overwrite imf[])
    for (int i = tid - 32; i < N; i += NT - 32) park_old[i] = imf[i];
  } else if (kPlace == kPlaceBorrow || kPlace == kPlaceBorrow2 || kPlace == kPlacePark) {
    // park the proto-IMF while warp 0 mirrors; the PCR buffers overwrite it
    real* save = borrow_save(slab);
    for (int i = tid - 32; i < N; i += kThreads - 32) save[i] = imf[i];
  }
  ps.bad = __syncthreads_or(bad || mbad) != 0;
  EMDB_PH(&C, 1);
  const int kb0 = C.kbase[0], kb1 = C.kbase[1], kn0 = C.kcnt[0], kn1 = C.kcnt[1];
  solve_splines<NT, kInt && EMDB_SETUP_TAB>(K, kb0, kb1, kn0, kn1, tid,
                                             EMDB_LOAD_CLOCKS ? &C : nullptr);
  const real* oldv = kWide ? park_old
                     : (kPlace == kPlaceBorrow || kPlace == kPlaceBorrow2 || kPlace == kPlacePark)
                            ? borrow_save(slab) : imf;

  SideView sv0, sv1;
  sv0.x = K.X[0] + kb0; sv0.y = K.Y[0] + kb0; sv0.M = K.M[0]; sv0.R = K.R[0];
  sv0.n = kn0; sv0.nl = NB - kb0; sv0.nt = e.n_max;
  sv1.x = K.X[1] + kb1; sv1.y = K.Y[1] + kb1; sv1.M = K.M[1]; sv1.R = K.R[1];
  sv1.n = kn1; sv1.nl = NB - kb1; sv1.nt = e.n_min;

  ps.sq = ps.dsq = ps.osq = ps.std_ = 0.0;
  ps.omax = -1e30;
  ps.omin = 1e30;
  bool oor = false;
  // O(1) segments: for a strictly increasing knot list (nbsym <= 2, no flat
  // runs -- a plateau extremum sits at the run's midpoint, not at its flagged
  // first sample) the reference's binary search returns (number of knots at
  // or left of t) - 1, clamped to [0, n-2].  Otherwise run the search.
  const bool fast = NB <= 2 && !e.trig;
  const int nch = (N + 31) >> 5;
  // chunk c = (tid>>5) + 4j is scanned by warp wc(c); its rank offset is woff[wc] + pre[c]
  // mirrored knots of both envelopes, for the O(1) segment count (nbsym <= 2)
  constexpr real kInf = __builtin_huge_val();
  const real l00 = sv0.nl > 0 ? sv0.x[0] : kInf, l01 = sv0.nl > 1 ? sv0.x[1] : kInf;
  const real l10 = sv1.nl > 0 ? sv1.x[0] : kInf, l11 = sv1.nl > 1 ? sv1.x[1] : kInf;
  const int nr0 = sv0.n - sv0.nl - sv0.nt, nr1 = sv1.n - sv1.nl - sv1.nt;
  const real r00 = nr0 > 0 ? sv0.x[sv0.nl + sv0.nt] : kInf, r01 = nr0 > 1 ? sv0.x[sv0.nl + sv0.nt + 1] : kInf;
  const real r10 = nr1 > 0 ? sv1.x[sv1.nl + sv1.nt] : kInf, r11 = nr1 > 1 ? sv1.x[sv1.nl + sv1.nt + 1] : kInf;
  (void)nch;
  const unsigned incl = lane == 31 ? kFull : ((2u << lane) - 1u);
  // knot segment of sample i for both envelopes
  auto segs = [&](int i, real t, int& lo0, int& lo1) {
    lo0 = 0;
    lo1 = 0;
    if (fast) {
      // knots at or left of t: mirrored ones compared directly, true ones
      // counted from the scan's ballot masks (global chunk prefix + popc)
      const int c = i >> 5;
      int k0 = min((int)L.pmax[c] + __popc(L.mmax[c] & incl), sv0.nt);
      int k1 = min((int)L.pmin[c] + __popc(L.mmin[c] & incl), sv1.nt);
      k0 += (l00 <= t) + (l01 <= t) + (r00 <= t) + (r01 <= t);
      k1 += (l10 <= t) + (l11 <= t) + (r10 <= t) + (r11 <= t);
      lo0 = min(max(k0 - 1, 0), sv0.n - 2);
      lo1 = min(max(k1 - 1, 0), sv1.n - 2);
    } else {
      if (sv0.n >= 4) lo0 = EMDB_SEARCH_RARE(sv0, t);
      if (sv1.n >= 4) lo1 = EMDB_SEARCH_RARE(sv1, t);
    }
  };
  // T is strictly increasing, so the knot spans cover every sample iff they
  // cover the first and the last one
  if (N > 0) {
    const real t0 = T(0), tN = T(N - 1);
    oor = (t0 < sv0.x[0]) || (tN > sv0.x[sv0.n - 1]) || (t0 < sv1.x[0]) || (tN > sv1.x[sv1.n - 1]);
  }
  // two samples per trip (i, i+NT): independent evaluation chains overlap;
  // each lane still accumulates its samples in increasing order
  for (int i = tid; i < N; i += (1 + EMDB_EVAL_PAIR) * NT) {
    const int i2 = i + NT;
    const bool has2 = EMDB_EVAL_PAIR && i2 < N;
    const real t = T(i);
    const real t2 = has2 ? T(i2) : t;
    int lo0, lo1, lo0b, lo1b;
    segs(i, t, lo0, lo1);
    if (has2) segs(i2, t2, lo0b, lo1b); else { lo0b = lo0; lo1b = lo1; }
#if EMDB_FAST_DIV
    bool slow = false;
    real emax, emin, emax2 = 0.0, emin2 = 0.0;
#if !EMDB_F32
    // (the FP32 build has no integer-axis shortcut: a float quotient formed
    // in double from the table's RN(1/h) would be rounded twice)
    if (kInt) {
      emax = eval_seg_int(sv0, t, lo0, slow, fast);
      emin = eval_seg_int(sv1, t, lo1, slow, fast);
      if (has2) {
        emax2 = eval_seg_int(sv0, t2, lo0b, slow, fast);
        emin2 = eval_seg_int(sv1, t2, lo1b, slow, fast);
      }
    } else
#endif
    {
      emax = eval_seg_q(sv0, t, lo0, slow);
      emin = eval_seg_q(sv1, t, lo1, slow);
      if (has2) {
        emax2 = eval_seg_q(sv0, t2, lo0b, slow);
        emin2 = eval_seg_q(sv1, t2, lo1b, slow);
      }
    }
    if (slow) {
      emax = EMDB_EVAL_RARE(sv0, t, lo0);
      emin = EMDB_EVAL_RARE(sv1, t, lo1);
      emax2 = EMDB_EVAL_RARE(sv0, t2, lo0b);
      emin2 = EMDB_EVAL_RARE(sv1, t2, lo1b);
    }
#else
    const real emax = eval_seg(sv0, t, lo0);
    const real emin = eval_seg(sv1, t, lo1);
    const real emax2 = eval_seg(sv0, t2, lo0b);
    const real emin2 = eval_seg(sv1, t2, lo1b);
#endif
    if (kWide) {
      // the update, and accumulate()'s quotient from the same operands
      const real old = oldv[i];
      const real mean = 0.5 * (emax + emin);
      const real nw = old - mean;
      imf[i] = nw;
      qbuf[i] = (nw - old) / nw;
      continue;
    }
    {
      const real mean = 0.5 * (emax + emin);
      const real old = oldv[i];
      const real nw = old - mean;
      imf[i] = nw;
      accumulate(ps, old, nw);
    }
    if (has2) {
      const real mean = 0.5 * (emax2 + emin2);
      const real old = oldv[i2];
      const real nw = old - mean;
      imf[i2] = nw;
      accumulate(ps, old, nw);
    }
  }
  // per-lane partial sums, then the reference's 128-lane trees on warp 0
  real* red = kPlace == kPlaceSlab ? L.red : K.red;
  if constexpr (kWide && !EMDB_WIDE_OVERLAP) {
    __syncthreads();
    EMDB_PH(&C, 5);
    wide_lane_sums<NT>(red, oldv, imf, qbuf, N, tid);
  } else if (kWide) {
    // the reference's 128 lanes, each summing its samples in increasing order;
    // meanwhile the other warps run the next pass's extrema count on the
    // updated proto-IMF (both only read it)
    __syncthreads();
    EMDB_PH(&C, 5);
    if (tid < kThreads) {
      for (int i = tid; i < N; i += kThreads) {
        const real old = oldv[i], nw = imf[i], qd = qbuf[i];
        const real diff = nw - old;
        ps.sq += nw * nw;
        ps.dsq += diff * diff;
        ps.osq += old * old;
        ps.std_ += qd * qd;
        ps.omax = fmax(ps.omax, old);
        ps.omin = fmin(ps.omin, old);
      }
    } else if (EMDB_WIDE_OVERLAP) {
      extrema_count<scan_slots<NT>()>(L, N, warp - scan_warp0<NT>(), lane);
    }
    if (EMDB_WIDE_OVERLAP && tid == 0) C.chunk_bad = 0;
  }
  if (!kWide || (EMDB_WIDE_OVERLAP && tid < kThreads)) {
    red[tid] = ps.sq; red[128 + tid] = ps.dsq; red[256 + tid] = ps.osq;
    red[384 + tid] = ps.std_; red[512 + tid] = ps.omax; red[640 + tid] = ps.omin;
  }
  __syncthreads();
  EMDB_PH(&C, kWide ? 6 : 5);
#if EMDB_TREE_SPLIT
  // the six trees spread over the warps (warp w: sum w; warps 0/1 also the
  // max / min tree); the next extrema scan's barrier publishes C.sums
  if (!kWide || warp < kWarps) {
    const real a = lane_tree(red + 128 * warp, lane, 0);
    if (lane == 0) C.sums[warp] = a;
    if (warp < 2) {
      const real b = lane_tree(red + 128 * (4 + warp), lane, 1 + warp);
      if (lane == 0) C.sums[4 + warp] = b;
    }
  }
  // overlapped scan: this barrier publishes C.sums (the scan's would have)
  if (kWide && EMDB_WIDE_OVERLAP) __syncthreads();
#else
  if (warp == 0) {
    real a0 = lane_tree(red, lane, 0);
    real a1 = lane_tree(red + 128, lane, 0);
    real a2 = lane_tree(red + 256, lane, 0);
    real a3 = lane_tree(red + 384, lane, 0);
    real a4 = lane_tree(red + 512, lane, 1);
    real a5 = lane_tree(red + 640, lane, 2);
    if (lane == 0) {
      C.sums[0] = a0; C.sums[1] = a1; C.sums[2] = a2;
      C.sums[3] = a3; C.sums[4] = a4; C.sums[5] = a5;
    }
  }
#endif
  return (ps.bad ? 1 : 0) | (oor ? 2 : 0);
}

}  // namespace

// ---------------------------------------------------------------------------
// The sift kernel.
// ---------------------------------------------------------------------------
// Chunk completion for the host-memory pipeline (emdb_run_host): after the
// barrier that follows every output write of trace b, thread 0 raises its
// chunk's row maximum to the trace's count of rows that may hold data (rows
// beyond it are zero) and counts the trace in the chunk's device counter; the CTA that
// completes the chunk publishes it with one store of 1 + the chunk's row
// maximum to the chunk's flag in mapped host memory, so the host can copy just
// those rows of that chunk back while the rest of the batch sifts.  The device
// fence before the count and the system fence before the flag order all the
// chunk's output writes (from every CTA that counted) before the flag.
__device__ __forceinline__ void mark_trace_done(const SiftParams& p, int b, int tid, int nim) {
  if (p.chunk_count == nullptr || tid != 0) return;
  const int c = b / p.chunk_traces;
  atomicMax(p.chunk_rows + c, (unsigned)max(nim, 0));
  __threadfence();
  const unsigned need = (unsigned)min(p.chunk_traces, p.chunk_span - c * p.chunk_traces);
  if (atomicAdd(p.chunk_count + c, 1u) + 1u == need) {
    const unsigned rows = atomicMax(p.chunk_rows + c, 0u);
    __threadfence_system();
    *reinterpret_cast<volatile unsigned*>(p.chunk_flag + c) = 1u + rows;
  }
}

// NT threads per CTA: 128 (the reference's lanes), or 512 for the wide
// instance that gives one long trace a whole SM.  kMinBlocks is the
// register-budget variant: the compiler fits the kernel into
// 65536 / (NT * kMinBlocks) registers so that many CTAs can be resident.
// kGImf (wide only): the proto-IMF in the global slab, for traces longer than
// shared memory holds.
// kTail: the build that takes part in tail migration -- a 128/256-thread
// instance that hands its last traces over, or the 512-thread instance that
// resumes them (p.resume).  The other builds carry none of its code.
template <int NT, int kMinBlocks, bool kInt, bool kGImf = false, bool kTail = false>
__global__ void __launch_bounds__(NT, kMinBlocks) emd_sift_kernel(SiftParams p) {
  constexpr bool kWide = NT > kThreads;
  static_assert(!kGImf || kWide, "the global proto-IMF is built for the wide instance");
  extern __shared__ __align__(16) char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int NB = p.nbsym;
  const int MAXI = p.max_imfs;
  Ctl* Cs = reinterpret_cast<Ctl*>(smem);
  char* slab = p.slab + (size_t)blockIdx.x * p.slab_stride;
  // wide instance: the parked proto-IMF and the stop-test quotients (and the
  // proto-IMF itself for kGImf), past the knot slab in this CTA's stride
  real* park_old = kWide ? reinterpret_cast<real*>(slab + p.park_off) : nullptr;
  real* qbuf = kWide ? reinterpret_cast<real*>(slab + p.q_off) : nullptr;
  real* gimf = kGImf ? reinterpret_cast<real*>(slab + p.imf_off) : nullptr;

  // this launch may hand over its tail / resumes another launch's tail
  const bool migrate = kTail && !kWide && p.cont_buf != nullptr;
  const bool resume = kTail && kWide && p.resume != 0;
  for (;;) {
    if (tid == 0) Cs->job = atomicAdd(resume ? p.cont_ticket : p.queue, 1);
    __syncthreads();
    const int job = Cs->job;
    // a resume launch takes the continuation records instead of the queue
    const ContHead* rec = nullptr;
    if (resume) {
      if (job >= p.cont_cap) break;
      if (!p.cont_valid[job]) {
        __syncthreads();          // every thread has read Cs->job before it is reused
        continue;
      }
      rec = reinterpret_cast<const ContHead*>(p.cont_buf + (size_t)job * p.cont_stride);
    } else if (job >= p.batch) {
      break;
    }
    const int b = rec ? rec->b : p.order ? p.order[job] : job;
    const int64_t off = p.offsets ? p.offsets[b] : (int64_t)b * p.dense_n;
    const int N = p.offsets ? (int)(p.offsets[b + 1] - off) : p.dense_n;
    const real* S = p.values + off;
    real* out = p.imfs + (int64_t)MAXI * off;
    TimeAxis T;
    T.arange = p.t_mode == kTArange;
    T.T = p.t_mode == kTShared ? p.T : (p.t_mode == kTPerTrace ? p.T + off : nullptr);

    if (fixed_bytes<NT, kGImf>(N) + kRedBytes + 64 > (size_t)p.arena_bytes ||
        (kWide && p.q_off + (size_t)N * sizeof(real) > p.slab_stride) ||
        (kGImf && p.imf_off + (size_t)N * sizeof(real) > p.slab_stride)) {
      // cannot hold this trace: report, leave outputs flagged
      if (tid == 0) {
        atomicOr(p.status, kStatusTooLong);
        p.n_imfs[b] = 0;
        p.overflow[b] = 1;
      }
      for (int k = tid; k < MAXI; k += NT) {
        p.dbg_n[(int64_t)b * MAXI + k] = -1;
        p.dbg_ext[(int64_t)b * MAXI + k] = -1;
        p.dbg_nzm[(int64_t)b * MAXI + k] = -1;
      }
      __syncthreads();
      mark_trace_done(p, b, tid, MAXI);     // rows unwritten: the host copies them all
      continue;
    }
    SmemLayout L = carve<NT, kGImf>(smem, N, p.arena_bytes, gimf);
    Ctl& C = *L.ctl;
    real* imf = L.imf;
    if (migrate && tid == 0) atomicAdd(p.active, 1);
    for (int k = tid; k < MAXI; k += NT) {
      C.dbg_n[k] = rec ? rec->dbg[0][k] : -1;
      C.dbg_e[k] = rec ? rec->dbg[1][k] : -1;
      C.dbg_z[k] = rec ? rec->dbg[2][k] : -1;
    }
#if EMDB_LOAD_CLOCKS
    const long long clk_trace0 = clock64();
#endif
    {
      // a resumed trace restarts from its parked proto-IMF
      const real* src = rec ? reinterpret_cast<const real*>(reinterpret_cast<const char*>(rec) +
                                                          cont_data_off())
                            : S;
      for (int i = tid; i < N; i += NT) imf[i] = src[i];
    }
    __syncthreads();
#if EMDB_LOAD_CLOCKS
    if (tid == 0 && p.counters)
      atomicAdd(p.counters + 2, (unsigned long long)(clock64() - clk_trace0));
    if (tid == 0) {
      for (int k = 0; k < kPhases; ++k) C.ph[k] = 0;
      C.ph_last = clock64();
    }
#endif

    bool ovf = rec ? rec->ovf != 0 : false;
    int imf_count = rec ? rec->imf_count : 0;
    bool finished = false;
    int extNo_last = rec ? rec->extNo_last : -1;
    bool stale = rec ? rec->stale != 0 : false;
    int n_resume = rec ? rec->n : 0;
    bool yielded = false;
    int n_yield = 0;
    unsigned long long passes = 0, spilled = 0;

    ExtInfo e = extrema_scan<NT>(L, N, tid, warp, lane, p.max_extrema);
    ovf |= e.overflow;

    while (!finished && imf_count < MAXI - 1) {
      int n = n_resume;
      n_resume = 0;
      for (;;) {
        if (migrate && (n & 3) == 0) {
          // every trace has started and few remain: hand this one to the
          // 512-thread instance at this pass boundary (checked every fourth
          // pass: the two L2 reads and the barrier cost ~1 % per pass)
          int want = 0;
          if (tid == 0)
            want = *reinterpret_cast<volatile int*>(p.queue) >= p.batch &&
                   *reinterpret_cast<volatile int*>(p.active) <= p.yield_below;
          if (__syncthreads_or(want)) {
            yielded = true;
            n_yield = n;
            break;
          }
        }
        ++n;
        if (n >= p.max_iteration) {
          ovf = true;
          if (tid == 0) { C.dbg_n[imf_count] = n; C.dbg_e[imf_count] = -1; C.dbg_z[imf_count] = -1; }
          break;
        }
        const int extNo = e.n_max + e.n_min;
        if (!(extNo > 2 && e.n_max >= 1 && e.n_min >= 1)) {
          extNo_last = extNo;
          finished = true;
          break;
        }
        const int kc0 = e.n_max + 2 * NB + 2, kc1 = e.n_min + 2 * NB + 2;
        int flags;
#if EMDB_MERGED_PLACE
        {
          // the wide instance's stride also holds the parked proto-IMF and the
          // quotients: its knots may use only the part before them
          const int place = choose_place(N, L.arena_bytes, kWide ? p.park_off : p.slab_stride,
                                         kc0, kc1, kGImf);
          if (EMDB_MERGED_PLACE == 2)
            flags = sift_pass<NT, kAnyPlace, kInt>(L, slab, e, N, NB, T, tid, warp, lane, place,
                                                   park_old, qbuf);
          else if (place == kPlaceSmem || place == kPlaceBorrow || place == kPlaceBorrow2)
            flags = sift_pass<NT, kOnChip, kInt>(L, slab, e, N, NB, T, tid, warp, lane, place,
                                                 park_old, qbuf);
          else
            flags = sift_pass<NT, kOffChip, kInt>(L, slab, e, N, NB, T, tid, warp, lane, place,
                                                  park_old, qbuf);
          spilled += place != kPlaceSmem;
        }
#else
        {
          const int place = choose_place(N, L.arena_bytes, kWide ? p.park_off : p.slab_stride,
                                         kc0, kc1, kGImf);
          if (place == kPlaceSmem)
            flags = sift_pass<NT, kPlaceSmem, kInt>(L, slab, e, N, NB, T, tid, warp, lane,
                                                    place, park_old, qbuf);
          else if (place == kPlaceBorrow)
            flags = sift_pass<NT, kPlaceBorrow, kInt>(L, slab, e, N, NB, T, tid, warp, lane,
                                                      place, park_old, qbuf);
          else if (place == kPlaceBorrow2)
            flags = sift_pass<NT, kPlaceBorrow2, kInt>(L, slab, e, N, NB, T, tid, warp, lane,
                                                       place, park_old, qbuf);
          else if (place == kPlaceSplit)
            flags = sift_pass<NT, kPlaceSplit, kInt>(L, slab, e, N, NB, T, tid, warp, lane,
                                                     place, park_old, qbuf);
          else if (place == kPlacePark)
            flags = sift_pass<NT, kPlacePark, kInt>(L, slab, e, N, NB, T, tid, warp, lane,
                                                    place, park_old, qbuf);
          else
            flags = sift_pass<NT, kPlaceSlab, kInt>(L, slab, e, N, NB, T, tid, warp, lane,
                                                    place, park_old, qbuf);
          spilled += place != kPlaceSmem;
        }
#endif
        ++passes;
        const bool pass_bad = (flags & 1) != 0;
        stale |= (flags & 2) != 0;
        // ---- post-update extrema scan (also next pass's pre-scan); the
        // wide instances ran its count inside the pass ----
        if (kWide && EMDB_WIDE_OVERLAP) e = extrema_finish<NT>(L, N, tid, warp, p.max_extrema);
        else e = extrema_scan<NT>(L, N, tid, warp, lane, p.max_extrema);
        EMDB_PH(&C, 7);
        ovf |= e.overflow;
        const int extNo2 = e.n_max + e.n_min;
        const int nzm2 = e.n_zer;
        const bool f2 = abs(extNo2 - nzm2) < 2;
        bool f1 = false;
        if (!pass_bad) {
          real sum_new_sq = C.sums[0], diff_sq = C.sums[1], old_sq = C.sums[2];
          real std_sum = C.sums[3], omax = C.sums[4], omin = C.sums[5];
          if (sum_new_sq < kSumNewSqMin) f1 = false;
          else if (diff_sq / (omax - omin) < kSvarThr) f1 = true;
          else if (std_sum < kStdThr) f1 = true;
          else if (diff_sq / old_sq < kEnergyRatioThr) f1 = true;
        }
        extNo_last = extNo2;
        if (f1 && f2) {
          if (tid == 0) { C.dbg_n[imf_count] = n; C.dbg_e[imf_count] = extNo2; C.dbg_z[imf_count] = nzm2; }
          break;
        }
      }
      if (yielded) break;
      // ---- emit IMF row, running residue into the next row, end condition ----
      EMDB_PH(&C, 9);
      {
        const real* rsrc = imf_count == 0 ? S : out + (int64_t)imf_count * N;
        real* row = out + (int64_t)imf_count * N;
        real* rnext = out + (int64_t)(imf_count + 1) * N;
        real gmax = -1e30, gmin = 1e30, gabs = 0.0;
        // the reference's 128 lanes (a wider CTA's other threads wait: once per IMF)
        for (int i = tid; i < (!kWide || tid < kThreads ? N : 0); i += kThreads) {
          real r = rsrc[i];
          real v = imf[i];
          row[i] = v;
          real rn = r - v;
          rnext[i] = rn;
          gmax = fmax(gmax, rn);
          gmin = fmin(gmin, rn);
          gabs += fabs(rn);
        }
        real* red = L.red;
        if (!kWide || tid < kThreads) { red[tid] = gmax; red[128 + tid] = gmin; red[256 + tid] = gabs; }
        __syncthreads();
        if (warp == 0) {
          real a0 = lane_tree(red, lane, 1);
          real a1 = lane_tree(red + 128, lane, 2);
          real a2 = lane_tree(red + 256, lane, 0);
          if (lane == 0) { C.sums[6] = a0 - a1; C.sums[7] = a2; }
        }
        __syncthreads();
        ++imf_count;
        if (C.sums[6] < kRangeThr || C.sums[7] < kTotalPowerThr) finished = true;
      }
      if (!finished && imf_count < MAXI - 1) {
        const real* rsrc = out + (int64_t)imf_count * N;
        for (int i = tid; i < N; i += NT) imf[i] = rsrc[i];
        __syncthreads();
        e = extrema_scan<NT>(L, N, tid, warp, lane, p.max_extrema);
        ovf |= e.overflow;
      }
      EMDB_PH(&C, 8);
    }

    if (yielded) {
      // continuation record in this CTA's slot (a CTA hands over at most one
      // trace: the queue is empty when it does)
      ContHead* h = reinterpret_cast<ContHead*>(p.cont_buf + (size_t)blockIdx.x * p.cont_stride);
      real* dst = reinterpret_cast<real*>(reinterpret_cast<char*>(h) + cont_data_off());
      for (int i = tid; i < N; i += NT) dst[i] = imf[i];
      for (int k = tid; k < kMaxImfsCap; k += NT) {
        h->dbg[0][k] = C.dbg_n[k];
        h->dbg[1][k] = C.dbg_e[k];
        h->dbg[2][k] = C.dbg_z[k];
      }
      if (tid == 0) {
        h->b = b;
        h->n = n_yield;
        h->imf_count = imf_count;
        h->extNo_last = extNo_last;
        h->ovf = ovf ? 1 : 0;
        h->stale = stale ? 1 : 0;
        p.cont_valid[blockIdx.x] = 1;
        atomicSub(p.active, 1);
        if (p.counters) {
          atomicAdd(p.counters, passes);
          atomicAdd(p.counters + 1, spilled);
        }
      }
      __syncthreads();
      continue;
    }

    // ---- epilogue: trend removal, residue ~ 0 test, zero unused rows ----
    const int last_row = imf_count;   // row holding the running residue (or none if 0 IMFs)
    const bool trend = extNo_last <= 2 && imf_count > 0;
    if (trend) imf_count -= 1;
    const real* rres = last_row == 0 ? S : out + (int64_t)last_row * N;
    real amax = 0.0;
    for (int i = tid; i < (!kWide || tid < kThreads ? N : 0); i += kThreads) {
      real r = rres[i];
      if (trend) r = r + imf[i];
      amax = fmax(amax, fabs(r));
    }
    real* red = L.red;
    if (!kWide || tid < kThreads) red[tid] = amax;
    __syncthreads();
    if (warp == 0) {
      real a = lane_tree(red, lane, 1);
      if (lane == 0) C.sums[0] = a;
    }
    __syncthreads();
    const bool rzero = C.sums[0] <= kResidueZeroAtol;
    const int nim = rzero ? imf_count : imf_count + 1;
    for (int i = tid; i < N; i += NT) {
      if (trend) {
        real r = rres[i] + imf[i];
        if (!rzero) out[(int64_t)imf_count * N + i] = r;
        out[(int64_t)last_row * N + i] = 0.0;
      } else {
        if (rzero && last_row < MAXI) out[(int64_t)last_row * N + i] = 0.0;
        else if (last_row == 0) out[i] = S[i];
      }
    }
    const int first_zero = last_row + 1;
    for (int64_t k = (int64_t)first_zero * N + tid; k < (int64_t)MAXI * N; k += NT) out[k] = 0.0;
    if (tid == 0) {
      p.n_imfs[b] = nim;
      p.overflow[b] = ovf ? 1 : 0;
      if (p.counters) {
        atomicAdd(p.counters, passes);
        atomicAdd(p.counters + 1, spilled);
      }
      if (migrate) atomicSub(p.active, 1);
    }
    if (stale) atomicOr(p.status, kStatusStaleEnvelope);
    for (int k = tid; k < MAXI; k += NT) {
      p.dbg_n[(int64_t)b * MAXI + k] = C.dbg_n[k];
      p.dbg_ext[(int64_t)b * MAXI + k] = C.dbg_e[k];
      p.dbg_nzm[(int64_t)b * MAXI + k] = C.dbg_z[k];
    }
    __syncthreads();
#if EMDB_LOAD_CLOCKS
    if (tid == 0 && p.counters) {
      atomicAdd(p.counters + 3, (unsigned long long)(clock64() - clk_trace0));
      for (int k = 0; k < kPhases; ++k) atomicAdd(p.counters + 4 + k, C.ph[k]);
    }
#endif
    // rows that may hold data: n_imfs, plus the dropped trend row that a
    // ~zero residue leaves in place (as the reference does)
    mark_trace_done(p, b, tid, nim + ((trend && rzero) ? 1 : 0));
  }
}

// ---------------------------------------------------------------------------
// Envelope-only diagnostic (envelope_batch_kernel, kernels.py:1100-1166):
// extrema + mirroring + both envelopes on raw traces, no sift loop.  The
// reference scans with find_extrema_serial here; the extrema lists are the
// same as the sift scan's (plateau rule included) and n_zer is not reported.
// ---------------------------------------------------------------------------
template <bool kSmem>
__device__ __forceinline__ void envelope_pass(const SmemLayout& L, char* slab, const ExtInfo& e,
                                              int N, int NB, const TimeAxis& T, int tid, int warp,
                                              int lane, real* emax_out, real* emin_out,
                                              real* kp[2], real* kv[2], int mbuf, int nk[2],
                                              int* status) {
  Ctl& C = *L.ctl;
  const int kc0 = e.n_max + 2 * NB + 2, kc1 = e.n_min + 2 * NB + 2;
  Knots K = place_knots(kSmem ? L.arena : slab, kc0, kc1);
  fill_true_knots<kWarps>(L, K, e, N, NB, T, warp, lane);
  __syncthreads();
  if (warp == 0) mirror_both(L, K, e, N, NB, T, lane);
  __syncthreads();
  const int kb0 = C.kbase[0], kb1 = C.kbase[1], kn0 = C.kcnt[0], kn1 = C.kcnt[1];
  solve_splines<kThreads>(K, kb0, kb1, kn0, kn1, tid);
  SideView sv[2];
  sv[0].x = K.X[0] + kb0; sv[0].y = K.Y[0] + kb0; sv[0].M = K.M[0]; sv[0].R = K.R[0]; sv[0].n = kn0;
  sv[0].nl = NB - kb0; sv[0].nt = e.n_max;
  sv[1].x = K.X[1] + kb1; sv[1].y = K.Y[1] + kb1; sv[1].M = K.M[1]; sv[1].R = K.R[1]; sv[1].n = kn1;
  sv[1].nl = NB - kb1; sv[1].nt = e.n_min;
  nk[0] = kn0;
  nk[1] = kn1;
  const int kcnt[2] = {kn0, kn1};
  bool oor = false;
  for (int i = tid; i < N; i += kThreads) {
    real t = T(i);
    int lo0 = sv[0].n >= 4 ? search_seg(sv[0], t) : 0;
    int lo1 = sv[1].n >= 4 ? search_seg(sv[1], t) : 0;
    bool r0 = !(t < sv[0].x[0] || t > sv[0].x[sv[0].n - 1]);
    bool r1 = !(t < sv[1].x[0] || t > sv[1].x[sv[1].n - 1]);
    real a = eval_seg(sv[0], t, lo0);
    real c = eval_seg(sv[1], t, lo1);
    emax_out[i] = r0 ? a : 0.0;
    emin_out[i] = r1 ? c : 0.0;
    oor |= !(r0 && r1);
  }
  if (oor) atomicOr(status, kStatusStaleEnvelope);
  for (int q = 0; q < 2; ++q)
    for (int k = tid; k < mbuf; k += kThreads) {
      kp[q][k] = k < kcnt[q] ? sv[q].x[k] : 0.0;
      kv[q][k] = k < kcnt[q] ? sv[q].y[k] : 0.0;
    }
}

__global__ void __launch_bounds__(kThreads, 4) emd_envelope_kernel(EnvParams p) {
  extern __shared__ __align__(16) char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int NB = p.nbsym;
  Ctl* Cs = reinterpret_cast<Ctl*>(smem);
  char* slab = p.slab + (size_t)blockIdx.x * p.slab_stride;
  for (;;) {
    if (tid == 0) Cs->job = atomicAdd(p.queue, 1);
    __syncthreads();
    const int b = Cs->job;
    if (b >= p.batch) break;
    const int64_t off = p.offsets ? p.offsets[b] : (int64_t)b * p.dense_n;
    const int N = p.offsets ? (int)(p.offsets[b + 1] - off) : p.dense_n;
    const real* S = p.values + off;
    real* emax_out = p.max_env + off;
    real* emin_out = p.min_env + off;
    real* kp[2] = {p.max_kpos + (int64_t)b * p.mbuf, p.min_kpos + (int64_t)b * p.mbuf};
    real* kv[2] = {p.max_kval + (int64_t)b * p.mbuf, p.min_kval + (int64_t)b * p.mbuf};
    TimeAxis T;
    T.arange = p.t_mode == kTArange;
    T.T = p.t_mode == kTShared ? p.T : (p.t_mode == kTPerTrace ? p.T + off : nullptr);
    if (fixed_bytes(N) + kRedBytes + 64 > (size_t)p.arena_bytes) {
      if (tid == 0) {
        atomicOr(p.status, kStatusTooLong);
        p.degenerate[b] = 1;
        p.n_extrema[2 * b] = 0; p.n_extrema[2 * b + 1] = 0;
        p.n_mirrored[2 * b] = 0; p.n_mirrored[2 * b + 1] = 0;
      }
      __syncthreads();
      continue;
    }
    SmemLayout L = carve<kThreads>(smem, N, p.arena_bytes);
    for (int i = tid; i < N; i += kThreads) L.imf[i] = S[i];
    __syncthreads();
    ExtInfo e = extrema_scan<kThreads>(L, N, tid, warp, lane, p.max_extrema);
    const bool degenerate = !(e.n_max + e.n_min > 2 && e.n_max >= 1 && e.n_min >= 1);
    int nk[2] = {0, 0};
    if (!degenerate) {
      const int kc0 = e.n_max + 2 * NB + 2, kc1 = e.n_min + 2 * NB + 2;
      if (knot_bytes(kc0, kc1) <= (size_t)L.arena_bytes)
        envelope_pass<true>(L, slab, e, N, NB, T, tid, warp, lane, emax_out, emin_out, kp, kv,
                            p.mbuf, nk, p.status);
      else
        envelope_pass<false>(L, slab, e, N, NB, T, tid, warp, lane, emax_out, emin_out, kp, kv,
                             p.mbuf, nk, p.status);
    } else {
      for (int i = tid; i < N; i += kThreads) { emax_out[i] = 0.0; emin_out[i] = 0.0; }
      for (int q = 0; q < 2; ++q)
        for (int k = tid; k < p.mbuf; k += kThreads) { kp[q][k] = 0.0; kv[q][k] = 0.0; }
    }
    if (tid == 0) {
      p.degenerate[b] = degenerate ? 1 : 0;
      p.n_extrema[2 * b] = e.n_max;
      p.n_extrema[2 * b + 1] = e.n_min;
      p.n_mirrored[2 * b] = nk[0];
      p.n_mirrored[2 * b + 1] = nk[1];
    }
    __syncthreads();
  }
}

#if !EMDB_F32
// ---------------------------------------------------------------------------
// Self-test of div_rn against the hardware division.  mode 0: every integer
// pair 0 <= a <= b <= n (the operands of A and B on the default time axis,
// where knot spacings are integers <= 2N); mode 1: n pseudo-random pairs with
// significands and exponents spread over [2^-600, 2^600] plus numerators
// formed like the spline's h^2-scaled term over 6.  Counts mismatching bits.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void div_check_kernel(int mode, long long n, unsigned long long seed,
                                 unsigned long long* mismatches) {
  unsigned long long bad0 = 0, bad1 = 0, bad2 = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (mode == 0) {
    // pairs indexed by b in [1, n]: thread grid-strides over b, loops over a
    for (long long bb = 1 + blockIdx.x * (long long)blockDim.x + threadIdx.x; bb <= n; bb += stride) {
      const double b = (double)bb;
      const double y = 1.0 / b;
      for (long long aa = 0; aa <= bb; ++aa) {
        const double a = (double)aa;
        if (__double_as_longlong(div_rn(a, b, y)) != __double_as_longlong(a / b)) ++bad0;
      }
    }
#if EMDB_PCR_NB || EMDB_ACC_NB || EMDB_SETUP_NB
  } else if (mode == 2) {
    // div_nb: [0] random a/b over [2^-1100, 2^1100] (zeros, subnormals, infinities
    // through the fallback), [1] all-ones / power-of-two significands of b,
    // [2] PCR-like |a| <= |b| within 2^+-40 of 1
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
      uint64_t h1 = mix64(seed ^ (uint64_t)i), h2 = mix64(h1 ^ 0x5bd1e995ull);
      double ma = __longlong_as_double((long long)((h1 >> 12) | 0x3ff0000000000000ull));
      double mb = __longlong_as_double((long long)((h2 >> 12) | 0x3ff0000000000000ull));
      double a = ldexp(ma, (int)(h1 % 2201) - 1100), b = ldexp(mb, (int)(h2 % 2201) - 1100);
      if (h1 & 1) a = -a;
      if (h2 & 2) b = -b;
      bool slow = false;
      double q = div_nb(a, b, slow);
      if (slow) q = div_slow(a, b);
      if (__double_as_longlong(q) != __double_as_longlong(div_slow(a, b))) ++bad0;
      const int eb2 = (int)((h2 >> 20) % 161) - 80;
      double b2 = (h2 & 4) ? ldexp(__longlong_as_double(0x3fffffffffffffffll), eb2) : ldexp(1.0, eb2);
      if (h2 & 8) b2 = -b2;
      slow = false;
      q = div_nb(a, b2, slow);
      if (slow) q = div_slow(a, b2);
      if (__double_as_longlong(q) != __double_as_longlong(div_slow(a, b2))) ++bad1;
      double b3 = ldexp(mb, (int)((h2 >> 30) % 81) - 40);
      double a3 = b3 * ((double)((h1 >> 11) & 0xfffffffffffffull) * 0x1p-52);
      if (h1 & 16) a3 = -a3;
      slow = false;
      q = div_nb(a3, b3, slow);
      if (slow) q = div_slow(a3, b3);
      if (__double_as_longlong(q) != __double_as_longlong(div_slow(a3, b3))) ++bad2;
    }
#endif
  } else {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
      uint64_t h1 = mix64(seed ^ (uint64_t)i), h2 = mix64(h1 ^ 0x5bd1e995ull);
      // significands in [1,2), exponents in [-300, 300] (quotients stay in range), random signs
      double ma = __longlong_as_double((long long)((h1 >> 12) | 0x3ff0000000000000ull));
      double mb = __longlong_as_double((long long)((h2 >> 12) | 0x3ff0000000000000ull));
      int ea = (int)(h1 % 601) - 300, eb = (int)(h2 % 601) - 300;
      double a = ldexp(ma, ea), b = ldexp(mb, eb);
      if (h1 & 1) a = -a;
      if (h2 & 2) b = -b;
      if (__double_as_longlong(div_rn(a, b, 1.0 / b)) != __double_as_longlong(a / b)) ++bad0;
      // division by 6 (the spline term's divisor)
      if (__double_as_longlong(div_rn(a, 6.0, kInv6)) != __double_as_longlong(a / 6.0)) ++bad1;
      // segment quotients: 0 <= a <= b, b a spacing in [1, 65536] with a random fraction
      double bi = (double)((h2 >> 40) % 65536 + 1) + (double)((h2 >> 8) & 0xffff) * 0x1p-16;
      double ai = bi * ((double)((h1 >> 11) & 0xfffffffffffffull) * 0x1p-52);
      if (__double_as_longlong(div_rn(ai, bi, 1.0 / bi)) != __double_as_longlong(ai / bi)) ++bad2;
    }
  }
  if (bad0) atomicAdd(mismatches, bad0);
  if (bad1) atomicAdd(mismatches + 1, bad1);
  if (bad2) atomicAdd(mismatches + 2, bad2);
}

cudaError_t launch_div_check(int mode, long long n, unsigned long long seed,
                             unsigned long long* mismatches, cudaStream_t stream) {
  div_check_kernel<<<148 * 8, 256, 0, stream>>>(mode, n, seed, mismatches);
  return cudaGetLastError();
}
#endif

#if EMDB_F32
// ---------------------------------------------------------------------------
// Self-test of the float quotients (div_q, div_nb above) against the float
// division.  mode 0: every integer pair 0 <= a <= b <= n through div_q with
// y = RN(1/b) (the segment quotients on the default time axis); mode 1: n
// pseudo-random pairs, [0] div_q with y = RN(1/b), significands random and
// exponents in [-40, 40]; [1] div_nb with exponents in [-140, 140] (zeros,
// subnormals and the range edges through the fallback); [2] div_nb on
// PCR-like rows, |a| <= |b| within 2^+-40 of 1.  Counts mismatching bits.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64f(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ float rnd_float(uint64_t h, int e_lo, int e_hi) {
  const float m = __int_as_float((int)((h >> 41) | 0x3f800000u));     // [1, 2)
  const float v = ldexpf(m, (int)(h % (uint64_t)(e_hi - e_lo + 1)) + e_lo);
  return (h & (1ull << 20)) ? -v : v;
}

__global__ void div_check_f32_kernel(int mode, long long n, unsigned long long seed,
                                     unsigned long long* mismatches) {
  unsigned long long bad0 = 0, bad1 = 0, bad2 = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (mode == 0) {
    for (long long bb = 1 + blockIdx.x * (long long)blockDim.x + threadIdx.x; bb <= n; bb += stride) {
      const float b = (float)bb;
      const float y = 1.0f / b;
      for (long long aa = 0; aa <= bb; ++aa) {
        const float a = (float)aa;
        bool slow = false;
        float q = div_q(a, b, y, slow);
        if (slow) q = div_slow(a, b);
        if (__float_as_int(q) != __float_as_int(div_slow(a, b))) ++bad0;
      }
    }
  } else {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
      const uint64_t h1 = mix64f(seed ^ (uint64_t)i), h2 = mix64f(h1 ^ 0x5bd1e995ull);
      const uint64_t h3 = mix64f(h2 ^ 0x9e3779b9ull), h4 = mix64f(h3 ^ 0x7f4a7c15ull);
      {
        const float a = rnd_float(h1, -40, 40), b = rnd_float(h2, -40, 40);
        bool slow = false;
        float q = div_q(a, b, 1.0f / b, slow);
        if (slow) q = div_slow(a, b);
        if (__float_as_int(q) != __float_as_int(div_slow(a, b))) ++bad0;
      }
      {
        float a = rnd_float(h3, -140, 140), b = rnd_float(h4, -140, 140);
        if ((h3 & 0xff) == 0) a = 0.0f;
        bool slow = false;
        float q = div_nb(a, b, slow);
        if (slow) q = div_slow(a, b);
        if (__float_as_int(q) != __float_as_int(div_slow(a, b))) ++bad1;
      }
      {
        const float b = rnd_float(h2 ^ h3, -40, 40);
        const float f = __int_as_float((int)((h4 >> 41) | 0x3f800000u)) - 1.0f;   // [0, 1)
        const float a = ((h1 & 2) ? -f : f) * b;
        bool slow = false;
        float q = div_nb(a, b, slow);
        if (slow) q = div_slow(a, b);
        if (__float_as_int(q) != __float_as_int(div_slow(a, b))) ++bad2;
      }
    }
  }
  if (bad0) atomicAdd(mismatches, bad0);
  if (bad1) atomicAdd(mismatches + 1, bad1);
  if (bad2) atomicAdd(mismatches + 2, bad2);
}

cudaError_t launch_div_check(int mode, long long n, unsigned long long seed,
                             unsigned long long* mismatches, cudaStream_t stream) {
  div_check_f32_kernel<<<148 * 8, 256, 0, stream>>>(mode, n, seed, mismatches);
  return cudaGetLastError();
}
#endif

size_t sift_fixed_smem(int N, int variant, bool imf_global) {
  const int nt = variant_threads(variant);
  if (nt <= kThreads) return fixed_bytes(N) + kRedBytes;
  if (nt == kHalfWideThreads) return fixed_bytes<kHalfWideThreads>(N) + kRedBytes;
  return (imf_global ? fixed_bytes<kWideThreads, true>(N) : fixed_bytes<kWideThreads>(N)) +
         kRedBytes;
}

int sift_pass_placement(int N, int arena_total, size_t slab_stride, int kc0, int kc1) {
  const size_t fixed = fixed_bytes(std::max(N, 1));
  if (arena_total < 0 || (size_t)arena_total < fixed + kRedBytes + 64) return -1;
  return choose_place(N, arena_total - (int)fixed, slab_stride, kc0, kc1);
}

size_t sift_slab_bytes(int max_extrema, int nbsym) {
  const long long kc = (long long)max_extrema + 2LL * nbsym + 2;
  const size_t cap = (size_t)(2 * kc);
  const size_t red_extra = (EMDB_FAST_DIV != 1 && 4 * cap >= (size_t)kRedDoubles) ? 0 : kRedBytes;
  return align16(10 * cap * sizeof(real) + red_extra);
}

namespace {
// kInt: the kernel build for the integer time axis (T = arange), whose
// segment quotients use the reciprocal table.
template <int NT, int V, bool kInt, bool kG = false>
cudaError_t occupancy_vt(int arena_bytes, int* ctas_per_sm) {
  cudaError_t e = cudaFuncSetAttribute(emd_sift_kernel<NT, V, kInt, kG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, arena_bytes);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm,
                                                       emd_sift_kernel<NT, V, kInt, kG>, NT,
                                                       arena_bytes);
}
// CTAs per SM that both builds reach (the smaller), so a plan's grid fits either
template <int NT, int V, bool kG = false>
cudaError_t occupancy_v(int arena_bytes, int* ctas_per_sm) {
  int a = 0, b = 0;
  cudaError_t e = occupancy_vt<NT, V, true, kG>(arena_bytes, &a);
  if (e == cudaSuccess) e = occupancy_vt<NT, V, false, kG>(arena_bytes, &b);
  *ctas_per_sm = a < b ? a : b;
  return e;
}
template <int NT, int V, bool kInt, bool kG = false, bool kT = false>
cudaError_t launch_vt(const SiftParams& p, int grid, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(emd_sift_kernel<NT, V, kInt, kG, kT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, p.arena_bytes);
  if (e != cudaSuccess) return e;
  emd_sift_kernel<NT, V, kInt, kG, kT><<<grid, NT, p.arena_bytes, stream>>>(p);
  return cudaGetLastError();
}
template <int NT, int V, bool kG = false, bool kT = false>
cudaError_t launch_v(const SiftParams& p, int grid, cudaStream_t stream) {
  return p.t_mode == kTArange ? launch_vt<NT, V, true, kG, kT>(p, grid, stream)
                              : launch_vt<NT, V, false, kG, kT>(p, grid, stream);
}
}  // namespace

#if !EMDB_F32
bool sift_variant_ok(int v) { return v == 1 || v == 2 || v == 4 || v == 5 || v == 6; }

int variant_threads(int v) {
  return v == 1 ? kWideThreads : v == 2 ? kHalfWideThreads : kThreads;
}
#endif

cudaError_t sift_occupancy(int arena_bytes, int variant, int* ctas_per_sm, bool imf_global) {
  switch (variant) {
    case 1: return imf_global ? occupancy_v<kWideThreads, 1, true>(arena_bytes, ctas_per_sm)
                              : occupancy_v<kWideThreads, 1>(arena_bytes, ctas_per_sm);
    case 2: return occupancy_v<kHalfWideThreads, 2>(arena_bytes, ctas_per_sm);
    case 5: return occupancy_v<kThreads, 5>(arena_bytes, ctas_per_sm);
    case 6: return occupancy_v<kThreads, 6>(arena_bytes, ctas_per_sm);
    default: return occupancy_v<kThreads, 4>(arena_bytes, ctas_per_sm);
  }
}

cudaError_t launch_sift(const SiftParams& p, int grid, cudaStream_t stream) {
  // tail migration (p.cont_buf): the 128 x 4 build that hands over, the
  // 512-thread build that resumes
  if (p.cont_buf != nullptr) {
    switch (p.variant) {
      case 1: return launch_v<kWideThreads, 1, false, true>(p, grid, stream);
      case 4: return launch_v<kThreads, 4, false, true>(p, grid, stream);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (p.variant) {
    case 1: return p.imf_off ? launch_v<kWideThreads, 1, true>(p, grid, stream)
                             : launch_v<kWideThreads, 1>(p, grid, stream);
    case 2: return launch_v<kHalfWideThreads, 2>(p, grid, stream);
    case 5: return launch_v<kThreads, 5>(p, grid, stream);
    case 6: return launch_v<kThreads, 6>(p, grid, stream);
    default: return launch_v<kThreads, 4>(p, grid, stream);
  }
}

cudaError_t envelope_occupancy(int arena_bytes, int* ctas_per_sm) {
  cudaError_t e = cudaFuncSetAttribute(emd_envelope_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, arena_bytes);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, emd_envelope_kernel, kThreads,
                                                       arena_bytes);
}

cudaError_t launch_envelope(const EnvParams& p, int grid, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(emd_envelope_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, p.arena_bytes);
  if (e != cudaSuccess) return e;
  emd_envelope_kernel<<<grid, kThreads, p.arena_bytes, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace emdb
