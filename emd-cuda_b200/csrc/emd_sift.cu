// Batched FP64 EMD sift for sm_100a -- the hot path behind GPUBatchEMD.
//
// Behaviour follows the reference's emd_batch_kernel (SeismicFlow/emd-cuda,
// kernels.py:834-1080) and its device functions, re-built for B200:
//
//  * one 128-thread CTA per trace, persistent: CTAs pull trace tickets from an
//    atomic work queue (FIFO, or a caller-given order), so a long trace never
//    holds a wave back and CSR batches of mixed length run in one launch;
//  * the proto-IMF lives in shared memory for the whole decomposition; the
//    running residue lives in the output rows (each row is written once,
//    the residue row is rewritten once per IMF);
//  * extrema: one warp-contiguous scan per sift pass computes ballot masks,
//    zero-crossing counts and the serial-fallback trigger; the masks are
//    compacted (popc ranks) straight into the knot arrays of both envelopes.
//    The post-update scan of pass n is reused as the pre-scan of pass n+1
//    (the reference scans the same data twice, kernels.py:930 vs 965);
//  * boundary mirroring runs on one warp while the knot arrays are filled;
//  * the upper and lower not-a-knot systems are solved concurrently by
//    parallel cyclic reduction (ping-pong buffers, one barrier per level);
//  * envelope evaluation, the mean update and the six stop-test partial
//    sums are one fused pass; sums are formed in the reference's order
//    (128 strided lanes + halving tree), and this file is compiled with
//    -fmad=false, so every value equals the reference algorithm's FP64
//    result bit for bit (the CPU oracle checks this).
//
// Per-iteration knot/PCR storage is carved from the CTA's shared-memory
// arena and spills to a per-CTA global slab only when a trace has more
// knots than the arena holds.  All spin-free: no waits on other CTAs.

#include "emdb_internal.cuh"

namespace emdb {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// reference thresholds (kernels.py:81-85, 814, 1069)
constexpr double kEnergyRatioThr = 0.2;
constexpr double kStdThr = 0.2;
constexpr double kSvarThr = 0.001;
constexpr double kTotalPowerThr = 0.005;
constexpr double kRangeThr = 0.001;
constexpr double kSumNewSqMin = 1e-10;
constexpr double kResidueZeroAtol = 1e-8;
constexpr int kLocalExtBuf = 64;  // kernels.py:206 (serial-fallback trigger)

struct Ctl {
  int job;
  int w_max[kWarps], w_min[kWarps], w_zc[kWarps], w_zre[kWarps], w_trig[kWarps];
  int head[2][kMaxNbsym + 1];  // first NB+1 extrema indices per side (0 = max, 1 = min)
  int tail[2][kMaxNbsym + 1];  // tail[q][k] = index of extremum n_q-1-k
  int kbase[2], kcnt[2];
  int mlist[4][kMaxNbsym + 1], mcnt[4], lsym, rsym;
  int dbg_n[kMaxImfsCap], dbg_e[kMaxImfsCap], dbg_z[kMaxImfsCap];
  int chunk_bad;
  double sums[8];
};

struct SmemLayout {
  Ctl* ctl;
  double* red;        // [6][128]
  double* imf;        // [N]
  uint32_t* mmax;     // [nch]
  uint32_t* mmin;
  uint16_t* pmax;     // per-chunk exclusive prefix within the warp's range
  uint16_t* pmin;
  char* arena;        // knot arena start
  int arena_bytes;    // bytes left for the knot arena
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t fixed_bytes(int N) {
  size_t nch = (size_t)(N + 31) / 32;
  size_t b = align16(sizeof(Ctl));
  b += align16(6 * kThreads * sizeof(double));
  b += align16((size_t)N * sizeof(double));
  b += align16(nch * 4) * 2 + align16(nch * 2) * 2;
  return b;
}

__device__ inline SmemLayout carve(char* base, int N, int arena_total) {
  SmemLayout L;
  size_t nch = (size_t)(N + 31) / 32;
  char* p = base;
  L.ctl = reinterpret_cast<Ctl*>(p); p += align16(sizeof(Ctl));
  L.red = reinterpret_cast<double*>(p); p += align16(6 * kThreads * sizeof(double));
  L.imf = reinterpret_cast<double*>(p); p += align16((size_t)N * sizeof(double));
  L.mmax = reinterpret_cast<uint32_t*>(p); p += align16(nch * 4);
  L.mmin = reinterpret_cast<uint32_t*>(p); p += align16(nch * 4);
  L.pmax = reinterpret_cast<uint16_t*>(p); p += align16(nch * 2);
  L.pmin = reinterpret_cast<uint16_t*>(p); p += align16(nch * 2);
  L.arena = p;
  L.arena_bytes = arena_total - (int)(p - base);
  return L;
}

// Knot / PCR storage for one sift pass (both envelopes).
struct Knots {
  double* X[2];
  double* Y[2];
  double* M[2];
  double* P[2];   // ping-pong PCR buffers: a | b | c | d, each `cap` rows
  int cap;        // PCR row capacity per buffer array
};

__device__ inline size_t knot_bytes(int kc0, int kc1) {
  // X, Y, M per side + 2 buffers x 4 arrays x (kc0+kc1) rows
  return (size_t)(3 * (kc0 + kc1) + 8 * (kc0 + kc1)) * sizeof(double);
}

__device__ inline Knots place_knots(char* base, int kc0, int kc1) {
  Knots K;
  double* p = reinterpret_cast<double*>(base);
  K.X[0] = p; p += kc0;
  K.Y[0] = p; p += kc0;
  K.M[0] = p; p += kc0;
  K.X[1] = p; p += kc1;
  K.Y[1] = p; p += kc1;
  K.M[1] = p; p += kc1;
  K.cap = kc0 + kc1;
  K.P[0] = p; p += 4 * K.cap;
  K.P[1] = p;
  return K;
}

struct TimeAxis {
  const double* T;
  bool arange;
  __device__ inline double operator()(int i) const { return arange ? (double)i : T[i]; }
};

// ---------------------------------------------------------------------------
// Extrema: count pass (find_extrema_parallel semantics, kernels.py:231-349,
// with the serial scan's plateau rule, kernels.py:157-200).
// ---------------------------------------------------------------------------
__device__ void extrema_count(const SmemLayout& L, int N, int warp, int lane) {
  const double* imf = L.imf;
  int nch = (N + 31) >> 5;
  int c0 = (warp * nch) / kWarps, c1 = ((warp + 1) * nch) / kWarps;
  int rmax = 0, rmin = 0, zc = 0, zre = 0;
  bool trig = false;
  for (int c = c0; c < c1; ++c) {
    int i = (c << 5) + lane;
    double v = (i < N) ? imf[i] : 0.0;
    double vp = __shfl_up_sync(kFull, v, 1);
    double vn = __shfl_down_sync(kFull, v, 1);
    if (lane == 0) vp = (i >= 1 && i - 1 < N) ? imf[i - 1] : 0.0;
    if (lane == 31) vn = (i + 1 < N) ? imf[i + 1] : 0.0;
    bool interior = (i >= 1) && (i <= N - 2);
    double dp = v - vp, dn = vn - v;
    bool strict = interior && (dp * dn < 0.0);
    bool ismin = strict && (dp < 0.0);
    bool ismax = strict && !(dp < 0.0);
    if (interior && dn == 0.0 && dp != 0.0) {
      // true left edge of a flat run: classify by the slopes around the run
      int j = i;
      while (j + 1 < N && imf[j + 1] == v) ++j;
      if (j + 1 < N) {
        double da = imf[j + 1] - imf[j];
        if (dp > 0.0 && da < 0.0) ismax = true;
        else if (dp < 0.0 && da > 0.0) ismin = true;
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
    Ctl& C = *L.ctl;
    C.w_max[warp] = rmax; C.w_min[warp] = rmin;
    C.w_zc[warp] = zc; C.w_zre[warp] = zre; C.w_trig[warp] = trig ? 1 : 0;
  }
}

struct ExtInfo {
  int tot_max, tot_min;   // true counts
  int n_max, n_min;       // stored (capped) counts
  int n_zer;
  int off_max, off_min;   // this warp's rank offsets
  bool overflow;
};

// After the count pass + barrier.  Reproduces the parallel/serial split of
// find_extrema_parallel: without a fallback trigger the zero-crossing count is
// sign changes only; with one, the serial count adds one per zero run that
// ends before N (kernels.py:123-143, 273-276).
__device__ ExtInfo extrema_totals(const SmemLayout& L, int N, int warp, int max_extrema) {
  const Ctl& C = *L.ctl;
  ExtInfo e;
  e.tot_max = e.tot_min = 0;
  int zc = 0, zre = 0;
  bool trig = false;
  e.off_max = e.off_min = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    if (w < warp) { e.off_max += C.w_max[w]; e.off_min += C.w_min[w]; }
    e.tot_max += C.w_max[w]; e.tot_min += C.w_min[w];
    zc += C.w_zc[w]; zre += C.w_zre[w];
    trig |= C.w_trig[w] != 0;
  }
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
// so it is evaluated in that rare case only.  Ends with a barrier.
__device__ void chunk_fallback_check(const SmemLayout& L, int N, int tid) {
  Ctl& C = *L.ctl;
  const double* s = L.imf;
  int cs = (N + kThreads - 1) / kThreads;
  int start = tid * cs, end = min(start + cs, N);
  int lo = max(start, 1), hi = min(end, N - 1);
  int nmx = 0, nmn = 0;
  for (int i = lo; i < hi; ++i) {
    double dp = s[i] - s[i - 1], dn = s[i + 1] - s[i];
    if (dp * dn < 0.0) { if (dp < 0.0) ++nmn; else ++nmx; }
  }
  int bad = __syncthreads_or(nmx > kLocalExtBuf || nmn > kLocalExtBuf);
  if (tid == 0) C.chunk_bad = bad;
  __syncthreads();
}

// One extrema scan = count pass + totals.  Ends after a barrier with every
// thread holding the same totals.
__device__ ExtInfo extrema_scan(const SmemLayout& L, int N, int tid, int warp, int lane,
                                int max_extrema) {
  extrema_count(L, N, warp, lane);
  if (tid == 0) L.ctl->chunk_bad = 0;
  __syncthreads();
  ExtInfo e = extrema_totals(L, N, warp, max_extrema);
  if (N > kThreads * 128 && L.imf[0] == 0.0) {
    bool trig = false;
    for (int w = 0; w < kWarps; ++w) trig |= L.ctl->w_trig[w] != 0;
    if (!trig) {
      chunk_fallback_check(L, N, tid);
      e = extrema_totals(L, N, warp, max_extrema);
    }
  }
  return e;
}

// ---------------------------------------------------------------------------
// Knot fill: compacted true extrema -> X/Y at offset NB (both sides).
// Returns this thread's "bad envelope sign" vote for true knots.
// ---------------------------------------------------------------------------
__device__ bool fill_true_knots(const SmemLayout& L, const Knots& K, const ExtInfo& e, int N,
                                int NB, const TimeAxis& T, int warp, int lane) {
  Ctl& C = *L.ctl;
  const double* imf = L.imf;
  int nch = (N + 31) >> 5;
  int c0 = (warp * nch) / kWarps, c1 = ((warp + 1) * nch) / kWarps;
  unsigned lt = (1u << lane) - 1u;
  bool bad = false;
  for (int c = c0; c < c1; ++c) {
    uint32_t bm = L.mmax[c], bn = L.mmin[c];
    if ((bm | bn) == 0u) continue;
    bool ismax = (bm >> lane) & 1u, ismin = (bn >> lane) & 1u;
    if (!(ismax || ismin)) continue;
    int i = (c << 5) + lane;
    int ii = i;
    double v = imf[i];
    double dp = v - imf[i - 1], dn = imf[i + 1] - v;
    if (!(dp * dn < 0.0)) {       // plateau extremum: report the run's midpoint
      int j = i;
      while (j + 1 < N && imf[j + 1] == v) ++j;
      ii = (i + j) / 2;
    }
    int q = ismax ? 0 : 1;
    int rank = q == 0 ? e.off_max + L.pmax[c] + __popc(bm & lt)
                      : e.off_min + L.pmin[c] + __popc(bn & lt);
    int nq = q == 0 ? e.n_max : e.n_min;
    if (rank < nq) {
      double y = imf[ii];
      K.X[q][NB + rank] = T(ii);
      K.Y[q][NB + rank] = y;
      bad |= q == 0 ? (y < 0.0) : (y > 0.0);
      if (rank <= NB) C.head[q][rank] = ii;
      int fe = nq - 1 - rank;
      if (fe <= NB) C.tail[q][fe] = ii;
    }
  }
  return bad;
}

// ---------------------------------------------------------------------------
// Boundary mirroring (mirror_one_side, kernels.py:360-558) for both sides.
// Runs on warp 0; lane 0 makes the O(nbsym) decisions, lanes write knots.
// Knot positions are strictly increasing whenever T is (the host checks T),
// so the reference's adjacent-duplicate removal never drops a knot and is
// not needed here.  Returns lane 0's "bad sign" vote for mirrored knots.
// ---------------------------------------------------------------------------
__device__ bool mirror_both(const SmemLayout& L, const Knots& K, const ExtInfo& e, int N, int NB,
                            const TimeAxis& T, int lane) {
  Ctl& C = *L.ctl;
  const double* S = L.imf;
  const int nM = e.n_max, nm = e.n_min;
  // list q: 0 lmax, 1 lmin, 2 rmax, 3 rmin
  int lst[4][kMaxNbsym + 1];
  int cnt[4];
  int lsym = 0, rsym = 0;
  if (lane == 0) {
    auto IM = [&](int k) { return k <= NB ? C.head[0][k] : C.tail[0][nM - 1 - k]; };
    auto Im = [&](int k) { return k <= NB ? C.head[1][k] : C.tail[1][nm - 1 - k]; };
    // ---- left bound ----
    if (IM(0) < Im(0)) {
      if (S[0] > S[Im(0)]) {
        cnt[0] = 0; for (int k = min(nM, NB + 1) - 1; k >= 1; --k) lst[0][cnt[0]++] = IM(k);
        cnt[1] = 0; for (int k = min(nm, NB) - 1; k >= 0; --k) lst[1][cnt[1]++] = Im(k);
        lsym = IM(0);
      } else {
        cnt[0] = 0; for (int k = min(nM, NB) - 1; k >= 0; --k) lst[0][cnt[0]++] = IM(k);
        cnt[1] = 0; for (int k = min(nm, NB - 1) - 1; k >= 0; --k) lst[1][cnt[1]++] = Im(k);
        lst[1][cnt[1]++] = 0;
        lsym = 0;
      }
    } else {
      if (S[0] < S[IM(0)]) {
        cnt[0] = 0; for (int k = min(nM, NB) - 1; k >= 0; --k) lst[0][cnt[0]++] = IM(k);
        cnt[1] = 0; for (int k = min(nm, NB + 1) - 1; k >= 1; --k) lst[1][cnt[1]++] = Im(k);
        lsym = Im(0);
      } else {
        cnt[0] = 0; for (int k = min(nM, NB - 1) - 1; k >= 0; --k) lst[0][cnt[0]++] = IM(k);
        lst[0][cnt[0]++] = 0;
        cnt[1] = 0; for (int k = min(nm, NB) - 1; k >= 0; --k) lst[1][cnt[1]++] = Im(k);
        lsym = 0;
      }
    }
    // ---- right bound ----
    if (IM(nM - 1) < Im(nm - 1)) {
      if (S[N - 1] < S[IM(nM - 1)]) {
        cnt[2] = 0; for (int k = nM - 1; k >= max(nM - NB, 0); --k) lst[2][cnt[2]++] = IM(k);
        cnt[3] = 0; for (int k = nm - 2; k >= max(nm - NB - 1, 0); --k) lst[3][cnt[3]++] = Im(k);
        rsym = Im(nm - 1);
      } else {
        cnt[2] = 0; lst[2][cnt[2]++] = N - 1;
        for (int k = max(nM - NB + 1, 0); k < nM; ++k) lst[2][cnt[2]++] = IM(k);
        cnt[3] = 0; for (int k = nm - 1; k >= max(nm - NB, 0); --k) lst[3][cnt[3]++] = Im(k);
        rsym = N - 1;
      }
    } else {
      if (S[N - 1] > S[Im(nm - 1)]) {
        cnt[2] = 0; for (int k = nM - 2; k >= max(nM - NB - 1, 0); --k) lst[2][cnt[2]++] = IM(k);
        cnt[3] = 0; for (int k = nm - 1; k >= max(nm - NB, 0); --k) lst[3][cnt[3]++] = Im(k);
        rsym = IM(nM - 1);
      } else {
        cnt[2] = 0; for (int k = nM - 1; k >= max(nM - NB, 0); --k) lst[2][cnt[2]++] = IM(k);
        cnt[3] = 0; lst[3][cnt[3]++] = N - 1;
        for (int k = max(nm - NB + 1, 0); k < nm; ++k) lst[3][cnt[3]++] = Im(k);
        rsym = N - 1;
      }
    }
    // An empty list falls back to the whole index list (kernels.py:456-459,
    // 523-531); that only happens when the side has exactly one extremum,
    // so the whole list is that one index.
    if (cnt[0] == 0) { lst[0][0] = IM(0); cnt[0] = 1; }
    if (cnt[1] == 0) { lst[1][0] = Im(0); cnt[1] = 1; }
    if (cnt[2] == 0) { lst[2][0] = IM(nM - 1); cnt[2] = 1; }
    if (cnt[3] == 0) { lst[3][0] = Im(nm - 1); cnt[3] = 1; }
    // ---- mirrored point does not reach the boundary (kernels.py:469-503) ----
    double tl = T(lsym);
    double tlmin0 = 2.0 * tl - T(lst[1][0]);
    double tlmax0 = 2.0 * tl - T(lst[0][0]);
    double T0 = T(0), TN = T(N - 1);
    if (tlmin0 > T0 || tlmax0 > T0) {
      if (lsym == IM(0)) {
        cnt[0] = 0; for (int k = min(nM, NB) - 1; k >= 0; --k) lst[0][cnt[0]++] = IM(k);
      } else {
        cnt[1] = 0; for (int k = min(nm, NB) - 1; k >= 0; --k) lst[1][cnt[1]++] = Im(k);
      }
      lsym = 0;
    }
    double tr = T(rsym);
    double trmin = 2.0 * tr - T(lst[3][cnt[3] - 1]);
    double trmax = 2.0 * tr - T(lst[2][cnt[2] - 1]);
    if (trmin < TN || trmax < TN) {
      if (rsym == IM(nM - 1)) {
        cnt[2] = 0; for (int k = nM - 1; k >= max(nM - NB, 0); --k) lst[2][cnt[2]++] = IM(k);
      } else {
        cnt[3] = 0; for (int k = nm - 1; k >= max(nm - NB, 0); --k) lst[3][cnt[3]++] = Im(k);
      }
      rsym = N - 1;
    }
    C.kbase[0] = NB - cnt[0];
    C.kbase[1] = NB - cnt[1];
    C.kcnt[0] = cnt[0] + nM + cnt[2];
    C.kcnt[1] = cnt[1] + nm + cnt[3];
    for (int q = 0; q < 4; ++q) {
      C.mcnt[q] = cnt[q];
      for (int j = 0; j < cnt[q]; ++j) C.mlist[q][j] = lst[q][j];
    }
    C.lsym = lsym;
    C.rsym = rsym;
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
    double pos = 2.0 * T(left ? C.lsym : C.rsym) - T(idx);
    double val = S[idx];
    int nside = side == 0 ? nM : nm;
    int slot = left ? (NB - cq + j) : (NB + nside + j);
    K.X[side][slot] = pos;
    K.Y[side][slot] = val;
    bad |= side == 0 ? (val < 0.0) : (val > 0.0);
  }
  return bad;
}

// ---------------------------------------------------------------------------
// Not-a-knot spline: reduced system + PCR + moments (kernels.py:607-697).
// ---------------------------------------------------------------------------
__device__ inline void setup_row(const double* x, const double* y, int n, int k, int m,
                                 double& a, double& b, double& c, double& d) {
  if (k == 0) {
    double h0 = x[1] - x[0], h1 = x[2] - x[1];
    double rhs1 = 6.0 * ((y[2] - y[1]) / h1 - (y[1] - y[0]) / h0);
    a = 0.0; b = h0 + 2.0 * h1; c = h1 - h0; d = h1 * rhs1 / (h0 + h1);
  } else if (k == m - 1) {
    double hnm3 = x[n - 2] - x[n - 3], hnm2 = x[n - 1] - x[n - 2];
    double rhs = 6.0 * ((y[n - 1] - y[n - 2]) / hnm2 - (y[n - 2] - y[n - 3]) / hnm3);
    a = hnm3 - hnm2; b = 2.0 * hnm3 + hnm2; c = 0.0; d = hnm3 * rhs / (hnm3 + hnm2);
  } else {
    int i = k + 1;
    double h_im1 = x[i] - x[i - 1], h_i = x[i + 1] - x[i];
    a = h_im1; b = 2.0 * (h_im1 + h_i); c = h_i;
    d = 6.0 * ((y[i + 1] - y[i]) / h_i - (y[i] - y[i - 1]) / h_im1);
  }
}

struct SideView {
  const double* x;
  const double* y;
  const double* M;
  int n;
};

__device__ void solve_splines(const Knots& K, const int kbase[2], const int kcnt[2], int tid) {
  int m[2];
  m[0] = kcnt[0] >= 4 ? kcnt[0] - 2 : 0;
  m[1] = kcnt[1] >= 4 ? kcnt[1] - 2 : 0;
  const int mt = m[0] + m[1];
  const int cap = K.cap;
  // setup -> P[0]
  for (int r = tid; r < mt; r += kThreads) {
    int q = r < m[0] ? 0 : 1;
    int k = q == 0 ? r : r - m[0];
    const double* x = K.X[q] + kbase[q];
    const double* y = K.Y[q] + kbase[q];
    double a, b, c, d;
    setup_row(x, y, kcnt[q], k, m[q], a, b, c, d);
    double* P = K.P[0];
    P[r] = a; P[cap + r] = b; P[2 * cap + r] = c; P[3 * cap + r] = d;
  }
  __syncthreads();
  int mmax = max(m[0], m[1]);
  int cur = 0;
  int fin[2] = {0, 0};
  for (int s = 1; s < mmax; s *= 2) {
    const double* Pa = K.P[cur];
    double* Pn = K.P[cur ^ 1];
    for (int r = tid; r < mt; r += kThreads) {
      int q = r < m[0] ? 0 : 1;
      int mq = m[q];
      if (s >= mq) continue;
      int k = q == 0 ? r : r - m[0];
      bool hl = k - s >= 0, hr = k + s < mq;
      int rl = r - s, rr = r + s;
      double ak = Pa[r], bk = Pa[cap + r], ck = Pa[2 * cap + r], dk = Pa[3 * cap + r];
      double b_left = hl ? Pa[cap + rl] : 1.0;
      double b_right = hr ? Pa[cap + rr] : 1.0;
      double alpha = hl ? ak / b_left : 0.0;
      double beta = hr ? ck / b_right : 0.0;
      double a_left = hl ? Pa[rl] : 0.0;
      double c_left = hl ? Pa[2 * cap + rl] : 0.0;
      double d_left = hl ? Pa[3 * cap + rl] : 0.0;
      double a_right = hr ? Pa[rr] : 0.0;
      double c_right = hr ? Pa[2 * cap + rr] : 0.0;
      double d_right = hr ? Pa[3 * cap + rr] : 0.0;
      Pn[r] = -alpha * a_left;
      Pn[2 * cap + r] = -beta * c_right;
      Pn[cap + r] = bk - alpha * c_left - beta * a_right;
      Pn[3 * cap + r] = dk - alpha * d_left - beta * d_right;
    }
    if (s < m[0]) fin[0] ^= 1;
    if (s < m[1]) fin[1] ^= 1;
    cur ^= 1;
    __syncthreads();
  }
  // diagonal solve + end-moment recovery (M[0], M[n-1] by the owners of the end rows)
  for (int r = tid; r < mt; r += kThreads) {
    int q = r < m[0] ? 0 : 1;
    int k = q == 0 ? r : r - m[0];
    int mq = m[q];
    int n = kcnt[q];
    const double* Pf = K.P[fin[q]];
    double* M = K.M[q];
    double Mk1 = Pf[3 * cap + r] / Pf[cap + r];
    M[k + 1] = Mk1;
    if (k == 0) {
      const double* x = K.X[q] + kbase[q];
      double M2 = Pf[3 * cap + r + 1] / Pf[cap + r + 1];
      double h0 = x[1] - x[0], h1 = x[2] - x[1];
      M[0] = ((h0 + h1) * Mk1 - h0 * M2) / h1;
    }
    if (k == mq - 1) {
      const double* x = K.X[q] + kbase[q];
      double Mnm3 = Pf[3 * cap + r - 1] / Pf[cap + r - 1];
      double hnm3 = x[n - 2] - x[n - 3], hnm2 = x[n - 1] - x[n - 2];
      M[n - 1] = ((hnm3 + hnm2) * Mk1 - hnm2 * Mnm3) / hnm3;
    }
  }
  __syncthreads();
}

// Envelope value at t (kernels.py:702-734); `inr` reports the t-range mask.
__device__ inline double eval_env(const SideView& s, double t, bool& inr) {
  const double* x = s.x;
  const double* y = s.y;
  int n = s.n;
  inr = !(t < x[0] || t > x[n - 1]);
  if (n == 2) {
    double slope = (y[1] - y[0]) / (x[1] - x[0]);
    return y[0] + slope * (t - x[0]);
  }
  if (n == 3) {
    double l0 = (t - x[1]) * (t - x[2]) / ((x[0] - x[1]) * (x[0] - x[2]));
    double l1 = (t - x[0]) * (t - x[2]) / ((x[1] - x[0]) * (x[1] - x[2]));
    double l2 = (t - x[0]) * (t - x[1]) / ((x[2] - x[0]) * (x[2] - x[1]));
    return y[0] * l0 + y[1] * l1 + y[2] * l2;
  }
  int lo = 0, hi = n - 2;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (x[mid] <= t) lo = mid; else hi = mid - 1;
  }
  double x0 = x[lo], x1 = x[lo + 1];
  double y0 = y[lo], y1 = y[lo + 1];
  double M0 = s.M[lo], M1 = s.M[lo + 1];
  double h = x1 - x0;
  double A = (x1 - t) / h;
  double B = (t - x0) / h;
  return A * y0 + B * y1 + ((A * A * A - A) * M0 + (B * B * B - B) * M1) * (h * h) / 6.0;
}

// 128-lane tree of the reference (kernels.py:794-804), on warp 0, for a value
// each thread has stored at red[q*128 + tid].  op 0: sum, 1: fmax, 2: fmin.
__device__ inline double lane_tree(const double* red, int lane, int op) {
  double v0 = red[lane], v1 = red[lane + 32], v2 = red[lane + 64], v3 = red[lane + 96];
  double r;
  if (op == 0) r = (v0 + v2) + (v1 + v3);
  else if (op == 1) r = fmax(fmax(v0, v2), fmax(v1, v3));
  else r = fmin(fmin(v0, v2), fmin(v1, v3));
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    double o = __shfl_down_sync(kFull, r, s);
    if (op == 0) r = r + o;
    else if (op == 1) r = fmax(r, o);
    else r = fmin(r, o);
  }
  return r;
}

}  // namespace

// ---------------------------------------------------------------------------
// The sift kernel.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 4) emd_sift_kernel(SiftParams p) {
  extern __shared__ __align__(16) char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int NB = p.nbsym;
  const int MAXI = p.max_imfs;
  Ctl* Cs = reinterpret_cast<Ctl*>(smem);
  char* slab = p.slab + (size_t)blockIdx.x * p.slab_stride;

  for (;;) {
    if (tid == 0) Cs->job = atomicAdd(p.queue, 1);
    __syncthreads();
    const int job = Cs->job;
    if (job >= p.batch) break;
    const int b = p.order ? p.order[job] : job;
    const int64_t off = p.offsets ? p.offsets[b] : (int64_t)b * p.dense_n;
    const int N = p.offsets ? (int)(p.offsets[b + 1] - off) : p.dense_n;
    const double* S = p.values + off;
    double* out = p.imfs + (int64_t)MAXI * off;
    TimeAxis T;
    T.arange = p.t_mode == kTArange;
    T.T = p.t_mode == kTShared ? p.T : (p.t_mode == kTPerTrace ? p.T + off : nullptr);

    if (fixed_bytes(N) + 64 > (size_t)p.arena_bytes) {
      // cannot hold this trace: report, leave outputs flagged
      if (tid == 0) {
        atomicOr(p.status, kStatusTooLong);
        p.n_imfs[b] = 0;
        p.overflow[b] = 1;
      }
      for (int k = tid; k < MAXI; k += kThreads) {
        p.dbg_n[(int64_t)b * MAXI + k] = -1;
        p.dbg_ext[(int64_t)b * MAXI + k] = -1;
        p.dbg_nzm[(int64_t)b * MAXI + k] = -1;
      }
      __syncthreads();
      continue;
    }
    SmemLayout L = carve(smem, N, p.arena_bytes);
    Ctl& C = *L.ctl;
    double* imf = L.imf;
    for (int k = tid; k < MAXI; k += kThreads) { C.dbg_n[k] = -1; C.dbg_e[k] = -1; C.dbg_z[k] = -1; }
    for (int i = tid; i < N; i += kThreads) imf[i] = S[i];
    __syncthreads();

    bool ovf = false;
    int imf_count = 0;
    bool finished = false;
    int extNo_last = -1;
    bool stale = false;

    ExtInfo e = extrema_scan(L, N, tid, warp, lane, p.max_extrema);
    ovf |= e.overflow;

    while (!finished && imf_count < MAXI - 1) {
      int n = 0;
      for (;;) {
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
        // ---- knot storage for this pass ----
        const int kc0 = e.n_max + 2 * NB + 2, kc1 = e.n_min + 2 * NB + 2;
        size_t need = knot_bytes(kc0, kc1);
        char* kb = need <= (size_t)L.arena_bytes ? L.arena : slab;
        Knots K = place_knots(kb, kc0, kc1);
        // ---- true knots, then mirrored knots ----
        bool bad = fill_true_knots(L, K, e, N, NB, T, warp, lane);
        bad = __syncthreads_or(bad);
        bool mbad = false;
        if (warp == 0) mbad = mirror_both(L, K, e, N, NB, T, lane);
        bad = __syncthreads_or(bad || mbad);
        int kbase[2] = {C.kbase[0], C.kbase[1]};
        int kcnt[2] = {C.kcnt[0], C.kcnt[1]};
        // ---- both not-a-knot systems ----
        solve_splines(K, kbase, kcnt, tid);
        // ---- fused: envelopes, mean, update, stop-test partial sums ----
        SideView sv[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          sv[q].x = K.X[q] + kbase[q];
          sv[q].y = K.Y[q] + kbase[q];
          sv[q].M = K.M[q];
          sv[q].n = kcnt[q];
        }
        double s_sq = 0.0, s_dsq = 0.0, s_osq = 0.0, s_std = 0.0;
        double s_max = -1e30, s_min = 1e30;
        bool oor = false;
        for (int i = tid; i < N; i += kThreads) {
          double t = T(i);
          bool r0, r1;
          double emax = eval_env(sv[0], t, r0);
          double emin = eval_env(sv[1], t, r1);
          oor |= !(r0 && r1);
          double mean = 0.5 * (emax + emin);
          double old = imf[i];
          double nw = old - mean;
          imf[i] = nw;
          double diff = nw - old;
          s_sq += nw * nw;
          s_dsq += diff * diff;
          s_osq += old * old;
          double qd = diff / nw;
          s_std += qd * qd;
          s_max = fmax(s_max, old);
          s_min = fmin(s_min, old);
        }
        stale |= oor;
        double* red = L.red;
        red[tid] = s_sq; red[128 + tid] = s_dsq; red[256 + tid] = s_osq;
        red[384 + tid] = s_std; red[512 + tid] = s_max; red[640 + tid] = s_min;
        __syncthreads();
        if (warp == 0) {
          double a0 = lane_tree(red, lane, 0);
          double a1 = lane_tree(red + 128, lane, 0);
          double a2 = lane_tree(red + 256, lane, 0);
          double a3 = lane_tree(red + 384, lane, 0);
          double a4 = lane_tree(red + 512, lane, 1);
          double a5 = lane_tree(red + 640, lane, 2);
          if (lane == 0) {
            C.sums[0] = a0; C.sums[1] = a1; C.sums[2] = a2;
            C.sums[3] = a3; C.sums[4] = a4; C.sums[5] = a5;
          }
        }
        // ---- post-update extrema scan (also next pass's pre-scan) ----
        e = extrema_scan(L, N, tid, warp, lane, p.max_extrema);
        ovf |= e.overflow;
        const int extNo2 = e.n_max + e.n_min;
        const int nzm2 = e.n_zer;
        const bool f2 = abs(extNo2 - nzm2) < 2;
        bool f1 = false;
        if (!bad) {
          double sum_new_sq = C.sums[0], diff_sq = C.sums[1], old_sq = C.sums[2];
          double std_sum = C.sums[3], omax = C.sums[4], omin = C.sums[5];
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
      // ---- emit IMF row, running residue into the next row, end condition ----
      {
        const double* rsrc = imf_count == 0 ? S : out + (int64_t)imf_count * N;
        double* row = out + (int64_t)imf_count * N;
        double* rnext = out + (int64_t)(imf_count + 1) * N;
        double gmax = -1e30, gmin = 1e30, gabs = 0.0;
        for (int i = tid; i < N; i += kThreads) {
          double r = rsrc[i];
          double v = imf[i];
          row[i] = v;
          double rn = r - v;
          rnext[i] = rn;
          gmax = fmax(gmax, rn);
          gmin = fmin(gmin, rn);
          gabs += fabs(rn);
        }
        double* red = L.red;
        red[tid] = gmax; red[128 + tid] = gmin; red[256 + tid] = gabs;
        __syncthreads();
        if (warp == 0) {
          double a0 = lane_tree(red, lane, 1);
          double a1 = lane_tree(red + 128, lane, 2);
          double a2 = lane_tree(red + 256, lane, 0);
          if (lane == 0) { C.sums[6] = a0 - a1; C.sums[7] = a2; }
        }
        __syncthreads();
        ++imf_count;
        if (C.sums[6] < kRangeThr || C.sums[7] < kTotalPowerThr) finished = true;
      }
      if (!finished && imf_count < MAXI - 1) {
        const double* rsrc = out + (int64_t)imf_count * N;
        for (int i = tid; i < N; i += kThreads) imf[i] = rsrc[i];
        __syncthreads();
        e = extrema_scan(L, N, tid, warp, lane, p.max_extrema);
        ovf |= e.overflow;
      }
    }

    // ---- epilogue: trend removal, residue ~ 0 test, zero unused rows ----
    const int last_row = imf_count;   // row holding the running residue (or none if 0 IMFs)
    const bool trend = extNo_last <= 2 && imf_count > 0;
    if (trend) imf_count -= 1;
    const double* rres = last_row == 0 ? S : out + (int64_t)last_row * N;
    double amax = 0.0;
    for (int i = tid; i < N; i += kThreads) {
      double r = rres[i];
      if (trend) r = r + imf[i];
      amax = fmax(amax, fabs(r));
    }
    double* red = L.red;
    red[tid] = amax;
    __syncthreads();
    if (warp == 0) {
      double a = lane_tree(red, lane, 1);
      if (lane == 0) C.sums[0] = a;
    }
    __syncthreads();
    const bool rzero = C.sums[0] <= kResidueZeroAtol;
    const int nim = rzero ? imf_count : imf_count + 1;
    for (int i = tid; i < N; i += kThreads) {
      if (trend) {
        double r = rres[i] + imf[i];
        if (!rzero) out[(int64_t)imf_count * N + i] = r;
        out[(int64_t)last_row * N + i] = 0.0;
      } else {
        if (rzero && last_row < MAXI) out[(int64_t)last_row * N + i] = 0.0;
        else if (last_row == 0) out[i] = S[i];
      }
    }
    const int first_zero = last_row + 1;
    for (int64_t k = (int64_t)first_zero * N + tid; k < (int64_t)MAXI * N; k += kThreads) out[k] = 0.0;
    if (tid == 0) {
      p.n_imfs[b] = nim;
      p.overflow[b] = ovf ? 1 : 0;
      if (stale) atomicOr(p.status, kStatusStaleEnvelope);
    }
    for (int k = tid; k < MAXI; k += kThreads) {
      p.dbg_n[(int64_t)b * MAXI + k] = C.dbg_n[k];
      p.dbg_ext[(int64_t)b * MAXI + k] = C.dbg_e[k];
      p.dbg_nzm[(int64_t)b * MAXI + k] = C.dbg_z[k];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Envelope-only diagnostic (envelope_batch_kernel, kernels.py:1100-1166):
// extrema + mirroring + both envelopes on raw traces, no sift loop.  The
// reference scans with find_extrema_serial here; the extrema lists are the
// same as the sift scan's (plateau rule included) and n_zer is not reported.
// ---------------------------------------------------------------------------
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
    const double* S = p.values + off;
    double* emax_out = p.max_env + off;
    double* emin_out = p.min_env + off;
    double* kp[2] = {p.max_kpos + (int64_t)b * p.mbuf, p.min_kpos + (int64_t)b * p.mbuf};
    double* kv[2] = {p.max_kval + (int64_t)b * p.mbuf, p.min_kval + (int64_t)b * p.mbuf};
    TimeAxis T;
    T.arange = p.t_mode == kTArange;
    T.T = p.t_mode == kTShared ? p.T : (p.t_mode == kTPerTrace ? p.T + off : nullptr);
    if (fixed_bytes(N) + 64 > (size_t)p.arena_bytes) {
      if (tid == 0) {
        atomicOr(p.status, kStatusTooLong);
        p.degenerate[b] = 1;
        p.n_extrema[2 * b] = 0; p.n_extrema[2 * b + 1] = 0;
        p.n_mirrored[2 * b] = 0; p.n_mirrored[2 * b + 1] = 0;
      }
      __syncthreads();
      continue;
    }
    SmemLayout L = carve(smem, N, p.arena_bytes);
    Ctl& C = *L.ctl;
    for (int i = tid; i < N; i += kThreads) L.imf[i] = S[i];
    __syncthreads();
    ExtInfo e = extrema_scan(L, N, tid, warp, lane, p.max_extrema);
    const bool degenerate = !(e.n_max + e.n_min > 2 && e.n_max >= 1 && e.n_min >= 1);
    int nk[2] = {0, 0};
    if (!degenerate) {
      const int kc0 = e.n_max + 2 * NB + 2, kc1 = e.n_min + 2 * NB + 2;
      char* kb = knot_bytes(kc0, kc1) <= (size_t)L.arena_bytes ? L.arena : slab;
      Knots K = place_knots(kb, kc0, kc1);
      fill_true_knots(L, K, e, N, NB, T, warp, lane);
      __syncthreads();
      if (warp == 0) mirror_both(L, K, e, N, NB, T, lane);
      __syncthreads();
      int kbase[2] = {C.kbase[0], C.kbase[1]};
      int kcnt[2] = {C.kcnt[0], C.kcnt[1]};
      solve_splines(K, kbase, kcnt, tid);
      SideView sv[2];
      for (int q = 0; q < 2; ++q) {
        sv[q].x = K.X[q] + kbase[q]; sv[q].y = K.Y[q] + kbase[q];
        sv[q].M = K.M[q]; sv[q].n = kcnt[q];
        nk[q] = kcnt[q];
      }
      bool oor = false;
      for (int i = tid; i < N; i += kThreads) {
        double t = T(i);
        bool r0, r1;
        double a = eval_env(sv[0], t, r0);
        double c = eval_env(sv[1], t, r1);
        emax_out[i] = r0 ? a : 0.0;
        emin_out[i] = r1 ? c : 0.0;
        oor |= !(r0 && r1);
      }
      if (oor) atomicOr(p.status, kStatusStaleEnvelope);
      for (int q = 0; q < 2; ++q)
        for (int k = tid; k < p.mbuf; k += kThreads) {
          kp[q][k] = k < kcnt[q] ? sv[q].x[k] : 0.0;
          kv[q][k] = k < kcnt[q] ? sv[q].y[k] : 0.0;
        }
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

size_t sift_fixed_smem(int N) { return fixed_bytes(N); }

size_t sift_slab_bytes(int max_extrema, int nbsym) {
  size_t kc = (size_t)max_extrema + 2 * (size_t)nbsym + 2;
  return align16((3 * 2 * kc + 8 * 2 * kc) * sizeof(double));
}

cudaError_t sift_occupancy(int arena_bytes, int* ctas_per_sm) {
  cudaError_t e = cudaFuncSetAttribute(emd_sift_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       arena_bytes);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, emd_sift_kernel, kThreads,
                                                       arena_bytes);
}

cudaError_t launch_sift(const SiftParams& p, int grid, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(emd_sift_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       p.arena_bytes);
  if (e != cudaSuccess) return e;
  emd_sift_kernel<<<grid, kThreads, p.arena_bytes, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace emdb
