"""CPU oracle for the batched EMD sift -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may
import it.  The product path (``cuda_emd``) never calls into it and fails
loudly when its CUDA library is missing.

What it restates
----------------
The reference (SeismicFlow/emd-cuda) keeps its whole algorithm inside the CUDA
string ``_CUDA_SOURCE`` of ``kernels.py``.  This file restates that algorithm in
FP64 NumPy, step for step, so that a GPU kernel built without FMA contraction
(``-fmad=false``) reproduces it bit for bit:

* extrema / zero crossings: ``find_extrema_parallel`` with its serial fallback
  (kernels.py:115-204, 231-349), including the fallback trigger and the
  leading-zero zero-crossing difference between the two paths;
* boundary mirroring and knot build with adjacent-duplicate removal
  (``mirror_one_side``, kernels.py:360-558);
* the not-a-knot spline: reduced (n-2) tridiagonal system, parallel cyclic
  reduction, end-moment recovery, per-sample binary search and evaluation
  (``notaknot_cubic_spline_block``, kernels.py:585-736);
* the stop tests (``check_imf_block``, kernels.py:742-821; f2 at kernels.py:970);
* the sift / outer loop, end condition, trend removal and residue-zero check
  (``emd_batch_kernel``, kernels.py:834-1080);
* T normalisation (emd.py:83-88).

Floating-point order
--------------------
Every sum the reference forms with a block reduction is formed here in the
same order: thread ``t`` of ``LANES`` (=THREADS=128, kernels.py:75) adds
samples ``t, t+LANES, ...`` sequentially, then a tree halves the lanes
(``red[t] += red[t+s]`` for s = LANES/2 .. 1).  Products, quotients and sums
are written in the reference's association order.  NumPy never fuses a
multiply-add, so this equals a CUDA build with FMA contraction off.

Parity pinning: ``tests/golden/`` holds outputs of the reference's own
``emd_batch_kernel`` (compiled from kernels.py by ``oracle/build_ref.py`` and
run on a B200); ``tests/test_oracle_golden.py`` checks this oracle against them.

REAL_T = float
---------------
The reference's kernel source is written over ``REAL_T`` (kernels.py:78),
substituted when it is built (kernels.py:1277-1285).  With
``OracleConfig(real_t="float")`` every array and REAL_T variable here is
float32 and the source's double literals keep their C++ meaning: a float
expression that meets one is evaluated in double and rounded once when it is
stored (the mirrored positions ``2.0 * T[a] - T[b]``, kernels.py:471-489,
528-553; the spline rows' ``h0 + 2.0 * h1``, kernels.py:551, 558; the
evaluation's ``... * (h * h) / 6.0``, kernels.py:733), and the two tests
against double literals compare in double (``sum_new_sq < 1e-10``,
kernels.py:814; ``<= 1e-8``, kernels.py:1069).  Where float arithmetic and that
double detour give the same value (a product by 2.0 or 6.0 of a float, a
float compared with 0.0) the float form is used.  NumPy's float32 operations
round every step (NEP 50 keeps Python scalars weak), as a CUDA build without
FMA contraction does.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import math

import numpy as np

# PyEMD default thresholds hard-coded in the reference (kernels.py:81-85).
ENERGY_RATIO_THR = 0.2
STD_THR = 0.2
SVAR_THR = 0.001
TOTAL_POWER_THR = 0.005
RANGE_THR = 0.001
# Σ new² early-out (kernels.py:814) and residue ~ 0 test (kernels.py:1069).
SUM_NEW_SQ_MIN = 1e-10
RESIDUE_ZERO_ATOL = 1e-8
# Per-thread extrema buffer of the parallel scan (kernels.py:206).
LOCAL_EXT_BUF = 64


@dataclass
class OracleConfig:
    """Mirror of the reference's ``EMDKernelConfig`` fields (kernels.py:1170-1176),
    plus the REAL_T its kernel source is built with."""

    max_extrema: int = 1024
    nbsym: int = 2
    max_iteration: int = 1000
    max_imfs: int = 16
    threads_per_block: int = 128
    real_t: str = "double"

    @property
    def rtype(self):
        return np.float32 if self.real_t == "float" else np.float64


@dataclass
class Extrema:
    ind_max: np.ndarray
    ind_min: np.ndarray
    n_zer: int
    overflow: bool
    serial: bool  # True when the reference would have taken its serial fallback


@dataclass
class SignalResult:
    imfs: np.ndarray        # [max_imfs, N]
    n_imfs: int
    overflow: int
    debug_n: np.ndarray     # [max_imfs] int32
    debug_extno: np.ndarray
    debug_nzm: np.ndarray
    stats: dict = field(default_factory=dict)


# ---------------------------------------------------------------------------
# Reductions in the reference's block order
# ---------------------------------------------------------------------------

def lane_sum(x: np.ndarray, lanes: int = 128) -> float:
    """Σx formed like the reference's strided-accumulate + halving tree
    (e.g. kernels.py:777-804, 1016-1033).  Terms must be >= 0 or NaN (all the
    reference's sums are), so the zero padding is exact."""
    n = x.shape[0]
    dt = x.dtype if x.dtype == np.float32 else np.float64
    rows = -(-n // lanes) if n else 1
    buf = np.zeros(rows * lanes, dtype=dt)
    buf[:n] = x
    grid = buf.reshape(rows, lanes)
    acc = np.zeros(lanes, dtype=dt)
    for r in range(rows):
        acc = acc + grid[r]
    s = lanes // 2
    while s > 0:
        acc[:s] = acc[:s] + acc[s:2 * s]
        s //= 2
    return acc[0] if dt == np.float32 else float(acc[0])


def _scalar(v, dt):
    return v if dt == np.float32 else float(v)


def lane_max(x: np.ndarray, init: float = -1e30):
    """max over samples with the reference's -1e30 seed (a REAL_T); CUDA max is fmax."""
    dt = x.dtype.type
    return _scalar(np.fmax.reduce(x, initial=dt(init)) if x.size else dt(init), dt)


def lane_min(x: np.ndarray, init: float = 1e30):
    dt = x.dtype.type
    return _scalar(np.fmin.reduce(x, initial=dt(init)) if x.size else dt(init), dt)


# ---------------------------------------------------------------------------
# Extrema detection (kernels.py:115-349)
# ---------------------------------------------------------------------------

def _extrema_serial(S: np.ndarray, max_extrema: int):
    """Literal restatement of find_extrema_serial (kernels.py:115-204)."""
    N = S.shape[0]
    # float32 samples stay float32 scalars (their differences and products
    # round to float, as REAL_T = float does); float64 ones become Python floats
    s = list(S) if S.dtype == np.float32 else S.tolist()
    n_zer = 0
    in_zero_run = False
    for i in range(N):
        is_zero = s[i] == 0.0
        if is_zero and not in_zero_run:
            in_zero_run = True
        if (not is_zero) and in_zero_run:
            n_zer += 1
            in_zero_run = False
        if (not is_zero) and i + 1 < N and s[i] * s[i + 1] < 0.0:
            n_zer += 1
    imax: list[int] = []
    imin: list[int] = []
    nmax = nmin = 0  # true counts (the reference saturates its stored count)
    i = 1
    while i < N - 1:
        dprev = s[i] - s[i - 1]
        dnext = s[i + 1] - s[i]
        if dprev * dnext < 0.0:
            if dprev < 0.0:
                nmin += 1
                if len(imin) < max_extrema:
                    imin.append(i)
            else:
                nmax += 1
                if len(imax) < max_extrema:
                    imax.append(i)
        elif dnext == 0.0 and dprev != 0.0:
            j = i
            while j + 1 < N and s[j + 1] == s[i]:
                j += 1
            if j + 1 < N:
                d_after = s[j + 1] - s[j]
                mid = (i + j) // 2
                if dprev > 0.0 and d_after < 0.0:
                    nmax += 1
                    if len(imax) < max_extrema:
                        imax.append(mid)
                elif dprev < 0.0 and d_after > 0.0:
                    nmin += 1
                    if len(imin) < max_extrema:
                        imin.append(mid)
            i = j
        i += 1
    overflow = len(imax) >= max_extrema or len(imin) >= max_extrema
    return (np.asarray(imax, dtype=np.int64), np.asarray(imin, dtype=np.int64),
            n_zer, overflow)


def find_extrema(S: np.ndarray, max_extrema: int = 1024, threads: int = 128) -> Extrema:
    """Effective behaviour of find_extrema_parallel (kernels.py:231-349).

    The parallel scan hands the whole job to the serial scan when any interior
    sample i in [1, N-2] has S[i]==0 or a zero forward/backward difference, or
    a thread's chunk holds more than LOCAL_EXT_BUF maxima or minima
    (kernels.py:264-288).  Otherwise extrema are the strict ones
    (dprev*dnext < 0, kernels.py:265-271) and zero crossings are counted as
    ``S[i] != 0 && S[i]*S[i+1] < 0`` over i in [0, N-2] (kernels.py:273-276) --
    which, unlike the serial count, does not count a leading exact zero.
    """
    N = S.shape[0]
    if N < 3:
        # Interior range empty: the parallel scan never falls back.
        nz = 0
        for i in range(N - 1):
            if S[i] != 0.0 and S[i] * S[i + 1] < 0.0:
                nz += 1
        e = np.zeros(0, dtype=np.int64)
        return Extrema(e, e, nz, max_extrema <= 0, False)
    d = S[1:] - S[:-1]
    dprev = d[:-1]
    dnext = d[1:]
    fallback = bool(np.any(dprev == 0.0) or np.any(dnext == 0.0) or np.any(S[1:-1] == 0.0))
    with np.errstate(all="ignore"):
        prod = dprev * dnext
    strict = prod < 0.0
    is_min = strict & (dprev < 0.0)
    is_max = strict & ~(dprev < 0.0)
    if not fallback:
        chunk = -(-N // threads)
        # extrema positions i in [1, N-2] -> chunk id i // chunk
        idx = np.arange(1, N - 1)
        cid = idx // chunk
        cmax = np.bincount(cid[is_max], minlength=threads)
        cmin = np.bincount(cid[is_min], minlength=threads)
        if cmax.max(initial=0) > LOCAL_EXT_BUF or cmin.max(initial=0) > LOCAL_EXT_BUF:
            fallback = True
    if fallback:
        imax, imin, n_zer, ovf = _extrema_serial(S, max_extrema)
        return Extrema(imax, imin, n_zer, ovf, True)
    with np.errstate(all="ignore"):
        zc = (S[:-1] != 0.0) & (S[:-1] * S[1:] < 0.0)
    n_zer = int(np.count_nonzero(zc))
    imax = np.flatnonzero(is_max) + 1
    imin = np.flatnonzero(is_min) + 1
    ovf = imax.size >= max_extrema or imin.size >= max_extrema
    return Extrema(imax[:max_extrema], imin[:max_extrema], n_zer, bool(ovf), False)


# ---------------------------------------------------------------------------
# Boundary mirroring + knot lists (kernels.py:360-558)
# ---------------------------------------------------------------------------

def mirror_knots(T: np.ndarray, S: np.ndarray, ind_max: np.ndarray, ind_min: np.ndarray,
                 nbsym: int = 2):
    """Both envelopes' knot lists, as the two mirror_one_side calls build them.

    Returns ``((pos_max, val_max), (pos_min, val_min), info)``; ``info`` holds
    lsym/rsym and the mirrored index lists for stage-level tests.
    """
    N = S.shape[0]
    im = [int(v) for v in ind_max]
    iN = [int(v) for v in ind_min]
    n_max, n_min = len(im), len(iN)
    NB = nbsym
    # ---- left bound (kernels.py:383-413) ----
    if im[0] < iN[0]:
        if S[0] > S[iN[0]]:
            lmax = [im[k] for k in range(min(n_max, NB + 1) - 1, 0, -1)]
            lmin = [iN[k] for k in range(min(n_min, NB) - 1, -1, -1)]
            lsym = im[0]
        else:
            lmax = [im[k] for k in range(min(n_max, NB) - 1, -1, -1)]
            lmin = [iN[k] for k in range(min(n_min, NB - 1) - 1, -1, -1)] + [0]
            lsym = 0
    else:
        if S[0] < S[im[0]]:
            lmax = [im[k] for k in range(min(n_max, NB) - 1, -1, -1)]
            lmin = [iN[k] for k in range(min(n_min, NB + 1) - 1, 0, -1)]
            lsym = iN[0]
        else:
            lmax = [im[k] for k in range(min(n_max, NB - 1) - 1, -1, -1)] + [0]
            lmin = [iN[k] for k in range(min(n_min, NB) - 1, -1, -1)]
            lsym = 0
    # ---- right bound (kernels.py:415-454) ----
    if im[n_max - 1] < iN[n_min - 1]:
        if S[N - 1] < S[im[n_max - 1]]:
            rmax = [im[k] for k in range(n_max - 1, max(n_max - NB, 0) - 1, -1)]
            rmin = [iN[k] for k in range(n_min - 2, max(n_min - NB - 1, 0) - 1, -1)]
            rsym = iN[n_min - 1]
        else:
            rmax = [N - 1] + [im[k] for k in range(max(n_max - NB + 1, 0), n_max)]
            rmin = [iN[k] for k in range(n_min - 1, max(n_min - NB, 0) - 1, -1)]
            rsym = N - 1
    else:
        if S[N - 1] > S[iN[n_min - 1]]:
            rmax = [im[k] for k in range(n_max - 2, max(n_max - NB - 1, 0) - 1, -1)]
            rmin = [iN[k] for k in range(n_min - 1, max(n_min - NB, 0) - 1, -1)]
            rsym = im[n_max - 1]
        else:
            rmax = [im[k] for k in range(n_max - 1, max(n_max - NB, 0) - 1, -1)]
            rmin = [N - 1] + [iN[k] for k in range(max(n_min - NB + 1, 0), n_min)]
            rsym = N - 1
    lmin_fb, rmin_fb = len(lmin) == 0, len(rmin) == 0
    lmax_fb, rmax_fb = len(lmax) == 0, len(rmax) == 0
    # ---- "mirrored point does not reach the boundary" (kernels.py:469-503) ----
    R = T.dtype.type
    # REAL_T x = 2.0 * T[a] - T[b]: formed in double, stored as REAL_T
    mpos = lambda a, b: R(2.0 * float(T[a]) - float(T[b]))
    lmin_first = iN[0] if lmin_fb else lmin[0]
    lmax_first = im[0] if lmax_fb else lmax[0]
    tlmin0 = mpos(lsym, lmin_first)
    tlmax0 = mpos(lsym, lmax_first)
    if tlmin0 > T[0] or tlmax0 > T[0]:
        if lsym == im[0]:
            lmax = [im[k] for k in range(min(n_max, NB) - 1, -1, -1)]
            lmax_fb = False
        else:
            lmin = [iN[k] for k in range(min(n_min, NB) - 1, -1, -1)]
            lmin_fb = False
        lsym = 0
    rmin_last = iN[n_min - 1] if rmin_fb else rmin[-1]
    rmax_last = im[n_max - 1] if rmax_fb else rmax[-1]
    trmin_last = mpos(rsym, rmin_last)
    trmax_last = mpos(rsym, rmax_last)
    if trmin_last < T[N - 1] or trmax_last < T[N - 1]:
        if rsym == im[n_max - 1]:
            rmax = [im[k] for k in range(n_max - 1, max(n_max - NB, 0) - 1, -1)]
            rmax_fb = False
        else:
            rmin = [iN[k] for k in range(n_min - 1, max(n_min - NB, 0) - 1, -1)]
            rmin_fb = False
        rsym = N - 1

    def build(true_idx, lbuf, l_fb, rbuf, r_fb):
        li = true_idx if l_fb else lbuf
        ri = true_idx if r_fb else rbuf
        li = np.asarray(li, dtype=np.int64)
        ri = np.asarray(ri, dtype=np.int64)
        ti = np.asarray(true_idx, dtype=np.int64)
        T64 = T.astype(np.float64)
        pos = np.concatenate([(2.0 * T64[lsym] - T64[li]).astype(R), T[ti],
                              (2.0 * T64[rsym] - T64[ri]).astype(R)])
        val = np.concatenate([S[li], S[ti], S[ri]])
        # keep a knot unless its position equals the previous one (kernels.py:521-556)
        keep = np.ones(pos.shape[0], dtype=bool)
        keep[1:] = pos[1:] != pos[:-1]
        return pos[keep], val[keep]

    kmax = build(im, lmax, lmax_fb, rmax, rmax_fb)
    kmin = build(iN, lmin, lmin_fb, rmin, rmin_fb)
    info = dict(lsym=lsym, rsym=rsym, lmax=lmax, lmin=lmin, rmax=rmax, rmin=rmin,
                lmax_fb=lmax_fb, lmin_fb=lmin_fb, rmax_fb=rmax_fb, rmin_fb=rmin_fb)
    return kmax, kmin, info


# ---------------------------------------------------------------------------
# Not-a-knot spline (kernels.py:585-736)
# ---------------------------------------------------------------------------

def spline_moments(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Second-derivative moments M[0..n-1] for n >= 4 knots: reduced system
    setup (kernels.py:613-636), PCR (kernels.py:648-677), diagonal solve
    (kernels.py:683-689) and end recovery (kernels.py:691-696)."""
    n = x.shape[0]
    m = n - 2
    R = x.dtype.type
    a = np.empty(m, dtype=R)
    b = np.empty(m, dtype=R)
    c = np.empty(m, dtype=R)
    d = np.empty(m, dtype=R)
    with np.errstate(all="ignore"):
        # interior rows k in [1, m-2] -> original row i = k+1
        if m > 2:
            i = np.arange(2, m)  # original rows of k = 1..m-2
            h_im1 = x[i] - x[i - 1]
            h_i = x[i + 1] - x[i]
            a[1:m - 1] = h_im1
            b[1:m - 1] = 2.0 * (h_im1 + h_i)
            c[1:m - 1] = h_i
            d[1:m - 1] = 6.0 * ((y[i + 1] - y[i]) / h_i - (y[i] - y[i - 1]) / h_im1)
        h0 = x[1] - x[0]
        h1 = x[2] - x[1]
        rhs1 = 6.0 * ((y[2] - y[1]) / h1 - (y[1] - y[0]) / h0)
        a[0] = 0.0
        b[0] = R(float(h0) + 2.0 * float(h1))          # double literal: formed in double
        c[0] = h1 - h0
        d[0] = h1 * rhs1 / (h0 + h1)
        hnm3 = x[n - 2] - x[n - 3]
        hnm2 = x[n - 1] - x[n - 2]
        rhs_nm2 = 6.0 * ((y[n - 1] - y[n - 2]) / hnm2 - (y[n - 2] - y[n - 3]) / hnm3)
        a[m - 1] = hnm3 - hnm2
        b[m - 1] = R(2.0 * float(hnm3) + float(hnm2))
        c[m - 1] = 0.0
        d[m - 1] = hnm3 * rhs_nm2 / (hnm3 + hnm2)
        if m == 1:  # unreachable for n >= 4; kept for shape safety
            pass
        k = np.arange(m)
        s = 1
        while s < m:
            hl = k - s >= 0
            hr = k + s < m
            kl = np.where(hl, k - s, 0)
            kr = np.where(hr, k + s, 0)
            b_left = np.where(hl, b[kl], 1.0)
            b_right = np.where(hr, b[kr], 1.0)
            alpha = np.where(hl, a / b_left, 0.0)
            beta = np.where(hr, c / b_right, 0.0)
            a_left = np.where(hl, a[kl], 0.0)
            c_left = np.where(hl, c[kl], 0.0)
            d_left = np.where(hl, d[kl], 0.0)
            a_right = np.where(hr, a[kr], 0.0)
            c_right = np.where(hr, c[kr], 0.0)
            d_right = np.where(hr, d[kr], 0.0)
            na = -alpha * a_left
            nc = -beta * c_right
            nb = b - alpha * c_left - beta * a_right
            nd = d - alpha * d_left - beta * d_right
            a, b, c, d = na, nb, nc, nd
            s *= 2
        M = np.empty(n, dtype=R)
        M[1:n - 1] = d / b
        M[0] = ((h0 + h1) * M[1] - h0 * M[2]) / h1
        M[n - 1] = ((hnm3 + hnm2) * M[n - 2] - hnm2 * M[n - 3]) / hnm3
    return M


def spline_eval(T: np.ndarray, x: np.ndarray, y: np.ndarray, M: np.ndarray | None):
    """Evaluate at every T sample (kernels.py:702-734).  Returns (env, in_range):
    samples outside [x[0], x[n-1]] are skipped by the reference, which leaves
    its pool value stale; ``in_range`` marks the evaluated ones."""
    n = x.shape[0]
    t = T
    in_range = ~((t < x[0]) | (t > x[n - 1]))
    out = np.zeros(t.shape[0], dtype=x.dtype)
    with np.errstate(all="ignore"):
        if n == 2:
            slope = (y[1] - y[0]) / (x[1] - x[0])
            out = y[0] + slope * (t - x[0])
        elif n == 3:
            l0 = (t - x[1]) * (t - x[2]) / ((x[0] - x[1]) * (x[0] - x[2]))
            l1 = (t - x[0]) * (t - x[2]) / ((x[1] - x[0]) * (x[1] - x[2]))
            l2 = (t - x[0]) * (t - x[1]) / ((x[2] - x[0]) * (x[2] - x[1]))
            out = y[0] * l0 + y[1] * l1 + y[2] * l2
        else:
            lo = np.zeros(t.shape[0], dtype=np.int64)
            hi = np.full(t.shape[0], n - 2, dtype=np.int64)
            while True:
                act = lo < hi
                if not act.any():
                    break
                mid = (lo + hi + 1) // 2
                cond = x[mid] <= t
                lo = np.where(act & cond, mid, lo)
                hi = np.where(act & ~cond, mid - 1, hi)
            x0 = x[lo]
            x1 = x[lo + 1]
            y0 = y[lo]
            y1 = y[lo + 1]
            M0 = M[lo]
            M1 = M[lo + 1]
            h = x1 - x0
            A = (x1 - t) / h
            B = (t - x0) / h
            if x.dtype == np.float32:
                # "... * (h * h) / 6.0": the quotient and the final sum in
                # double, one rounding to REAL_T at the store
                num = ((A * A * A - A) * M0 + (B * B * B - B) * M1) * (h * h)
                out = ((A * y0 + B * y1).astype(np.float64)
                       + num.astype(np.float64) / 6.0).astype(np.float32)
            else:
                out = A * y0 + B * y1 + ((A * A * A - A) * M0 + (B * B * B - B) * M1) * (h * h) / 6.0
    return out, in_range


def envelope(T: np.ndarray, pos: np.ndarray, val: np.ndarray):
    n = pos.shape[0]
    if n < 2:
        raise AssertionError("fewer than two knots: unreachable for the reference's mirroring")
    M = spline_moments(pos, val) if n >= 4 else None
    return spline_eval(T, pos, val, M)


# ---------------------------------------------------------------------------
# Stop tests (kernels.py:742-821, 970)
# ---------------------------------------------------------------------------

def check_imf(imf_new: np.ndarray, imf_old: np.ndarray, any_bad_sign: bool,
              lanes: int = 128) -> bool:
    if any_bad_sign:
        return False
    with np.errstate(all="ignore"):
        diff = imf_new - imf_old
        sum_new_sq = lane_sum(imf_new * imf_new, lanes)
        diff_sq_sum = lane_sum(diff * diff, lanes)
        old_sq_sum = lane_sum(imf_old * imf_old, lanes)
        q = diff / imf_new
        std_sum = lane_sum(q * q, lanes)
        old_max = lane_max(imf_old)
        old_min = lane_min(imf_old)
        R = imf_new.dtype.type
        # double literal: compared in double (kernels.py:814)
        if float(sum_new_sq) < SUM_NEW_SQ_MIN:
            return False
        # the thresholds are REAL_T functions (kernels.py:81-85)
        svar = diff_sq_sum / (old_max - old_min)
        if svar < R(SVAR_THR):
            return True
        if std_sum < R(STD_THR):
            return True
        energy_ratio = diff_sq_sum / old_sq_sum
        if energy_ratio < R(ENERGY_RATIO_THR):
            return True
    return False


# ---------------------------------------------------------------------------
# One signal (kernels.py:834-1080)
# ---------------------------------------------------------------------------

def emd_signal(S: np.ndarray, T: np.ndarray, cfg: OracleConfig | None = None,
               collect_stats: bool = False) -> SignalResult:
    cfg = cfg or OracleConfig()
    R = cfg.rtype
    S = np.ascontiguousarray(S, dtype=R)
    T = np.ascontiguousarray(T, dtype=R)
    N = S.shape[0]
    lanes = cfg.threads_per_block
    MAXI = cfg.max_imfs
    imfs = np.zeros((MAXI, N), dtype=R)
    dbg_n = np.full(MAXI, -1, dtype=np.int32)
    dbg_e = np.full(MAXI, -1, dtype=np.int32)
    dbg_z = np.full(MAXI, -1, dtype=np.int32)
    overflow = False
    stale = False
    residue = S.copy()
    imf_count = 0
    finished = False
    extNo_last = -1
    imf = residue.copy()
    stats = {"iters": [], "knots": [], "serial_scans": 0} if collect_stats else None

    while (not finished) and imf_count < MAXI - 1:
        imf = residue.copy()
        n = 0
        ext = None
        while True:
            n += 1
            if n >= cfg.max_iteration:
                overflow = True
                if imf_count < MAXI:
                    dbg_n[imf_count] = n
                    dbg_e[imf_count] = -1
                    dbg_z[imf_count] = -1
                break
            # The post-update scan of the previous pass saw this same imf.
            if ext is None:
                ext = find_extrema(imf, cfg.max_extrema, lanes)
                overflow |= ext.overflow
                if stats is not None and ext.serial:
                    stats["serial_scans"] += 1
            n_max, n_min = ext.ind_max.size, ext.ind_min.size
            extNo = n_max + n_min
            if extNo > 2 and n_max >= 1 and n_min >= 1:
                (pmax, vmax), (pmin, vmin), _ = mirror_knots(T, imf, ext.ind_max, ext.ind_min,
                                                             cfg.nbsym)
                bad = bool(np.any(vmax < 0.0) or np.any(vmin > 0.0))
                env_max, r1 = envelope(T, pmax, vmax)
                env_min, r2 = envelope(T, pmin, vmin)
                if not (r1.all() and r2.all()):
                    stale = True
                if stats is not None:
                    stats["knots"].append((pmax.size, pmin.size))
                mean = 0.5 * (env_max + env_min)
                imf_old = imf
                imf = imf - mean
                ext = find_extrema(imf, cfg.max_extrema, lanes)
                overflow |= ext.overflow
                if stats is not None and ext.serial:
                    stats["serial_scans"] += 1
                extNo2 = ext.ind_max.size + ext.ind_min.size
                nzm2 = ext.n_zer
                f2 = abs(extNo2 - nzm2) < 2
                f1 = check_imf(imf, imf_old, bad, lanes)
                extNo_last = extNo2
                if f1 and f2:
                    if imf_count < MAXI:
                        dbg_n[imf_count] = n
                        dbg_e[imf_count] = extNo2
                        dbg_z[imf_count] = nzm2
                    break
            else:
                extNo_last = extNo
                finished = True
                break
        if stats is not None:
            stats["iters"].append(n)
        imfs[imf_count] = imf
        residue = residue - imf
        imf_count += 1
        gmax = lane_max(residue)
        gmin = lane_min(residue)
        gabs = lane_sum(np.abs(residue), lanes)
        if (gmax - gmin) < R(RANGE_THR) or gabs < R(TOTAL_POWER_THR):
            finished = True

    if extNo_last <= 2 and imf_count > 0:
        imf_count -= 1
        residue = residue + imf
    absmax = float(np.fmax.reduce(np.abs(residue), initial=R(0.0)))
    residue_is_zero = absmax <= RESIDUE_ZERO_ATOL      # double literal: compared in double
    if not residue_is_zero:
        imfs[imf_count] = residue
    n_imfs = imf_count if residue_is_zero else imf_count + 1
    st = stats or {}
    st["stale_envelope"] = stale
    return SignalResult(imfs, n_imfs, int(overflow), dbg_n, dbg_e, dbg_z, st)


def normalise_T(T: np.ndarray | None, N: int) -> np.ndarray:
    """emd.py:83-88: arange(N) by default, else (T - T[0]) / min(diff(T))."""
    if T is None:
        return np.arange(N, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    d = np.diff(T)
    return (T - T[0]) / np.min(d)


def emd_batch(signals: np.ndarray, T: np.ndarray | None = None,
              cfg: OracleConfig | None = None):
    """Whole-batch oracle with the reference's outputs
    (imfs, n_imfs, overflow, debug_n, debug_extno, debug_nzm), kernels.py:1343-1372."""
    cfg = cfg or OracleConfig()
    signals = np.atleast_2d(np.asarray(signals, dtype=np.float64))
    B, N = signals.shape
    Tn = normalise_T(T, N)
    imfs = np.zeros((B, cfg.max_imfs, N))
    n_imfs = np.zeros(B, dtype=np.int32)
    ovf = np.zeros(B, dtype=np.int32)
    dn = np.full((B, cfg.max_imfs), -1, dtype=np.int32)
    de = np.full((B, cfg.max_imfs), -1, dtype=np.int32)
    dz = np.full((B, cfg.max_imfs), -1, dtype=np.int32)
    for b in range(B):
        r = emd_signal(signals[b], Tn, cfg)
        imfs[b] = r.imfs
        n_imfs[b] = r.n_imfs
        ovf[b] = r.overflow
        dn[b], de[b], dz[b] = r.debug_n, r.debug_extno, r.debug_nzm
    return imfs, n_imfs, ovf, dn, de, dz


def emd_ragged(values: np.ndarray, offsets: np.ndarray, cfg: OracleConfig | None = None):
    """Per-trace oracle for CSR batches (each trace has its own length and
    T = arange(N_i)).  Returns per-trace SignalResult list."""
    cfg = cfg or OracleConfig()
    out = []
    for b in range(offsets.shape[0] - 1):
        s = values[offsets[b]:offsets[b + 1]]
        out.append(emd_signal(s, np.arange(s.shape[0], dtype=np.float64), cfg))
    return out


def flop_count(N: int, iters: int, knots: list[tuple[int, int]], n_imfs: int) -> float:
    """Algorithmic FP64 operation count used for the roofline: 65 per sample per
    sift pass, 20 per knot per envelope, 4 per sample per IMF."""
    k = sum(a + b for a, b in knots)
    return 65.0 * N * iters + 20.0 * k + 4.0 * N * n_imfs


__all__ = [
    "OracleConfig", "Extrema", "SignalResult", "lane_sum", "find_extrema", "mirror_knots",
    "spline_moments", "spline_eval", "envelope", "check_imf", "emd_signal", "emd_batch",
    "emd_ragged", "normalise_T", "flop_count", "math",
]
