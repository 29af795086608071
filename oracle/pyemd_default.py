"""PyEMD's default EMD restated in FP64 NumPy/SciPy -- TEST INFRASTRUCTURE ONLY.

This module is a checker, never the product: only ``tests/`` and the audit
script beside it use it.

What it restates
----------------
PyEMD (the ``EMD-signal`` package, class ``PyEMD.EMD``) is the method the
reference claims to reproduce (README.md:5, 72-91; kernels.py:44-50,
558-564).  The reference does not vendor or pin it, and it is not installed
here, so this file restates its published default algorithm -- ``EMD()`` with
``spline_kind="cubic"``, ``nbsym=2``, ``extrema_detection="simple"``,
``FIXE=0``, ``FIXE_H=0``, ``MAX_ITERATION=1000``, ``energy_ratio_thr=0.2``,
``std_thr=0.2``, ``svar_thr=0.001``, ``total_power_thr=0.005``,
``range_thr=0.001`` -- in code written for this project:

* extrema ("simple" mode): strict local maxima / minima from the signs of the
  first differences; flat runs classified by the differences before and
  after the run and reported at the run's midpoint rounded half to even, a
  run touching the last sample ignored; PyEMD's left-edge test looks at the
  run starting at difference index 1 (a one-based check carried over from
  the MATLAB original), so a run starting at index 0 is classified with the
  last difference as its "before" slope and a run starting at index 1 is
  ignored;
* zero crossings: sign changes between neighbours plus one per run of exact
  zeros (an isolated zero is a run of one), wherever the run lies;
* boundary mirroring (``prepare_points_simple``): nbsym extrema reflected
  about the first / last extremum or the end sample by the four-way rule,
  re-reflected about the end sample when a mirrored point does not reach past
  it, adjacent knots with equal positions merged;
* envelopes: the not-a-knot cubic spline through the knots
  (``scipy.interpolate.CubicSpline(bc_type="not-a-knot")``; PyEMD calls
  SciPy's ``interp1d(kind="cubic")``, the same spline from another solver)
  and, for exactly three knots, PyEMD's natural cubic spline through them;
* the sift: mean of the envelopes subtracted until the stop tests
  (``check_imf``: envelope signs, sum of squares, scaled variance, standard
  deviation, energy ratio) and |extrema - zero crossings| < 2 both hold, or
  MAX_ITERATION passes;
* the outer loop: the residue S - (sum of the IMFs) is sifted again until its
  range < range_thr or its absolute sum < total_power_thr; if the last sift
  saw <= 2 extrema its row is dropped as the trend; the residue is appended
  unless it is all within 1e-8 of zero (``np.allclose``);
* in "simple" mode PyEMD replaces any given time axis by arange(N).

Divergence switches
-------------------
Each documented difference between PyEMD and the reference's kernel can be
switched, one at a time, to the reference's behaviour (``PyEMDOptions``).  The
audit (tests/test_pyemd_audit.py, oracle/audit_pyemd.py) attributes every
trace whose discrete outputs differ from the reference's to the switch that
removes the difference; a difference that no switch removes must sit on a
floating-point tie (two neighbouring samples within 1e-12 x range, or a stop
quantity within 1e-9 relative of its threshold), which the run records.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.interpolate import CubicSpline

ENERGY_RATIO_THR = 0.2
STD_THR = 0.2
SVAR_THR = 0.001
TOTAL_POWER_THR = 0.005
RANGE_THR = 0.001
SUM_NEW_SQ_MIN = 1e-10
ALLCLOSE_ATOL = 1e-8       # np.allclose(residue, 0): |r| <= atol


@dataclass
class PyEMDOptions:
    nbsym: int = 2
    max_iteration: int = 1000
    max_imf: int = -1               # PyEMD default: no limit
    # -- switches towards the reference kernel (all off = PyEMD) --------------
    ref_plateau_floor: bool = False   # plateau extremum at floor((i+j)/2), not round-half-even
    ref_flat_edges: bool = False      # flat runs from sample 0 dropped, from sample 1 classified
    ref_zero_count: bool = False      # the reference's zero-crossing count (kernels.py:115-144, 273-276)
    ref_three_knots: bool = False     # 3 knots: the not-a-knot parabola, not the natural spline
    ref_running_residue: bool = False  # residue r_k = r_(k-1) - imf_k (kernels.py:994-997)
    ref_time_axis: bool = False       # use the given (normalised) time axis
    ref_caps: bool = False            # first max_extrema extrema per side; at most max_imfs - 1 IMFs
    max_extrema: int = 1024
    max_imfs: int = 16

    def with_(self, **kw) -> "PyEMDOptions":
        d = dict(self.__dict__)
        d.update(kw)
        return PyEMDOptions(**d)


SWITCHES = ("ref_time_axis", "ref_caps", "ref_plateau_floor", "ref_flat_edges", "ref_zero_count",
            "ref_three_knots", "ref_running_residue")


@dataclass
class PyEMDResult:
    rows: np.ndarray          # [n_rows, N]: IMFs, then the residue if it is not ~0
    n_imfs: int               # rows, the reference's n_imfs
    debug_n: list             # per IMF: sift passes at exit (MAX_ITERATION at the cap; -1 trend)
    debug_extno: list         # per IMF: extrema after the last update (-1 at the cap / trend)
    debug_nzm: list
    hit_cap: bool             # some IMF reached MAX_ITERATION
    over_extrema: bool        # some scan had >= max_extrema maxima or minima
    raised: str = ""          # where PyEMD itself would raise (empty if nowhere)
    min_gap: float = np.inf   # smallest |S[i+1]-S[i]| / range over every scan and mirror test
    min_thr_margin: float = np.inf  # smallest |q / thr - 1| over every stop decision
    passes: int = 0

    @property
    def overflow(self) -> int:
        return int(self.hit_cap or self.over_extrema)


@dataclass
class _Trace:
    rng: float
    min_gap: float = np.inf
    min_thr: float = np.inf
    raised: str = ""
    over_extrema: bool = False

    def gap(self, d: np.ndarray) -> None:
        if d.size and self.rng > 0:
            self.min_gap = min(self.min_gap, float(np.min(np.abs(d))) / self.rng)

    def thr(self, q: float, t: float) -> None:
        if np.isfinite(q):
            self.min_thr = min(self.min_thr, abs(q / t - 1.0))


def simple_extrema(S: np.ndarray, opt: PyEMDOptions, tr: _Trace | None = None):
    """(ind_max, ind_min, n_zer) of PyEMD's "simple" extrema detection."""
    N = S.shape[0]
    d = np.diff(S)
    if tr is not None:
        tr.gap(d)
    if N >= 3:
        d1, d2 = d[:-1], d[1:]
        with np.errstate(invalid="ignore"):
            strict = d1 * d2 < 0
        imax = list(np.flatnonzero(strict & (d1 > 0)) + 1)
        imin = list(np.flatnonzero(strict & (d1 < 0)) + 1)
    else:
        imax, imin = [], []
    if np.any(d == 0):
        flat = (d == 0).astype(np.int8)
        edge = np.diff(np.concatenate([[0], flat, [0]]))
        first = np.flatnonzero(edge == 1)      # first zero difference of each run
        after = np.flatnonzero(edge == -1)     # one past its last: the run's last sample
        keep = np.ones(first.size, dtype=bool)
        if first.size:
            # left edge: PyEMD tests index 1; the reference drops the run from
            # sample 0 and classifies the one from sample 1
            lead = 0 if opt.ref_flat_edges else 1
            if first[0] == lead:
                keep[0] = False
            if after[-1] == N - 1:             # run reaching the last sample
                keep[-1] = False
        for a, b in zip(first[keep], after[keep]):
            before = d[a - 1]                  # a == 0 wraps to the last difference (PyEMD)
            mid = (a + b) // 2 if opt.ref_plateau_floor else int(np.round((a + b) / 2.0))
            if before > 0:
                if d[b] < 0:
                    imax.append(mid)
            elif d[b] > 0:
                imin.append(mid)
        imax.sort()
        imin.sort()
    ind_max = np.asarray(imax, dtype=np.int64)
    ind_min = np.asarray(imin, dtype=np.int64)
    return ind_max, ind_min, zero_crossings(S, opt)


def zero_crossings(S: np.ndarray, opt: PyEMDOptions) -> int:
    """PyEMD: sign changes plus one per run of exact zeros.  With
    ref_zero_count, the reference's count: its serial scan (taken when an
    interior sample is zero or has a zero difference) leaves out a zero run
    that reaches the last sample; its parallel scan counts sign changes only."""
    N = S.shape[0]
    with np.errstate(invalid="ignore"):
        sc = int(np.count_nonzero(S[:-1] * S[1:] < 0)) if N > 1 else 0
    z = (S == 0).astype(np.int8)
    runs_start = np.flatnonzero(np.diff(np.concatenate([[0], z])) == 1)
    if not opt.ref_zero_count:
        return sc + int(runs_start.size)
    if N < 3:
        return sc
    d = np.diff(S)
    serial = bool(np.any(d[:-1] == 0) or np.any(d[1:] == 0) or np.any(S[1:-1] == 0))
    if not serial:
        return sc
    runs_end = np.flatnonzero(np.diff(np.concatenate([z, [0]])) == -1)   # last zero of a run
    return sc + int(np.count_nonzero(runs_end < N - 1))


def mirror_points(T: np.ndarray, S: np.ndarray, ind_max: np.ndarray, ind_min: np.ndarray,
                  nbsym: int, tr: _Trace | None = None):
    """PyEMD's prepare_points_simple: knot positions and values of both
    envelopes, nbsym mirrored extrema per side.  Returns
    ((tmax, zmax), (tmin, zmin), raised)."""
    N = S.shape[0]
    nM, nm = ind_max.size, ind_min.size
    last = N - 1
    rev = lambda a: a[::-1]
    if tr is not None:
        # the end samples are compared with the nearest extremum of the other kind
        tr.gap(np.array([S[0] - S[ind_min[0] if ind_max[0] < ind_min[0] else ind_max[0]],
                         S[-1] - S[ind_max[-1] if ind_max[-1] < ind_min[-1] else ind_min[-1]]]))
    # left end: reflect about the first extremum, or about sample 0
    if ind_max[0] < ind_min[0]:
        if S[0] > S[ind_min[0]]:
            lmax, lmin, lsym = rev(ind_max[1:min(nM, nbsym + 1)]), rev(ind_min[:min(nm, nbsym)]), ind_max[0]
        else:
            lmax = rev(ind_max[:min(nM, nbsym)])
            lmin = np.concatenate([rev(ind_min[:min(nm, nbsym - 1)]), [0]])
            lsym = 0
    else:
        if S[0] < S[ind_max[0]]:
            lmax, lmin, lsym = rev(ind_max[:min(nM, nbsym)]), rev(ind_min[1:min(nm, nbsym + 1)]), ind_min[0]
        else:
            lmax = np.concatenate([rev(ind_max[:min(nM, nbsym - 1)]), [0]])
            lmin = rev(ind_min[:min(nm, nbsym)])
            lsym = 0
    # right end: reflect about the last extremum, or about the last sample
    if ind_max[-1] < ind_min[-1]:
        if S[-1] < S[ind_max[-1]]:
            rmax = rev(ind_max[max(nM - nbsym, 0):])
            rmin = rev(ind_min[max(nm - nbsym - 1, 0):-1])
            rsym = ind_min[-1]
        else:
            rmax = rev(np.concatenate([ind_max[max(nM - nbsym + 1, 0):], [last]]))
            rmin = rev(ind_min[max(nm - nbsym, 0):])
            rsym = last
    else:
        if S[-1] > S[ind_min[-1]]:
            rmax = rev(ind_max[max(nM - nbsym - 1, 0):-1])
            rmin = rev(ind_min[max(nm - nbsym, 0):])
            rsym = ind_max[-1]
        else:
            rmax = rev(ind_max[max(nM - nbsym, 0):])
            rmin = rev(np.concatenate([ind_min[max(nm - nbsym + 1, 0):], [last]]))
            rsym = last
    # an empty side list falls back to every extremum of that kind
    lmin = lmin if lmin.size else ind_min
    rmin = rmin if rmin.size else ind_min
    lmax = lmax if lmax.size else ind_max
    rmax = rmax if rmax.size else ind_max
    lmin, lmax, rmin, rmax = (np.asarray(a, dtype=np.int64) for a in (lmin, lmax, rmin, rmax))
    raised = ""
    tl = lambda idx: 2 * T[lsym] - T[idx]
    trr = lambda idx: 2 * T[rsym] - T[idx]
    if tl(lmin)[0] > T[0] or tl(lmax)[0] > T[0]:
        # the mirrored points do not reach past the start: reflect about sample 0
        if lsym == ind_max[0]:
            lmax = rev(ind_max[:min(nM, nbsym)])
        else:
            lmin = rev(ind_min[:min(nm, nbsym)])
        if lsym == 0:
            raised = "left edge"
        lsym = 0
    if trr(rmin)[-1] < T[-1] or trr(rmax)[-1] < T[-1]:
        if rsym == ind_max[-1]:
            rmax = rev(ind_max[max(nM - nbsym, 0):])
        else:
            rmin = rev(ind_min[max(nm - nbsym, 0):])
        if rsym == last:
            raised = raised or "right edge"
        rsym = last
    tmax = np.concatenate([tl(lmax), T[ind_max], trr(rmax)])
    zmax = np.concatenate([S[lmax], S[ind_max], S[rmax]])
    tmin = np.concatenate([tl(lmin), T[ind_min], trr(rmin)])
    zmin = np.concatenate([S[lmin], S[ind_min], S[rmin]])

    # merge knots whose position equals the previous one's (keep the first)
    def dedup(t, z):
        keep = np.concatenate([[True], t[1:] != t[:-1]])
        return t[keep], z[keep]
    return dedup(tmax, zmax), dedup(tmin, zmin), raised


def natural_three(x: np.ndarray, y: np.ndarray, t: np.ndarray) -> np.ndarray:
    """The natural cubic spline through three knots (zero second derivative
    at both ends), PyEMD's choice when an envelope has exactly three knots:
    knot slopes from the 3x3 slope system, Hermite form on each piece."""
    h0, h1 = x[1] - x[0], x[2] - x[1]
    s0, s1 = (y[1] - y[0]) / h0, (y[2] - y[1]) / h1
    A = np.array([[2.0 / h0, 1.0 / h0, 0.0],
                  [1.0 / h0, 2.0 * (1.0 / h0 + 1.0 / h1), 1.0 / h1],
                  [0.0, 1.0 / h1, 2.0 / h1]])
    rhs = np.array([3.0 * s0 / h0, 3.0 * s0 / h0 + 3.0 * s1 / h1, 3.0 * s1 / h1])
    k = np.linalg.solve(A, rhs)
    out = np.empty_like(t)
    for lo, (xa, xb, ya, yb, ka, kb) in enumerate(((x[0], x[1], y[0], y[1], k[0], k[1]),
                                                   (x[1], x[2], y[1], y[2], k[1], k[2]))):
        m = (t >= xa) & ((t < xb) if lo == 0 else (t <= xb))
        h = xb - xa
        u = (t[m] - xa) / h
        a = ka * h - (yb - ya)
        b = -kb * h + (yb - ya)
        out[m] = (1 - u) * ya + u * yb + u * (1 - u) * (a * (1 - u) + b * u)
    return out


def envelope(T: np.ndarray, x: np.ndarray, y: np.ndarray, opt: PyEMDOptions) -> np.ndarray:
    """Spline through the knots, evaluated on the time axis (the knots span
    it: mirroring reaches past both ends)."""
    if x.size >= 4 or (x.size == 3 and opt.ref_three_knots):
        return CubicSpline(x, y, bc_type="not-a-knot")(T)
    if x.size == 3:
        return natural_three(x, y, T)
    return y[0] + (y[1] - y[0]) / (x[1] - x[0]) * (T - x[0])      # 2 knots (PyEMD would raise)


def check_imf(new: np.ndarray, old: np.ndarray, zmax: np.ndarray, zmin: np.ndarray,
              tr: _Trace | None = None) -> bool:
    """PyEMD's default stop test on one sift update."""
    if np.any(zmax < 0) or np.any(zmin > 0):
        return False
    if np.sum(new * new) < SUM_NEW_SQ_MIN:
        return False
    diff = new - old
    dsq = np.sum(diff * diff)
    with np.errstate(divide="ignore", invalid="ignore"):
        svar = dsq / (np.max(old) - np.min(old))
        if tr is not None:
            tr.thr(svar, SVAR_THR)
        if svar < SVAR_THR:
            return True
        std = np.sum((diff / new) ** 2)
        if tr is not None:
            tr.thr(std, STD_THR)
        if std < STD_THR:
            return True
        er = dsq / np.sum(old * old)
        if tr is not None:
            tr.thr(er, ENERGY_RATIO_THR)
        return bool(er < ENERGY_RATIO_THR)


def emd(S: np.ndarray, T: np.ndarray | None = None, opt: PyEMDOptions | None = None) -> PyEMDResult:
    """Decompose one signal as PyEMD's EMD().emd(S, T) does."""
    opt = opt or PyEMDOptions()
    S = np.ascontiguousarray(S, dtype=np.float64)
    N = S.shape[0]
    if T is None or not opt.ref_time_axis:
        T = np.arange(N, dtype=np.float64)
    else:
        T = np.asarray(T, dtype=np.float64)
        T = (T - T[0]) / np.min(np.diff(T)) if N > 1 else T - T[0]
    tr = _Trace(rng=float(np.ptp(S)) if N else 0.0)
    imfs: list[np.ndarray] = []
    dbg_n: list[int] = []
    dbg_e: list[int] = []
    dbg_z: list[int] = []
    hit_cap = False
    passes = 0
    running = S.copy()
    extNo = -1
    finished = False
    max_rows = opt.max_imfs - 1 if opt.ref_caps else None

    def scan(x):
        imx, imn, nz = simple_extrema(x, opt, tr)
        if imx.size >= opt.max_extrema or imn.size >= opt.max_extrema:
            tr.over_extrema = True
            if opt.ref_caps:
                imx, imn = imx[:opt.max_extrema], imn[:opt.max_extrema]
        return imx, imn, nz

    while not finished:
        if max_rows is not None and len(imfs) >= max_rows:
            break
        if opt.ref_running_residue:
            residue = running.copy()
        else:
            residue = S - np.sum(np.array(imfs), axis=0) if imfs else S.copy()
        imf = residue.copy()
        n = 0
        slot = (-1, -1, -1)
        while True:
            n += 1
            if n >= opt.max_iteration:
                hit_cap = True
                slot = (n, -1, -1)
                break
            imx, imn, nz = scan(imf)
            extNo = imx.size + imn.size
            if extNo > 2:
                if imx.size == 0 or imn.size == 0:
                    tr.raised = tr.raised or "one-sided extrema"
                    finished = True
                    break
                (tmx, zmx), (tmn, zmn), raised = mirror_points(T, imf, imx, imn, opt.nbsym, tr)
                tr.raised = tr.raised or raised
                mean = 0.5 * (envelope(T, tmx, zmx, opt) + envelope(T, tmn, zmn, opt))
                old = imf.copy()
                imf = imf - mean
                passes += 1
                imx2, imn2, nz2 = scan(imf)
                extNo = imx2.size + imn2.size
                f1 = check_imf(imf, old, zmx, zmn, tr)
                f2 = abs(extNo - nz2) < 2
                if f1 and f2:
                    slot = (n, extNo, nz2)
                    break
            else:
                finished = True
                break
        imfs.append(imf.copy())
        dbg_n.append(slot[0])
        dbg_e.append(slot[1])
        dbg_z.append(slot[2])
        running = running - imf
        tmp = running if opt.ref_running_residue else S - np.sum(np.array(imfs), axis=0)
        rng, pw = np.max(tmp) - np.min(tmp), np.sum(np.abs(tmp))
        tr.thr(rng, RANGE_THR)
        tr.thr(pw, TOTAL_POWER_THR)
        if rng < RANGE_THR or pw < TOTAL_POWER_THR or len(imfs) == opt.max_imf:
            finished = True
    if extNo <= 2 and imfs:
        # the last sift saw <= 2 extrema: that row is the trend, back into the residue
        running = running + imfs.pop()
    if opt.ref_running_residue:
        res = running
    else:
        res = S - np.sum(np.array(imfs), axis=0) if imfs else S.copy()
    amax = float(np.max(np.abs(res))) if N else 0.0
    if amax > 0:
        tr.thr(amax, ALLCLOSE_ATOL)
    rows = list(imfs)
    if not np.allclose(res, 0):
        rows.append(res)
    R = np.array(rows) if rows else np.zeros((0, N))
    return PyEMDResult(R, len(rows), dbg_n, dbg_e, dbg_z, hit_cap, tr.over_extrema, tr.raised,
                       tr.min_gap, tr.min_thr, passes)
