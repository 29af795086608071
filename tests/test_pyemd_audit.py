"""The reference audited against PyEMD's default EMD (oracle/pyemd_default.py).

PyEMD is the method the reference claims to reproduce (README.md:72-91,
kernels.py:44-50, 558-564).  Parity bar: n_imfs, overflow and the per-IMF
sift / extrema / zero-crossing counts identical, IMF values within 1e-9 x
signal range -- except on traces listed here with their cause: a behaviour
in which the reference departs from PyEMD on purpose or by construction
(each a switch of PyEMDOptions that, turned on alone, reproduces the
reference exactly), or an extremum tie (two neighbouring samples within
1e-12 x range).  The B200 kernel is bit-identical to the reference's
algorithm (tests/test_gpu_parity.py), so the same table holds for it; the GPU
test at the end checks it against the PyEMD oracle directly.
"""
import numpy as np
import pytest
from scipy.interpolate import CubicSpline, interp1d

from oracle import audit_pyemd as A
from oracle import pyemd_default as P

IMF_RTOL = 1e-9

# Every golden trace whose discrete outputs differ from PyEMD's, with the
# cause the audit finds (one of the divergence switches of
# oracle/pyemd_default.py, each a documented difference of the reference).
EXPECTED = {
    ("tiny6", 0): "ref_zero_count",        # leading exact zero: the parallel scan does not count it
    ("edge512", 0): "ref_zero_count",      # pure tone sin(2 pi 0.05 t): an exact zero at t = 0
    ("edge512", 3): "ref_flat_edges",      # quantised tone: a flat run from sample 1
    ("chirp6000", 0): "ref_caps",          # > max_extrema extrema: the reference truncates
    ("nonuniformT", 0): "ref_time_axis",   # PyEMD's simple mode replaces T by arange(N)
    ("nonuniformT", 1): "ref_time_axis",
    ("nonuniformT", 2): "ref_time_axis",
    ("nonuniformT", 3): "ref_time_axis",
    **{("small_cfg", b): "ref_caps" for b in (0, 1, 2, 3, 4, 5, 7)},   # max_extrema 128
}
# discrete outputs agree, values apart because of an extremum tie
EXPECTED_VALUE_TIES = {("edge512", 2)}   # two tones: sin(2 pi 0.02 t) peaks between samples


@pytest.fixture(scope="module")
def golden_audit():
    return A.run(A.golden_cases())


def test_golden_mismatches_are_listed(golden_audit):
    found = {(r["group"], r["index"]): r["cause"] for r in golden_audit if not r["match"]}
    assert found == EXPECTED


def test_golden_values_within_tolerance(golden_audit):
    for r in golden_audit:
        if r["imf_err"] is None:
            continue
        key = (r["group"], r["index"])
        if key in EXPECTED_VALUE_TIES:
            assert r["imf_err"] > IMF_RTOL and r["min_gap"] < A.GAP_TIE
            assert "extremum tie" in r["value_cause"]
        else:
            assert r["imf_err"] <= IMF_RTOL, (key, r["imf_err"])


def test_benchmark_kinds_match_pyemd():
    # seeded traces of every benchmark kind: discrete-identical to PyEMD's
    # default EMD, IMF values within 1e-9 x range, or an extremum tie
    rows = A.run(A.restatement_cases(6, seed=11))
    for r in rows:
        key = (r["group"], r["index"])
        if not r["match"]:
            assert "tie" in (r["cause"] or ""), (key, r["cause"])
        elif r["imf_err"] > IMF_RTOL:
            assert "tie" in r.get("value_cause", ""), (key, r["imf_err"])


def test_not_a_knot_envelope_equals_pyemd_interp1d():
    # PyEMD evaluates envelopes with interp1d(kind="cubic"); the oracle uses
    # CubicSpline(bc_type="not-a-knot"): the same spline
    rng = np.random.default_rng(3)
    x = np.cumsum(rng.integers(3, 40, size=30)).astype(np.float64) - 50
    y = rng.normal(size=30)
    t = np.arange(x[0], x[-1] + 1)
    a = P.envelope(t, x, y, P.PyEMDOptions())
    b = interp1d(x, y, kind="cubic")(t)
    assert np.max(np.abs(a - b)) <= 1e-12 * np.ptp(y)


def test_three_knot_envelope_is_the_natural_spline():
    x = np.array([-7.0, 4.0, 19.0])
    y = np.array([0.3, -1.2, 0.8])
    t = np.arange(-7.0, 20.0)
    got = P.envelope(t, x, y, P.PyEMDOptions())
    want = CubicSpline(x, y, bc_type="natural")(t)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-13)
    # with the switch: the reference's not-a-knot parabola
    par = P.envelope(t, x, y, P.PyEMDOptions(ref_three_knots=True))
    np.testing.assert_allclose(par, np.polyval(np.polyfit(x, y, 2), t), atol=1e-12)


def test_flat_runs_and_zero_crossings():
    opt = P.PyEMDOptions()
    S = np.array([0.0, 1.0, 3.0, 3.0, 1.0, 0.5, 2.0, -1.0])
    imx, imn, nz = P.simple_extrema(S, opt)
    assert list(imx) == [2, 6] and list(imn) == [5]
    # plateau of even length: midpoint rounded half to even (PyEMD) vs floor
    S = np.array([0.0, 1.0, 3.0, 3.0, 3.0, 3.0, 1.0, -1.0])        # run over samples 2..5
    assert list(P.simple_extrema(S, opt)[0]) == [4]                # round(3.5) = 4
    assert list(P.simple_extrema(S, opt.with_(ref_plateau_floor=True))[0]) == [3]
    # zero crossings: sign changes + one per zero run, wherever it lies
    S = np.array([0.0, 1.0, -1.0, 0.0, 0.0, 2.0, -3.0, 0.0])
    assert P.zero_crossings(S, opt) == 2 + 3
    # the reference's serial scan leaves out a zero run that reaches the end
    assert P.zero_crossings(S, opt.with_(ref_zero_count=True)) == 2 + 2


def test_known_answers():
    t = np.arange(1024, dtype=np.float64)
    # a linear trend: no IMF, the residue is the whole signal
    r = P.emd(0.01 * t + 0.3)
    assert r.n_imfs == 1 and np.allclose(r.rows[0], 0.01 * t + 0.3)
    # two separated tones: IMFs whose sum (with the residue) is the signal
    x = np.sin(2 * np.pi * 0.011 * t) + 0.6 * np.sin(2 * np.pi * 0.13 * t + 0.3)
    r = P.emd(x)
    assert r.n_imfs >= 2
    assert np.max(np.abs(r.rows.sum(0) - x)) < 1e-10


@pytest.mark.gpu
def test_b200_kernel_against_pyemd():
    import torch
    from cuda_emd import GPUBatchEMD, workloads as W
    X = np.concatenate([W.sinusoid_batch(24, 1024, seed=71), W.seismic_batch(8, 2048, seed=72)[:, :1024]])
    emd = GPUBatchEMD()
    imfs, n_imfs, ovf = emd(torch.from_numpy(X).cuda())
    torch.cuda.synchronize()
    imfs, n_imfs, ovf = imfs.cpu().numpy(), n_imfs.cpu().numpy(), ovf.cpu().numpy()
    dn, de, dz = (x.cpu().numpy() for x in emd.last_debug)
    for b in range(X.shape[0]):
        r = P.emd(X[b])
        d = (int(n_imfs[b]), int(ovf[b]), dn[b].astype(np.int64), de[b].astype(np.int64),
             dz[b].astype(np.int64))
        if not A.same(A.discrete(r, 16), d):
            assert r.min_gap < A.GAP_TIE, f"trace {b}: differs from PyEMD without a tie"
            continue
        err = np.max(np.abs(r.rows - imfs[b, :r.n_imfs])) / np.ptp(X[b])
        assert err <= IMF_RTOL or r.min_gap < A.GAP_TIE, (b, err)
