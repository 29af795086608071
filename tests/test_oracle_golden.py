"""Pin the CPU oracle against the reference's own kernel.

``tests/golden/ref_golden.npz`` was produced by ``tests/golden/make_golden.py``
on a B200 from the reference's ``emd_batch_kernel`` (kernels.py:834-1080),
compiled from kernels.py by ``oracle/build_ref.py``:

* against the ``-fmad=false`` build the oracle must be bit-identical (SHA-256
  of each signal's full [MAX_IMFS, N] output block) and equal in every
  discrete output;
* against the stock build (FMA contraction on, as NVRTC compiles it) the
  discrete outputs must be equal and IMF values within 1e-9 x signal range.
"""
import hashlib

import numpy as np
import pytest

import cases
from oracle import emd_oracle as O

IMF_RTOL = 1e-9  # x signal range (the stated tolerance for IMF values)


def _sha(block):
    return hashlib.sha256(np.ascontiguousarray(block, dtype="<f8").tobytes()).hexdigest().encode()


GROUPS = [g["name"] for g in cases.groups()]


@pytest.mark.parametrize("name", GROUPS)
def test_oracle_matches_reference(golden, name):
    X = golden[f"{name}__signals"]
    T = golden[f"{name}__T"]
    c = golden[f"{name}__cfg"]
    cfg = O.OracleConfig(max_extrema=int(c[0]), nbsym=int(c[1]), max_iteration=int(c[2]),
                         max_imfs=int(c[3]), threads_per_block=int(c[4]))
    sel = list(golden[f"{name}__stock__sel"]) if f"{name}__stock__sel" in golden else []
    rows = golden[f"{name}__stock__rows"] if sel else None
    flat = golden[f"{name}__stock__imfs"] if sel else None
    row_off = np.concatenate([[0], np.cumsum(rows)]) if sel else None
    for b in range(X.shape[0]):
        r = O.emd_signal(X[b], T, cfg)
        for tag in ("nofma", "stock"):
            assert r.n_imfs == golden[f"{name}__{tag}__n_imfs"][b], (name, b, tag)
            assert r.overflow == golden[f"{name}__{tag}__overflow"][b], (name, b, tag)
            np.testing.assert_array_equal(r.debug_n, golden[f"{name}__{tag}__dbg_n"][b])
            np.testing.assert_array_equal(r.debug_extno, golden[f"{name}__{tag}__dbg_ext"][b])
            np.testing.assert_array_equal(r.debug_nzm, golden[f"{name}__{tag}__dbg_nzm"][b])
        assert _sha(r.imfs) == golden[f"{name}__nofma__sha"][b], (name, b, "bit-exact vs -fmad=false")
        if b in sel:
            j = sel.index(b)
            ref_rows = flat[row_off[j]:row_off[j + 1]]
            rng = float(np.ptp(X[b])) or 1.0
            err = np.max(np.abs(r.imfs[:ref_rows.shape[0]] - ref_rows)) if ref_rows.size else 0.0
            assert err <= IMF_RTOL * rng, (name, b, err)


def test_oracle_envelope_stage(golden):
    """Extrema + mirroring + spline on raw signals vs the reference's
    envelope_batch_kernel (kernels.py:1100-1166), which uses the serial scan."""
    name = cases.ENVELOPE_GROUP
    X = golden[f"{name}__signals"]
    T = golden[f"{name}__T"]
    for b in range(X.shape[0]):
        imax, imin, _, _ = O._extrema_serial(X[b], 1024)
        nm = golden[f"{name}__env__n_extrema"][b]
        assert (imax.size, imin.size) == tuple(nm)
        deg = golden[f"{name}__env__degenerate"][b]
        if imax.size + imin.size <= 2 or imax.size < 1 or imin.size < 1:
            assert deg == 1
            continue
        assert deg == 0
        (pmax, vmax), (pmin, vmin), _ = O.mirror_knots(T, X[b], imax, imin, 2)
        nmir = golden[f"{name}__env__n_mirrored"][b]
        assert (pmax.size, pmin.size) == tuple(nmir)
        np.testing.assert_array_equal(pmax, golden[f"{name}__env__max_kpos"][b][:pmax.size])
        np.testing.assert_array_equal(vmax, golden[f"{name}__env__max_kval"][b][:pmax.size])
        np.testing.assert_array_equal(pmin, golden[f"{name}__env__min_kpos"][b][:pmin.size])
        np.testing.assert_array_equal(vmin, golden[f"{name}__env__min_kval"][b][:pmin.size])
        emax, _ = O.envelope(T, pmax, vmax)
        emin, _ = O.envelope(T, pmin, vmin)
        rng = float(np.ptp(X[b])) or 1.0
        assert np.max(np.abs(emax - golden[f"{name}__env__max_env"][b])) <= IMF_RTOL * rng
        assert np.max(np.abs(emin - golden[f"{name}__env__min_env"][b])) <= IMF_RTOL * rng


# ---------------------------------------------------------------------------
# REAL_T = float: the oracle in float32 against the reference source built
# with REAL_T = float (tests/golden/ref_golden_f32.npz, make_golden.py --real
# float).  Bit-identical to the -fmad=false build, equal discrete outputs.
# ---------------------------------------------------------------------------

def _sha32(block):
    return hashlib.sha256(np.ascontiguousarray(block, dtype="<f4").tobytes()).hexdigest().encode()


@pytest.fixture(scope="module")
def golden32():
    import os
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                "ref_golden_f32.npz"))


@pytest.mark.parametrize("name", GROUPS)
def test_oracle_f32_matches_reference_f32(golden32, name):
    X = golden32[f"{name}__signals"]
    T = golden32[f"{name}__T"]
    assert X.dtype == np.float32 and T.dtype == np.float32
    c = golden32[f"{name}__cfg"]
    cfg = O.OracleConfig(max_extrema=int(c[0]), nbsym=int(c[1]), max_iteration=int(c[2]),
                         max_imfs=int(c[3]), threads_per_block=int(c[4]), real_t="float")
    for b in range(X.shape[0]):
        r = O.emd_signal(X[b], T, cfg)
        assert r.imfs.dtype == np.float32
        assert r.n_imfs == golden32[f"{name}__nofma__n_imfs"][b], (name, b)
        assert r.overflow == golden32[f"{name}__nofma__overflow"][b], (name, b)
        np.testing.assert_array_equal(r.debug_n, golden32[f"{name}__nofma__dbg_n"][b])
        np.testing.assert_array_equal(r.debug_extno, golden32[f"{name}__nofma__dbg_ext"][b])
        np.testing.assert_array_equal(r.debug_nzm, golden32[f"{name}__nofma__dbg_nzm"][b])
        assert _sha32(r.imfs) == golden32[f"{name}__nofma__sha"][b], (name, b, "bit-exact")
