"""GPU parity of the FP32 path (EMDKernelConfig(real_t="float")).

The pin is the reference's own kernel source built with REAL_T = float and
-fmad=false (``oracle/build_ref.py``), whose outputs on the parity groups are
``tests/golden/ref_golden_f32.npz`` (``tests/golden/make_golden.py --real
float``): the B200 FP32 kernels must give the same bits (SHA-256 of each
trace's float32 [MAX_IMFS, N] block) and the same discrete outputs, on every
kernel instance and both time-axis builds; fresh inputs against the oracle
run in float32; the public API's dtype rules.
"""
import hashlib
import os

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _sha(block):
    return hashlib.sha256(np.ascontiguousarray(block, dtype="<f4").tobytes()).hexdigest().encode()


@pytest.fixture(scope="module")
def golden32():
    return np.load(os.path.join(HERE, "golden", "ref_golden_f32.npz"))


def _cfg(c, **kw):
    from cuda_emd import EMDKernelConfig
    return EMDKernelConfig(max_extrema=int(c[0]), nbsym=int(c[1]), max_iteration=int(c[2]),
                           max_imfs=int(c[3]), threads_per_block=int(c[4]), real_t="float", **kw)


def _run(cfg, X, T, variant=0):
    import torch
    L = cfg.build()
    if variant:
        L._plan.set_variant(variant)
    out = L.run(torch.from_numpy(np.ascontiguousarray(X)).cuda(),
                None if T is None else torch.from_numpy(np.ascontiguousarray(T)).cuda())
    L.check_status()
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize("variant", [4, 2, 1])
@pytest.mark.parametrize("name", [g["name"] for g in cases.groups()])
def test_f32_golden_bitexact(golden32, name, variant):
    X = golden32[f"{name}__signals"]
    T = golden32[f"{name}__T"]
    assert X.dtype == np.float32 and T.dtype == np.float32
    axes = [T]
    if np.array_equal(T, np.arange(X.shape[1], dtype=np.float32)):
        axes.append(None)                      # the integer-axis build too
    for Tx in axes:
        imfs, n_imfs, ovf, dn, de, dz = _run(_cfg(golden32[f"{name}__cfg"]), X, Tx, variant)
        assert imfs.dtype == np.float32
        for b in range(X.shape[0]):
            assert n_imfs[b] == golden32[f"{name}__nofma__n_imfs"][b], (name, b)
            assert ovf[b] == golden32[f"{name}__nofma__overflow"][b], (name, b)
            np.testing.assert_array_equal(dn[b], golden32[f"{name}__nofma__dbg_n"][b])
            np.testing.assert_array_equal(de[b], golden32[f"{name}__nofma__dbg_ext"][b])
            np.testing.assert_array_equal(dz[b], golden32[f"{name}__nofma__dbg_nzm"][b])
            assert _sha(imfs[b]) == golden32[f"{name}__nofma__sha"][b], (name, b, variant)


def test_f32_envelope_only_golden(golden32):
    import torch
    from cuda_emd import EMDKernelConfig
    name = cases.ENVELOPE_GROUP
    X = golden32[f"{name}__signals"]
    T = golden32[f"{name}__T"]
    L = EMDKernelConfig(real_t="float").build()
    out = [o.cpu().numpy() for o in L.run_envelope_only(torch.from_numpy(X).cuda(),
                                                         torch.from_numpy(T).cuda())]
    keys = ("max_env", "min_env", "n_extrema", "degenerate", "max_kpos", "max_kval",
            "min_kpos", "min_kval", "n_mirrored")
    for k, v in zip(keys, out):
        ref = golden32[f"{name}__env__{k}"]
        if k in ("max_env", "min_env"):
            # the fixture's envelopes come from the stock build (FMA
            # contraction on), which rounds differently in the last bit:
            # within 4 float ulps of the signal range
            for b in range(X.shape[0]):
                if golden32[f"{name}__env__degenerate"][b]:
                    continue
                rng = float(np.ptp(X[b])) or 1.0
                assert np.max(np.abs(v[b] - ref[b])) <= 4 * 2.0 ** -23 * rng, (k, b)
        else:
            np.testing.assert_array_equal(v, ref, err_msg=k)


def test_f32_fresh_inputs_match_oracle():
    """Fresh seeded inputs against the oracle run with REAL_T = float, dense
    and ragged (per-trace time axes), on the 128- and 512-thread instances."""
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    from oracle import emd_oracle as O
    cfg = EMDKernelConfig(real_t="float")
    ocfg = O.OracleConfig(real_t="float")
    X = np.concatenate([W.sinusoid_batch(6, 1024, seed=200),
                        W.seismic_batch(3, 1024, seed=201)]).astype(np.float32)
    T = np.arange(1024, dtype=np.float32)
    refs = [O.emd_signal(X[b], T, ocfg) for b in range(X.shape[0])]
    for variant in (4, 1):
        for Tx in (T, None):
            imfs, n_imfs, ovf, dn, de, dz = _run(cfg, X, Tx, variant)
            for b, r in enumerate(refs):
                assert n_imfs[b] == r.n_imfs and ovf[b] == r.overflow, (variant, b)
                np.testing.assert_array_equal(dn[b], r.debug_n)
                np.testing.assert_array_equal(dz[b], r.debug_nzm)
                assert _sha(imfs[b]) == _sha(r.imfs), (variant, b)
    # ragged, each trace with its own non-uniform axis
    vals, offs, _ = W.ragged_mix(10, lo=100, hi=1500, seed=202)
    vals = vals.astype(np.float32)
    rng = np.random.default_rng(203)
    Tr = np.empty(vals.shape[0], dtype=np.float32)
    for b in range(10):
        n = offs[b + 1] - offs[b]
        t = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 2.0, n - 1))])
        Tr[offs[b]:offs[b + 1]] = (t / np.min(np.diff(t))).astype(np.float32)
    L = cfg.build()
    out = L.run_ragged(torch.from_numpy(vals).cuda(), torch.from_numpy(offs).cuda(),
                       T=torch.from_numpy(Tr).cuda(), t_per_trace=True)
    L.check_status()
    imfs, n_imfs = out[0].cpu().numpy(), out[1].cpu().numpy()
    assert imfs.dtype == np.float32
    for b in range(10):
        n = int(offs[b + 1] - offs[b])
        r = O.emd_signal(vals[offs[b]:offs[b + 1]], Tr[offs[b]:offs[b + 1]], ocfg)
        assert n_imfs[b] == r.n_imfs, b
        assert np.array_equal(imfs[16 * offs[b]:16 * offs[b + 1]].reshape(16, n), r.imfs), b


def test_f32_public_api_dtype_rules():
    import torch
    from cuda_emd import EMDKernelConfig, GPUBatchEMD, workloads as W
    emd = GPUBatchEMD(EMDKernelConfig(real_t="float"))
    assert emd.config.dtype == np.float32 and emd.config.real_t_name == "float"
    assert emd.config.itemsize == 4
    emd.warmup()
    X = W.sinusoid_batch(4, 512, seed=210)
    with pytest.raises(ValueError):
        emd(torch.from_numpy(X).cuda())                     # float64 into a float launcher
    with pytest.raises(ValueError):
        GPUBatchEMD(EMDKernelConfig())(torch.from_numpy(X.astype(np.float32)).cuda())
    x32 = torch.from_numpy(X.astype(np.float32)).cuda()
    imfs, n_imfs, ovf = emd(x32)
    assert imfs.dtype == torch.float32 and imfs.shape == (4, 16, 512)
    # T given in float64 is normalised in float64, then rounded to float
    t = 0.002 * np.arange(512) + 7.0
    imfs_t, n_t, _ = emd(x32, torch.from_numpy(t).cuda())
    assert torch.equal(imfs_t, imfs) and torch.equal(n_t, n_imfs)
    # an axis whose normalised span passes 2^22 cannot keep every mirrored
    # knot distinct in float: refused
    t_bad = np.concatenate([[0.0, 1.0], 1.0 + 1e5 * np.arange(1, 511)])
    with pytest.raises(ValueError):
        emd(x32, torch.from_numpy(t_bad).cuda())
    # a queue order changes no bit
    order = torch.from_numpy(np.random.default_rng(211).permutation(4).astype(np.int32)).cuda()
    imfs_o, n_o, _ = emd(x32, order=order)
    assert torch.equal(imfs_o, imfs) and torch.equal(n_o, n_imfs)


def test_f32_long_trace_beyond_shared_memory_matches_oracle():
    """A float trace longer than the 512-thread instance holds in shared
    memory (proto-IMF in the global slab) against the float oracle; the
    iteration cap is lowered to keep the oracle's run to seconds."""
    from cuda_emd import EMDKernelConfig
    from oracle import emd_oracle as O
    N = 60000
    t = np.arange(N, dtype=np.float64)
    x = (np.sin(2 * np.pi * t / 9000.0) + 0.4 * np.sin(2 * np.pi * t / 1300.0 + 0.5)
         + 1e-5 * t).astype(np.float32)
    r = O.emd_signal(x, np.arange(N, dtype=np.float32),
                     O.OracleConfig(real_t="float", max_iteration=20))
    imfs, n_imfs, ovf, dn, de, dz = _run(EMDKernelConfig(real_t="float", max_iteration=20),
                                         x[None, :], None)
    assert n_imfs[0] == r.n_imfs and ovf[0] == r.overflow
    np.testing.assert_array_equal(dn[0], r.debug_n)
    assert _sha(imfs[0]) == _sha(r.imfs)


def test_f32_branch_free_divisions_match_hardware():
    """The FP32 kernels' float quotients (Markstein from an IEEE reciprocal in
    the evaluation; the branch-free division in the PCR rows) equal the IEEE
    float division bit for bit: every integer pair 0 <= a <= b <= 65536 and
    4e8 seeded random cases of each kind."""
    from cuda_emd import _native
    assert _native.check_division(3, 65536) == (0, 0, 0)
    assert _native.check_division(4, 400_000_000, seed=7) == (0, 0, 0)
