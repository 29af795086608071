"""GPU parity: the B200 kernels (through the C ABI) against the reference's
own kernel outputs (golden fixtures), the CPU oracle, and -- when
``oracle/_ref`` is built -- the reference kernel run live on the same GPU.

Bar: bit-identical IMFs (SHA-256 of each trace's [MAX_IMFS, N] block) and
identical discrete outputs against the ``-fmad=false`` reference build and
the oracle; against the stock reference build (FMA contraction on) identical
discrete outputs and IMF values within 1e-9 x signal range.
"""
import hashlib

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

IMF_RTOL = 1e-9


def _sha(block):
    return hashlib.sha256(np.ascontiguousarray(block, dtype="<f8").tobytes()).hexdigest().encode()


def _cfg(c):
    from cuda_emd import EMDKernelConfig
    return EMDKernelConfig(max_extrema=int(c[0]), nbsym=int(c[1]), max_iteration=int(c[2]),
                           max_imfs=int(c[3]), threads_per_block=int(c[4]))


def _run_np(cfg, X, T, axis="given"):
    """Run the dense launcher.  axis="given" passes T as an array (the general
    time-axis kernel); axis="arange" passes None, which selects the kernel
    build for the integer axis T = arange(N) -- only valid when T is that."""
    import torch
    L = cfg.build()
    sig = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    if axis == "arange":
        assert np.array_equal(T, np.arange(X.shape[1], dtype=np.float64))
        Td = None
    else:
        Td = torch.from_numpy(np.ascontiguousarray(T)).cuda()
    out = L.run(sig, Td)
    L.check_status()
    return [o.cpu().numpy() for o in out]


def _axes(T, N):
    """Both kernel builds when T is arange(N), else the general one."""
    return ("given", "arange") if np.array_equal(T, np.arange(N, dtype=np.float64)) else ("given",)


@pytest.mark.parametrize("name", [g["name"] for g in cases.groups()])
@pytest.mark.parametrize("axis", ["given", "arange"])
def test_golden_bitexact(golden, name, axis):
    X = golden[f"{name}__signals"]
    T = golden[f"{name}__T"]
    if axis not in _axes(T, X.shape[1]):
        pytest.skip("time axis is not arange")
    imfs, n_imfs, ovf, dn, de, dz = _run_np(_cfg(golden[f"{name}__cfg"]), X, T, axis)
    for b in range(X.shape[0]):
        assert n_imfs[b] == golden[f"{name}__nofma__n_imfs"][b], (name, b)
        assert ovf[b] == golden[f"{name}__nofma__overflow"][b], (name, b)
        np.testing.assert_array_equal(dn[b], golden[f"{name}__nofma__dbg_n"][b])
        np.testing.assert_array_equal(de[b], golden[f"{name}__nofma__dbg_ext"][b])
        np.testing.assert_array_equal(dz[b], golden[f"{name}__nofma__dbg_nzm"][b])
        assert _sha(imfs[b]) == golden[f"{name}__nofma__sha"][b], (name, b)
        # the stock (FMA) reference build: same discrete outputs
        assert n_imfs[b] == golden[f"{name}__stock__n_imfs"][b]
        np.testing.assert_array_equal(dn[b], golden[f"{name}__stock__dbg_n"][b])


def test_golden_values_vs_stock(golden):
    for name in ("edge512", "cfg0", "cfg1", "tiny6", "nonuniformT"):
        X = golden[f"{name}__signals"]
        T = golden[f"{name}__T"]
        imfs = _run_np(_cfg(golden[f"{name}__cfg"]), X, T)[0]
        sel = list(golden[f"{name}__stock__sel"])
        rows = golden[f"{name}__stock__rows"]
        flat = golden[f"{name}__stock__imfs"]
        off = np.concatenate([[0], np.cumsum(rows)])
        for j, b in enumerate(sel):
            ref = flat[off[j]:off[j + 1]]
            rng = float(np.ptp(X[b])) or 1.0
            assert np.max(np.abs(imfs[b, :ref.shape[0]] - ref)) <= IMF_RTOL * rng


def test_envelope_only_golden(golden):
    import torch
    from cuda_emd import EMDKernelConfig
    name = cases.ENVELOPE_GROUP
    X = golden[f"{name}__signals"]
    T = golden[f"{name}__T"]
    L = EMDKernelConfig().build()
    out = [o.cpu().numpy() for o in L.run_envelope_only(torch.from_numpy(X).cuda(),
                                                         torch.from_numpy(T).cuda())]
    emax, emin, next_, deg, kp0, kv0, kp1, kv1, nmir = out
    np.testing.assert_array_equal(next_, golden[f"{name}__env__n_extrema"])
    np.testing.assert_array_equal(deg, golden[f"{name}__env__degenerate"])
    np.testing.assert_array_equal(nmir, golden[f"{name}__env__n_mirrored"])
    np.testing.assert_array_equal(kp0, golden[f"{name}__env__max_kpos"])
    np.testing.assert_array_equal(kv0, golden[f"{name}__env__max_kval"])
    np.testing.assert_array_equal(kp1, golden[f"{name}__env__min_kpos"])
    np.testing.assert_array_equal(kv1, golden[f"{name}__env__min_kval"])
    for b in range(X.shape[0]):
        rng = float(np.ptp(X[b])) or 1.0
        assert np.max(np.abs(emax[b] - golden[f"{name}__env__max_env"][b])) <= IMF_RTOL * rng
        assert np.max(np.abs(emin[b] - golden[f"{name}__env__min_env"][b])) <= IMF_RTOL * rng


def test_oracle_fresh_inputs():
    """Fresh seeded inputs (not in the fixtures) against the oracle, bit for bit."""
    from cuda_emd import EMDKernelConfig, workloads as W
    from oracle import emd_oracle as O
    for X in (W.sinusoid_batch(12, 1024, seed=100), W.seismic_batch(4, 2048, seed=101)):
        T = np.arange(X.shape[1], dtype=np.float64)
        refs = [O.emd_signal(X[b], T) for b in range(X.shape[0])]
        for axis in ("given", "arange"):
            imfs, n_imfs, ovf, dn, de, dz = _run_np(EMDKernelConfig(), X, T, axis)
            for b, r in enumerate(refs):
                assert n_imfs[b] == r.n_imfs and ovf[b] == r.overflow
                np.testing.assert_array_equal(dn[b], r.debug_n)
                np.testing.assert_array_equal(de[b], r.debug_extno)
                np.testing.assert_array_equal(dz[b], r.debug_nzm)
                assert _sha(imfs[b]) == _sha(r.imfs), (axis, b)


def test_long_knot_spacing_matches_oracle():
    """Smooth long traces: knot spacings beyond the integer axis's reciprocal
    table (16384 samples; these reach ~23,800) take the exact fallback inside
    that build; both builds equal the oracle bit for bit."""
    from cuda_emd import EMDKernelConfig
    from oracle import emd_oracle as O
    N = 24000
    t = np.arange(N, dtype=np.float64)
    X = np.stack([np.sin(2 * np.pi * t / 30000.0) + 0.2 * np.sin(2 * np.pi * t / 2500.0 + 0.3) + 1e-5 * t,
                  np.cos(2 * np.pi * t / 24000.0) + 0.1 * np.sin(2 * np.pi * t / 700.0)])
    refs = [O.emd_signal(X[b], t) for b in range(2)]
    for axis in ("given", "arange"):
        imfs, n_imfs, ovf, dn, de, dz = _run_np(EMDKernelConfig(), X, t, axis)
        for b, r in enumerate(refs):
            assert n_imfs[b] == r.n_imfs and ovf[b] == r.overflow
            np.testing.assert_array_equal(dn[b], r.debug_n)
            assert _sha(imfs[b]) == _sha(r.imfs), (axis, b)


def test_ragged_matches_oracle_and_order():
    """CSR batch of mixed lengths in one launch: every trace equals the oracle
    bit for bit, and a permuted queue order changes nothing."""
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    from oracle import emd_oracle as O
    vals, offs, kinds = W.ragged_mix(24, lo=64, hi=2048, seed=5)
    L = EMDKernelConfig().build()
    v = torch.from_numpy(vals).cuda()
    o = torch.from_numpy(offs).cuda()
    a = [x.cpu().numpy() for x in L.run_ragged(v, o)]
    L.check_status()
    perm = torch.from_numpy(np.random.default_rng(0).permutation(24).astype(np.int32)).cuda()
    b_ = [x.cpu().numpy() for x in L.run_ragged(v, o, order=perm)]
    for x, y in zip(a, b_):
        np.testing.assert_array_equal(x, y)
    imfs, n_imfs, ovf, dn, de, dz = a
    mi = 16
    for b in range(24):
        N = int(offs[b + 1] - offs[b])
        r = O.emd_signal(vals[offs[b]:offs[b + 1]], np.arange(N, dtype=np.float64))
        blk = imfs[mi * offs[b]: mi * offs[b + 1]].reshape(mi, N)
        assert n_imfs[b] == r.n_imfs and ovf[b] == r.overflow
        np.testing.assert_array_equal(dn[b], r.debug_n)
        assert _sha(blk) == _sha(r.imfs), b


def test_api_errors_and_overflow_warning():
    import torch
    from cuda_emd import GPUBatchEMD, EMDKernelConfig
    emd = GPUBatchEMD()
    with pytest.raises(ValueError):
        emd(torch.zeros((2, 64), dtype=torch.float32, device="cuda"))
    emd_small = GPUBatchEMD(EMDKernelConfig(max_extrema=128, max_iteration=6))
    x = torch.from_numpy(np.random.default_rng(3).normal(size=(2, 512))).cuda()
    with pytest.warns(UserWarning):
        imfs, n_imfs, ovf = emd_small(x)
    assert int(ovf.sum()) == 2
    emd.warmup()
    imfs, n_imfs, ovf = emd(x)
    k = emd.unpack(imfs, n_imfs, 0)
    assert k.shape == (int(n_imfs[0]), 512)
    # NumPy in -> NumPy out; 1-D input is promoted
    out = emd(np.sin(np.arange(256) * 0.3))
    assert isinstance(out[0], np.ndarray) and out[0].shape == (1, 16, 256)


@pytest.mark.skipif(not __import__("refkernel").have_ref(), reason="oracle/_ref not built")
def test_live_reference_kernel_cfg1_subsample():
    """cfg1-type traces (2048 samples) through the reference's own kernel on the
    same GPU: bit-identical to its -fmad=false build, discrete-identical and
    within tolerance of its stock build."""
    import torch
    from refkernel import RefKernel
    from cuda_emd import EMDKernelConfig, workloads as W
    X = W.seismic_batch(256, 2048, seed=77)
    T = np.arange(2048, dtype=np.float64)
    mine = _run_np(EMDKernelConfig(), X, T)
    nofma = RefKernel("libemd_ref_nofma.so").run(X, T)
    stock = RefKernel("libemd_ref.so").run(X, T)
    for k in range(1, 6):
        np.testing.assert_array_equal(mine[k], nofma[k])
    np.testing.assert_array_equal(mine[0], nofma[0])
    for k in range(1, 6):
        np.testing.assert_array_equal(mine[k], stock[k])
    rng = np.ptp(X, axis=1)
    err = np.abs(mine[0] - stock[0]).max(axis=(1, 2))
    assert np.all(err <= IMF_RTOL * rng)


@pytest.mark.parametrize("nbsym", [1, 3])
def test_nbsym_variants_match_oracle(nbsym):
    """nbsym != 2: nbsym=3 yields unsorted right-boundary knot lists (the
    reference's own ordering), which the kernel evaluates with the reference's
    binary search; both must equal the oracle bit for bit."""
    from cuda_emd import EMDKernelConfig, workloads as W
    from oracle import emd_oracle as O
    X = W.sinusoid_batch(8, 512, seed=200 + nbsym)
    T = np.arange(512, dtype=np.float64)
    cfg = EMDKernelConfig(nbsym=nbsym)
    ocfg = O.OracleConfig(nbsym=nbsym)
    refs = [O.emd_signal(X[b], T, ocfg) for b in range(X.shape[0])]
    for axis in ("given", "arange"):
        imfs, n_imfs, ovf, dn, de, dz = _run_np(cfg, X, T, axis)
        for b, r in enumerate(refs):
            assert n_imfs[b] == r.n_imfs and ovf[b] == r.overflow
            np.testing.assert_array_equal(dn[b], r.debug_n)
            assert _sha(imfs[b]) == _sha(r.imfs), (nbsym, axis, b)


@pytest.mark.parametrize("arena", [0, 26000, 232448])
def test_arena_sizes_same_results(arena):
    """Knot storage in shared memory or spilled to the global slab gives the
    same bits (small arena forces the slab path)."""
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    X = W.seismic_batch(24, 2048, seed=300)
    L = EMDKernelConfig().build()
    ref = [o.cpu() for o in L.run(torch.from_numpy(X).cuda(), None)]
    if arena:
        L._plan.set_arena(arena)
    out = [o.cpu() for o in L.run(torch.from_numpy(X).cuda(), None)]
    L.check_status()
    for a, b in zip(ref, out):
        assert torch.equal(a, b)


@pytest.mark.parametrize("N,arena", [(8192, 76800), (4096, 57344)])
def test_park_placement_same_results(N, arena):
    """Long traces with many knots (seismic noise past max_extrema, a chirp):
    at 3-4 CTAs/SM their passes park the proto-IMF in the slab and put PCR
    buffer 1 in its place; at one CTA/SM the knots stay on-chip.  Same bits."""
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    rng = np.random.default_rng(311)
    X = np.concatenate([W.seismic_batch(5, N, seed=310), W.chirp_trace(rng, N)[None, :]])
    L = EMDKernelConfig().build()
    L._plan.set_arena(232448)
    ref = [o.cpu() for o in L.run(torch.from_numpy(X).cuda(), None)]
    L._plan.set_arena(arena)
    out = [o.cpu() for o in L.run(torch.from_numpy(X).cuda(), None)]
    L.check_status()
    for a, b in zip(ref, out):
        assert torch.equal(a, b)


@pytest.mark.parametrize("N,arena", [(16384, 232448), (8192, 115712)])
def test_compact_borrow_same_results(N, arena):
    """Long traces whose knots need the compact borrow placement (moments
    beside X | Y at the arena's end, both PCR buffers in the parked proto-IMF's
    space) give the same bits as with every knot in the slab (smallest
    arena)."""
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    rng = np.random.default_rng(312)
    X = np.concatenate([W.seismic_batch(3, N, seed=313), W.chirp_trace(rng, N)[None, :]])
    L = EMDKernelConfig().build()
    L._plan.set_arena(L._plan.min_arena(N))
    ref = [o.cpu() for o in L.run(torch.from_numpy(X).cuda(), None)]
    L._plan.set_arena(arena)
    out = [o.cpu() for o in L.run(torch.from_numpy(X).cuda(), None)]
    L.check_status()
    for a, b in zip(ref, out):
        assert torch.equal(a, b)


def test_arena_too_small_raises():
    import torch
    from cuda_emd import EMDKernelConfig
    L = EMDKernelConfig().build()
    L._plan.set_arena(20000)
    with pytest.raises(ValueError):
        L.run(torch.zeros((2, 2048), dtype=torch.float64, device="cuda"), None)


@pytest.mark.parametrize("variant", [5, 6])
def test_register_variants_same_results(variant):
    """The 5- and 6-CTA/SM register-budget builds compute the same bits."""
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    X = torch.from_numpy(W.seismic_batch(40, 2048, seed=400)).cuda()
    L = EMDKernelConfig().build()
    ref = [o.cpu() for o in L.run(X, None)]
    L._plan.set_variant(variant)
    out = [o.cpu() for o in L.run(X, None)]
    L.check_status()
    for a, b in zip(ref, out):
        assert torch.equal(a, b)


def test_division_matches_hardware():
    """The reciprocal-based division used in envelope evaluation equals the
    IEEE division bit for bit: exhaustively over every integer pair
    0 <= a <= b <= 65536 (all A/B operands on the default time axis for traces
    up to 32768 samples) and on 4e8 pseudo-random pairs."""
    from cuda_emd import _native
    assert _native.check_division(0, 65536) == (0, 0, 0)
    for seed in range(4):
        assert _native.check_division(1, 100_000_000, seed=seed) == (0, 0, 0)


def test_branch_free_division_matches_hardware():
    """The PCR rows' division without a reciprocal at hand (approximate
    reciprocal, two Newton steps, one Markstein correction, then the nearer of
    two neighbours by exact remainders, with a flagged fallback) equals the
    IEEE division bit for bit on 4e8 seeded cases across every exponent range,
    special significands and PCR-like operands."""
    from cuda_emd import _native
    for seed in range(4):
        assert _native.check_division(2, 100_000_000, seed=seed) == (0, 0, 0)
