"""GPU parity of the wide sift instances (plan variant 1: one 512-thread CTA
per SM on one trace; variant 2: two 256-thread CTAs per SM) and of the
long-trace form (proto-IMF in global memory).
It must give the same bits as the 128-thread instance and the oracle on every
path: the golden groups (both time-axis builds), long traces past
max_extrema with every knot placement forced by the arena size, ragged CSR
batches with per-trace time axes, and traces longer than shared memory holds
(32,768 to 65,536 samples, against oracle fixtures)."""
import hashlib
import os

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

WIDE = 1
HERE = os.path.dirname(os.path.abspath(__file__))


def _sha(block):
    return hashlib.sha256(np.ascontiguousarray(block, dtype="<f8").tobytes()).hexdigest().encode()


def _launcher(cfg, variant=WIDE, arena=0):
    L = cfg.build()
    L._plan.set_variant(variant)
    if arena:
        L._plan.set_arena(arena)
    return L


def _run(L, X, T=None):
    import torch
    out = L.run(torch.from_numpy(np.ascontiguousarray(X)).cuda(),
                None if T is None else torch.from_numpy(np.ascontiguousarray(T)).cuda())
    L.check_status()
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("name", [g["name"] for g in cases.groups()])
def test_wide_golden_bitexact(golden, name, variant):
    from cuda_emd import EMDKernelConfig
    X = golden[f"{name}__signals"]
    T = golden[f"{name}__T"]
    c = golden[f"{name}__cfg"]
    cfg = EMDKernelConfig(max_extrema=int(c[0]), nbsym=int(c[1]), max_iteration=int(c[2]),
                          max_imfs=int(c[3]))
    L = _launcher(cfg, variant=variant)
    axes = [T]
    if np.array_equal(T, np.arange(X.shape[1], dtype=np.float64)):
        axes.append(None)                      # the integer-axis build too
    for Tx in axes:
        imfs, n_imfs, ovf, dn, de, dz = _run(L, X, Tx)
        for b in range(X.shape[0]):
            assert n_imfs[b] == golden[f"{name}__nofma__n_imfs"][b], (name, b)
            assert ovf[b] == golden[f"{name}__nofma__overflow"][b], (name, b)
            np.testing.assert_array_equal(dn[b], golden[f"{name}__nofma__dbg_n"][b])
            np.testing.assert_array_equal(de[b], golden[f"{name}__nofma__dbg_ext"][b])
            np.testing.assert_array_equal(dz[b], golden[f"{name}__nofma__dbg_nzm"][b])
            assert _sha(imfs[b]) == golden[f"{name}__nofma__sha"][b], (name, b)


@pytest.mark.parametrize("N", [4096, 8192])
def test_wide_equals_narrow_on_long_overflowing_traces(N):
    # seismic traces past max_extrema (knot lists at the cap), chirps and
    # tones, with the wide instance at the full arena (knots on-chip) and at
    # arenas small enough to force the split / park / slab placements
    from cuda_emd import EMDKernelConfig, workloads as W
    cfg = EMDKernelConfig(max_iteration=50)
    rng = np.random.default_rng(N)
    X = np.concatenate([W.seismic_batch(5, N, seed=N + 1),
                        np.stack([W.chirp_trace(rng, N) for _ in range(2)]),
                        W.sinusoid_batch(3, N, seed=N + 2)])
    ref = _run(_launcher(cfg, variant=4), X)
    assert ref[2][:5].any()                    # seismic traces past max_extrema
    full = 232448
    floor = cfg.build()._plan.min_arena(N) + 1024     # the wide fixed part is a little larger
    for arena in (full, (full + floor) // 2 & ~127, (floor + 8192) & ~127, (floor + 127) & ~127):
        out = _run(_launcher(cfg, arena=arena), X)
        for a, b in zip(ref, out):
            assert np.array_equal(a, b), (N, arena)
    # two 256-thread CTAs per SM, automatic (half-SM) arena
    out = _run(_launcher(cfg, variant=2), X)
    for a, b in zip(ref, out):
        assert np.array_equal(a, b), (N, "half-wide")


def test_wide_ragged_per_trace_time_axis_matches_oracle():
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    from oracle import emd_oracle as O
    vals, offs, _ = W.ragged_mix(24, lo=200, hi=6000, seed=41)
    rng = np.random.default_rng(42)
    T = np.empty_like(vals)
    for b in range(24):
        n = offs[b + 1] - offs[b]
        t = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 2.0, n - 1))])
        T[offs[b]:offs[b + 1]] = (t - t[0]) / np.min(np.diff(t))
    L = _launcher(EMDKernelConfig())
    out = L.run_ragged(torch.from_numpy(vals).cuda(), torch.from_numpy(offs).cuda(),
                       T=torch.from_numpy(T).cuda(), t_per_trace=True)
    L.check_status()
    imfs, n_imfs, ovf, dn, de, dz = (o.cpu().numpy() for o in out)
    for b in range(24):
        n = int(offs[b + 1] - offs[b])
        r = O.emd_signal(vals[offs[b]:offs[b + 1]], T[offs[b]:offs[b + 1]])
        blk = imfs[16 * offs[b]:16 * offs[b + 1]].reshape(16, n)
        assert n_imfs[b] == r.n_imfs and ovf[b] == r.overflow, b
        np.testing.assert_array_equal(dn[b], r.debug_n)
        assert np.array_equal(blk, r.imfs), b


def test_wide_20000_samples_equals_narrow():
    # the longest traces the 128-thread instance holds at one CTA per SM
    from cuda_emd import EMDKernelConfig, workloads as W
    cfg = EMDKernelConfig(max_iteration=20)
    X = W.seismic_batch(2, 20000, seed=51)
    a = _run(_launcher(cfg, variant=4), X)
    b = _run(_launcher(cfg), X)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_traces_longer_than_shared_memory_match_oracle_fixtures():
    # 32,768 - 65,536 samples: the proto-IMF lives in global memory; any plan
    # falls back to that instance by itself (here through GPUBatchEMD and the
    # ragged path), bit-identical to the oracle (tests/golden/make_long.py)
    import torch
    from cuda_emd import EMDKernelConfig, GPUBatchEMD
    sys_path = os.path.join(HERE, "golden")
    import sys
    if sys_path not in sys.path:
        sys.path.insert(0, sys_path)
    from make_long import long_cases
    z = np.load(os.path.join(HERE, "golden", "long_golden.npz"))
    for name, x, mi in long_cases():
        emd = GPUBatchEMD(EMDKernelConfig(max_iteration=mi))
        imfs, n_imfs, ovf = emd(torch.from_numpy(x[None, :]).cuda())
        dn = emd.last_debug[0].cpu().numpy()[0]
        assert int(n_imfs[0]) == int(z[f"{name}__n_imfs"]), name
        assert int(ovf[0]) == int(z[f"{name}__overflow"]), name
        np.testing.assert_array_equal(dn, z[f"{name}__dbg_n"])
        assert _sha(imfs[0].cpu().numpy()) == z[f"{name}__sha"].item(), name
    # a ragged batch mixing a long and a short trace: the launch for the
    # longest trace's length runs both
    name, x, mi = long_cases()[0]
    short = np.sin(np.arange(700) * 0.05)
    vals = np.concatenate([short, x])
    offs = np.array([0, 700, 700 + x.shape[0]], dtype=np.int64)
    emd = GPUBatchEMD(EMDKernelConfig(max_iteration=mi))
    imfs, n_imfs, ovf = emd.ragged(torch.from_numpy(vals).cuda(), torch.from_numpy(offs).cuda())
    blk = imfs[16 * 700:].cpu().numpy().reshape(16, x.shape[0])
    assert _sha(blk) == z[f"{name}__sha"].item()
