"""Seeded randomized parity sweep: the B200 path against the CPU oracle, bit
for bit, over configurations and inputs the fixed cases touch lightly --
small max_extrema (overflow and truncation), small max_iteration (the
iteration cap), few output rows, nbsym 1-3, lengths from 3 to thousands of
samples, plateaus and exact zeros (the serial-scan path), the integer and the
general time-axis builds, and tight shared-memory arenas that force every
knot placement (shared, borrow, compact borrow, split, park, slab)."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_CASES = 120


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def make_case(k):
    """Case k: (config fields, signals [B, N], T or None, arena mode)."""
    from cuda_emd import workloads as W
    rng = np.random.default_rng(1000 + k)
    N = int(rng.choice([3, 7, 64, 300, 1000, 2048, 4500]))
    cfg = dict(max_extrema=int(rng.choice([16, 64, 256, 1024])), nbsym=int(rng.choice([1, 2, 3])),
               max_iteration=int(rng.choice([5, 50] if N >= 1000 else [5, 50, 1000])),
               max_imfs=int(rng.choice([3, 6, 16])))
    rows = []
    for _ in range(int(rng.integers(2, 6))):
        kind = rng.integers(0, 6)
        if kind == 0 or N < 64:
            x = W.sinusoid_trace(rng, N)
        elif kind == 1:
            x = W.seismic_trace(rng, N)
        elif kind == 2 and N <= 1000:
            x = W.chirp_trace(rng, N)
        elif kind == 3:
            x = np.cumsum(rng.standard_normal(N))            # random walk
        elif kind == 4:
            x = np.round(W.sinusoid_trace(rng, N) * 4.0) / 4.0  # plateaus and exact zeros
        else:
            x = np.zeros(N)
            x[N // 3:] = rng.standard_normal(N - N // 3)
        rows.append(np.asarray(x, dtype=np.float64))
    X = np.stack(rows)
    T = None if rng.random() < 0.5 else np.cumsum(rng.uniform(0.5, 1.5, N))
    arena = "tight" if rng.random() < 0.4 else "auto"
    return cfg, X, T, arena


@pytest.mark.parametrize("k", range(N_CASES))
def test_random_case_matches_oracle(k):
    import torch
    from cuda_emd import EMDKernelConfig
    from oracle import emd_oracle as O
    cfg, X, T, arena = make_case(k)
    B, N = X.shape
    c = EMDKernelConfig(threads_per_block=128, **cfg)
    L = c.build()
    if arena == "tight":
        # room for the trace plus ~24 knots: most passes go to the slab or split
        L._plan.set_arena(L._plan.min_arena(N) + 24 * 80)
    Tn = None if T is None else O.normalise_T(T, N)
    sig = torch.from_numpy(X).cuda()
    out = L.run(sig, None if Tn is None else torch.from_numpy(Tn).cuda())
    L.check_status()
    imfs, n_imfs, ovf, dn, de, dz = (o.cpu().numpy() for o in out)
    ocfg = O.OracleConfig(threads_per_block=128, **cfg)
    Tor = np.arange(N, dtype=np.float64) if Tn is None else Tn
    for b in range(B):
        r = O.emd_signal(X[b], Tor, ocfg)
        ctx = (k, cfg, N, arena, T is None, b)
        assert n_imfs[b] == r.n_imfs and ovf[b] == r.overflow, ctx
        np.testing.assert_array_equal(dn[b], r.debug_n, err_msg=str(ctx))
        np.testing.assert_array_equal(de[b], r.debug_extno, err_msg=str(ctx))
        np.testing.assert_array_equal(dz[b], r.debug_nzm, err_msg=str(ctx))
        assert _sha(imfs[b]) == _sha(r.imfs), ctx


N_RAGGED = 24


@pytest.mark.parametrize("k", range(N_RAGGED))
def test_random_ragged_case_matches_oracle(k):
    """CSR batches of mixed lengths in one launch, with a per-trace time axis
    (each normalised on its own) or none, a random queue order and a random
    configuration: every trace equals the oracle bit for bit."""
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    from oracle import emd_oracle as O
    rng = np.random.default_rng(5000 + k)
    cfg = dict(max_extrema=int(rng.choice([32, 256, 1024])), nbsym=int(rng.choice([1, 2, 3])),
               max_iteration=int(rng.choice([10, 100])), max_imfs=int(rng.choice([4, 16])))
    lens = rng.integers(3, 1500, size=int(rng.integers(3, 12)))
    rows = [W.sinusoid_trace(rng, int(n)) if rng.random() < 0.5 else
            np.cumsum(rng.standard_normal(int(n))) for n in lens]
    per_T = rng.random() < 0.5
    Ts = [O.normalise_T(np.cumsum(rng.uniform(0.5, 1.5, int(n))), int(n)) if per_T
          else np.arange(int(n), dtype=np.float64) for n in lens]
    offs = np.zeros(len(rows) + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    v = torch.from_numpy(np.concatenate(rows)).cuda()
    o = torch.from_numpy(offs).cuda()
    Td = torch.from_numpy(np.concatenate(Ts)).cuda() if per_T else None
    order = torch.from_numpy(rng.permutation(len(rows)).astype(np.int32)).cuda()
    L = EMDKernelConfig(threads_per_block=128, **cfg).build()
    imfs, n_imfs, ovf, dn, de, dz = (x.cpu().numpy() for x in
                                     L.run_ragged(v, o, order=order, T=Td, t_per_trace=True))
    L.check_status()
    mi = cfg["max_imfs"]
    ocfg = O.OracleConfig(threads_per_block=128, **cfg)
    for b, x in enumerate(rows):
        r = O.emd_signal(x, Ts[b], ocfg)
        ctx = (k, cfg, int(lens[b]), per_T, b)
        assert n_imfs[b] == r.n_imfs and ovf[b] == r.overflow, ctx
        np.testing.assert_array_equal(dn[b], r.debug_n, err_msg=str(ctx))
        block = imfs[mi * offs[b]: mi * offs[b + 1]].reshape(mi, int(lens[b]))
        assert _sha(block) == _sha(r.imfs), ctx
