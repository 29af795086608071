"""GPU tests of the ragged runner's end-to-end path (RaggedRunner.run_host):
host CSR traces in, host results out.  The rows it copies back (rows 0..n_imfs
of each trace, gathered by emdb_pack_rows) must equal the device path's rows
bit for bit, every later row of the device output must be zero, and the
counts must match -- with FIFO queues and with a learned order, on two calls
in a row, and after the batch layout changes in the same buffers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(n, seed, lo=64, hi=3000):
    from cuda_emd import workloads as W
    vals, offs, _ = W.ragged_mix(n, lo=lo, hi=hi, seed=seed)
    return vals, offs


def _check(res, dev_out, offs, mi):
    imfs = dev_out[0].cpu().numpy()
    n_imfs = dev_out[1].cpu().numpy()
    assert np.array_equal(res.n_imfs.numpy(), n_imfs)
    assert np.array_equal(res.overflow.numpy(), dev_out[2].cpu().numpy())
    for k in range(3):
        assert np.array_equal(res.debug[k].numpy(), dev_out[3 + k].cpu().numpy())
    for b in range(offs.shape[0] - 1):
        n = int(offs[b + 1] - offs[b])
        blk = imfs[mi * offs[b]: mi * offs[b + 1]].reshape(mi, n)
        k = int(res.n_rows[b])
        assert k == min(int(n_imfs[b]) + 1, mi)
        assert np.array_equal(res.rows(b), blk[:k]), f"trace {b}"
        assert not blk[k:].any(), f"trace {b}: nonzero row past n_imfs + 1"


def test_run_host_matches_device_fifo_and_learned():
    import torch
    from cuda_emd import EMDKernelConfig, scheduler as S
    from cuda_emd.ragged import RaggedRunner
    cfg = EMDKernelConfig()
    vals, offs = _batch(300, 31)
    v, o = torch.from_numpy(vals).cuda(), torch.from_numpy(offs).cuda()
    runner = RaggedRunner(cfg, cache_path=None, autotune=False)
    ref = [x.clone() for x in runner.run(v, o)]
    # a small cost model is enough: order never changes a result
    cm = S.CostModel(seed=0)
    cm.fit(S.features(v, o), S.labels_from_debug(ref[3], ref[1]), epochs=2, batch=128)
    vp, op = torch.from_numpy(vals).pin_memory(), torch.from_numpy(offs).pin_memory()
    for model in (None, cm, cm):
        res = runner.run_host(vp, op, model=model)
        _check(res, ref, offs, cfg.max_imfs)
    # another layout in the same-size buffers (the traces in another order:
    # same count and total length): the runner must plan again
    perm = np.random.default_rng(33).permutation(offs.shape[0] - 1)
    rows = [vals[offs[b]:offs[b + 1]] for b in perm]
    vals2 = np.concatenate(rows)
    offs2 = np.zeros_like(offs)
    np.cumsum([r.shape[0] for r in rows], out=offs2[1:])
    assert not np.array_equal(offs2, offs)
    v2, o2 = torch.from_numpy(vals2).cuda(), torch.from_numpy(offs2).cuda()
    ref2 = [x.clone() for x in RaggedRunner(cfg, cache_path=None, autotune=False).run(v2, o2)]
    res2 = runner.run_host(torch.from_numpy(vals2), torch.from_numpy(offs2), model=cm)
    _check(res2, ref2, offs2, cfg.max_imfs)


def test_pack_rows_kernel_against_numpy():
    import ctypes
    import torch
    from cuda_emd import _native
    L = _native.load()
    rng = np.random.default_rng(5)
    lens = rng.integers(0, 700, size=97)
    offs = np.zeros(98, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    mi = 16
    imfs = rng.normal(size=mi * int(offs[-1]))
    n_rows = rng.integers(-2, 20, size=97).astype(np.int32)     # clamped to [0, 16]
    k = np.clip(n_rows, 0, mi).astype(np.int64)
    row_off = np.zeros(97, dtype=np.int64)
    row_off[1:] = np.cumsum(k * lens)[:-1]
    packed = torch.full((int((k * lens).sum()) + 5,), float("nan"), dtype=torch.float64, device="cuda")
    d = lambda a: torch.from_numpy(a).cuda()
    I, O, NR, RO = d(imfs), d(offs), d(n_rows), d(row_off)
    rc = L.emdb_pack_rows(I.data_ptr(), O.data_ptr(), NR.data_ptr(), RO.data_ptr(), 97, mi,
                          packed.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, _native.last_error()
    got = packed.cpu().numpy()
    for b in range(97):
        n = int(lens[b])
        want = imfs[mi * offs[b]: mi * offs[b] + k[b] * n]
        assert np.array_equal(got[row_off[b]: row_off[b] + k[b] * n], want), b
    assert np.isnan(got[-5:]).all()


def test_public_ragged_with_per_trace_time_axes():
    # GPUBatchEMD.ragged with one time axis per trace (each normalised as the
    # reference normalises its single T) against the oracle per trace
    import torch
    from cuda_emd import GPUBatchEMD, workloads as W
    from oracle import emd_oracle as O
    vals, offs, _ = W.ragged_mix(16, lo=100, hi=2500, seed=61)
    rng = np.random.default_rng(62)
    T = np.empty_like(vals)
    for b in range(16):
        n = offs[b + 1] - offs[b]
        T[offs[b]:offs[b + 1]] = 3.0 + np.concatenate([[0.0], np.cumsum(rng.uniform(0.2, 0.9, n - 1))])
    emd = GPUBatchEMD()
    imfs, n_imfs, ovf = emd.ragged(torch.from_numpy(vals).cuda(), torch.from_numpy(offs).cuda(),
                                   T=torch.from_numpy(T).cuda())
    imfs, n_imfs = imfs.cpu().numpy(), n_imfs.cpu().numpy()
    for b in range(16):
        n = int(offs[b + 1] - offs[b])
        Tb = O.normalise_T(T[offs[b]:offs[b + 1]], n)
        r = O.emd_signal(vals[offs[b]:offs[b + 1]], Tb)
        assert n_imfs[b] == r.n_imfs, b
        assert np.array_equal(imfs[16 * offs[b]:16 * offs[b + 1]].reshape(16, n), r.imfs), b


def test_learned_tier_choice_changes_no_bit():
    # the cost model also picks the tier: predicted-heavy traces of the long
    # tiers run on the wide instance in their own capped launch; every output
    # equals the FIFO single-tier run
    import torch
    from cuda_emd import EMDKernelConfig, scheduler as S
    from cuda_emd.ragged import RaggedRunner
    cfg = EMDKernelConfig(max_iteration=120)
    vals, offs = _batch(160, 71, lo=1500, hi=8192)
    v, o = torch.from_numpy(vals).cuda(), torch.from_numpy(offs).cuda()
    ref = [x.clone() for x in cfg.build().run_ragged(v, o)]
    cm = S.CostModel(seed=0)
    cm.fit(S.features(v, o), S.labels_from_debug(ref[3], ref[1]), epochs=3, batch=64)
    runner = RaggedRunner(cfg, cache_path=None, autotune=False, heavy_passes=50.0)
    for graph in (False, True, True):
        out = runner.run_learned(v, o, cm, use_graph=graph, offsets_host=offs, split_heavy=True)
        torch.cuda.synchronize()
        runner.check_status()
        assert any(t.variant == 1 for t in runner._prep[1])     # some traces went wide
        for a, b in zip(ref, out):
            assert torch.equal(a, b)
