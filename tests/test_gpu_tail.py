"""GPU tests of tail migration (emdb_plan_set_tail): the traces still in flight
when a launch's queue runs dry stop at a sift-pass boundary, park their state
and finish on the 512-thread instance.  Every output must equal the run
without migration bit for bit -- dense and ragged, FP64 and FP32, with the
integer and a given time axis, when a few traces move and when every trace
moves (a batch smaller than the grid hands over all of them after their
first pass)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _launcher(real="double", tail=0):
    from cuda_emd import EMDKernelConfig
    L = EMDKernelConfig(real_t=real).build()
    L._plan.set_variant(4)
    L._plan.set_tail(tail)
    return L


def _dense(L, X, T=None):
    import torch
    out = L.run(torch.from_numpy(np.ascontiguousarray(X)).cuda(),
                None if T is None else torch.from_numpy(np.ascontiguousarray(T)).cuda())
    L.check_status()
    return [o.cpu().numpy() for o in out]


def _same(a, b):
    for x, y in zip(a, b):
        assert x.dtype == y.dtype and np.array_equal(x, y)


@pytest.mark.parametrize("real", ["double", "float"])
def test_tail_migration_changes_no_bit_dense(real):
    from cuda_emd import workloads as W
    rng = np.random.default_rng(5)
    dt = np.float32 if real == "float" else np.float64
    # a batch that keeps the grid busy, with slow chirps queued last
    X = np.concatenate([W.seismic_batch(900, 2048, seed=6),
                        np.stack([W.chirp_trace(rng, 2048) for _ in range(8)])]).astype(dt)
    T = (np.arange(2048) * 1.0).astype(dt)
    ref = _dense(_launcher(real), X)
    for tail in (-1, 300, 1 << 30):
        L = _launcher(real, tail)
        L._plan.counters(reset=True)
        out = _dense(L, X)
        _same(ref, out)
        _same(ref, _dense(L, X, T))                   # the given-axis build
    # every pass is counted once whichever instance ran it
    L0 = _launcher(real)
    L0._plan.counters(reset=True)
    _dense(L0, X)
    p0 = L0._plan.counters(reset=True)[0]
    L1 = _launcher(real, 1 << 30)
    L1._plan.counters(reset=True)
    _dense(L1, X)
    assert L1._plan.counters(reset=True)[0] == p0


def test_tail_migration_small_batch_moves_every_trace():
    # fewer traces than CTAs: the queue is dry at once, every trace moves to
    # the 512-thread instance after its first pass
    from cuda_emd import workloads as W
    X = np.concatenate([W.seismic_batch(40, 4096, seed=8), W.sinusoid_batch(40, 4096, seed=9)])
    ref = _dense(_launcher(), X)
    _same(ref, _dense(_launcher(tail=-1), X))


def test_tail_migration_ragged_per_trace_axes():
    import torch
    from cuda_emd import workloads as W
    vals, offs, _ = W.ragged_mix(700, lo=200, hi=3000, seed=10)
    rng = np.random.default_rng(11)
    T = np.empty_like(vals)
    for b in range(offs.shape[0] - 1):
        n = offs[b + 1] - offs[b]
        t = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 2.0, n - 1))])
        T[offs[b]:offs[b + 1]] = t / np.min(np.diff(t))
    v, o, Td = (torch.from_numpy(a).cuda() for a in (vals, offs, T))

    def run(L):
        out = L.run_ragged(v, o, T=Td, t_per_trace=True)
        L.check_status()
        return [x.cpu().numpy() for x in out]
    ref = run(_launcher())
    _same(ref, run(_launcher(tail=-1)))
    _same(ref, run(_launcher(tail=1 << 30)))


@pytest.mark.parametrize("real", ["double", "float"])
def test_tail_migration_golden_groups(real):
    # every parity group (zeros, plateaus, tiny traces, both caps, a
    # non-uniform axis, the small config) with every trace handed over: the
    # reference's bits (the -fmad=false fixtures), FP64 and FP32
    import hashlib
    import os
    import cases
    from cuda_emd import EMDKernelConfig
    here = os.path.dirname(os.path.abspath(__file__))
    z = np.load(os.path.join(here, "golden", "ref_golden_f32.npz" if real == "float"
                             else "ref_golden.npz"))
    code = "<f4" if real == "float" else "<f8"
    for g in cases.groups():
        name = g["name"]
        X, T, c = z[f"{name}__signals"], z[f"{name}__T"], z[f"{name}__cfg"]
        cfg = EMDKernelConfig(max_extrema=int(c[0]), nbsym=int(c[1]), max_iteration=int(c[2]),
                              max_imfs=int(c[3]), real_t=real)
        L = cfg.build()
        L._plan.set_variant(4)
        L._plan.set_tail(1 << 30)
        imfs, n_imfs, ovf, dn, de, dz = _dense(L, X, T)
        for b in range(X.shape[0]):
            assert n_imfs[b] == z[f"{name}__nofma__n_imfs"][b], (name, b)
            assert ovf[b] == z[f"{name}__nofma__overflow"][b], (name, b)
            np.testing.assert_array_equal(dn[b], z[f"{name}__nofma__dbg_n"][b])
            np.testing.assert_array_equal(de[b], z[f"{name}__nofma__dbg_ext"][b])
            sha = hashlib.sha256(np.ascontiguousarray(imfs[b], dtype=code).tobytes()).hexdigest()
            assert sha.encode() == z[f"{name}__nofma__sha"][b], (name, b)


def test_tail_migration_nbsym_and_small_caps():
    # other mirror widths and a config that overflows both caps early, with
    # hand-overs in the middle of IMFs (a batch larger than the threshold)
    from cuda_emd import EMDKernelConfig, workloads as W
    X = np.concatenate([W.seismic_batch(600, 1024, seed=12), W.sinusoid_batch(200, 1024, seed=13)])
    for kw in (dict(nbsym=1), dict(nbsym=3), dict(max_extrema=128, max_iteration=6)):
        ref = _dense(_moved(EMDKernelConfig(**kw), 0), X)
        _same(ref, _dense(_moved(EMDKernelConfig(**kw), 300), X))


def _moved(cfg, tail):
    L = cfg.build()
    L._plan.set_variant(4)
    L._plan.set_tail(tail)
    return L
