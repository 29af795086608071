"""GPU tests of the learned queue order: feature kernel and MLP kernels against
the NumPy oracle (oracle/sched_oracle.py), training convergence, and the
invariant that a learned order changes no output bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _traces():
    from cuda_emd import workloads as W
    vals, offs, kinds = W.ragged_mix(64, lo=16, hi=3000, seed=21)
    return vals, offs


def test_features_match_oracle():
    import torch
    from cuda_emd import scheduler as S
    from oracle import sched_oracle as SO
    vals, offs = _traces()
    f = S.features(torch.from_numpy(vals).cuda(), torch.from_numpy(offs).cuda()).cpu().numpy()
    for b in range(offs.shape[0] - 1):
        ref = SO.trace_features(vals[offs[b]:offs[b + 1]])
        np.testing.assert_allclose(f[b], ref, rtol=2e-5, atol=2e-6, err_msg=f"trace {b}")
    X = np.random.default_rng(1).normal(size=(5, 777))
    fd = S.features(torch.from_numpy(X).cuda()).cpu().numpy()
    for b in range(5):
        np.testing.assert_allclose(fd[b], SO.trace_features(X[b]), rtol=2e-5, atol=2e-6)


def _model_with(params_np, mu, sd):
    import torch
    from cuda_emd.scheduler import CostModel
    cm = CostModel()
    cm.params = torch.from_numpy(params_np.astype(np.float32)).cuda()
    cm.params_bf16 = cm.params.to(torch.bfloat16)
    cm.mu = torch.from_numpy(mu.astype(np.float32)).cuda()
    cm.sd = torch.from_numpy(sd.astype(np.float32)).cuda()
    return cm


def _flat(p):
    return np.concatenate([p["W1"].ravel(), p["b1"], p["W2"].ravel(), p["b2"], p["W3"].ravel(), p["b3"]])


def test_mlp_gradients_match_oracle():
    import torch
    from oracle import sched_oracle as SO
    rng = np.random.default_rng(2)
    p = SO.init_params(3)
    for k in ("b1", "b2", "b3"):
        p[k] = rng.normal(0, 0.1, size=p[k].shape)
    B = 300
    Xraw = rng.normal(size=(B, 32)) * 3 + 1
    mu, sd = Xraw.mean(0), Xraw.std(0)
    Xs = (Xraw - mu) / sd
    T = rng.normal(size=(B, 2))
    cm = _model_with(_flat(p), mu, sd)
    Xd = torch.from_numpy(Xraw.astype(np.float32)).cuda()
    Y, acts = cm.forward_train(Xd)
    grads, loss = cm.backward(Xd, acts, Y, torch.from_numpy(T.astype(np.float32)).cuda())
    yref, _ = SO.forward(p, Xs)
    lref, gref = SO.loss_and_grads(p, Xs, T)
    np.testing.assert_allclose(Y.cpu().numpy(), yref, rtol=1e-3, atol=1e-3)
    assert abs(float(loss.item()) - lref) <= 1e-3 * max(1.0, lref)
    g = grads.cpu().numpy()
    gflat = _flat(gref)
    scale = np.abs(gflat).max()
    np.testing.assert_allclose(g, gflat, rtol=1e-3, atol=1e-4 * scale)


def test_adam_matches_oracle():
    import ctypes
    import torch
    from cuda_emd import scheduler as S
    from oracle import sched_oracle as SO
    rng = np.random.default_rng(4)
    n = 1000
    w = rng.normal(size=n)
    g = rng.normal(size=n)
    m = rng.normal(size=n) * 0.1
    v = np.abs(rng.normal(size=n)) * 0.01
    L = S._lib()
    wd, gd, md, vd = (torch.from_numpy(a.astype(np.float32)).cuda() for a in (w, g, m, v))
    bf = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    rc = L.emdb_mlp_adam(wd.data_ptr(), gd.data_ptr(), md.data_ptr(), vd.data_ptr(), n, 1e-3, 0.9,
                         0.999, 1e-8, 3, bf.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    P, G, M, V = {"w": w.copy()}, {"w": g}, {"w": m.copy()}, {"w": v.copy()}
    SO.adam_step(P, G, M, V, 3)
    np.testing.assert_allclose(wd.cpu().numpy(), P["w"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(bf.float().cpu().numpy(), P["w"], rtol=1e-2, atol=1e-2)


def test_bf16_inference_close_to_fp32():
    import torch
    from oracle import sched_oracle as SO
    rng = np.random.default_rng(5)
    p = SO.init_params(6)
    Xraw = rng.normal(size=(1000, 32))
    cm = _model_with(_flat(p), np.zeros(32), np.ones(32))
    y = cm.predict(torch.from_numpy(Xraw.astype(np.float32)).cuda()).cpu().numpy()
    yref, _ = SO.forward(p, Xraw)
    err = np.abs(y - yref).max() / (np.abs(yref).max() + 1e-9)
    assert err < 3e-2, err


def test_training_learns_and_order_is_output_neutral():
    """Train on logged counts of a ragged batch; the loss falls; LPT order
    from the model gives bit-identical outputs to FIFO."""
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    from cuda_emd import scheduler as S
    vals, offs, kinds = W.ragged_mix(512, lo=128, hi=2048, seed=31)
    v = torch.from_numpy(vals).cuda()
    o = torch.from_numpy(offs).cuda()
    L = EMDKernelConfig().build()
    fifo = L.run_ragged(v, o)
    feats = S.features(v, o)
    T = S.labels_from_debug(fifo[3], fifo[1])
    cm = S.CostModel(seed=0)
    hist = cm.fit(feats, T, epochs=30, batch=128)
    assert hist[-1] < 0.7 * hist[0], hist
    lengths = o[1:] - o[:-1]
    order = S.lpt_order(S.predicted_cost(cm, feats, lengths))
    lpt = L.run_ragged(v, o, order=order)
    for a, b in zip(fifo, lpt):
        assert torch.equal(a, b)


def test_learned_order_gains_on_a_tail_heavy_batch():
    """What the trained network gains over the plain method: a batch with
    several waves of medium traces (4,736 seismic, N = 1024) and 48 expensive
    chirps (N = 4096) at the end of the queue.  FIFO starts the chirps last, so
    they run alone at the end; ordering by the network's predicted cost (N x
    predicted passes, trained on a different mixed batch) starts them first.
    The makespan drops clearly (the true-cost order reaches ~1.5x on B200) and
    the outputs stay bit-identical."""
    import numpy as np
    import torch
    from cuda_emd import EMDKernelConfig, workloads as W
    from cuda_emd import scheduler as S
    L = EMDKernelConfig().build()
    tv, to, _ = W.ragged_mix(4096, lo=256, hi=4096, seed=43)
    tv, to = torch.from_numpy(tv).cuda(), torch.from_numpy(to).cuda()
    lab = L.run_ragged(tv, to)
    cm = S.CostModel(seed=0)
    cm.fit(S.features(tv, to), S.labels_from_debug(lab[3], lab[1]), epochs=20, batch=1024)

    rng = np.random.default_rng(7)
    rows = list(W.seismic_batch(4736, 1024, seed=3)) + [W.chirp_trace(rng, 4096) for _ in range(48)]
    offs = np.zeros(len(rows) + 1, dtype=np.int64)
    np.cumsum([r.size for r in rows], out=offs[1:])
    v = torch.from_numpy(np.concatenate(rows)).cuda()
    o = torch.from_numpy(offs).cuda()
    order = S.lpt_order(S.predicted_cost(cm, S.features(v, o), o[1:] - o[:-1]))

    def best_ms(order):
        out = L.run_ragged(v, o, order=order)
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out = L.run_ragged(v, o, order=order)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best, out

    t_fifo, fifo = best_ms(None)
    t_learned, learned = best_ms(order)
    print(f"FIFO {t_fifo:.1f} ms, learned order {t_learned:.1f} ms ({t_fifo / t_learned:.2f}x)")
    assert t_learned < 0.85 * t_fifo, (t_fifo, t_learned)
    for a, b in zip(fifo, learned):
        assert torch.equal(a, b)
