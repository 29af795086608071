"""GPU tests of the batching layers: tiered ragged launches (with and without
CUDA-graph capture) and the continuous-batching server, which must return for
every request exactly what the request gets when served alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _csr(n, lo, hi, seed):
    import torch
    from cuda_emd import workloads as W
    vals, offs, kinds = W.ragged_mix(n, lo=lo, hi=hi, seed=seed)
    return vals, offs, torch.from_numpy(vals).cuda(), torch.from_numpy(offs).cuda()


def test_tiered_ragged_equals_single_launch(tmp_path):
    import torch
    from cuda_emd import EMDKernelConfig
    from cuda_emd.ragged import RaggedRunner
    vals, offs, v, o = _csr(96, 200, 9000, seed=41)
    single = EMDKernelConfig().build().run_ragged(v, o)
    rr = RaggedRunner(cache_path=str(tmp_path / "tune.json"))
    tiers = rr.run(v, o)
    torch.cuda.synchronize()
    rr.check_status()
    for a, b in zip(single, tiers):
        assert torch.equal(a, b)
    # graph-captured replay of the same tier launches: same bits
    g = rr.run(v, o, use_graph=True)
    g = rr.run(v, o, outs=g, use_graph=True)
    torch.cuda.synchronize()
    for a, b in zip(single, g):
        assert torch.equal(a, b)
    # a cost-ordered queue changes nothing either
    cost = torch.rand(96, device="cuda")
    c = rr.run(v, o, cost=cost)
    torch.cuda.synchronize()
    for a, b in zip(single, c):
        assert torch.equal(a, b)


def test_server_alone_equals_in_mix():
    import torch
    from cuda_emd.serving import EMDServer, make_requests, run_open_loop, Request
    rng = np.random.default_rng(5)
    reqs = make_requests(12, rng, lo=256, hi=4096, max_traces=16)
    # each request alone
    alone = []
    for r in reqs:
        srv = EMDServer(slots=1, short_slots=0)
        rr = Request(r.rid, r.traces)
        srv.submit(rr)
        srv.drain(timeout_s=120)
        alone.append(rr.result)
    # all of them in one open-loop run with overlapping arrivals
    srv = EMDServer(slots=3, max_batch_traces=16)
    mix = [Request(r.rid, r.traces) for r in reqs]
    arr = np.cumsum(np.full(len(mix), 0.002))
    rep = run_open_loop(srv, mix, arr, timeout_s=300)
    srv.check_status()
    assert rep["requests"] == 12 and rep["p99_ms"] >= rep["p50_ms"] > 0
    for a, m in zip(alone, mix):
        rows_a, n_a, o_a = a
        rows_m, n_m, o_m = m.result
        np.testing.assert_array_equal(n_a, n_m)
        np.testing.assert_array_equal(o_a, o_m)
        for x, y in zip(rows_a, rows_m):
            np.testing.assert_array_equal(x, y)
    # two launches ran on the device at the same time: their start / end
    # events (device clock) overlap
    iv = srv.device_intervals()
    assert len(iv) >= 2
    assert any(a[1] < b[2] and b[1] < a[2] for i, a in enumerate(iv) for b in iv[i + 1:]), iv


def test_server_hbm_budget_limits_admission():
    from cuda_emd.serving import EMDServer, make_requests
    rng = np.random.default_rng(6)
    reqs = make_requests(6, rng, lo=1024, hi=2048, max_traces=8)
    one = max(EMDServer._cost_bytes(sum(t.shape[0] for t in r.traces), len(r.traces), 16) for r in reqs)
    srv = EMDServer(slots=4, hbm_budget_bytes=one + 1)
    for r in reqs:
        srv.submit(r)
    srv.step()
    assert len(srv.flights) == 1          # the budget admits one request at a time
    srv.drain(timeout_s=120)
    assert all(r.result is not None for r in reqs)


def test_short_request_is_not_held_by_a_long_one():
    """Two requests admitted into one launch: one long chirp (thousands of
    extrema, a long sift) and one short trace.  Each trace raises its own
    completion flag, the tiers run side by side, and the short request is
    delivered as soon as its trace is done -- long before the launch ends --
    with the same results as when served alone."""
    from cuda_emd import workloads as W
    from cuda_emd.serving import EMDServer, Request
    rng = np.random.default_rng(8)
    long_tr, short_tr = W.chirp_trace(rng, 8192), W.sinusoid_trace(rng, 256)
    alone = EMDServer(slots=1, short_slots=0)
    solo = Request(9, [short_tr])
    alone.submit(solo)
    alone.drain(timeout_s=120)
    srv = EMDServer(slots=1, short_slots=0)       # one lane: both in one launch
    a, b = Request(0, [long_tr]), Request(1, [short_tr])
    srv.submit(a)
    srv.submit(b)
    srv.drain(timeout_s=120)
    srv.check_status()
    assert a.admitted == b.admitted                 # one launch for both
    la, lb = a.delivered - a.admitted, b.delivered - b.admitted
    print(f"long request {la * 1e3:.1f} ms, short request {lb * 1e3:.1f} ms")
    assert lb < 0.5 * la, (la, lb)
    for x, y in zip(solo.result[0], b.result[0]):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(solo.result[1], b.result[1])


def test_short_lane_is_not_blocked_by_long_requests():
    """Length lanes: a short request arriving while long requests hold every
    long-lane slot is admitted at once into the short lane and delivered long
    before them, with the same results as alone."""
    from cuda_emd import workloads as W
    from cuda_emd.serving import EMDServer, Request
    rng = np.random.default_rng(9)
    longs = [Request(i, [W.chirp_trace(rng, 8192)]) for i in range(3)]
    short = Request(10, [W.sinusoid_trace(rng, 512)])
    srv = EMDServer(slots=2, short_slots=1, max_batch_traces=1)
    for r in longs:
        srv.submit(r)
    srv.step()                                       # two long launches, one waiting
    srv.submit(short)
    srv.drain(timeout_s=120)
    assert short.admitted <= min(r.done for r in longs)
    assert short.delivered < min(r.delivered for r in longs)
    solo = EMDServer(slots=1, short_slots=0)
    s2 = Request(11, short.traces)
    solo.submit(s2)
    solo.drain(timeout_s=60)
    for x, y in zip(s2.result[0], short.result[0]):
        np.testing.assert_array_equal(x, y)


def test_cancel_and_deadline_on_the_device():
    """A request cancelled while running and one whose deadline passes while
    waiting are not delivered; the others are, unchanged, and every slot
    and byte of budget is released."""
    from cuda_emd.serving import EMDServer, Request, make_requests
    rng = np.random.default_rng(12)
    reqs = make_requests(6, rng, lo=512, hi=2048, max_traces=4)
    srv = EMDServer(slots=1, short_slots=1, max_batch_traces=4)
    for r in reqs:
        srv.submit(r)
    srv.step()
    running = [r for r in reqs if r.status == "running"]
    assert running and srv.cancel(running[0].rid)
    waiting = [r for r in reqs if r.status == "pending"]
    waiting[-1].deadline = srv.now() - 1.0           # already past
    srv.drain(timeout_s=120)
    assert running[0].status == "cancelled" and running[0].result is None
    assert waiting[-1].status == "timeout" and waiting[-1].result is None
    rest = [r for r in reqs if r not in (running[0], waiting[-1])]
    assert all(r.status == "delivered" and r.result is not None for r in rest)
    assert srv.in_use == 0 and srv.adm.nslots == 2 and srv.adm.running == 0
