"""Host logic of the serving loop that needs no GPU: the load-sized arena of a
tier launch (largest arena that keeps every trace in flight resident at 1 or 2
CTAs per SM, else the plan's own rule) and the admission cost per batch."""
import pytest

from cuda_emd import serving

SM = 148
SMEM_SM = 233472         # B200: 228 KB of shared memory per SM
OPTIN = 232448           # largest dynamic shared memory per block


def _server(adaptive=True, min_arena=None):
    s = object.__new__(serving.EMDServer)      # no device: only the fields _tier_arena reads
    s.adaptive_arena = adaptive
    s.num_sms = SM
    s.smem_sm = SMEM_SM
    s.smem_optin = OPTIN
    s.min_arena = dict(min_arena or {})
    return s


MIN = {1024: 17000, 2048: 31000, 4096: 48000, 8192: 77000, 16384: 146000}


@pytest.mark.parametrize("in_flight,edge,want", [
    (1, 8192, OPTIN),              # one trace: an SM to itself, the largest arena
    (SM, 8192, OPTIN),             # still one CTA per SM
    (SM + 1, 8192, 115712),        # two per SM: 228 KB / 2 - 1 KB, in 128-byte units
    (2 * SM, 2048, 115712),
    (2 * SM + 1, 2048, 0),         # three or more per SM: the plan's rule
    (10000, 16384, 0),
    (SM + 1, 16384, 0),            # a 16384-sample trace does not fit two per SM
])
def test_tier_arena_by_load(in_flight, edge, want):
    s = _server(min_arena=MIN)
    assert s._tier_arena(edge, in_flight) == want


def test_tier_arena_off_uses_plan_rule():
    s = _server(adaptive=False, min_arena=MIN)
    assert s._tier_arena(8192, 1) == 0


def test_tier_arena_is_128_byte_aligned_and_within_optin():
    s = _server(min_arena=MIN)
    for n in range(1, 2 * SM + 1, 7):
        a = s._tier_arena(1024, n)
        assert a % 128 == 0 and 0 < a <= OPTIN


def test_cost_bytes_counts_inputs_outputs_and_counts():
    mi = 16
    b = serving.EMDServer._cost_bytes(1000, 3, mi)
    assert b == 1000 * 8 * (1 + mi) + 3 * (4 * 3 * mi + 24)


# -- admission policy (lanes, budget, cancel, deadlines): host logic only --------

def _req(rid, lens):
    import numpy as np
    return serving.Request(rid, [np.zeros(n) for n in lens])


def _adm(short=1, long=2, budget=1 << 40, max_batch=64):
    return serving.Admission(short, long, budget, max_batch, short_max=4096, max_imfs=16)


def test_lanes_route_by_longest_trace():
    a = _adm()
    assert a.lane_of(_req(0, [100, 4096])) == "short"
    assert a.lane_of(_req(1, [100, 4097])) == "long"
    assert _adm(short=0).lane_of(_req(2, [100])) == "long"      # no short lane: one queue


def test_short_requests_pass_long_ones_that_hold_every_long_slot():
    a = _adm(short=1, long=1, max_batch=1)
    for i in range(3):
        a.submit(_req(i, [8192]))
    first = a.next_batches(False)
    assert [(lane, [r.rid for r in b]) for _, lane, b, _ in first] == [("long", [0])]
    a.submit(_req(9, [512]))                       # long lane full, two long ones waiting
    nxt = a.next_batches(True)
    assert [(lane, [r.rid for r in b]) for _, lane, b, _ in nxt] == [("short", [9])]
    assert a.pending() == 2


def test_budget_batches_and_release():
    one = serving.cost_bytes(1000, 1, 16)
    a = _adm(short=2, long=0, budget=2 * one)
    for i in range(4):
        a.submit(_req(i, [1000]))
    b = a.next_batches(False)
    assert len(b) == 1 and [r.rid for r in b[0][2]] == [0, 1]    # two fit the budget together
    assert a.next_batches(True) == []                            # the budget is spent
    slot, lane, reqs, nbytes = b[0]
    assert nbytes == serving.cost_bytes(2000, 2, 16) and a.in_use == nbytes
    a.release(slot, lane, nbytes)
    assert a.in_use == 0 and [r.rid for r in a.next_batches(False)[0][2]] == [2, 3]


def test_oversized_request_runs_alone_when_the_device_is_idle():
    a = _adm(short=2, long=0, budget=10)
    a.submit(_req(0, [1000]))
    assert a.next_batches(True) == []              # something in flight: wait
    b = a.next_batches(False)
    assert len(b) == 1 and b[0][2][0].rid == 0


def test_cancel_and_expire_waiting_requests():
    a = _adm(short=1, long=1)
    r0, r1, r2 = _req(0, [100]), _req(1, [9000]), _req(2, [100])
    r2.deadline = 5.0
    for r in (r0, r1, r2):
        a.submit(r)
    assert a.cancel(1) is r1 and r1.status == "cancelled"
    assert a.cancel(1) is None                     # not waiting any more
    assert a.expire(4.0) == []
    assert a.expire(6.0) == [r2] and r2.status == "timeout"
    b = a.next_batches(False)
    assert [r.rid for _, _, rs, _ in b for r in rs] == [0] and r0.status == "running"


@pytest.mark.parametrize("in_flight,edge,want", [
    (1, 8192, (1, 0)),             # one SM per trace: the 512-thread instance
    (SM, 16384, (1, 0)),
    (SM + 1, 8192, (2, 0)),        # two per SM: two 256-thread CTAs per SM
    (2 * SM, 4096, (2, 0)),
    (2 * SM + 1, 8192, (4, 0)),    # denser: the 128-thread instance, plan rule
    (1, 2048, (4, OPTIN)),         # short tiers keep the 128-thread instance
])
def test_tier_instance_by_load(in_flight, edge, want):
    s = _server(min_arena=MIN)
    s.wide_from = 4096
    assert s._tier_instance(edge, in_flight) == want
