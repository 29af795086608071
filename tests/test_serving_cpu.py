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
