"""Host logic of the ragged runner that needs no GPU: length tiers and the
autotuner's candidate (register variant, arena) pairs -- the largest arena
that keeps k CTAs per SM resident for k = 6..1, in 128-byte units, kept when
it holds a trace of the tier's length with every knot spilled."""
import ctypes

import pytest

from cuda_emd import _native
from cuda_emd import ragged as R


class _FakePlan:
    """The three plan calls candidates() makes; min_arena is the library's own
    (device-free) emdb_min_arena."""

    def __init__(self):
        self.variant = None
        self.arena = None

    def set_variant(self, v):
        self.variant = v

    def set_arena(self, a):
        self.arena = a

    def min_arena(self, n):
        out = ctypes.c_int()
        assert _native.load().emdb_min_arena(int(n), ctypes.byref(out)) == 0
        return out.value


def test_tier_edges():
    assert R.tier_of(1) == 1024 and R.tier_of(1024) == 1024
    assert R.tier_of(1025) == 2048 and R.tier_of(8192) == 8192
    assert R.tier_of(8193) == 16384
    # past the listed edges: powers of two (the long-trace instance runs them)
    assert R.tier_of(R.TIER_EDGES[-1] + 1) == 65536
    assert R.tier_of(65537) == 131072 and R.tier_of(1 << 20) == 1 << 20


@pytest.mark.parametrize("n", [256, 2048, 4096, 8192, 16384, 32768])
def test_candidates(n):
    p = _FakePlan()
    cands = R.candidates(p, n)
    floor = p.min_arena(n)
    assert p.variant == 4 and p.arena == 0          # reset before the floor query
    # the wide instance (one 512-thread CTA per SM, automatic arena) is offered
    # for long tiers, last
    wide = [c for c in cands if c[0] == R.WIDE]
    assert wide == ([(R.WIDE, 0)] if n >= R.WIDE_FROM else [])
    if wide:
        assert cands[-1] == (R.WIDE, 0)
    # and two 256-thread CTAs per SM for tiers from 2048 samples that fit half an SM
    half = [c for c in cands if c[0] == R.HALF_WIDE]
    fits_half = (233472 // 2 - 1024) & ~127 >= floor + 1024
    assert half == ([(R.HALF_WIDE, 0)] if n >= R.HALF_WIDE_FROM and fits_half else [])
    cands = [c for c in cands if c[0] not in (R.WIDE, R.HALF_WIDE)]
    if floor > 232448:
        # the proto-IMF alone exceeds a block's shared memory (N = 32768:
        # 256 KB): only the wide instance, which keeps it in global memory
        assert cands == [], n
        return
    assert cands, n
    arenas = [a for _, a in cands]
    assert arenas == sorted(arenas)                  # k = 6..1: growing arenas
    for v, a in cands:
        assert a % 128 == 0 and floor <= a <= 232448
        assert v >= 4
    # every CTA count whose share holds the trace is offered, the others not
    offered = {min((233472 // k - 1024) & ~127, 232448) for k in range(1, 7)}
    assert set(arenas) == {a for a in offered if a >= floor}
    if n <= 2048:
        assert (6, min((233472 // 6 - 1024) & ~127, 232448)) in cands
    if n == 16384:
        assert arenas == [232448]                    # only one CTA per SM holds it
