"""Knot placement of a sift pass (emdb_pass_placement, the function the kernel
itself calls), checked on the CPU against a separate statement of each
layout's memory footprint: the chosen placement must fit the CTA's knot
arena, the proto-IMF region it may borrow and the per-CTA slab, and it must be
the first fitting one in the order shared, borrow, compact borrow, split,
park, slab.  A wrong choice here would make a pass write past its arena or
slab, so the sweep covers every CTA count's arena, short to long traces and
knot counts up to the max_extrema cap."""
import itertools

import pytest

from cuda_emd import _native as N
from cuda_emd.kernels import EMDKernelConfig

RED = 6 * 128 * 8            # the six 128-lane reduction arrays
SHARED, SPLIT, SLAB, BORROW, PARK, BORROW2 = 0, 1, 2, 3, 4, 5
ORDER = [SHARED, BORROW, BORROW2, SPLIT, PARK, SLAB]


def a16(x):
    return (x + 15) & ~15


def knot_bytes(cap):
    # X, Y and two PCR buffers of a | b | c | d per knot slot; the reduction
    # lanes need their own room only when buffer 1 is smaller than them
    return 10 * cap * 8 + (0 if 4 * cap >= 6 * 128 else RED)


def fits(place, n, arena, slab, cap):
    """Footprint of each layout, from its description: arena = knot arena
    after the fixed part, region = proto-IMF + knot arena (contiguous)."""
    imf = a16(8 * n)
    region = imf + arena
    if place == SHARED:
        return knot_bytes(cap) <= arena
    if place == BORROW:      # X | Y | P0 at the arena's end, P1 over the parked proto-IMF
        return 6 * cap * 8 <= arena and 10 * cap * 8 <= region and imf + RED <= slab
    if place == BORROW2:     # X | Y | M at the arena's end, P0 | P1 over the parked proto-IMF
        return 3 * cap * 8 <= arena and 11 * cap * 8 <= region and imf + RED <= slab
    if place == SPLIT:       # X | Y | P0 in the arena, P1 in the slab
        return 6 * cap * 8 <= arena and 4 * cap * 8 <= slab
    if place == PARK:        # P1 over the parked proto-IMF, X | Y | P0 in the slab after it
        return 4 * cap * 8 <= region and imf + 6 * cap * 8 <= slab
    return knot_bytes(cap) <= slab


def _cases():
    for cfg_kw in ({}, {"nbsym": 3}, {"max_extrema": 128}):
        cfg = EMDKernelConfig(**cfg_kw)
        for n in (6, 256, 1000, 2048, 4096, 5000, 8192, 12000, 16384, 24000):
            yield cfg, n


@pytest.mark.parametrize("cfg,n", list(_cases()),
                         ids=lambda v: v if isinstance(v, int) else f"me{v.max_extrema}nb{v.nbsym}")
def test_placement_fits_and_is_first_fitting(cfg, n):
    c = cfg.to_c()
    kcm = cfg.max_extrema + 2 * cfg.nbsym + 2
    slab = a16(knot_bytes(2 * kcm))
    m = N.load()
    import ctypes
    ma = ctypes.c_int()
    assert m.emdb_min_arena(n, ctypes.byref(ma)) == 0
    fixed = ma.value - RED - 64                   # control block, masks, proto-IMF
    arenas = {min(233472 // k - 1024, 232448) & ~127 for k in range(1, 7)} | {ma.value, ma.value - 16}
    counts = sorted({0, 1, 3, 50, 200, 340, 500, 700, cfg.max_extrema} & set(range(cfg.max_extrema + 1)))
    seen = set()
    for arena, (nmax, nmin) in itertools.product(sorted(arenas), itertools.product(counts, counts)):
        p = N.pass_placement(c, n, arena, nmax, nmin)
        if arena < fixed + RED + 64:
            assert p == -1, (n, arena)
            continue
        cap = (nmax + 2 * cfg.nbsym + 2) + (nmin + 2 * cfg.nbsym + 2)
        knot_arena = arena - fixed
        assert p in ORDER, p
        assert fits(p, n, knot_arena, slab, cap), (n, arena, nmax, nmin, N.PLACEMENTS[p])
        first = next(q for q in ORDER if fits(q, n, knot_arena, slab, cap))
        assert p == first, (n, arena, nmax, nmin, N.PLACEMENTS[p], N.PLACEMENTS[first])
        seen.add(p)
    assert SLAB in seen or SHARED in seen


def test_placement_examples():
    """The cases the placements were built for."""
    c = EMDKernelConfig().to_c()
    assert N.pass_placement(c, 2048, 57344, 100, 100) == SHARED        # cfg1, short knot lists
    assert N.pass_placement(c, 2048, 57344, 300, 300) == BORROW        # cfg1, dense extrema
    assert N.pass_placement(c, 8192, 76800, 1024, 1024) == PARK        # overflowed, 3 CTAs/SM
    assert N.pass_placement(c, 16384, 232448, 1024, 1024) == BORROW2   # overflowed, 1 CTA/SM
    assert N.pass_placement(c, 8192, 232448, 1024, 1024) == BORROW     # overflowed, 1 CTA/SM
    assert N.pass_placement(c, 8192, 20000, 10, 10) == -1              # arena below the trace


def test_placement_rejects_bad_arguments():
    c = EMDKernelConfig().to_c()
    with pytest.raises(ValueError):
        N.pass_placement(c, 2048, 57344, 2000, 10)                      # above max_extrema
    with pytest.raises(ValueError):
        N.pass_placement(c, 0, 57344, 10, 10)
