"""The automatic shared-memory arena of untuned launches (dense runs, the host
pipeline, the serving loop).  The 128-thread instance: the most CTAs per SM
whose arena holds the trace plus room for ~2 x 96 knots, but never fewer than
3 CTAs/SM while a 3-CTA arena still holds the trace.  Measured on B200 with
seismic batches: 4 CTAs/SM for 2048 samples, 3 for 4096 (88 ms vs 109 ms at
4) and 3 for 8192 (679 ms vs 865 ms at 2).  A plan with no instance set picks
one by trace length: 128 threads x 4 per SM up to 2048 samples, 256 x 2 up to
4096, one 512-thread CTA per SM beyond."""
import pytest

pytestmark = pytest.mark.gpu


def test_auto_arena_choices():
    import torch
    from cuda_emd import EMDKernelConfig
    props = torch.cuda.get_device_properties(0)
    smem = getattr(props, "shared_memory_per_multiprocessor", None)
    if smem != 233472:
        pytest.skip(f"rule measured on B200 (228 KB shared memory per SM), this device has {smem}")
    plan = EMDKernelConfig().build()._plan
    by_length = {256: 4, 2048: 4, 2049: 2, 4096: 2, 4097: 1, 8192: 1, 16384: 1}
    for n, ctas in by_length.items():
        arena, per_sm, grid = plan.query(n)
        assert per_sm == ctas, (n, arena, per_sm)
        assert grid == per_sm * props.multi_processor_count
    plan.set_variant(4)
    want = {256: 4, 2048: 4, 4096: 3, 8192: 3, 16384: 1}
    for n, ctas in want.items():
        arena, per_sm, grid = plan.query(n)
        assert per_sm == ctas, (n, arena, per_sm)
        assert grid == per_sm * props.multi_processor_count
        assert arena >= plan.min_arena(n), (n, arena)
        assert arena % 128 == 0
