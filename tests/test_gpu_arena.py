"""The automatic shared-memory arena of untuned launches (dense runs, the host
pipeline, the serving loop): the most CTAs per SM whose arena holds the trace
plus room for ~2 x 96 knots, but never fewer than 3 CTAs/SM while a 3-CTA arena
still holds the trace.  Measured on B200 with seismic batches: 4 CTAs/SM for
2048 samples, 3 for 4096 (88 ms vs 109 ms at 4) and 3 for 8192 (679 ms vs
865 ms at 2)."""
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
    want = {256: 4, 2048: 4, 4096: 3, 8192: 3, 16384: 1}
    for n, ctas in want.items():
        arena, per_sm, grid = plan.query(n)
        assert per_sm == ctas, (n, arena, per_sm)
        assert grid == per_sm * props.multi_processor_count
        assert arena >= plan.min_arena(n), (n, arena)
        assert arena % 128 == 0
