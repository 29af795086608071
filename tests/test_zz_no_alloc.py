"""The no-allocation entry point, emdb_run_noalloc, through the C ABI.

Some callers cannot allocate device memory: code that runs while a stream is
being captured into a CUDA graph, services that reserve the whole device up
front and forbid allocations on their request path, and hosts whose own
allocator owns the device.  For them the library keeps its sift scratch in
one file-scope device array instead of a plan.  This file checks that its
results equal the planned entry point's (emdb_run) bit for bit -- the
tolerance every parity test here uses -- on two calls in a row (the second
call reuses the array the first one left behind), and that a config whose
per-CTA scratch cannot fit the array is refused.  It is named to be
collected last, and passes alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _outputs_like(ref):
    import torch
    # poison every output so that an element the kernel fails to write shows up
    return [torch.full_like(r, -7) if r.dtype == torch.int32 else torch.full_like(r, float("nan"))
            for r in ref]


def test_noalloc_equals_planned_entry_on_two_calls():
    import torch
    from cuda_emd import EMDKernelConfig, _native, workloads as W
    L = _native.load()
    cfg = EMDKernelConfig()
    X = torch.from_numpy(np.concatenate([W.seismic_batch(200, 2048, seed=901),
                                         W.sinusoid_batch(56, 2048, seed=902)])).cuda()
    B, N = X.shape
    ref = cfg.build().run(X, None)              # emdb_run through a plan
    torch.cuda.synchronize()
    c = cfg.to_c()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        outs = _outputs_like(ref)
        rc = L.emdb_run_noalloc(ctypes.byref(c), X.data_ptr(), None, B, N,
                                *[o.data_ptr() for o in outs], stream)
        assert rc == 0, _native.last_error()
        torch.cuda.synchronize()
        for a, b in zip(ref, outs):
            assert torch.equal(a, b), f"call {call}: no-allocation result differs"


def test_noalloc_rejects_oversized_scratch():
    import torch
    from cuda_emd import EMDKernelConfig, _native
    L = _native.load()
    c = EMDKernelConfig(max_extrema=400000).to_c()   # ~64 MB of spill per CTA > 32 MiB
    X = torch.zeros((2, 256), dtype=torch.float64, device="cuda")
    outs = [torch.empty((2, 16, 256), dtype=torch.float64, device="cuda")] + \
           [torch.empty(s, dtype=torch.int32, device="cuda") for s in ((2,), (2,), (2, 16), (2, 16), (2, 16))]
    rc = L.emdb_run_noalloc(ctypes.byref(c), X.data_ptr(), None, 2, 256, *[o.data_ptr() for o in outs],
                            torch.cuda.current_stream().cuda_stream)
    assert rc == _native.EMDB_ERR_UNSUPPORTED
    assert "no-allocation" in _native.last_error()
