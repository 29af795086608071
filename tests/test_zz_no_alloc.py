"""The no-allocation entry point, emdb_run_noalloc, through the C ABI.

Some callers cannot allocate device memory: services that reserve the whole
device up front and forbid allocations on their request path, hosts whose own
allocator owns the device, and paths that cannot afford cudaMalloc/cudaFree
(they may synchronise the device).  For them the library keeps its sift
scratch in one file-scope device array instead of a plan.  This file checks
that its results equal the planned entry point's (emdb_run) bit for bit -- the
tolerance every parity test here uses -- on two calls in a row (the second
call reuses the array the first one left behind), with the default time axis,
with a given non-uniform time axis, and on long traces whose sift passes keep
their knots in the array's spill slab; that the status word is read and
cleared; and that a config whose per-CTA scratch cannot fit the array is
refused.  It is named to be collected last, and passes alone in a fresh
process as well.
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


def _two_calls_equal(X, T=None, cfg=None):
    import torch
    from cuda_emd import EMDKernelConfig, _native
    L = _native.load()
    cfg = cfg or EMDKernelConfig()
    B, N = X.shape
    ref = cfg.build().run(X, T)                 # emdb_run through a plan
    torch.cuda.synchronize()
    c = cfg.to_c()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        outs = _outputs_like(ref)
        rc = L.emdb_run_noalloc(ctypes.byref(c), X.data_ptr(), None if T is None else T.data_ptr(),
                                B, N, *[o.data_ptr() for o in outs], stream)
        assert rc == 0, _native.last_error()
        torch.cuda.synchronize()
        for a, b in zip(ref, outs):
            assert torch.equal(a, b), f"call {call}: no-allocation result differs"
    st = ctypes.c_int(-1)
    assert L.emdb_noalloc_status(ctypes.byref(st), stream) == 0, _native.last_error()
    assert st.value == 0, f"status word {st.value}"
    return ref


def test_noalloc_equals_planned_entry_on_two_calls():
    import torch
    from cuda_emd import workloads as W
    X = torch.from_numpy(np.concatenate([W.seismic_batch(200, 2048, seed=901),
                                         W.sinusoid_batch(56, 2048, seed=902)])).cuda()
    _two_calls_equal(X)


def test_noalloc_given_time_axis():
    import torch
    from cuda_emd import workloads as W
    from cuda_emd.emd import _normalise_T
    N = 1536
    X = torch.from_numpy(W.seismic_batch(64, N, seed=903)).cuda()
    steps = np.random.default_rng(904).uniform(0.5, 2.0, N - 1)
    T = np.concatenate([[0.0], np.cumsum(steps)])
    Tn = _normalise_T(torch.from_numpy(T).cuda(), N, torch.cuda.current_device())
    _two_calls_equal(X, Tn.contiguous())


def test_noalloc_long_traces_use_the_slab():
    # 8192-sample seismic traces exceed max_extrema: at the automatic arena
    # (3 CTAs/SM) their passes keep knots and PCR buffers in the spill slab
    import torch
    from cuda_emd import EMDKernelConfig, _native, workloads as W
    cfg = EMDKernelConfig(max_iteration=40)          # keeps the test short
    X = torch.from_numpy(W.seismic_batch(6, 8192, seed=905)).cuda()
    plan = cfg.build()._plan
    plan.set_variant(4)                              # the no-allocation entry's instance
    arena, _, _ = plan.query(8192)
    assert _native.pass_placement(cfg.to_c(), 8192, arena, cfg.max_extrema, cfg.max_extrema) in (2, 4)
    ref = _two_calls_equal(X, cfg=cfg)
    assert int(ref[2].sum()) == X.shape[0]           # every trace overflowed


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
