"""CPU checks of the C ABI: the library loads without a GPU and exports every
symbol include/emdb200.h declares; the Python mirror exposes the reference's
API surface (emd.py:53-114, kernels.py:1170-1407)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "emdb200.h")).read()
    return sorted(set(re.findall(r"^int\s+(emdb_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_header_symbols():
    from cuda_emd import _native
    L = _native.load()
    declared = _declared()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(_native.EXPORTS) == declared
    assert L.emdb_version() >= 10000


def test_plan_create_without_gpu_reports_error():
    import ctypes
    from cuda_emd import _native
    L = _native.load()
    cfg = _native.EmdbConfig(1024, 2, 1000, 16, 128)
    h = ctypes.c_void_p()
    rc = L.emdb_plan_create(ctypes.byref(cfg), 0, ctypes.byref(h))
    import torch
    if torch.cuda.is_available():
        assert rc == 0
        L.emdb_plan_destroy(h)
    else:
        assert rc != 0 and _native.last_error()


def test_config_validation_codes():
    import ctypes
    from cuda_emd import _native
    L = _native.load()
    h = ctypes.c_void_p()
    bad = [_native.EmdbConfig(1024, 0, 1000, 16, 128), _native.EmdbConfig(1024, 2, 0, 16, 128),
           _native.EmdbConfig(1024, 2, 1000, 1, 128), _native.EmdbConfig(2, 2, 1000, 16, 128)]
    for c in bad:
        assert L.emdb_plan_create(ctypes.byref(c), 0, ctypes.byref(h)) == _native.EMDB_ERR_INVALID
    c = _native.EmdbConfig(1024, 2, 1000, 16, 256)
    assert L.emdb_plan_create(ctypes.byref(c), 0, ctypes.byref(h)) == _native.EMDB_ERR_UNSUPPORTED
    with pytest.raises(ValueError):
        _native.check(_native.EMDB_ERR_INVALID, "x")


def test_reference_api_surface():
    from cuda_emd import GPUBatchEMD, EMDKernelConfig, EMDBatchLauncher
    cfg = EMDKernelConfig()
    assert (cfg.max_extrema, cfg.nbsym, cfg.max_iteration, cfg.max_imfs, cfg.threads_per_block) == \
        (1024, 2, 1000, 16, 128)
    assert cfg.real_t_name == "double" and cfg.itemsize == 8
    assert cfg.shared_mem_bytes() == (1024 + 4) * 56 + 256
    assert cfg.static_shared_mem_bytes() == 12 * 128 + 4
    for m in ("warmup", "unpack", "ragged"):
        assert hasattr(GPUBatchEMD, m)
    for m in ("run", "run_envelope_only", "run_ragged"):
        assert hasattr(EMDBatchLauncher, m)


def test_cpu_only_call_fails_loudly():
    import numpy as np
    import torch
    from cuda_emd import GPUBatchEMD, EMDKernelConfig
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(Exception):
        GPUBatchEMD(EMDKernelConfig())(np.zeros((1, 64)))


def test_noalloc_checks_config_before_any_device_work():
    # the no-allocation entry point applies the plan's config rules (max_extrema
    # in [4, 2^20], nbsym in [1, 8], ...) before it touches the device, so an
    # out-of-range value is refused here, on a machine without a GPU, with the
    # same code as emdb_plan_create gives
    import ctypes
    from cuda_emd import _native
    L = _native.load()
    nul = [None] * 6
    for c in (_native.EmdbConfig((1 << 20) + 1, 2, 1000, 16, 128),
              _native.EmdbConfig(429496726, 1, 1000, 16, 128),
              _native.EmdbConfig(1024, 9, 1000, 16, 128),
              _native.EmdbConfig(1024, 2, 1000, 65, 128)):
        rc = L.emdb_run_noalloc(ctypes.byref(c), None, None, 4, 256, *nul, None)
        assert rc == _native.EMDB_ERR_INVALID, (c.max_extrema, rc)
    c = _native.EmdbConfig(1024, 2, 1000, 16, 256)
    assert L.emdb_run_noalloc(ctypes.byref(c), None, None, 4, 256, *nul, None) == \
        _native.EMDB_ERR_UNSUPPORTED


def test_slab_bytes_do_not_wrap():
    # the largest accepted max_extrema still sizes a positive, monotone slab
    from cuda_emd import _native
    cfg = _native.EmdbConfig(1 << 20, 8, 1000, 16, 128)
    p = _native.pass_placement(cfg, 8192, 76800, 1 << 20, 1 << 20)
    assert p == 2          # every knot in the slab, never a wrapped "fits"
