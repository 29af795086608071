"""Host-memory pipeline (emdb_run_host, GPUBatchEMD on NumPy / CPU torch
input): one launch whose finished chunks of traces are copied back while the
rest sift.  Its results must equal the device path's bit for bit, whatever the
chunking (one partial chunk, many chunks with a ragged last one), with and
without a time axis, into caller-supplied page-locked buffers, and on calls
repeated on one plan (the chunk flags are reset per call)."""
import numpy as np
import pytest
import torch

from cuda_emd.emd import GPUBatchEMD
from cuda_emd import workloads as W


def _device(emd, X, T=None):
    d = torch.from_numpy(X).cuda()
    imfs, n, o = emd(d, T=None if T is None else torch.from_numpy(T).cuda())
    dbg = tuple(x.cpu().numpy() for x in emd.last_debug)
    return (imfs.cpu().numpy(), n.cpu().numpy(), o.cpu().numpy()) + dbg


def _same(a, b):
    for x, y in zip(a, b):
        x = np.asarray(x)
        y = np.asarray(y)
        assert x.shape == y.shape
        assert x.tobytes() == y.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("batch,N", [(37, 500), (1000, 1024), (4099, 256)])
def test_host_numpy_equals_device(batch, N):
    emd = GPUBatchEMD()
    X = W.seismic_batch(batch, N, seed=batch) if N >= 512 else W.sinusoid_batch(batch, N, seed=batch)
    ref = _device(emd, X)
    for _ in range(2):
        imfs, n, o = emd(X)
        assert isinstance(imfs, np.ndarray)
        _same((imfs, n, o) + tuple(emd.last_debug), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [300, 2000])      # one launch; four input groups
def test_host_with_time_axis_and_out_buffers(batch):
    emd = GPUBatchEMD()
    rng = np.random.default_rng(11)
    X = W.sinusoid_batch(batch, 700, seed=4)
    T = np.cumsum(rng.uniform(0.5, 1.5, 700))
    ref = _device(emd, X, T)
    xin = torch.from_numpy(X).pin_memory()
    mi = emd.config.max_imfs
    out = (torch.full((batch, mi, 700), np.nan, dtype=torch.float64).pin_memory(),
           torch.full((batch,), -7, dtype=torch.int32).pin_memory(),
           torch.full((batch,), -7, dtype=torch.int32).pin_memory())
    imfs, n, o = emd(xin, T=T, out=out)
    assert imfs.data_ptr() == out[0].data_ptr()
    _same((imfs.numpy(), n.numpy(), o.numpy()) + tuple(x.numpy() for x in emd.last_debug), ref)


@pytest.mark.gpu
def test_host_rejects_bad_out():
    emd = GPUBatchEMD()
    X = W.sinusoid_batch(8, 100, seed=1)
    with pytest.raises(ValueError):
        emd(X, out=(np.zeros((8, 3, 100)), np.zeros(8, np.int32), np.zeros(8, np.int32)))
    with pytest.raises(ValueError):
        emd(torch.from_numpy(X).cuda(), out=(None, None, None))


@pytest.mark.gpu
def test_host_edge_signals_equal_device():
    """Signals whose outputs end oddly -- a pure tone (residue dropped), a
    trend alone, a tone over a trend, all zeros, an overflowing chirp -- over
    several chunks: the host path copies only the rows that may hold data
    (including the dropped trend row a ~zero residue leaves in place) and
    writes the rest as zeros; every element must equal the device path."""
    emd = GPUBatchEMD()
    N = 512
    t = np.arange(N, dtype=np.float64)
    kinds = [np.sin(2 * np.pi * t / 64.0),
             1e-3 * t - 0.2,
             np.sin(2 * np.pi * t / 40.0) + 2e-3 * t,
             np.zeros(N),
             np.sin(2 * np.pi * (0.001 + 0.2 * t / N) * t),
             np.cos(2 * np.pi * t / 128.0) * np.exp(-t / 300.0)]
    X = np.stack([kinds[i % len(kinds)] * (1.0 + 0.01 * (i // len(kinds))) for i in range(600)])
    ref = _device(emd, X)
    imfs, n, o = emd(X)
    _same((imfs, n, o) + tuple(emd.last_debug), ref)


@pytest.mark.gpu
def test_host_bytes_reported():
    """emdb_host_bytes: the inputs up, and at most the dense outputs down
    (only rows that may hold data cross the link)."""
    emd = GPUBatchEMD()
    X = W.seismic_batch(512, 1024, seed=9)
    emd(X)
    h2d, d2h = emd._get_launcher()._plan.host_bytes()
    mi = emd.config.max_imfs
    dense = 512 * mi * 1024 * 8 + 2 * 512 * 4 + 3 * 512 * mi * 4
    assert h2d == 512 * 1024 * 8
    assert 0 < d2h <= dense
