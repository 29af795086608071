"""Trace-file ingest (cuda_emd.ingest.decompose_file): a float64 .npy of
traces streamed batch by batch -- input pages locked in place, outputs through
double-buffered staging into a memory-mapped .npy -- must give exactly the
device path's results, with a partial last batch and with a time axis."""
import numpy as np
import pytest
import torch

from cuda_emd import workloads as W
from cuda_emd.emd import GPUBatchEMD
from cuda_emd.ingest import decompose_file

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("with_T", [False, True])
def test_decompose_file_equals_device(tmp_path, with_T):
    X = W.seismic_batch(300, 1024, seed=21)
    T = np.cumsum(np.random.default_rng(3).uniform(0.5, 1.5, 1024)) if with_T else None
    src, dst = str(tmp_path / "in.npy"), str(tmp_path / "out.npy")
    np.save(src, X)
    res = decompose_file(src, dst, batch=128, T=T)
    emd = GPUBatchEMD()
    imfs, n, o = emd(torch.from_numpy(X).cuda(),
                     T=None if T is None else torch.from_numpy(T).cuda())
    got = np.load(dst, mmap_mode="r")
    assert got.shape == tuple(imfs.shape)
    assert np.array_equal(np.asarray(got), imfs.cpu().numpy())
    assert np.array_equal(res["n_imfs"], n.cpu().numpy())
    assert np.array_equal(res["overflow"], o.cpu().numpy())
    for k, d in zip(("debug_n", "debug_extno", "debug_nzm"), emd.last_debug):
        assert np.array_equal(res[k], d.cpu().numpy())
    print("batches read in place:", res["batches_in_place"], "of 3;", res["register_error"])


def test_decompose_file_rejects_bad_input(tmp_path):
    src = str(tmp_path / "bad.npy")
    np.save(src, np.zeros((4, 16), dtype=np.float32))
    with pytest.raises(ValueError):
        decompose_file(src, str(tmp_path / "o.npy"))
