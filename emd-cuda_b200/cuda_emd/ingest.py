"""Trace-file ingest: decompose every trace of a float64 ``.npy`` file
``[ntraces, N]`` into a memory-mapped output ``.npy`` ``[ntraces, max_imfs,
N]`` plus the per-trace counts, batch by batch through the host pipeline
(``emdb_run_host``).

* Input: the file is memory-mapped read-only.  Each batch's range is
  page-locked in place (``emdb_host_register``) so the host pipeline's copies
  read the page cache by DMA with no staging copy.  Where the operating system
  refuses to pin file pages (recent Linux kernels refuse long-term pins of
  file-backed memory), a reader thread copies batch k+1 into one of two
  page-locked input buffers while the GPU works on batch k.
* Output goes through two page-locked staging buffers: while the GPU works on
  batch k+1, a writer thread copies batch k's IMF rows into the output
  mapping (the OS writes them back to the file).

The reference has no ingest step (its API takes arrays already in memory);
this is the step before the hot path for file-based workloads.
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes
import mmap

import numpy as np

from . import _native
from .emd import _normalise_T
from .kernels import EMDKernelConfig

_PAGE = mmap.PAGESIZE


def _page_range(ptr: int, nbytes: int) -> tuple[int, int]:
    """The page-aligned range enclosing [ptr, ptr + nbytes)."""
    lo = ptr & ~(_PAGE - 1)
    hi = (ptr + nbytes + _PAGE - 1) & ~(_PAGE - 1)
    return lo, hi - lo


def decompose_file(in_path: str, out_path: str, batch: int = 16384, T=None,
                   config: EMDKernelConfig | None = None, device: int | None = None,
                   writers: int = 4) -> dict:
    """Decompose every trace of ``in_path`` into ``out_path`` (a new .npy of
    IMF rows); returns ``{"n_imfs", "overflow", "debug_n", "debug_extno",
    "debug_nzm"}`` as NumPy arrays plus ``"batches_in_place"``, the number of
    batches whose input pages were locked and read in place, and
    ``"register_error"``, why they were not (None if they were).  ``T`` as for
    GPUBatchEMD (None = arange).  Raises like GPUBatchEMD; warns
    (UserWarning) if any trace overflowed."""
    import torch
    X = np.load(in_path, mmap_mode="r")
    if X.ndim != 2 or X.dtype != np.float64 or not X.flags.c_contiguous:
        raise ValueError("input must be a C-contiguous float64 .npy of shape [ntraces, N]")
    ntr, N = X.shape
    cfg = config or EMDKernelConfig.for_device(device)
    launcher = cfg.build(device)
    L, plan = launcher._plan.L, launcher._plan
    mi = cfg.max_imfs
    Tn = _normalise_T(T, N, launcher.device)
    Th = None if Tn is None else Tn.detach().cpu().contiguous()
    out = np.lib.format.open_memmap(out_path, mode="w+", dtype=np.float64, shape=(ntr, mi, N))
    res = {k: np.empty((ntr,) if k in ("n_imfs", "overflow") else (ntr, mi), dtype=np.int32)
           for k in ("n_imfs", "overflow", "debug_n", "debug_extno", "debug_nzm")}
    batch = max(1, min(batch, ntr)) if ntr else 1
    stage = [(torch.empty((batch, mi, N), dtype=torch.float64).pin_memory(),
              [torch.empty(s, dtype=torch.int32).pin_memory()
               for s in ((batch,), (batch,), (batch, mi), (batch, mi), (batch, mi))])
             for _ in range(2)]
    stream = torch.cuda.current_stream(launcher.device).cuda_stream
    x_ptr = X.ctypes.data if ntr else 0
    bounds = [(s, min(ntr, s + batch)) for s in range(0, ntr, batch)]

    # in place if the first batch's pages can be locked, else staged
    reg_error = None
    in_place_ok = False
    if bounds:
        lo, nb = _page_range(x_ptr, (bounds[0][1] - bounds[0][0]) * N * 8)
        if L.emdb_host_register(ctypes.c_void_p(lo), nb, 1) == _native.EMDB_OK:
            _native.check(L.emdb_host_unregister(ctypes.c_void_p(lo)), "emdb_host_unregister")
            in_place_ok = True
        else:
            reg_error = _native.last_error()
    stage_in = None if in_place_ok else [torch.empty((batch, N), dtype=torch.float64).pin_memory()
                                         for _ in range(2)]

    def load(k: int, s: int, e: int) -> None:
        dst = stage_in[k].numpy()[: e - s]
        parts = np.array_split(np.arange(e - s), max(1, min(writers, e - s)))
        with cf.ThreadPoolExecutor(max_workers=len(parts)) as ex:
            list(ex.map(lambda p: np.copyto(dst[p[0]: p[-1] + 1], X[s + p[0]: s + p[-1] + 1])
                        if p.size else None, parts))

    def write_back(k: int, s: int, e: int) -> None:
        imfs, small = stage[k]
        src = imfs.numpy()[: e - s]
        # split the copy over rows so numpy's release of the GIL lets threads overlap
        parts = np.array_split(np.arange(e - s), max(1, min(writers, e - s)))
        with cf.ThreadPoolExecutor(max_workers=len(parts)) as ex:
            list(ex.map(lambda p: np.copyto(out[s + p[0]: s + p[-1] + 1], src[p[0]: p[-1] + 1])
                        if p.size else None, parts))
        for name, t in zip(("n_imfs", "overflow", "debug_n", "debug_extno", "debug_nzm"), small):
            res[name][s:e] = t.numpy()[: e - s]

    pending = [None, None]
    in_place = 0
    with cf.ThreadPoolExecutor(max_workers=1) as writer, \
            cf.ThreadPoolExecutor(max_workers=1) as reader:
        loaded = None if in_place_ok or not bounds else reader.submit(load, 0, *bounds[0])
        for bi, (s, e) in enumerate(bounds):
            k = bi % 2
            if pending[k] is not None:
                pending[k].result()          # output staging buffer k free again
            registered = False
            if in_place_ok:
                ptr = x_ptr + s * N * 8
                lo, nb = _page_range(ptr, (e - s) * N * 8)
                registered = L.emdb_host_register(ctypes.c_void_p(lo), nb, 1) == _native.EMDB_OK
                in_place += int(registered)
            else:
                loaded.result()              # batch bi is in stage_in[k]
                ptr = stage_in[k].data_ptr()
                if bi + 1 < len(bounds):     # its buffer's last reader (batch bi-1) has returned
                    loaded = reader.submit(load, (bi + 1) % 2, *bounds[bi + 1])
            try:
                imfs, small = stage[k]
                _native.check(L.emdb_run_host(
                    plan.handle, ctypes.c_void_p(ptr),
                    Th.data_ptr() if Th is not None else None, e - s, N, imfs.data_ptr(),
                    *[t.data_ptr() for t in small], stream), "emdb_run_host")
            finally:
                if registered:
                    _native.check(L.emdb_host_unregister(ctypes.c_void_p(lo)),
                                  "emdb_host_unregister")
            launcher.check_status()
            pending[k] = writer.submit(write_back, k, s, e)
        for f in pending:
            if f is not None:
                f.result()
    out.flush()
    del out
    n_hit = int((res["overflow"] != 0).sum())
    if n_hit:
        import warnings
        warnings.warn(
            f"{n_hit}/{ntr} signal(s) hit MAX_EXTREMA or MAX_ITERATION during sifting -- their "
            "output is not a verified decomposition. Check the `overflow` array to find which, "
            "and raise EMDKernelConfig.max_extrema / max_iteration for those.", stacklevel=2)
    res["batches_in_place"] = in_place
    res["register_error"] = reg_error
    return res
