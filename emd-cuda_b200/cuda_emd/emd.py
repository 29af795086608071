"""GPUBatchEMD -- drop-in for the reference's host wrapper
(SeismicFlow/emd-cuda emd.py:53-114) over the B200 kernels.

    from cuda_emd.emd import GPUBatchEMD
    gpu_emd = GPUBatchEMD()
    gpu_emd.warmup()
    imfs, n_imfs, overflow = gpu_emd(signals)      # signals [batch, N] float64

``imfs`` is [batch, MAX_IMFS, N] float64, ``n_imfs`` / ``overflow`` [batch]
int32, ``last_debug`` holds (debug_n, debug_extno, debug_nzm) [batch, MAX_IMFS].
Results are returned in the caller's array framework (torch, CuPy or NumPy).

Beyond the reference: ``ragged(values, offsets, T=None, order=None)``
decomposes a CSR batch of mixed-length traces, each with its own time axis
if given, in one launch.
"""
from __future__ import annotations

import warnings

import numpy as np

try:
    from .kernels import EMDKernelConfig
except ImportError:  # flat layout: emd.py and kernels.py side by side
    from kernels import EMDKernelConfig  # type: ignore


# FP32 path: the largest normalised time a float axis may hold, so that every
# sample time and mirrored knot position (up to about twice the last time)
# keeps a spacing of at least one ulp.  The reference drops a knot whose
# position equals its neighbour's (kernels.py:521-556); with such an axis that
# never happens, as in double.
F32_MAX_TIME = float(1 << 22)


def _as_f64_axis(T, device: int, f32: bool):
    # the reference normalises T in float64 whatever it was given
    # (cp.asarray(T, dtype=cp.float64), emd.py:85); the FP64 launcher keeps
    # its dtype rule (float64 only), the FP32 one also takes float32 T
    from ._arrays import as_device_f64, _to_torch
    if not f32:
        return as_device_f64(T, device)[0]
    import torch
    t, _ = _to_torch(T, device)
    if t.dtype not in (torch.float32, torch.float64):
        raise ValueError(f"T must be float32 or float64, got {t.dtype}")
    return t.to(torch.float64)


def _to_real(Tn, f32: bool):
    """The normalised axis in the kernels' type; for float it must stay
    strictly increasing and below F32_MAX_TIME."""
    if not f32:
        return Tn
    import torch
    Tf = Tn.to(torch.float32)
    if Tf.numel() > 1 and not bool((Tf[1:] > Tf[:-1]).all()):
        raise ValueError("T must normalise to an axis that stays strictly increasing in float32")
    if Tf.numel() and float(Tf.abs().max().item()) >= F32_MAX_TIME:
        raise ValueError(f"normalised T must stay below {F32_MAX_TIME:.0f} for REAL_T=float")
    return Tf


def _normalise_T(T, N: int, device: int, f32: bool = False):
    """emd.py:83-88: arange(N) if T is None, else (T - T[0]) / min(diff(T)).
    None stays None (the kernel then uses arange without a buffer).  The
    normalised axis must be finite and strictly increasing; the reference
    would read stale envelope values otherwise, so this build refuses it.
    f32: normalised in float64 as the reference does, then rounded to float."""
    if T is None:
        return None
    import torch
    Td = _as_f64_axis(T, device, f32)
    if Td.dim() != 1 or Td.shape[0] != N:
        raise ValueError(f"T must be 1-D of length {N}")
    if N < 2:
        return _to_real(Td - Td[0] if N == 1 else Td, f32)
    d = Td[1:] - Td[:-1]
    Tn = (Td - Td[0]) / torch.min(d)
    dn = Tn[1:] - Tn[:-1]
    if not bool(torch.isfinite(Tn).all()) or not bool((dn > 0).all()):
        raise ValueError("T must normalise to a finite, strictly increasing axis")
    return _to_real(Tn, f32)


def _normalise_T_csr(T, offsets, device: int, f32: bool = False):
    """Per-trace _normalise_T of CSR-aligned time axes, on the device:
    (T_b - T_b[0]) / min(diff(T_b)) for every trace b."""
    import torch
    from ._arrays import as_device_i64
    Td = _as_f64_axis(T, device, f32)
    offs = as_device_i64(offsets, device)
    if Td.dim() != 1 or Td.shape[0] != int(offs[-1].item()):
        raise ValueError("T must be 1-D and aligned with values (length offsets[-1])")
    B = offs.shape[0] - 1
    lens = offs[1:] - offs[:-1]
    trace = torch.repeat_interleave(torch.arange(B, device=Td.device), lens)
    first = Td[offs[:-1]]
    d = Td[1:] - Td[:-1]
    # steps that stay inside one trace
    inner = trace[1:] == trace[:-1]
    big = torch.full((B,), float("inf"), dtype=torch.float64, device=Td.device)
    big = big.scatter_reduce(0, trace[1:][inner], d[inner], reduce="amin")
    step = torch.where(torch.isinf(big), torch.ones_like(big), big)
    Tn = (Td - first[trace]) / step[trace]
    dn = Tn[1:] - Tn[:-1]
    if not bool(torch.isfinite(Tn).all()) or not bool((dn[inner] > 0).all()):
        raise ValueError("each trace's T must normalise to a finite, strictly increasing axis")
    if f32:
        Tf = Tn.to(torch.float32)
        if not bool((Tf[1:] > Tf[:-1])[inner].all()):
            raise ValueError("each trace's T must stay strictly increasing in float32")
        if Tf.numel() and float(Tf.abs().max().item()) >= F32_MAX_TIME:
            raise ValueError(f"normalised T must stay below {F32_MAX_TIME:.0f} for REAL_T=float")
        return Tf
    return Tn


class GPUBatchEMD:
    def __init__(self, config: "EMDKernelConfig | None" = None):
        self._config = config or EMDKernelConfig.for_device()
        self._launcher = None
        self.last_debug = None

    @property
    def config(self) -> EMDKernelConfig:
        return self._config

    def warmup(self, N: int = 64) -> None:
        """One tiny real call (an all-zero trace, emd.py:58-64) so that plan
        creation and first-launch costs land here, not in a timed call."""
        import torch
        dt = torch.float32 if self._config.f32 else torch.float64
        self(torch.zeros((1, N), dtype=dt, device="cuda"))

    def _get_launcher(self):
        if self._launcher is None:
            self._launcher = self._config.build()
        return self._launcher

    def _overflow_warning(self, overflow, batch: int) -> None:
        import torch
        ov = overflow if isinstance(overflow, torch.Tensor) else torch.as_tensor(np.asarray(overflow))
        n_hit = int(ov.sum().item())
        if n_hit:
            warnings.warn(
                f"{n_hit}/{batch} signal(s) hit MAX_EXTREMA or MAX_ITERATION during "
                "sifting -- their output is not a verified decomposition. Check the "
                "`overflow` array to find which, and raise EMDKernelConfig.max_extrema "
                "/ max_iteration for those.",
                stacklevel=3,
            )

    def __call__(self, signals, T=None, out=None, order=None):
        """Decompose signals [batch, N] (or [N]).  Device input (torch CUDA,
        CuPy) gives device results.  Host input (NumPy, CPU torch) runs the
        host pipeline: one launch whose finished traces are copied back while
        the rest sift, results in host memory; ``out`` = optional
        (imfs, n_imfs, overflow) host buffers to fill.  ``order`` (device
        input only): an int32 permutation of the batch giving the work
        queue's order (e.g. scheduler.learned_order's longest-predicted-first);
        it changes when each trace runs, never a result."""
        if signals.ndim == 1:
            signals = signals[None, :]
        dt = np.dtype(str(signals.dtype).replace("torch.", ""))
        if dt != self._config.dtype:
            raise ValueError(
                f"GPUBatchEMD (this build) is {self._config.dtype} only, got {signals.dtype}. "
                f"Cast explicitly first, e.g. signals.astype({self._config.dtype}) -- this "
                f"class won't silently do that for you."
            )
        launcher = self._get_launcher()
        batch, N = signals.shape
        Tn = _normalise_T(T, N, launcher.device, self._config.f32)
        from ._arrays import kind_of
        if kind_of(signals) in ("numpy", "torch_cpu"):
            if order is not None:
                raise ValueError("order= is for device input")
            imfs, n_imfs, overflow, dn, de, dz = launcher.run_host(signals, Tn, out=out)
        elif out is not None:
            raise ValueError("out= is for host input; device input returns device arrays")
        elif order is not None:
            imfs, n_imfs, overflow, dn, de, dz = self._run_ordered(launcher, signals, Tn, order)
        else:
            imfs, n_imfs, overflow, dn, de, dz = launcher.run(signals, Tn)
        self.last_debug = (dn, de, dz)
        launcher.check_status()
        self._overflow_warning(overflow, batch)
        return imfs, n_imfs, overflow

    @staticmethod
    def _run_ordered(launcher, signals, Tn, order):
        """A dense batch through the CSR launch (offsets b*N), whose queue
        takes an order: trace b's rows land at b*max_imfs*N, the dense layout."""
        import torch
        from ._arrays import _to_torch
        sig, _ = _to_torch(signals, launcher.device)
        B, N = sig.shape
        offs = torch.arange(0, (B + 1) * N, N, dtype=torch.int64, device=sig.device)
        res = launcher.run_ragged(sig.reshape(-1), offs, order=order, T=Tn,
                                  t_per_trace=False, max_n=N)
        mi = launcher.config.max_imfs
        return (res[0].reshape(B, mi, N),) + tuple(res[1:])

    def ragged(self, values, offsets, T=None, order=None, max_n: int | None = None):
        """Decompose a CSR batch (values f64 [total], offsets int64 [batch+1]) in
        one launch.  ``T``: None = arange(N_b) per trace; else CSR-aligned time
        axes (f64 [total], trace b's at T[offsets[b]:offsets[b+1]]), each
        normalised as emd.py:83-88 does for a single T -- this lifts the
        reference's one-shared-T restriction (emd.py:28-30).  ``order`` (int32
        permutation) only sets the queue order.  Returns (imfs_csr, n_imfs,
        overflow)."""
        launcher = self._get_launcher()
        Tn = None if T is None else _normalise_T_csr(T, offsets, launcher.device, self._config.f32)
        imfs, n_imfs, overflow, dn, de, dz = launcher.run_ragged(values, offsets, order=order,
                                                                 T=Tn, t_per_trace=True,
                                                                 max_n=max_n)
        self.last_debug = (dn, de, dz)
        launcher.check_status()
        self._overflow_warning(overflow, n_imfs.shape[0])
        return imfs, n_imfs, overflow

    def unpack(self, imfs, n_imfs, i: int):
        """Signal i's rows [n_imfs[i], N] as a NumPy array (emd.py:109-114)."""
        k = int(n_imfs[i].item() if hasattr(n_imfs[i], "item") else n_imfs[i])
        x = imfs[i, :k, :]
        if hasattr(x, "cpu"):
            return x.cpu().numpy()
        if hasattr(x, "get"):
            return x.get()
        return np.asarray(x)
