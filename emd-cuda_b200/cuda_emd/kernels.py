"""EMDKernelConfig and EMDBatchLauncher -- the reference's config/launch layer
(SeismicFlow/emd-cuda kernels.py:1170-1407) over the B200 C ABI.

Same fields, properties, sizing helpers and return tuples as the reference;
the launch goes to ``libemdb200.so`` (hand-written sm_100a CUDA) instead of a
CuPy RawModule.  Arrays may be torch tensors (CUDA or CPU), CuPy arrays or
NumPy arrays; outputs come back in the caller's framework (NumPy inputs are
copied to the device and the results copied back).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native
from ._arrays import (as_device_f64, as_device_real, as_device_i64, as_device_i32, to_caller,
                      device_of, stream_of, kind_of)

REAL_TYPES = {"double": np.float64, "float": np.float32}


@dataclass
class EMDKernelConfig:
    max_extrema: int = 1024
    nbsym: int = 2
    max_iteration: int = 1000
    max_imfs: int = 16
    threads_per_block: int = 128
    # The type the kernels compute in: the reference substitutes REAL_T into
    # its kernel source from this name (kernels.py:78, 1277-1285) and fixes
    # it to "double"; "float" selects the FP32 build of the B200 kernels.
    real_t: str = "double"

    def __post_init__(self):
        if self.real_t not in REAL_TYPES:
            raise ValueError(f"real_t must be one of {sorted(REAL_TYPES)}, got {self.real_t!r}")

    @property
    def dtype(self):
        return np.dtype(REAL_TYPES[self.real_t])

    @property
    def real_t_name(self) -> str:
        """The C type the kernels compute in (kernels.py:1182-1185)."""
        return self.real_t

    @property
    def f32(self) -> bool:
        return self.real_t == "float"

    @property
    def itemsize(self) -> int:
        return self.dtype.itemsize

    def static_shared_mem_bytes(self) -> int:
        """The reference kernel's static shared memory, 12*T + 4 bytes
        (kernels.py:1191-1203).  Kept for API parity; the B200 kernels carve
        everything from one dynamic arena (see ``arena_bytes``)."""
        return 3 * 4 * self.threads_per_block + 4

    @classmethod
    def for_device(cls, device=None, target_blocks_per_sm: int = 4,
                   min_max_extrema: int = 1024, real_t: str = "double") -> "EMDKernelConfig":
        """Same sizing arithmetic as the reference (kernels.py:1205-1271), so
        the default ``max_extrema`` -- which decides the overflow flag and the
        extrema truncation -- matches it on the same device (1024 on B200)."""
        import torch
        dev = torch.device("cuda", device if isinstance(device, int) else
                           (device.index if device is not None and hasattr(device, "index") and device.index is not None
                            else torch.cuda.current_device()))
        optin = _smem_optin(dev.index)
        cfg = cls(real_t=real_t)
        static_bytes = cfg.static_shared_mem_bytes()
        per_elem = 6 * cfg.itemsize + 2 * 4
        budget_occ = max(0, optin // target_blocks_per_sm - static_bytes)
        max_extrema_occ = max(0, budget_occ // per_elem - 2 * cfg.nbsym)
        desired = max(min_max_extrema, max_extrema_occ)
        hard_budget = max(0, int(optin * 0.95) - static_bytes)
        hard_max = max(64, hard_budget // per_elem - 2 * cfg.nbsym)
        cfg.max_extrema = min(desired, hard_max)
        return cfg

    def shared_mem_bytes(self) -> int:
        """The reference kernel's dynamic shared memory (kernels.py:1273-1275)."""
        m = self.max_extrema + 2 * self.nbsym
        return m * (6 * self.itemsize + 2 * 4) + 256

    def arena_bytes(self, max_n: int, device: int | None = None) -> int:
        """Dynamic shared memory per CTA the B200 kernel uses for traces up to max_n."""
        return self.build(device)._plan.query(max_n, f32=self.f32)[0]

    def to_c(self) -> _native.EmdbConfig:
        return _native.EmdbConfig(int(self.max_extrema), int(self.nbsym), int(self.max_iteration),
                                  int(self.max_imfs), int(self.threads_per_block))

    def build(self, device: int | None = None) -> "EMDBatchLauncher":
        return EMDBatchLauncher(self, device=device)


def _smem_optin(index: int) -> int:
    import torch
    props = torch.cuda.get_device_properties(index)
    v = getattr(props, "shared_memory_per_block_optin", None)
    return int(v) if v else 49152


class EMDBatchLauncher:
    """Owns the device plan (scratch + config) and launches the B200 kernels.
    Errors follow the reference: ValueError for bad dtypes or a config the
    device cannot hold, RuntimeError for CUDA failures (kernels.py:1304-1352)."""

    def __init__(self, config: EMDKernelConfig, device: int | None = None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("EMDBatchLauncher needs a CUDA device; there is no CPU path")
        self.config = config
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._plan = _native.Plan(config.to_c(), self.device)

    # -- helpers ------------------------------------------------------------
    def _check_dtype(self, signals, T):
        cfg = self.config
        sd = np.dtype(str(signals.dtype).replace("torch.", ""))
        td = np.dtype(str(T.dtype).replace("torch.", "")) if T is not None else cfg.dtype
        if sd != cfg.dtype or td != cfg.dtype:
            raise ValueError(
                f"This launcher computes in REAL_T={cfg.real_t_name} (dtype {cfg.dtype}), "
                f"but got signals.dtype={signals.dtype}, T.dtype={getattr(T, 'dtype', None)}. "
                f"Passing mismatched dtypes would silently reinterpret bytes rather than convert "
                f"them -- cast explicitly first.")

    def _raise_status(self, stream: int) -> None:
        st = self._plan.status(stream)
        if st & _native.STATUS_TOO_LONG:
            raise ValueError("a trace did not fit the kernel's shared-memory arena")
        if st & _native.STATUS_STALE_ENVELOPE:
            raise RuntimeError("a sample fell outside the envelope knot span (time axis not increasing)")

    # -- reference API ------------------------------------------------------
    def run(self, signals, T):
        """Dense batch: (imfs, n_imfs, overflow, debug_n, debug_extno, debug_nzm)
        (kernels.py:1343-1372)."""
        import torch
        self._check_dtype(signals, T)
        f32 = self.config.f32
        sig, kind = as_device_real(signals, self.device, f32)
        if sig.dim() != 2:
            raise ValueError("signals must be [batch, N]")
        Td = None if T is None else as_device_real(T, self.device, f32)[0]
        B, N = sig.shape
        mi = self.config.max_imfs
        imfs = torch.empty((B, mi, N), dtype=sig.dtype, device=sig.device)
        n_imfs = torch.empty(B, dtype=torch.int32, device=sig.device)
        ovf = torch.empty(B, dtype=torch.int32, device=sig.device)
        dn = torch.empty((B, mi), dtype=torch.int32, device=sig.device)
        de = torch.empty((B, mi), dtype=torch.int32, device=sig.device)
        dz = torch.empty((B, mi), dtype=torch.int32, device=sig.device)
        st = stream_of(sig.device)
        fn = self._plan.L.emdb_run_f32 if f32 else self._plan.L.emdb_run
        _native.check(fn(
            self._plan.handle, sig.data_ptr(), Td.data_ptr() if Td is not None else None, B, N,
            imfs.data_ptr(), n_imfs.data_ptr(), ovf.data_ptr(), dn.data_ptr(), de.data_ptr(),
            dz.data_ptr(), st), "emdb_run")
        self._keepalive = (sig, Td)
        return tuple(to_caller(x, kind) for x in (imfs, n_imfs, ovf, dn, de, dz))

    def run_host(self, signals, T, out=None):
        """Dense batch from and to host memory (NumPy or CPU torch) through
        emdb_run_host: one launch, each finished chunk's IMF rows copied back
        while the rest still sifts.  ``out`` = optional (imfs, n_imfs, overflow)
        host buffers to fill (page-locked ones keep the copies asynchronous);
        otherwise page-locked buffers are allocated.  Returns the same 6-tuple
        as run(), in the caller's framework."""
        import torch
        self._check_dtype(signals, T)
        if self.config.f32:
            raise ValueError("the host-memory pipeline computes in double; for REAL_T=float "
                             "copy the batch to the device and call run()")
        kind = kind_of(signals)
        if kind not in ("numpy", "torch_cpu"):
            raise ValueError("run_host takes host arrays (NumPy or CPU torch)")
        sig = signals if isinstance(signals, torch.Tensor) else torch.from_numpy(np.asarray(signals))
        sig = sig.contiguous()
        if sig.dim() != 2:
            raise ValueError("signals must be [batch, N]")
        B, N = sig.shape
        mi = self.config.max_imfs
        Th = None
        if T is not None:
            Th = (T.detach().cpu() if isinstance(T, torch.Tensor)
                  else torch.from_numpy(np.asarray(T, dtype=np.float64))).contiguous()

        def host(shape, dtype, given, what):
            if given is None:
                return torch.empty(shape, dtype=dtype, pin_memory=True)
            t = given if isinstance(given, torch.Tensor) else torch.from_numpy(given)
            if t.is_cuda or tuple(t.shape) != shape or t.dtype != dtype or not t.is_contiguous():
                raise ValueError(f"out {what} must be a contiguous host {dtype} array of shape {shape}")
            return t

        o = out if out is not None else (None, None, None)
        imfs = host((B, mi, N), torch.float64, o[0], "imfs")
        n_imfs = host((B,), torch.int32, o[1], "n_imfs")
        ovf = host((B,), torch.int32, o[2], "overflow")
        dn, de, dz = (torch.empty((B, mi), dtype=torch.int32, pin_memory=True) for _ in range(3))
        st = stream_of(torch.device("cuda", self.device))
        _native.check(self._plan.L.emdb_run_host(
            self._plan.handle, sig.data_ptr(), Th.data_ptr() if Th is not None else None, B, N,
            imfs.data_ptr(), n_imfs.data_ptr(), ovf.data_ptr(), dn.data_ptr(), de.data_ptr(),
            dz.data_ptr(), st), "emdb_run_host")
        res = (imfs, n_imfs, ovf, dn, de, dz)
        if kind == "numpy":
            return tuple(x.numpy() for x in res)
        return res

    def run_ragged(self, values, offsets, order=None, T=None, t_per_trace: bool = True,
                   max_n: int | None = None):
        """CSR batch of mixed lengths in one launch.  Returns
        (imfs_csr [max_imfs * total], n_imfs, overflow, debug_n, debug_extno, debug_nzm);
        trace b's rows are imfs_csr[max_imfs*off[b] : max_imfs*off[b+1]].reshape(max_imfs, N_b)."""
        import torch
        f32 = self.config.f32
        vals, kind = as_device_real(values, self.device, f32)
        offs = as_device_i64(offsets, self.device)
        B = offs.shape[0] - 1
        if max_n is None:
            max_n = int((offs[1:] - offs[:-1]).max().item()) if B > 0 else 0
        Td = None if T is None else as_device_real(T, self.device, f32)[0]
        od = None if order is None else as_device_i32(order, self.device)
        mi = self.config.max_imfs
        total = vals.shape[0]
        imfs = torch.empty(mi * total, dtype=vals.dtype, device=vals.device)
        n_imfs = torch.empty(B, dtype=torch.int32, device=vals.device)
        ovf = torch.empty(B, dtype=torch.int32, device=vals.device)
        dn = torch.empty((B, mi), dtype=torch.int32, device=vals.device)
        de = torch.empty((B, mi), dtype=torch.int32, device=vals.device)
        dz = torch.empty((B, mi), dtype=torch.int32, device=vals.device)
        st = stream_of(vals.device)
        fn = self._plan.L.emdb_run_ragged_f32 if f32 else self._plan.L.emdb_run_ragged
        _native.check(fn(
            self._plan.handle, vals.data_ptr(), offs.data_ptr(), B, int(max_n),
            Td.data_ptr() if Td is not None else None, 1 if t_per_trace else 0,
            od.data_ptr() if od is not None else None, imfs.data_ptr(), n_imfs.data_ptr(),
            ovf.data_ptr(), dn.data_ptr(), de.data_ptr(), dz.data_ptr(), st), "emdb_run_ragged")
        self._keepalive = (vals, offs, Td, od)
        return tuple(to_caller(x, kind) for x in (imfs, n_imfs, ovf, dn, de, dz))

    def run_envelope_only(self, signals, T):
        """Extrema + mirroring + spline without the sift loop, the reference's
        9-tuple (kernels.py:1374-1407)."""
        import torch
        self._check_dtype(signals, T)
        f32 = self.config.f32
        sig, kind = as_device_real(signals, self.device, f32)
        Td = None if T is None else as_device_real(T, self.device, f32)[0]
        B, N = sig.shape
        mbuf = self.config.max_extrema + 2 * self.config.nbsym
        dev = sig.device
        f = lambda *s: torch.empty(s, dtype=sig.dtype, device=dev)
        i = lambda *s: torch.empty(s, dtype=torch.int32, device=dev)
        outs = (f(B, N), f(B, N), i(B, 2), i(B), f(B, mbuf), f(B, mbuf), f(B, mbuf), f(B, mbuf), i(B, 2))
        st = stream_of(dev)
        fn = self._plan.L.emdb_envelope_f32 if f32 else self._plan.L.emdb_envelope
        _native.check(fn(
            self._plan.handle, sig.data_ptr(), Td.data_ptr() if Td is not None else None, B, N,
            *[o.data_ptr() for o in outs], st), "emdb_envelope")
        self._keepalive = (sig, Td)
        return tuple(to_caller(x, kind) for x in outs)

    def check_status(self) -> None:
        """Synchronise and raise if the kernel reported a status bit."""
        import torch
        self._raise_status(stream_of(torch.device("cuda", self.device)))
