"""Drive the reference's own ``emd_batch_kernel`` (built into ``oracle/_ref`` by
``oracle/build_ref.py``) from tests.  Checker infrastructure: GPU only, never
part of the product.  Device memory comes from torch."""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def ref_lib_path(name: str = "libemd_ref.so") -> str:
    return os.path.join(REF_DIR, name)


def have_ref(name: str = "libemd_ref.so") -> bool:
    return os.path.isfile(ref_lib_path(name))


def f32_name(name: str) -> str:
    """The REAL_T = float build of a reference variant:
    libemd_ref[_small][_nofma].so -> libemd_ref[_small]_f32[_nofma].so."""
    stem = name[:-3]
    if stem.endswith("_nofma"):
        return stem[:-6] + "_f32_nofma.so"
    return stem + "_f32.so"


class RefKernel:
    """ctypes handle on one reference build variant."""

    def __init__(self, name: str = "libemd_ref.so"):
        self.lib = ctypes.CDLL(ref_lib_path(name))
        P, I = ctypes.c_void_p, ctypes.c_int
        self.lib.ref_emd_launch.argtypes = [P, P, I, I, P, P, P, P, P, P, P, P]
        self.lib.ref_emd_launch.restype = I
        self.lib.ref_envelope_launch.argtypes = [P, P, I, I, P, P, P, P, P, P, P, P, P, P]
        self.lib.ref_envelope_launch.restype = I
        self.lib.ref_config.argtypes = [ctypes.POINTER(ctypes.c_int)]
        cfg = (ctypes.c_int * 5)()
        self.lib.ref_config(cfg)
        self.max_extrema, self.nbsym, self.max_iteration, self.max_imfs, self.threads = list(cfg)
        # REAL_T of the build (4: float); builds that predate the query are double
        nbytes = self.lib.ref_real_bytes() if hasattr(self.lib, "ref_real_bytes") else 8
        self.np_dtype = np.float32 if nbytes == 4 else np.float64

    @property
    def torch_dtype(self):
        import torch
        return torch.float32 if self.np_dtype == np.float32 else torch.float64

    def run_device(self, sig, T, stream=None):
        """sig [B,N] REAL_T cuda, T [N] REAL_T cuda -> the reference's 6-tuple
        (kernels.py:1343-1372), allocated and zero/−1-filled like run()."""
        import torch
        B, N = sig.shape
        dev = sig.device
        rt = self.torch_dtype
        pools = torch.empty(6 * B * N, dtype=rt, device=dev)
        imfs = torch.zeros((B, self.max_imfs, N), dtype=rt, device=dev)
        n_imfs = torch.zeros(B, dtype=torch.int32, device=dev)
        ovf = torch.zeros(B, dtype=torch.int32, device=dev)
        dn = torch.full((B, self.max_imfs), -1, dtype=torch.int32, device=dev)
        de = torch.full((B, self.max_imfs), -1, dtype=torch.int32, device=dev)
        dz = torch.full((B, self.max_imfs), -1, dtype=torch.int32, device=dev)
        st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        rc = self.lib.ref_emd_launch(sig.data_ptr(), T.data_ptr(), B, N, imfs.data_ptr(),
                                     n_imfs.data_ptr(), ovf.data_ptr(), pools.data_ptr(),
                                     dn.data_ptr(), de.data_ptr(), dz.data_ptr(), st)
        if rc != 0:
            raise RuntimeError(f"reference launch failed: cuda error {rc}")
        return imfs, n_imfs, ovf, dn, de, dz

    def run(self, signals: np.ndarray, T: np.ndarray):
        import torch
        sig = torch.from_numpy(np.ascontiguousarray(signals, dtype=self.np_dtype)).cuda()
        Td = torch.from_numpy(np.ascontiguousarray(T, dtype=self.np_dtype)).cuda()
        out = self.run_device(sig, Td)
        torch.cuda.synchronize()
        return tuple(o.cpu().numpy() for o in out)

    def envelope(self, signals: np.ndarray, T: np.ndarray):
        """run_envelope_only's 9-tuple (kernels.py:1374-1407)."""
        import torch
        sig = torch.from_numpy(np.ascontiguousarray(signals, dtype=self.np_dtype)).cuda()
        Td = torch.from_numpy(np.ascontiguousarray(T, dtype=self.np_dtype)).cuda()
        B, N = sig.shape
        mbuf = self.max_extrema + 2 * self.nbsym
        z = lambda *s, dt=self.torch_dtype: torch.zeros(s, dtype=dt, device="cuda")
        outs = [z(B, N), z(B, N), z(B, 2, dt=torch.int32), z(B, dt=torch.int32),
                z(B, mbuf), z(B, mbuf), z(B, mbuf), z(B, mbuf), z(B, 2, dt=torch.int32)]
        rc = self.lib.ref_envelope_launch(sig.data_ptr(), Td.data_ptr(), B, N,
                                          *[o.data_ptr() for o in outs],
                                          torch.cuda.current_stream().cuda_stream)
        if rc != 0:
            raise RuntimeError(f"reference envelope launch failed: cuda error {rc}")
        torch.cuda.synchronize()
        return tuple(o.cpu().numpy() for o in outs)
