"""B200-native batched FP64 EMD (drop-in for SeismicFlow/emd-cuda's GPUBatchEMD)."""
from .kernels import EMDKernelConfig, EMDBatchLauncher  # noqa: F401
from .emd import GPUBatchEMD  # noqa: F401

__all__ = ["GPUBatchEMD", "EMDKernelConfig", "EMDBatchLauncher"]
