"""Seeded synthetic trace generators for the benchmark workloads.

No public dataset is named for this path, so every workload is synthetic and
fully determined by its seed:

* ``sinusoid_batch``  -- three tones (0.005-0.05, 0.05-0.15, 0.15-0.4 cycles/sample,
  amplitudes U[0.5, 2], phases U[0, 2pi)) + linear trend (slope U[-1e-3, 1e-3])
  + Gaussian noise sigma 0.05.  256 x 1024 is the small CPU-checkable case.
* ``seismic_batch``   -- Ricker wavelet (peak 10-60 Hz) convolved with 20-80
  Laplace(0,1) reflectivity spikes at uniform positions, plus 5-100 Hz
  band-limited Gaussian noise (4th-order Butterworth, SOS form) at 10 dB SNR,
  dt = 2 ms.  16,384 x 2048 is the equal-length head-to-head case.
* ``chirp``           -- linear chirp 0.001 -> 0.45 cycles/sample, amplitude 1,
  noise sigma 0.01.
* ``ragged_mix``      -- lengths log-uniform in [lo, hi]; 60 % seismic, 38 %
  sinusoid, 2 % chirp; returned in CSR layout (values, offsets).
"""
from __future__ import annotations

import numpy as np

DT_SEISMIC = 0.002


def sinusoid_trace(rng: np.random.Generator, N: int) -> np.ndarray:
    t = np.arange(N, dtype=np.float64)
    f = np.array([rng.uniform(0.005, 0.05), rng.uniform(0.05, 0.15), rng.uniform(0.15, 0.4)])
    amp = rng.uniform(0.5, 2.0, size=3)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=3)
    slope = rng.uniform(-1e-3, 1e-3)
    x = (amp[:, None] * np.sin(2.0 * np.pi * f[:, None] * t[None, :] + ph[:, None])).sum(0)
    x = x + slope * t + rng.normal(0.0, 0.05, size=N)
    return x


def sinusoid_batch(n: int, N: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.stack([sinusoid_trace(rng, N) for _ in range(n)])


def _ricker(f: float, dt: float) -> np.ndarray:
    half = 1.5 / f
    t = np.arange(-half, half + dt / 2, dt)
    a = (np.pi * f * t) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


_SOS_CACHE: dict = {}


def _bandpass_sos(dt: float):
    key = round(dt, 9)
    if key not in _SOS_CACHE:
        from scipy.signal import butter
        _SOS_CACHE[key] = butter(4, [5.0, 100.0], btype="bandpass", fs=1.0 / dt, output="sos")
    return _SOS_CACHE[key]


def seismic_trace(rng: np.random.Generator, N: int, dt: float = DT_SEISMIC) -> np.ndarray:
    from scipy.signal import sosfilt
    f = rng.uniform(10.0, 60.0)
    k = int(rng.integers(20, 81))
    refl = np.zeros(N)
    pos = rng.integers(0, N, size=k)
    np.add.at(refl, pos, rng.laplace(0.0, 1.0, size=k))
    w = _ricker(f, dt)
    half = (w.shape[0] - 1) // 2
    # centred crop of the full convolution (= mode "same" when N >= len(w))
    sig = np.convolve(refl, w, mode="full")[half:half + N]
    noise = sosfilt(_bandpass_sos(dt), rng.normal(0.0, 1.0, size=N))
    ps = float(np.mean(sig * sig))
    pn = float(np.mean(noise * noise))
    if ps <= 0.0:
        ps = 1.0
    noise *= np.sqrt(ps / (10.0 * pn)) if pn > 0 else 0.0
    return sig + noise


def seismic_batch(n: int, N: int, seed: int = 1, dt: float = DT_SEISMIC) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.stack([seismic_trace(rng, N, dt) for _ in range(n)])


def chirp_trace(rng: np.random.Generator, N: int) -> np.ndarray:
    t = np.arange(N, dtype=np.float64)
    f0, f1 = 0.001, 0.45
    phase = 2.0 * np.pi * (f0 * t + 0.5 * (f1 - f0) * t * t / max(N - 1, 1))
    return np.sin(phase) + rng.normal(0.0, 0.01, size=N)


def ragged_lengths(rng: np.random.Generator, n: int, lo: int, hi: int) -> np.ndarray:
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=n)).astype(np.int64).clip(lo, hi)


def ragged_mix(n: int, lo: int = 256, hi: int = 8192, seed: int = 2):
    """CSR batch: (values f64 [sum N_i], offsets int64 [n+1], kinds int8 [n]).
    kind 0 = seismic, 1 = sinusoid, 2 = chirp."""
    rng = np.random.default_rng(seed)
    lens = ragged_lengths(rng, n, lo, hi)
    u = rng.uniform(size=n)
    kinds = np.where(u < 0.60, 0, np.where(u < 0.98, 1, 2)).astype(np.int8)
    offsets = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])
    values = np.empty(int(offsets[-1]), dtype=np.float64)
    for i in range(n):
        N = int(lens[i])
        if kinds[i] == 0:
            x = seismic_trace(rng, N)
        elif kinds[i] == 1:
            x = sinusoid_trace(rng, N)
        else:
            x = chirp_trace(rng, N)
        values[offsets[i]:offsets[i + 1]] = x
    return values, offsets, kinds


def pad_csr(values: np.ndarray, offsets: np.ndarray, N: int | None = None) -> np.ndarray:
    """Zero-pad a CSR batch to a dense [batch, max N] array (the reference's
    only way to take mixed lengths; padding changes the decomposition)."""
    lens = np.diff(offsets)
    N = int(N or lens.max())
    out = np.zeros((lens.shape[0], N))
    for i in range(lens.shape[0]):
        out[i, :lens[i]] = values[offsets[i]:offsets[i + 1]]
    return out
