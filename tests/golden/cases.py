"""Seeded parity cases shared by the golden-fixture generator and the tests.

Each group is one launch of the reference kernel (one N, one T, one config):
edge cases the reference's own comments record bugs for (exact zeros,
plateaus, a leading zero, tiny N, the all-zero warm-up signal, the extrema
cap, the iteration cap, non-uniform T) plus samples of the benchmark
workloads.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "emd-cuda_b200"))

from cuda_emd import workloads as W  # noqa: E402

DEFAULT_CFG = dict(max_extrema=1024, nbsym=2, max_iteration=1000, max_imfs=16, threads_per_block=128)
SMALL_CFG = dict(DEFAULT_CFG, max_extrema=128, max_iteration=6)


def _edge512() -> np.ndarray:
    N = 512
    t = np.arange(N, dtype=np.float64)
    rng = np.random.default_rng(11)
    rows = []
    rows.append(np.sin(2 * np.pi * 0.05 * t))                          # pure tone
    rows.append(0.01 * t + 0.3)                                         # linear trend
    rows.append(np.sin(2 * np.pi * 0.02 * t) + 0.5 * np.sin(2 * np.pi * 0.2 * t))  # two tones
    rows.append(np.round(4.0 * np.sin(2 * np.pi * 0.013 * t)) / 4.0)    # plateaus + zeros
    x = np.sin(2 * np.pi * 0.031 * t) + 0.3 * np.sin(2 * np.pi * 0.17 * t)
    x[0] = 0.0                                                          # leading exact zero only
    rows.append(x)
    x = np.sin(2 * np.pi * 0.021 * t) + 0.05 * rng.normal(size=N)
    x[[100, 250, 251, 400]] = 0.0                                       # interior exact zeros
    rows.append(x)
    rows.append(rng.normal(size=N))                                     # white noise
    x = np.sin(2 * np.pi * 0.04 * t) + 0.1 * rng.normal(size=N)
    x[300:306] = x[300]                                                 # interior plateau
    rows.append(x)
    return np.stack(rows)


def _tiny(N: int) -> np.ndarray:
    if N == 6:
        return np.array([[0.0, 1.0, -1.0, 1.0, -1.0, 0.5],
                         [1.0, 2.0, 1.0, 2.0, 1.0, 2.0],
                         [0.3, -0.2, 0.9, -0.4, 0.1, -0.7]])
    if N == 3:
        return np.array([[0.0, 1.0, 0.0], [1.0, -1.0, 2.0]])
    return np.array([[0.7]])


def groups() -> list[dict]:
    """Every parity group: name, signals [B,N], T [N] (normalised as emd.py does),
    config dict, and the reference build variants to run."""
    out = []

    def add(name, X, T=None, cfg=DEFAULT_CFG):
        X = np.atleast_2d(np.asarray(X, dtype=np.float64))
        N = X.shape[1]
        if T is None:
            Tn = np.arange(N, dtype=np.float64)
        else:
            d = np.diff(T)
            Tn = (T - T[0]) / np.min(d)
        small = cfg is SMALL_CFG
        out.append(dict(name=name, signals=X, T=Tn, cfg=cfg,
                        libs=("libemd_ref_small.so", "libemd_ref_small_nofma.so") if small
                        else ("libemd_ref.so", "libemd_ref_nofma.so")))

    add("warmup64", np.zeros((1, 64)))
    add("tiny1", _tiny(1))
    add("tiny3", _tiny(3))
    add("tiny6", _tiny(6))
    add("edge512", _edge512())
    add("cfg0", W.sinusoid_batch(16, 1024, seed=0))
    add("cfg1", W.seismic_batch(6, 2048, seed=1))
    rng = np.random.default_rng(7)
    add("chirp2048", np.stack([W.chirp_trace(rng, 2048) for _ in range(2)]))
    add("chirp6000", W.chirp_trace(np.random.default_rng(8), 6000)[None, :])
    rng = np.random.default_rng(9)
    Tj = np.cumsum(rng.uniform(0.5, 1.5, size=512))
    add("nonuniformT", W.sinusoid_batch(4, 512, seed=3), T=Tj)
    rng = np.random.default_rng(10)
    Xs = np.concatenate([rng.normal(size=(4, 512)), W.sinusoid_batch(4, 512, seed=4)])
    add("small_cfg", Xs, cfg=SMALL_CFG)
    return out


ENVELOPE_GROUP = "edge512"
