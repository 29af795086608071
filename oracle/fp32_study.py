"""FP32 against FP64: how often the reference algorithm's discrete outcome
changes when it runs with REAL_T = float -- TEST INFRASTRUCTURE ONLY.

Both runs are the oracle (``emd_oracle.emd_signal``), which is pinned bit for
bit to the reference's kernel built with REAL_T = double and with REAL_T =
float (``tests/golden/ref_golden*.npz``); the float run takes the double
input rounded to float32.  Per trace kind it reports the share of traces
whose IMF count, overflow flag and per-IMF sift counts (debug_n) agree, and
for traces with the same IMF count the largest difference of any IMF sample
relative to the trace's range.

Run: python oracle/fp32_study.py [traces per kind]   (a minute on 8 cores)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "emd-cuda_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def kinds(n: int):
    """(name, signals) per trace kind: the cfg0 three-tone mix, cfg1 seismic
    traces, and linear chirps (seeded workload generators)."""
    from cuda_emd import workloads as W
    rng = np.random.default_rng(77)
    return [("cfg0 three-tone 1024", W.sinusoid_batch(n, 1024, seed=70)),
            ("cfg1 seismic 2048", W.seismic_batch(n, 2048, seed=71)),
            ("chirp 2048", np.stack([W.chirp_trace(rng, 2048) for _ in range(max(1, n // 4))]))]


def compare(x: np.ndarray) -> dict:
    from oracle import emd_oracle as O
    T = np.arange(x.shape[0], dtype=np.float64)
    r64 = O.emd_signal(x, T, O.OracleConfig())
    r32 = O.emd_signal(x.astype(np.float32), T.astype(np.float32), O.OracleConfig(real_t="float"))
    same_n = r64.n_imfs == r32.n_imfs
    rng = float(np.ptp(x)) or 1.0
    err = None
    if same_n and r64.n_imfs:
        k = r64.n_imfs
        err = float(np.max(np.abs(r64.imfs[:k] - r32.imfs[:k].astype(np.float64)))) / rng
    return {"n_imfs": same_n, "overflow": r64.overflow == r32.overflow,
            "debug_n": bool(np.array_equal(r64.debug_n, r32.debug_n)), "err": err,
            "ovf32": int(r32.overflow), "ovf64": int(r64.overflow)}


def _chunk(args):
    X, = args
    return [compare(x) for x in X]


def study(n: int = 64, processes: int = 0) -> dict:
    import multiprocessing as mp
    out = {}
    procs = processes or min(8, os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(procs) as pool:
        for name, X in kinds(n):
            res = sum(pool.map(_chunk, [(p,) for p in np.array_split(X, procs) if p.shape[0]]), [])
            errs = [r["err"] for r in res if r["err"] is not None]
            out[name] = {
                "traces": len(res),
                "same_n_imfs": sum(r["n_imfs"] for r in res) / len(res),
                "same_overflow": sum(r["overflow"] for r in res) / len(res),
                "same_debug_n": sum(r["debug_n"] for r in res) / len(res),
                "overflow_f32_only": sum(r["ovf32"] and not r["ovf64"] for r in res),
                "max_rel_err_same_n": max(errs) if errs else None,
                "median_rel_err_same_n": float(np.median(errs)) if errs else None,
            }
    return out


if __name__ == "__main__":
    import json
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 64
    print(json.dumps(study(n), indent=1))
