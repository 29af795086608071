"""Generate tests/golden/long_golden.npz: oracle outputs for traces longer than
a CTA's shared memory holds (the wide instance keeps their proto-IMF in the
global slab), too slow to recompute inside a GPU test.

Each case is regenerated from its seed by ``long_cases()`` (the test imports
it); the fixture stores the discrete outputs and the SHA-256 of the oracle's
full [max_imfs, N] IMF block, which the B200 kernel must equal bit for bit.

Run: python tests/golden/make_long.py   (a few minutes on 8 cores)
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "emd-cuda_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

OUT = os.path.join(HERE, "long_golden.npz")


def long_cases():
    """(name, signal, max_iteration): smooth multi-tone traces of 32,768,
    65,536 and 40,000 samples (a few hundred extrema), and two that exceed
    max_extrema (a seismic-like trace and a chirp), with the iteration cap
    lowered to keep the oracle's run short."""
    from cuda_emd import workloads as W
    out = []
    for k, N in enumerate((32768, 65536, 40000)):
        rng = np.random.default_rng(500 + k)
        t = np.arange(N, dtype=np.float64)
        f = rng.uniform(0.0004, 0.004, size=3)
        a = rng.uniform(0.5, 2.0, size=3)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        x = (a[:, None] * np.sin(2 * np.pi * f[:, None] * t + ph[:, None])).sum(0) + 1e-5 * t
        out.append((f"tones{N}", x, 1000))
    out.append(("seismic36000", W.seismic_trace(np.random.default_rng(510), 36000), 12))
    out.append(("chirp50000", W.chirp_trace(np.random.default_rng(511), 50000), 8))
    return out


def _one(args):
    name, x, mi = args
    from oracle import emd_oracle as O
    cfg = O.OracleConfig(max_iteration=mi)
    r = O.emd_signal(x, np.arange(x.shape[0], dtype=np.float64), cfg)
    sha = hashlib.sha256(np.ascontiguousarray(r.imfs, dtype="<f8").tobytes()).hexdigest().encode()
    return name, r.n_imfs, r.overflow, r.debug_n, r.debug_extno, r.debug_nzm, sha


def main():
    import multiprocessing as mp
    cases = long_cases()
    with mp.get_context("spawn").Pool(min(len(cases), os.cpu_count() or 1)) as pool:
        res = pool.map(_one, cases)
    z = {}
    for name, n, o, dn, de, dz, sha in res:
        z[f"{name}__n_imfs"] = np.int32(n)
        z[f"{name}__overflow"] = np.int32(o)
        z[f"{name}__dbg_n"] = dn
        z[f"{name}__dbg_ext"] = de
        z[f"{name}__dbg_nzm"] = dz
        z[f"{name}__sha"] = np.bytes_(sha)
        print(name, n, o, dn[:8])
    np.savez(OUT, **z)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
