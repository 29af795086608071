"""Generate ``tests/golden/ref_golden.npz`` from the reference's own kernel.

Runs on a B200 box (needs CUDA and ``oracle/_ref/*.so`` from
``oracle/build_ref.py``).  For every group in ``cases.groups()`` it launches the
reference ``emd_batch_kernel`` (stock build and ``-fmad=false`` build) and
stores the inputs, the discrete outputs (n_imfs, overflow, debug arrays), a
SHA-256 of each signal's full [MAX_IMFS, N] IMF block, and -- for a few
signals -- the stock build's IMF rows.  It also stores the envelope-only
kernel's outputs for one group.  Finally it prints how the NumPy oracle
compares, so a run log shows the pinning result directly.

``--real float`` does the same with the reference source built with REAL_T =
float (``libemd_ref*_f32*.so``): inputs rounded to float32 (T normalised in
float64 first, as the product path does), IMF blocks hashed as float32, into
``tests/golden/ref_golden_f32.npz``.

Usage: python tests/golden/make_golden.py [--real double|float] [--out PATH]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, HERE)

import cases  # noqa: E402
from refkernel import RefKernel, f32_name  # noqa: E402

# signals whose stock-build IMF rows are stored in full (group -> indices)
STORE_ROWS = {"edge512": None, "cfg0": [0, 1], "cfg1": [0], "tiny6": None, "nonuniformT": [0]}


def sha(block: np.ndarray) -> bytes:
    """SHA-256 of an IMF block in its own precision (little-endian f8 or f4)."""
    code = "<f4" if block.dtype == np.float32 else "<f8"
    return hashlib.sha256(np.ascontiguousarray(block, dtype=code).tobytes()).hexdigest().encode()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--real", choices=("double", "float"), default="double")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    f32 = a.real == "float"
    if a.out is None:
        a.out = os.path.join(ROOT, "tests", "golden",
                             "ref_golden_f32.npz" if f32 else "ref_golden.npz")
    rdt = np.float32 if f32 else np.float64
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    libs = {}
    store = {}
    for g in cases.groups():
        name = g["name"]
        X, T = g["signals"].astype(rdt), g["T"].astype(rdt)
        store[f"{name}__signals"] = X
        store[f"{name}__T"] = T
        c = g["cfg"]
        store[f"{name}__cfg"] = np.array([c["max_extrema"], c["nbsym"], c["max_iteration"],
                                          c["max_imfs"], c["threads_per_block"]], dtype=np.int64)
        for lib, tag in zip(g["libs"], ("stock", "nofma")):
            lib = f32_name(lib) if f32 else lib
            k = libs.setdefault(lib, RefKernel(lib))
            t0 = time.time()
            imfs, n_imfs, ovf, dn, de, dz = k.run(X, T)
            dt = time.time() - t0
            store[f"{name}__{tag}__n_imfs"] = n_imfs
            store[f"{name}__{tag}__overflow"] = ovf
            store[f"{name}__{tag}__dbg_n"] = dn
            store[f"{name}__{tag}__dbg_ext"] = de
            store[f"{name}__{tag}__dbg_nzm"] = dz
            store[f"{name}__{tag}__sha"] = np.array([sha(imfs[b]) for b in range(X.shape[0])],
                                                    dtype="S64")
            if tag == "stock" and name in STORE_ROWS:
                sel = STORE_ROWS[name] or list(range(X.shape[0]))
                rows = [imfs[b, :max(int(n_imfs[b]), 1)] for b in sel]
                store[f"{name}__stock__sel"] = np.array(sel, dtype=np.int64)
                store[f"{name}__stock__rows"] = np.array([r.shape[0] for r in rows], dtype=np.int64)
                store[f"{name}__stock__imfs"] = np.concatenate(rows, axis=0)
            print(f"{name:12s} {tag:5s} B={X.shape[0]:3d} N={X.shape[1]:5d} n_imfs={n_imfs.tolist()} "
                  f"ovf={int(ovf.sum())} ({dt*1e3:.0f} ms)", flush=True)
        if name == cases.ENVELOPE_GROUP:
            env = libs[f32_name(g["libs"][0]) if f32 else g["libs"][0]].envelope(X, T)
            for key, v in zip(("max_env", "min_env", "n_extrema", "degenerate", "max_kpos",
                               "max_kval", "min_kpos", "min_kval", "n_mirrored"), env):
                store[f"{name}__env__{key}"] = v
    np.savez_compressed(a.out, **store)
    print("wrote", a.out, os.path.getsize(a.out), "bytes")

    # Pinning summary against the NumPy oracle.
    from oracle import emd_oracle as O
    for g in cases.groups():
        name = g["name"]
        cfg = O.OracleConfig(**g["cfg"], real_t=a.real)
        X, T = g["signals"].astype(rdt), g["T"].astype(rdt)
        exact = disc = 0
        for b in range(X.shape[0]):
            r = O.emd_signal(X[b], T, cfg)
            if sha(r.imfs) == store[f"{name}__nofma__sha"][b]:
                exact += 1
            ok = (r.n_imfs == store[f"{name}__stock__n_imfs"][b]
                  and r.overflow == store[f"{name}__stock__overflow"][b]
                  and np.array_equal(r.debug_n, store[f"{name}__stock__dbg_n"][b]))
            disc += int(ok)
        print(f"oracle vs ref  {name:12s} bit-exact(nofma) {exact}/{X.shape[0]}  "
              f"discrete==stock {disc}/{X.shape[0]}", flush=True)


if __name__ == "__main__":
    main()
