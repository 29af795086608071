"""Build recipe: compile the reference's own CUDA kernel into ``oracle/_ref/``.

TEST INFRASTRUCTURE ONLY (the checker, never the product).

The reference (SeismicFlow/emd-cuda) ships its kernels as the string
``_CUDA_SOURCE`` inside ``kernels.py`` (kernels.py:69-1167) and compiles them at
run time with CuPy/NVRTC (kernels.py:1296).  CuPy is not installed here, so this
recipe does the same job with nvcc:

1. read ``kernels.py`` from the reference checkout with ``ast`` (no import, so
   CuPy is not needed) and take the ``_CUDA_SOURCE`` literal unchanged;
2. apply the same ``%``-substitution as ``EMDKernelConfig.build``
   (kernels.py:1277-1286) with the default config;
3. append a small host launcher of our own (below) that opts into the
   kernel's dynamic shared memory and launches it with the reference's
   geometry: grid (batch,), block (THREADS,), ``shared_mem_bytes()`` bytes
   (kernels.py:1273-1275, 1365-1371);
4. compile in a temporary directory with ``-std=c++11`` (the reference's NVRTC
   option) for sm_100a, writing only the shared libraries into ``oracle/_ref/``:

   * ``libemd_ref.so``       -- stock build (FMA contraction on, as NVRTC does);
   * ``libemd_ref_nofma.so`` -- the same source with ``-fmad=false``, the
     arithmetic the NumPy oracle restates bit for bit;
   * ``libemd_ref_small[_nofma].so`` -- MAX_EXTREMA=128, MAX_ITERATION=6, so
     that short fixtures reach both overflow paths (extrema cap and
     iteration cap);
   * ``libemd_ref[_small]_f32[_nofma].so`` -- the same source with REAL_T =
     float (the substitution key the reference's build takes from
     ``EMDKernelConfig.real_t_name``, kernels.py:1284; its Python layer fixes
     it to double): the pin of the FP32 path.

The extracted source never lands in the repository.  Run:
``python oracle/build_ref.py --ref <reference checkout>`` (or set
``EMDB_REFERENCE_DIR``).
"""
from __future__ import annotations

import argparse
import ast
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
# the reference checkout: --ref, else this environment variable
DEFAULT_REF = os.environ.get("EMDB_REFERENCE_DIR", "")

DEFAULTS = dict(MAX_EXTREMA=1024, NBSYM=2, MAX_ITERATION=1000, MAX_IMFS=16, THREADS=128,
                REAL_T="double")
SMALL = dict(MAX_EXTREMA=128, MAX_ITERATION=6)
F32 = dict(REAL_T="float")
VARIANTS = (
    ("libemd_ref.so", {}, []),
    ("libemd_ref_nofma.so", {}, ["-fmad=false"]),
    ("libemd_ref_small.so", SMALL, []),
    ("libemd_ref_small_nofma.so", SMALL, ["-fmad=false"]),
    ("libemd_ref_f32.so", F32, []),
    ("libemd_ref_f32_nofma.so", F32, ["-fmad=false"]),
    ("libemd_ref_small_f32.so", dict(SMALL, **F32), []),
    ("libemd_ref_small_f32_nofma.so", dict(SMALL, **F32), ["-fmad=false"]),
)

# Host-side launcher written for this recipe (not part of the reference); its
# buffers are REAL_T, the type the reference source #defines (kernels.py:78).
LAUNCHER = r"""
#include <cuda_runtime.h>
#include <stddef.h>

static size_t ref_smem_bytes() {
    // EMDKernelConfig.shared_mem_bytes(): (MAX_EXTREMA + 2*NBSYM) * 56 + 256
    return (size_t)(MAX_EXTREMA + 2 * NBSYM) * 56 + 256;
}

extern "C" int ref_config(int* out5) {
    out5[0] = MAX_EXTREMA; out5[1] = NBSYM; out5[2] = MAX_ITERATION;
    out5[3] = MAX_IMFS; out5[4] = THREADS;
    return 0;
}

extern "C" int ref_real_bytes(void) { return (int)sizeof(REAL_T); }

extern "C" int ref_emd_launch(const REAL_T* signals, const REAL_T* T, int batch, int N,
                              REAL_T* imfs, int* n_imfs, int* overflow,
                              REAL_T* pools6, int* dbg_n, int* dbg_ext, int* dbg_nzm,
                              cudaStream_t stream) {
    size_t smem = ref_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(emd_batch_kernel,
                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    if (batch <= 0) return 0;
    size_t pn = (size_t)batch * (size_t)N;
    emd_batch_kernel<<<batch, THREADS, smem, stream>>>(
        signals, T, N, imfs, n_imfs, overflow,
        pools6, pools6 + pn, pools6 + 2 * pn, pools6 + 3 * pn, pools6 + 4 * pn, pools6 + 5 * pn,
        dbg_n, dbg_ext, dbg_nzm);
    return (int)cudaGetLastError();
}

extern "C" int ref_envelope_launch(const REAL_T* signals, const REAL_T* T, int batch, int N,
                                   REAL_T* max_env, REAL_T* min_env, int* n_extrema,
                                   int* degenerate, REAL_T* max_kpos, REAL_T* max_kval,
                                   REAL_T* min_kpos, REAL_T* min_kval, int* n_mirrored,
                                   cudaStream_t stream) {
    size_t smem = ref_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(envelope_batch_kernel,
                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    if (batch <= 0) return 0;
    envelope_batch_kernel<<<batch, THREADS, smem, stream>>>(
        signals, T, N, max_env, min_env, n_extrema, degenerate,
        max_kpos, max_kval, min_kpos, min_kval, n_mirrored);
    return (int)cudaGetLastError();
}
"""


def extract_source(ref_dir: str) -> str:
    path = os.path.join(ref_dir, "kernels.py")
    with open(path, "r", encoding="utf-8") as f:
        tree = ast.parse(f.read(), filename=path)
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(
                isinstance(t, ast.Name) and t.id == "_CUDA_SOURCE" for t in node.targets):
            return ast.literal_eval(node.value)
    raise RuntimeError(f"_CUDA_SOURCE not found in {path}")


def build(ref_dir: str = DEFAULT_REF, out_dir: str = OUT_DIR, quiet: bool = False) -> list[str]:
    if not os.path.isfile(os.path.join(ref_dir, "kernels.py")):
        raise FileNotFoundError(f"reference checkout not found at {ref_dir}")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    raw = extract_source(ref_dir)
    os.makedirs(out_dir, exist_ok=True)
    built = []
    with tempfile.TemporaryDirectory() as td:
        for name, over, extra in VARIANTS:
            cu = os.path.join(td, name + ".cu")
            with open(cu, "w") as f:
                f.write(raw % dict(DEFAULTS, **over))
                f.write(LAUNCHER)
            out = os.path.join(out_dir, name)
            cmd = [nvcc, "-std=c++11", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                   "-shared", "-Xcompiler", "-fPIC", *extra, "-o", out, cu, "-lcudart"]
            if not quiet:
                print(" ".join(cmd[:-2]), "...", file=sys.stderr)
            subprocess.run(cmd, check=True, cwd=td,
                           stdout=subprocess.DEVNULL if quiet else None,
                           stderr=subprocess.PIPE if quiet else None)
            built.append(out)
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("--out", default=OUT_DIR)
    a = ap.parse_args()
    for p in build(a.ref, a.out):
        print(p)
