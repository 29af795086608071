"""Benchmark: batched FP64 EMD on B200, one JSON line on rank 0.

Default workload (N=1 GPU): 16,384 seismic-like float64 traces of 2048
samples (Ricker wavelet * Laplace reflectivity + 5-100 Hz band-limited noise
at 10 dB SNR, dt = 2 ms), PyEMD-default EMD, MAX_IMFS 16, max_iteration 1000.
One step = one decomposition of the whole batch.

  value     signals/s with inputs resident in HBM (device-timed launches)
  e2e       signals/s through GPUBatchEMD with pinned host buffers: each step
            copies the traces in, decomposes, checks overflow, copies IMFs,
            n_imfs and overflow back
  roofline  the sift kernel's algorithmic FP64 rate (from the logged sift and
            extrema counts) against a cuBLAS DGEMM measured in this run, plus
            its HBM rate against MEASURED_PEAKS.json
  cpu_baseline  the CPU oracle on a bounded sample, all host cores

``--impl reference`` times the reference's algorithm on the host cores (the
CPU oracle restatement: the reference itself is CUDA-only and its CuPy
dependency is absent) and prints the same line with impl=reference.

Multi-GPU (torchrun, --gpus N): traces are independent, so each rank
decomposes its own batch (weak scaling, no data-path collective); timing is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "emd-cuda_b200"))
sys.path.insert(0, ROOT)

METRIC = "EMD signals/s (FP64)"
WORKLOADS = {
    "seismic16k": dict(n=16384, N=2048, desc="16384 seismic traces x 2048 samples, dt 2 ms"),
    "sinusoid256": dict(n=256, N=1024, desc="256 three-tone traces x 1024 samples"),
    "seismic1k": dict(n=1024, N=2048, desc="1024 seismic traces x 2048 samples (profiling size)"),
}


def make_workload(name: str, rank: int = 0):
    from cuda_emd import workloads as W
    w = WORKLOADS[name]
    if name.startswith("seismic"):
        X = W.seismic_batch(w["n"], w["N"], seed=1 + 1000 * rank)
    else:
        X = W.sinusoid_batch(w["n"], w["N"], seed=0 + 1000 * rank)
    return np.ascontiguousarray(X)


# ---------------------------------------------------------------------------
# CPU side: oracle on host cores (spawn pool, created before any CUDA use)
# ---------------------------------------------------------------------------

def _oracle_chunk(args):
    X, = args
    sys.path.insert(0, ROOT)
    from oracle import emd_oracle as O
    T = np.arange(X.shape[1], dtype=np.float64)
    t0 = time.perf_counter()
    for x in X:
        O.emd_signal(x, T)
    return X.shape[0], time.perf_counter() - t0


def cpu_oracle_rate(X: np.ndarray, pool, cores: int, sample: int):
    """signals/s of the oracle over `sample` traces split across `cores` processes."""
    sub = X[:sample]
    parts = [p for p in np.array_split(sub, cores) if p.shape[0]]
    t0 = time.perf_counter()
    res = pool.map(_oracle_chunk, [(p,) for p in parts])
    wall = time.perf_counter() - t0
    n = sum(r[0] for r in res)
    return n / wall, n, wall


# ---------------------------------------------------------------------------
# GPU helpers
# ---------------------------------------------------------------------------

class ClockSampler:
    def __init__(self, index: int, path: str):
        self.path = path
        self.proc = None
        try:
            self.f = open(path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dgemm_tflops(dev) -> float:
    """FP64 peak measured here: cuBLAS DGEMM 8192^3, best of 5."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def algorithmic_flops(N: int, n_imfs, dbg_n, dbg_ext) -> float:
    """65 flop/sample per sift pass + 20 flop/knot per envelope (knots ~ the
    logged extrema count + 2*nbsym mirrored) + 4 flop/sample per IMF."""
    dn = np.where(dbg_n > 0, dbg_n, 0).astype(np.float64)
    de = np.where(dbg_ext > 0, dbg_ext, 0).astype(np.float64)
    per_pass = 65.0 * N + 20.0 * (de + 8.0)
    return float((dn * per_pass).sum() + 4.0 * N * np.asarray(n_imfs, dtype=np.float64).sum())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="seismic16k", choices=list(WORKLOADS))
    ap.add_argument("--cpu-sample", type=int, default=0, help="traces for the CPU leg (0 = auto)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--arena", type=int, default=0, help="shared-memory arena per CTA (0 = auto)")
    a = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    # CPU pool first (spawn), before any CUDA context exists.
    pool = None
    want_cpu = (a.impl == "reference" or not a.no_cpu) and rank == 0
    if want_cpu:
        import multiprocessing as mp
        pool = mp.get_context("spawn").Pool(cores)

    if a.impl == "reference":
        run_reference(a, rank, world, pool, cores)
        return

    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    from cuda_emd import GPUBatchEMD, EMDKernelConfig

    X = make_workload(a.workload, rank)
    B, N = X.shape
    sig = torch.from_numpy(X).to(dev)
    cfg = EMDKernelConfig.for_device(local)
    emd = GPUBatchEMD(cfg)
    emd.warmup()
    launcher = emd._get_launcher()
    if a.arena:
        launcher._plan.set_arena(a.arena)
    arena_used, ctas_per_sm, grid_max = launcher._plan.query(N)

    # ---- device-resident throughput ----
    for _ in range(a.warmup):
        out = launcher.run(sig, None)
    torch.cuda.synchronize(dev)
    launcher.check_status()
    n_imfs, dbg_n, dbg_ext = out[1].cpu().numpy(), out[3].cpu().numpy(), out[4].cpu().numpy()
    ovf = int(out[2].sum().item())
    del out
    flops_per_step = algorithmic_flops(N, n_imfs, dbg_n, dbg_ext)
    hbm_bytes_per_step = 8.0 * B * N + 8.0 * B * cfg.max_imfs * N

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local, os.path.join(ROOT, "gpurun_out", f"clocks_r{rank}.csv")) \
        if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else None
    st = torch.cuda.current_stream(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(a.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(st)
    for k in range(a.steps):
        ev[k][0].record(st)
        out = launcher.run(sig, None)
        ev[k][1].record(st)
        del out
    t_end.record(st)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    elapsed = t_start.elapsed_time(t_end) * 1e-3
    per_launch = [e0.elapsed_time(e1) * 1e-3 for e0, e1 in ev]
    if world > 1:
        t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    total = B * a.steps * world
    value = total / elapsed
    ms_per_step = elapsed / a.steps * 1e3
    launch_s = statistics.mean(per_launch)

    # ---- end to end through the public API with pinned host buffers ----
    e2e = None
    if not a.no_e2e:
        host_in = torch.from_numpy(X).pin_memory()
        host_imfs = torch.empty((B, cfg.max_imfs, N), dtype=torch.float64).pin_memory()
        host_n = torch.empty(B, dtype=torch.int32).pin_memory()
        host_o = torch.empty(B, dtype=torch.int32).pin_memory()

        def e2e_step():
            d = host_in.to(dev, non_blocking=True)
            imfs, nim, of = emd(d)
            host_imfs.copy_(imfs, non_blocking=True)
            host_n.copy_(nim, non_blocking=True)
            host_o.copy_(of, non_blocking=True)
            del imfs
        for _ in range(max(1, min(a.warmup, 2))):
            e2e_step()
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(a.steps):
            e2e_step()
        e1.record(st)
        torch.cuda.synchronize(dev)
        te = e0.elapsed_time(e1) * 1e-3
        if world > 1:
            t = torch.tensor([te], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        e2e = {"value": B * a.steps * world / te, "unit": "signals/s",
               "h2d_bytes_per_step": int(8 * B * N),
               "d2h_bytes_per_step": int(8 * B * cfg.max_imfs * N + 8 * B)}
        del host_imfs

    # ---- roofline ----
    roofline = None
    if rank == 0:
        peaks = {}
        pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.isfile(pk):
            peaks = json.load(open(pk))
        fp64 = dgemm_tflops(dev)
        achieved = flops_per_step / launch_s / 1e12
        hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
        hbm_ach = hbm_bytes_per_step / launch_s / 1e9
        roofline = {"bound": "fp64", "achieved": round(achieved, 3), "peak": round(fp64, 3),
                    "unit": "TFLOP/s", "frac": round(achieved / fp64, 4), "traffic": None,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                    "kernel": "emd_sift_kernel",
                    "algorithmic_flop_per_launch": flops_per_step,
                    "launch_ms": round(launch_s * 1e3, 3),
                    "hbm": {"achieved": round(hbm_ach, 1), "peak": hbm_peak, "unit": "GB/s",
                            "frac": round(hbm_ach / hbm_peak, 5),
                            "bytes_per_launch": hbm_bytes_per_step,
                            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback"}}

    # ---- CPU baseline (rank 0) ----
    cpu = None
    if pool is not None:
        sample = a.cpu_sample or max(cores * 128, 64)
        rate, n, wall = cpu_oracle_rate(X, pool, cores, min(sample, B))
        cpu = {"value": round(rate, 2), "unit": "signals/s", "cores": cores, "kind": "port",
               "sample": f"first {n} traces of the workload, NumPy oracle, {cores} processes, "
                         f"{wall:.1f} s wall"}
        pool.close()

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "signals/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_per_step, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, see cuda_emd/workloads.py)",
            "config": {"workload": a.workload, "desc": WORKLOADS[a.workload]["desc"],
                       "batch_per_gpu": B, "N": N, "max_imfs": cfg.max_imfs,
                       "max_extrema": cfg.max_extrema, "max_iteration": cfg.max_iteration,
                       "queue": "FIFO persistent", "l2": "inputs+outputs larger than L2",
                       "arena_bytes": arena_used, "ctas_per_sm": ctas_per_sm,
                       "overflow_traces": ovf, "parallelism": f"replicas x{world}"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
            "gpu_launches": a.steps,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libemd_ref.so")


def run_reference(a, rank, world, pool, cores):
    """The reference's own emd_batch_kernel (kernels.py:834-1080, built from
    kernels.py into oracle/_ref by oracle/build_ref.py: CuPy is absent, so
    nvcc stands in for its NVRTC compile) on the same GPU and workload, with
    the reference's launch geometry and per-call pool allocation + zero-fill
    (kernels.py:1343-1372).  The CPU oracle on the host cores is reported as
    its cpu_baseline.  Without the built library or a GPU, the CPU oracle is
    the measured arm."""
    if rank != 0:
        return
    X = make_workload(a.workload, 0)
    B, N = X.shape
    sample = min(a.cpu_sample or max(cores * 16, 64), B)
    r, n, wall = cpu_oracle_rate(X, pool, cores, sample)
    pool.close()
    cpu = {"value": round(r, 2), "unit": "signals/s", "cores": cores, "kind": "port",
           "sample": f"first {n} traces of the workload, NumPy oracle, {cores} processes, "
                     f"{wall:.1f} s wall"}
    import torch
    line = {"impl": "reference", "metric": METRIC, "unit": "signals/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "cpu_baseline": cpu}
    if os.path.isfile(REF_LIB) and torch.cuda.is_available():
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from refkernel import RefKernel
        k = RefKernel("libemd_ref.so")
        dev = torch.device("cuda", 0)
        sig = torch.from_numpy(X).to(dev)
        Tn = torch.arange(N, dtype=torch.float64, device=dev)
        k.run_device(torch.zeros((1, 64), dtype=torch.float64, device=dev), Tn[:64])  # warmup()
        for _ in range(a.warmup):
            out = k.run_device(sig, Tn)
            del out
        torch.cuda.synchronize()
        st = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(a.steps):
            out = k.run_device(sig, Tn)
            del out
        e1.record(st)
        torch.cuda.synchronize()
        el = e0.elapsed_time(e1) * 1e-3
        value = B * a.steps / el
        host_in = torch.from_numpy(X).pin_memory()
        host_imfs = torch.empty((B, k.max_imfs, N), dtype=torch.float64).pin_memory()
        h_n = torch.empty(B, dtype=torch.int32).pin_memory()
        h_o = torch.empty(B, dtype=torch.int32).pin_memory()
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(a.steps):
            d = host_in.to(dev, non_blocking=True)
            imfs, nim, ovf, dn, de, dz = k.run_device(d, Tn)
            bool(ovf.any())                      # emd.py:95 read-back
            host_imfs.copy_(imfs, non_blocking=True)
            h_n.copy_(nim, non_blocking=True)
            h_o.copy_(ovf, non_blocking=True)
            del imfs
        e1.record(st)
        torch.cuda.synchronize()
        te = e0.elapsed_time(e1) * 1e-3
        line.update({
            "value": round(value, 2), "ms_per_step": round(el / a.steps * 1e3, 3),
            "config": {"workload": a.workload, "desc": WORKLOADS[a.workload]["desc"],
                       "batch_per_gpu": B, "N": N,
                       "reference_kernel": "emd_batch_kernel from kernels.py, nvcc -std=c++11 "
                                           "sm_100a (oracle/_ref/libemd_ref.so); grid (batch,), "
                                           "block 128, 57824 B dynamic smem",
                       "parallelism": "one GPU"},
            "e2e": {"value": round(B * a.steps / te, 2), "unit": "signals/s",
                    "h2d_bytes_per_step": int(8 * B * N),
                    "d2h_bytes_per_step": int(8 * B * k.max_imfs * N + 8 * B)},
        })
    else:
        line.update({
            "value": cpu["value"], "ms_per_step": round(B / max(r, 1e-9) * 1e3, 3),
            "config": {"workload": a.workload, "desc": WORKLOADS[a.workload]["desc"],
                       "batch_per_gpu": B, "N": N, "parallelism": "host cores",
                       "note": "reference kernel library not built here; CPU oracle measured"},
            "e2e": {"value": cpu["value"], "unit": "signals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        })
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
