"""Benchmark: batched FP64 EMD on B200, one JSON line on rank 0.

Default workload (N=1 GPU): the ragged batch -- 65,536 float64 traces with
lengths log-uniform in [256, 8192] (60 % seismic-like: Ricker wavelet *
Laplace reflectivity + 5-100 Hz band-limited noise at 10 dB SNR, dt 2 ms;
38 % three tones + trend + noise; 2 % linear chirps), CSR layout, PyEMD-
default EMD, MAX_IMFS 16, max_iteration 1000.  One step = one decomposition of
the whole batch: traces grouped into length tiers, one persistent sift launch
per tier, the sequence graph-captured.

  value     signals/s of the learned-scheduled step (features + BF16 MLP
            inference + longest-predicted-first queue per tier + the tier
            launches), inputs resident in HBM, device-timed
  plain     the same with FIFO queues; learned.speedup_vs_plain, and the
            ceiling of any ordering (queue ordered by the true logged cost)
  e2e       signals/s through RaggedRunner.run_host on pinned host CSR
            buffers: H2D, the learned step, rows with data gathered and
            copied back with the counts, every step
  roofline  the sift launches' algorithmic FP64 rate (from the logged sift and
            extrema counts) against a cuBLAS DGEMM measured in this run, plus
            the HBM rate against MEASURED_PEAKS.json
  cpu_baseline  the CPU oracle on a bounded random sample, all host cores
  serve     continuous-batching server under Poisson load: saturation and
            p50/p99/p99.9 latency at a few offered loads

Other workloads: --workload seismic16k (16,384 x 2048 seismic traces, the
equal-length head-to-head with the reference kernel), seismic8k, serve, ...

``--impl reference`` times the reference's algorithm on the host cores (the
CPU oracle restatement: the reference itself is CUDA-only and its CuPy
dependency is absent) and prints the same line with impl=reference; beside
it, the reference's own kernel on the same GPU (padded to max N).

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
# the headline metric: the ragged batch, learned order vs plain, with serving latency beside it
METRIC_HEADLINE = ("EMD signals/s (FP64) learned-scheduled vs plain on one B200; "
                   "p50/p99 serve latency")
# DRAM bytes per trace of emd_sift_kernel, keyed by (N, max_imfs): one ncu
# capture of the seismic1k launch (1024 traces x 2048 samples) read
# dram__bytes_read.sum 24.33 MB + dram__bytes_write.sum 240.00 MB.  Inputs and
# outputs are per trace and the spill slab stays in L2, so a launch's traffic
# is this figure times its traces.
NCU_DRAM_BYTES_PER_TRACE = {(2048, 16): 264329984 / 1024}
# DRAM bytes per sample of the ragged mix's tier launches: ncu
# dram__bytes_read.sum + dram__bytes_write.sum over the four tier launches of
# a learned step on a 4,096-trace sample of the batch (9.30 M samples), mean
# of 11 steps 1,120.8 MB: inputs and outputs are per sample, spills stay in L2
NCU_DRAM_BYTES_PER_SAMPLE_RAGGED = 1120837888.0 / 9298408
NCU_RAGGED_SOURCE = ("ncu dram__bytes_read+write of the tier launches of a 4096-trace "
                     "sample of the batch (120.5 B/sample) x samples per step")


def hbm_peak_gbs():
    """(GB/s, source): MEASURED_PEAKS.json's hbm_gbs, else the pool's fallback."""
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.isfile(pk):
        try:
            v = json.load(open(pk)).get("hbm_gbs")
            if v:
                return float(v), "MEASURED_PEAKS.json hbm_gbs"
        except Exception:
            pass
    return 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"
WORKLOADS = {
    "seismic16k": dict(n=16384, N=2048, desc="16384 seismic traces x 2048 samples, dt 2 ms"),
    "sinusoid256": dict(n=256, N=1024, desc="256 three-tone traces x 1024 samples"),
    "seismic1k": dict(n=1024, N=2048, desc="1024 seismic traces x 2048 samples (profiling size)"),
    "seismic8k": dict(n=2048, N=8192, desc="2048 seismic traces x 8192 samples (every trace overflows "
                                           "max_extrema)"),
    "seismic8k-prof": dict(n=296, N=8192, desc="296 seismic traces x 8192 samples (two per SM: the "
                                               "profiling size of seismic8k)"),
    "serve": dict(lo=512, hi=16384, max_traces=64,
                  desc="Poisson requests of 1-64 traces, N log-uniform [512, 16384], ragged mix; "
                       "offered load 10-110% of measured saturation"),
    "ragged64k": dict(n=65536, lo=256, hi=8192,
                      desc="65536 mixed traces, N log-uniform [256, 8192] (60% seismic, 38% "
                           "three-tone, 2% chirp), CSR; plain FIFO vs learned longest-first"),
}


def make_workload(name: str, rank: int = 0):
    from cuda_emd import workloads as W
    w = WORKLOADS[name]
    from cuda_emd.replicas import workload_seed
    if name.startswith("seismic"):
        X = W.seismic_batch(w["n"], w["N"], seed=workload_seed(1, rank))
    else:
        X = W.sinusoid_batch(w["n"], w["N"], seed=workload_seed(0, rank))
    return np.ascontiguousarray(X)


# ---------------------------------------------------------------------------
# CPU side: oracle on host cores (spawn pool, created before any CUDA use)
# ---------------------------------------------------------------------------

def _oracle_chunk(args):
    X, real_t = args
    sys.path.insert(0, ROOT)
    from oracle import emd_oracle as O
    cfg = O.OracleConfig(real_t=real_t)
    T = np.arange(X.shape[1], dtype=cfg.rtype)
    t0 = time.perf_counter()
    for x in X:
        O.emd_signal(x, T, cfg)
    return X.shape[0], time.perf_counter() - t0


def cpu_oracle_rate(X: np.ndarray, pool, cores: int, sample: int, real_t: str = "double"):
    """signals/s of the oracle over `sample` traces split across `cores` processes."""
    sub = X[:sample]
    parts = [p for p in np.array_split(sub, cores) if p.shape[0]]
    t0 = time.perf_counter()
    res = pool.map(_oracle_chunk, [(p, real_t) for p in parts])
    wall = time.perf_counter() - t0
    n = sum(r[0] for r in res)
    return n / wall, n, wall


# ---------------------------------------------------------------------------
# GPU helpers
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clock and throttle-reason samples every 200 ms while the
    timed region runs; kept in `path` when one is given, else a temp file."""

    def __init__(self, index: int, path: str | None = None):
        import tempfile
        self.temp = path is None
        if path is None:
            fd, path = tempfile.mkstemp(prefix="emdb_clocks_", suffix=".csv")
            os.close(fd)
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

    def _discard(self):
        f = getattr(self, "f", None)
        if f is not None and not f.closed:
            f.close()
        if self.temp and os.path.exists(self.path):
            os.unlink(self.path)

    def stop(self):
        if self.proc is None:
            self._discard()
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
        if self.temp:
            os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dgemm_tflops(dev, dtype=None) -> float:
    """FP64 peak measured here: cuBLAS DGEMM 8192^3, best of 5 (dtype float32:
    SGEMM with TF32 off, the FP32 pipe's peak)."""
    import torch
    dtype = dtype or torch.float64
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, dtype=dtype, device=dev)
    b = torch.randn(n, n, dtype=dtype, device=dev)
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
    ap.add_argument("--workload", default="ragged64k", choices=list(WORKLOADS))
    ap.add_argument("--cpu-sample", type=int, default=0, help="traces for the CPU leg (0 = auto)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--arena", type=int, default=0, help="shared-memory arena per CTA (0 = auto)")
    ap.add_argument("--clocks-csv", default=None,
                    help="keep the raw clock samples here ({rank} = rank); default: a temp file")
    ap.add_argument("--variant", type=int, default=0, help="kernel register variant: min CTAs/SM")
    ap.add_argument("--real", default="double", choices=["double", "float"],
                    help="dense workloads: the type the kernels compute in (REAL_T)")
    ap.add_argument("--order", default="fifo", choices=["fifo", "learned"],
                    help="dense workloads: queue order of the timed steps (learned: the cost "
                         "model, trained here on a disjoint seeded batch, orders each step's "
                         "queue longest-predicted-first; the FIFO rate is reported beside it)")
    ap.add_argument("--order-train", type=int, default=4,
                    help="--order learned: seeded batches of the workload to train on")
    ap.add_argument("--train-traces", type=int, default=200000, help="ragged64k: MLP training set")
    ap.add_argument("--eval-traces", type=int, default=0, help="ragged64k: batch size (0 = 65536)")
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--no-split", action="store_true",
                    help="ragged64k: the model only orders queues, tiers stay by length")
    ap.add_argument("--heavy-passes", type=float, default=600.0,
                    help="ragged64k: predicted sift passes from which a trace goes wide")
    ap.add_argument("--heavy-boost", type=float, default=1.0,
                    help="ragged64k: wide launches' SM share = predicted work share x this")
    ap.add_argument("--requests", type=int, default=160, help="serve: requests per load level")
    ap.add_argument("--loads", default="0.1,0.3,0.5,0.7,0.9,1.1", help="serve: offered loads")
    ap.add_argument("--slots", type=int, default=4,
                    help="serving: launch slots of the long-request lane")
    ap.add_argument("--short-slots", type=int, default=2,
                    help="serving: launch slots of the short-request lane (0 = one lane)")
    ap.add_argument("--serve-requests", type=int, default=160,
                    help="ragged64k: requests per load level of the serving sweep (0 = skip)")
    ap.add_argument("--serve-loads", default="0.3,0.7,1.1",
                    help="ragged64k: offered loads of the serving sweep")
    ap.add_argument("--ref-sample", type=int, default=4096,
                    help="reference arm, ragged64k: traces per padded GPU measurement")
    a = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    # CPU pool first (spawn), before any CUDA context exists.
    pool = None
    want_cpu = (a.impl == "reference" or not a.no_cpu) and rank == 0
    # the ragged and serving workloads are generated on the host: every rank
    # needs a pool for that, sharing the host's cores
    gen_pool = a.impl == "b200" and a.workload in ("ragged64k", "serve")
    if want_cpu or gen_pool:
        import multiprocessing as mp
        pool = mp.get_context("spawn").Pool(cores if rank == 0 and world == 1
                                            else max(2, cores // max(world, 1)))

    if a.impl == "reference":
        run_reference(a, rank, world, pool, cores)
        return
    if a.workload == "ragged64k":
        run_ragged(a, rank, world, pool, cores)
        return
    if a.workload == "serve":
        run_serve(a, rank, world, pool, cores)
        return

    import torch
    from cuda_emd import replicas as R
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    R.init(world, "nccl", dev)

    from cuda_emd import GPUBatchEMD, EMDKernelConfig

    import dataclasses
    f32 = a.real == "float"
    X = make_workload(a.workload, rank)
    if f32:
        X = X.astype(np.float32)
    B, N = X.shape
    isz = X.dtype.itemsize
    sig = torch.from_numpy(X).to(dev)
    # same config for both types (max_extrema as the FP64 sizing gives it)
    cfg = dataclasses.replace(EMDKernelConfig.for_device(local), real_t=a.real)
    emd = GPUBatchEMD(cfg)
    emd.warmup()
    launcher = emd._get_launcher()
    if a.variant:
        launcher._plan.set_variant(a.variant)
    if a.arena:
        launcher._plan.set_arena(a.arena)
    arena_used, ctas_per_sm, grid_max = launcher._plan.query(N, f32=f32)

    # ---- device-resident throughput ----
    for _ in range(a.warmup):
        out = launcher.run(sig, None)
    torch.cuda.synchronize(dev)
    launcher.check_status()
    n_imfs, dbg_n, dbg_ext = out[1].cpu().numpy(), out[3].cpu().numpy(), out[4].cpu().numpy()
    ovf = int(out[2].sum().item())
    del out
    launcher._plan.counters(reset=True)
    launcher.run(sig, None)
    passes_step, spilled_step = launcher._plan.counters(reset=True)
    flops_per_step = algorithmic_flops(N, n_imfs, dbg_n, dbg_ext)
    hbm_bytes_per_step = float(isz) * B * N + float(isz) * B * cfg.max_imfs * N

    R.barrier(world)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local, a.clocks_csv.replace("{rank}", str(rank)) if a.clocks_csv else None)
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
    R.barrier(world)
    clk = clocks.stop() if clocks else None
    elapsed = t_start.elapsed_time(t_end) * 1e-3
    per_launch = [e0.elapsed_time(e1) * 1e-3 for e0, e1 in ev]
    elapsed = R.max_over_ranks(elapsed, world, dev)
    value = R.whole_job_rate(B, a.steps, world, elapsed)
    ms_per_step = elapsed / a.steps * 1e3
    launch_s = statistics.mean(per_launch)

    # ---- learned queue order (dense): features + BF16 MLP + LPT + launch per step ----
    ordered = None
    if a.order == "learned":
        from cuda_emd import scheduler as S
        t_tr = time.perf_counter()
        emd_tr = GPUBatchEMD(dataclasses.replace(cfg, real_t="double")) if f32 else emd
        ltr = emd_tr._get_launcher()
        feats, labels, n_tr = [], [], 0
        for k in range(a.order_train):
            # same generator, seeds disjoint from the timed batch's
            xtr = torch.from_numpy(make_workload(a.workload, rank + 1000 * (k + 1))).to(dev)
            otr = ltr.run(xtr, None)
            feats.append(S.features(xtr))
            labels.append(S.labels_from_debug(otr[3], otr[1]))
            n_tr += xtr.shape[0]
            del otr, xtr
        cm = S.CostModel(local, seed=0)
        cm.fit(torch.cat(feats), torch.cat(labels), epochs=a.epochs, batch=256)
        cm.warmup()
        del feats, labels
        torch.cuda.synchronize(dev)
        train_s = time.perf_counter() - t_tr

        def learned_step():
            order = S.learned_order(cm, sig)
            return GPUBatchEMD._run_ordered(launcher, sig, None, order)

        true_cost = torch.from_numpy(np.where(dbg_n > 0, dbg_n, 0).sum(1).astype(np.float32)).to(dev)
        true_order = S.lpt_order(true_cost)

        def timed_order(fn):
            for _ in range(max(1, min(a.warmup, 2))):
                fn()
            torch.cuda.synchronize(dev)
            R.barrier(world)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(a.steps):
                fn()
            e1.record(st)
            torch.cuda.synchronize(dev)
            return R.max_over_ranks(e0.elapsed_time(e1) * 1e-3, world, dev)

        clocks2 = ClockSampler(local, None)
        el_learned = timed_order(learned_step)
        clk2 = clocks2.stop() if clocks2 else None
        el_true = timed_order(lambda: GPUBatchEMD._run_ordered(launcher, sig, None, true_order))
        chk = learned_step()
        assert all(torch.equal(x, y) for x, y in
                   zip(chk, launcher.run(sig, None))), "order changed a result"
        del chk
        ordered = {"plain_value": round(value, 2), "plain_ms_per_step": round(ms_per_step, 3),
                   "learned_ms_per_step": round(el_learned / a.steps * 1e3, 3),
                   "speedup_learned": round(elapsed / el_learned, 4),
                   "true_cost_ms_per_step": round(el_true / a.steps * 1e3, 3),
                   "speedup_true_cost": round(elapsed / el_true, 4),
                   "train": f"{n_tr} traces of the same generator (disjoint seeds), "
                            f"{a.epochs} epochs, {train_s:.1f} s",
                   "note": "learned step = features + BF16 inference + LPT order + the launch, "
                           "all inside the timed region; true-cost = the queue ordered by the "
                           "logged sift passes (known only afterwards): the ordering ceiling",
                   "clocks": clk2}
        value = R.whole_job_rate(B, a.steps, world, el_learned)
        ms_per_step = el_learned / a.steps * 1e3

    # ---- end to end through the public API with pinned host buffers ----
    e2e = None
    if not a.no_e2e:
        host_in = torch.from_numpy(X).pin_memory()
        host_imfs = torch.empty((B, cfg.max_imfs, N), dtype=sig.dtype).pin_memory()
        host_n = torch.empty(B, dtype=torch.int32).pin_memory()
        host_o = torch.empty(B, dtype=torch.int32).pin_memory()

        def e2e_step():
            if f32:
                # the FP32 path takes device arrays: the batch goes up, the
                # public call sifts it, every result row comes back
                d = host_in.to(dev, non_blocking=True)
                im, nn, oo = emd(d)
                host_imfs.copy_(im, non_blocking=True)
                host_n.copy_(nn, non_blocking=True)
                host_o.copy_(oo, non_blocking=True)
                return
            # host input -> host results through GPUBatchEMD: the library copies
            # the batch up, sifts it in one launch and copies each finished
            # chunk of traces back while the rest still sift
            emd(host_in, out=(host_imfs, host_n, host_o))
        for _ in range(max(1, min(a.warmup, 2))):
            e2e_step()
        torch.cuda.synchronize(dev)
        R.barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(a.steps):
            e2e_step()
        e1.record(st)
        torch.cuda.synchronize(dev)
        te = R.max_over_ranks(e0.elapsed_time(e1) * 1e-3, world, dev)
        if f32:
            h2d, d2h = isz * B * N, isz * B * cfg.max_imfs * N + 8 * B
        else:
            h2d, d2h = emd._get_launcher()._plan.host_bytes()     # what the last step moved
        e2e = {"value": R.whole_job_rate(B, a.steps, world, te), "unit": "signals/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "d2h_dense_bytes_per_step": int(isz * B * cfg.max_imfs * N + 8 * B
                                               + 3 * 4 * B * cfg.max_imfs),
               "note": ("device copy of the batch, GPUBatchEMD on it, every output row "
                        "copied back" if f32 else
                        "of each finished chunk only the rows that may hold data are "
                        "copied; the zero rows after them are written on the host, "
                        "inside the timed region")}
        del host_imfs

    # ---- roofline ----
    roofline = None
    if rank == 0:
        peaks = {}
        pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.isfile(pk):
            peaks = json.load(open(pk))
        fp64 = dgemm_tflops(dev, torch.float32 if f32 else torch.float64)
        achieved = flops_per_step / launch_s / 1e12
        hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
        hbm_ach = hbm_bytes_per_step / launch_s / 1e9
        per_trace = None if f32 else NCU_DRAM_BYTES_PER_TRACE.get((N, cfg.max_imfs))
        traffic = round(per_trace * B) if per_trace else None
        roofline = {"bound": "fp32" if f32 else "fp64", "achieved": round(achieved, 3),
                    "peak": round(fp64, 3),
                    "unit": "TFLOP/s", "frac": round(achieved / fp64, 4), "traffic": traffic,
                    "traffic_source": ("ncu dram__bytes_read+write per trace of a 1024-trace "
                                       "launch x traces per launch") if traffic else None,
                    "peak_source": ("cuBLAS SGEMM (TF32 off) 8192^3 measured in this run" if f32
                                    else "cuBLAS DGEMM 8192^3 measured in this run"),
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
        rate, n, wall = cpu_oracle_rate(X, pool, cores, min(sample, B), a.real)
        cpu = {"value": round(rate, 2), "unit": "signals/s", "cores": cores, "kind": "port",
               "sample": f"first {n} traces of the workload, NumPy oracle, {cores} processes, "
                         f"{wall:.1f} s wall"}
        pool.close()

    if rank == 0:
        line = {
            "metric": METRIC.replace("FP64", "FP32") if f32 else METRIC, "value": round(value, 2),
            "unit": "signals/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_per_step, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if f32 else "f64",
            "data": "synthetic (seeded generator, see cuda_emd/workloads.py)",
            "config": {"workload": a.workload, "desc": WORKLOADS[a.workload]["desc"],
                       "batch_per_gpu": B, "N": N, "max_imfs": cfg.max_imfs,
                       "max_extrema": cfg.max_extrema, "max_iteration": cfg.max_iteration,
                       "queue": ("learned longest-predicted-first" if ordered
                                 else "FIFO persistent"),
                       "l2": "inputs+outputs larger than L2",
                       "real_t": a.real,
                       "arena_bytes": arena_used, "ctas_per_sm": ctas_per_sm,
                       "sift_passes_per_step": passes_step,
                       "spilled_pass_frac": round(spilled_step / max(passes_step, 1), 4),
                       "overflow_traces": ovf, "parallelism": f"replicas x{world}"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
            "order": ordered,
            # each dense launch of the 128/256-thread instances is a pair
            # (tail migration's resume launch); learned steps add the
            # feature and inference kernels
            "gpu_launches": a.steps * ((2 if ctas_per_sm >= 2 else 1) + (2 if ordered else 0)),
        }
        print(json.dumps(line), flush=True)
    R.finish(world)


REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libemd_ref.so")


def cpu_reference_steps(X: np.ndarray, pool, cores: int, steps: int, warmup: int, per: int):
    """The reference arm's CPU timing: `warmup` untimed and `steps` timed steps,
    each the oracle on a bounded slice of `per` traces (successive slices,
    wrapping), all host cores.  Returns (signals/s, traces timed, wall s)."""
    B = X.shape[0]
    per = max(1, min(per, B))

    def step(k):
        s0 = (k * per) % B
        sl = X[s0:s0 + per] if s0 + per <= B else np.concatenate([X[s0:], X[:s0 + per - B]])
        return cpu_oracle_rate(sl, pool, cores, per)

    for k in range(warmup):
        step(k)
    n_tot, wall_tot = 0, 0.0
    for k in range(steps):
        _, n, wall = step(warmup + k)
        n_tot += n
        wall_tot += wall
    return n_tot / wall_tot, n_tot, wall_tot


def ref_gpu_time(k, X: np.ndarray, steps: int, warmup: int):
    """The reference's emd_batch_kernel on the same GPU, dense [B, N] input:
    device-timed launches with its per-call pool allocation and fills
    (kernels.py:1343-1372).  Returns seconds per launch."""
    import torch
    dev = torch.device("cuda", 0)
    B, N = X.shape
    sig = torch.from_numpy(np.ascontiguousarray(X)).to(dev)
    Tn = torch.arange(N, dtype=torch.float64, device=dev)
    k.run_device(torch.zeros((1, 64), dtype=torch.float64, device=dev), Tn[:64])  # warmup()
    for _ in range(warmup):
        out = k.run_device(sig, Tn)
        del out
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        out = k.run_device(sig, Tn)
        del out
    e1.record(st)
    torch.cuda.synchronize()
    del sig
    torch.cuda.empty_cache()
    return e0.elapsed_time(e1) * 1e-3 / steps


def run_reference(a, rank, world, pool, cores):
    """Reference arm.  The reference's path is a CUDA kernel with no CPU
    implementation, so its CPU arm is the oracle port (oracle/emd_oracle.py,
    bit-identical to the reference kernel built with -fmad=false) on all host
    cores: W untimed and K timed steps, each a bounded slice of the workload.
    That is the line's value, its cpu_baseline and its e2e (no host<->device
    bytes).  When oracle/_ref is built and a GPU is present, the reference's
    own emd_batch_kernel (kernels.py:834-1080, compiled from kernels.py by
    oracle/build_ref.py: CuPy is absent, nvcc stands in for NVRTC) on the same
    GPU and workload is reported beside it as ``reference_gpu_kernel``, with
    the reference's launch geometry and per-call pool allocation + fills."""
    if rank != 0:
        return
    if a.workload == "ragged64k":
        return run_reference_ragged(a, pool, cores)
    X = make_workload(a.workload, 0)
    B, N = X.shape
    # enough traces per step that the pool's dispatch is a small part of it
    per = min(a.cpu_sample or max(cores * 32, 64), B)
    r, n, wall = cpu_reference_steps(X, pool, cores, a.steps, a.warmup, per)
    pool.close()
    cpu = {"value": round(r, 2), "unit": "signals/s", "cores": cores, "kind": "port",
           "sample": f"{a.steps} steps of {per} traces of the workload (after {a.warmup} "
                     f"warm-up steps), NumPy oracle, {cores} processes, {wall:.1f} s timed"}
    line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": "signals/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(per / max(r, 1e-9) * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator)",
            "config": {"workload": a.workload, "desc": WORKLOADS[a.workload]["desc"],
                       "batch_per_gpu": B, "N": N, "parallelism": f"{cores} host processes",
                       "step": f"{per} traces of the workload per step"},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "signals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    import torch
    if os.path.isfile(REF_LIB) and torch.cuda.is_available():
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from refkernel import RefKernel
        k = RefKernel("libemd_ref.so")
        dev = torch.device("cuda", 0)
        el = ref_gpu_time(k, X, a.steps, a.warmup)
        Tn = torch.arange(N, dtype=torch.float64, device=dev)
        host_in = torch.from_numpy(X).pin_memory()
        host_imfs = torch.empty((B, k.max_imfs, N), dtype=torch.float64).pin_memory()
        h_n = torch.empty(B, dtype=torch.int32).pin_memory()
        h_o = torch.empty(B, dtype=torch.int32).pin_memory()
        st = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
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
        line["reference_gpu_kernel"] = {
            "value": round(B / el, 2), "unit": "signals/s", "ms_per_step": round(el * 1e3, 3),
            "kernel": "emd_batch_kernel from kernels.py, nvcc -std=c++11 sm_100a "
                      "(oracle/_ref/libemd_ref.so); grid (batch,), block 128, 57824 B dynamic smem",
            "e2e": {"value": round(B * a.steps / te, 2), "unit": "signals/s",
                    "h2d_bytes_per_step": int(8 * B * N),
                    "d2h_bytes_per_step": int(8 * B * k.max_imfs * N + 8 * B)}}
    print(json.dumps(line), flush=True)


def run_reference_ragged(a, pool, cores):
    """Reference on the ragged batch (cfg2 evaluation set).  CPU arm: the oracle
    on bounded slices, as run_reference.  GPU reference kernel, timing only
    (zero padding changes the decomposition): (1) the batch padded to its max
    N = 8192, as the reference API requires one N; (2) per length bucket
    (<=1024, 2048, 4096, 8192) padded to the bucket edge, the fairer number.
    Both on a seeded subsample of --ref-sample traces per measurement (the
    whole padded batch would hold ~100 GB and run for minutes); the rate of a
    bucket scales by its trace count, so (2) is sum(bucket traces) / sum(bucket
    traces / bucket rate)."""
    w = WORKLOADS["ragged64k"]
    n_eval = a.eval_traces or w["n"]
    vals, offs = gen_ragged(pool, n_eval, w["lo"], w["hi"], seed=2)
    lens = np.diff(offs)
    rng = np.random.default_rng(12345)
    per = a.cpu_sample or max(cores * 2, 32)
    # CPU arm: the oracle over bounded random slices of the batch, all cores
    pick = rng.permutation(n_eval)
    rows = [vals[offs[b]:offs[b + 1]] for b in pick[: per * (a.steps + a.warmup)]]
    t_cpu = 0.0
    n_cpu = 0
    for k in range(a.warmup + a.steps):
        chunk = rows[k * per:(k + 1) * per]
        parts = [chunk[i::cores] for i in range(cores)]
        t0 = time.perf_counter()
        res = pool.map(_oracle_rows, [(p,) for p in parts if p])
        wall = time.perf_counter() - t0
        if k >= a.warmup:
            t_cpu += wall
            n_cpu += sum(r for r in res)
    pool.close()
    r_cpu = n_cpu / t_cpu
    cpu = {"value": round(r_cpu, 2), "unit": "signals/s", "cores": cores, "kind": "port",
           "sample": f"{a.steps} steps of {per} random traces of the batch (after {a.warmup} "
                     f"warm-up steps), NumPy oracle, {cores} processes, {t_cpu:.1f} s timed"}
    line = {"impl": "reference", "metric": METRIC_HEADLINE, "value": cpu["value"],
            "unit": "signals/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(per / max(r_cpu, 1e-9) * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": "ragged64k", "desc": w["desc"], "batch_per_gpu": n_eval,
                       "parallelism": f"{cores} host processes"},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "signals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    import torch
    if os.path.isfile(REF_LIB) and torch.cuda.is_available():
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from refkernel import RefKernel
        k = RefKernel("libemd_ref.so")
        ns = a.ref_sample

        def padded(idx, width):
            P = np.zeros((idx.size, width), dtype=np.float64)
            for r, b in enumerate(idx):
                P[r, :lens[b]] = vals[offs[b]:offs[b + 1]]
            return P

        sub = np.sort(rng.choice(n_eval, size=min(ns, n_eval), replace=False))
        t_pad = ref_gpu_time(k, padded(sub, int(lens.max())), 1, 1)
        buckets = {}
        t_weighted = 0.0
        for lo, hi in ((0, 1024), (1024, 2048), (2048, 4096), (4096, 8192)):
            m = np.flatnonzero((lens > lo) & (lens <= hi))
            if m.size == 0:
                continue
            bs = np.sort(rng.choice(m, size=min(ns, m.size), replace=False))
            t_b = ref_gpu_time(k, padded(bs, hi), 1, 1)
            rate = bs.size / t_b
            buckets[str(hi)] = {"traces": int(m.size), "sampled": int(bs.size),
                                "signals_per_s": round(rate, 2)}
            t_weighted += m.size / rate
        line["reference_gpu_kernel"] = {
            "padded_to_max_n": {"value": round(sub.size / t_pad, 2), "unit": "signals/s",
                                "N": int(lens.max()), "sampled": int(sub.size)},
            "per_length_bucket": {"value": round(n_eval / t_weighted, 2), "unit": "signals/s",
                                  "buckets": buckets},
            "note": "timing only: zero padding changes the decomposition",
            "kernel": "emd_batch_kernel from kernels.py, nvcc -std=c++11 sm_100a (oracle/_ref)"}
    print(json.dumps(line), flush=True)


def _oracle_rows(args):
    rows, = args
    sys.path.insert(0, ROOT)
    from oracle import emd_oracle as O
    for x in rows:
        O.emd_signal(x, np.arange(x.shape[0], dtype=np.float64))
    return len(rows)


# ---------------------------------------------------------------------------
# Ragged batch: plain FIFO tiers vs learned longest-predicted-first order
# ---------------------------------------------------------------------------

def _gen_ragged_chunk(args):
    n, lo, hi, seed = args
    sys.path.insert(0, os.path.join(ROOT, "emd-cuda_b200"))
    from cuda_emd import workloads as W
    vals, offs, kinds = W.ragged_mix(n, lo=lo, hi=hi, seed=seed)
    return vals, np.diff(offs)


def gen_ragged(pool, n: int, lo: int, hi: int, seed: int, chunk: int = 2048):
    """Deterministic CSR batch built from independently seeded chunks."""
    parts = [(min(chunk, n - s), lo, hi, seed * 100003 + k)
             for k, s in enumerate(range(0, n, chunk))]
    res = pool.map(_gen_ragged_chunk, parts) if pool is not None else [_gen_ragged_chunk(p) for p in parts]
    vals = np.concatenate([r[0] for r in res])
    lens = np.concatenate([r[1] for r in res])
    offs = np.zeros(lens.shape[0] + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    return vals, offs


def algorithmic_flops_ragged(lens: np.ndarray, n_imfs, dbg_n, dbg_ext) -> float:
    """algorithmic_flops summed over traces of different lengths."""
    dn = np.where(dbg_n > 0, dbg_n, 0).astype(np.float64)
    de = np.where(dbg_ext > 0, dbg_ext, 0).astype(np.float64)
    L = np.asarray(lens, dtype=np.float64)
    per_pass = 65.0 * L[:, None] + 20.0 * (de + 8.0)
    return float((dn * per_pass).sum() + 4.0 * (L * np.asarray(n_imfs, dtype=np.float64)).sum())


def _oracle_rows_timed(args):
    rows, = args
    sys.path.insert(0, ROOT)
    from oracle import emd_oracle as O
    t0 = time.perf_counter()
    for x in rows:
        O.emd_signal(x, np.arange(x.shape[0], dtype=np.float64))
    return len(rows), time.perf_counter() - t0


def cpu_ragged_rate(pool, cores: int, vals, offs, per: int, seed: int = 12345):
    """The oracle on `per` random traces of a CSR batch, all host cores."""
    rng = np.random.default_rng(seed)
    B = offs.shape[0] - 1
    pick = rng.permutation(B)[:per]
    rows = [vals[offs[b]:offs[b + 1]] for b in pick]
    parts = [rows[i::cores] for i in range(cores)]
    t0 = time.perf_counter()
    res = pool.map(_oracle_rows_timed, [(q,) for q in parts if q])
    wall = time.perf_counter() - t0
    n = sum(r[0] for r in res)
    return n / wall, n, wall, int(sum(r.shape[0] for r in rows))


def run_ragged(a, rank, world, pool, cores):
    """The headline: the ragged batch (65,536 mixed traces) decomposed with
    length tiers in one graph-captured launch sequence, plain FIFO queues vs
    the learned longest-predicted-first order (cost model trained here on the
    plain method's logged counts), plus a short serving sweep."""
    import torch
    from cuda_emd import EMDKernelConfig
    from cuda_emd import replicas as R
    from cuda_emd import scheduler as S
    from cuda_emd.ragged import RaggedRunner
    w = WORKLOADS["ragged64k"]
    n_eval = a.eval_traces or w["n"]
    t0 = time.perf_counter()
    ev_vals, ev_offs = gen_ragged(pool, n_eval, w["lo"], w["hi"], seed=2 + 1000 * rank)
    tr_vals, tr_offs = gen_ragged(pool, a.train_traces, w["lo"], w["hi"], seed=3 + 1000 * rank)
    gen_s = time.perf_counter() - t0
    # CPU baseline (rank 0): the oracle on a bounded random sample of the batch
    cpu = None
    if pool is not None and rank == 0 and not a.no_cpu:
        per = a.cpu_sample or max(cores * 8, 64)
        rate, n, wall, nsamp = cpu_ragged_rate(pool, cores, ev_vals, ev_offs, per)
        cpu = {"value": round(rate, 3), "unit": "signals/s", "cores": cores, "kind": "port",
               "sample": f"{n} random traces of the batch ({nsamp} samples), NumPy oracle, "
                         f"{cores} processes, {wall:.1f} s wall"}
    # serving sweep requests (single-GPU runs only: the server is one process)
    serve_traces = gen_requests(pool, a.serve_requests) if a.serve_requests > 0 and world == 1 else None
    if pool is not None:
        pool.close()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    R.init(world, "nccl", dev)
    cfg = EMDKernelConfig.for_device(local)
    v = torch.from_numpy(ev_vals).to(dev)
    o = torch.from_numpy(ev_offs).to(dev)
    lens_h = np.diff(ev_offs)
    B = n_eval
    runner = RaggedRunner(cfg, device=local, heavy_passes=a.heavy_passes, heavy_boost=a.heavy_boost)
    st = torch.cuda.current_stream(dev)

    def timed(arm, steps, warm, clocks=None):
        """W warm-up and K timed steps of one arm; per-step events around the
        whole step and around its tier launches (the graph replay)."""
        outs = None
        for _ in range(max(warm, 1)):
            outs = arm(outs)
        torch.cuda.synchronize(dev)
        runner.check_status()
        R.barrier(world)
        torch.cuda.synchronize(dev)
        sampler = ClockSampler(local, None) if clocks is not None else None
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
        t_s, t_e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_s.record(st)
        for k in range(steps):
            ev[k][0].record(st)
            outs = arm(outs, ev[k][1])
            ev[k][2].record(st)
        t_e.record(st)
        torch.cuda.synchronize(dev)
        R.barrier(world)
        if sampler is not None:
            clocks.append(sampler.stop())
        runner.check_status()
        total = R.max_over_ranks(t_s.elapsed_time(t_e) * 1e-3, world, dev)
        launch = [e[1].elapsed_time(e[2]) * 1e-3 for e in ev]
        return outs, total / steps, statistics.mean(launch)

    def plain(outs, mark=None):
        tiers_, orders_ = runner.prepare(v, o, None, offsets_host=ev_offs)     # FIFO queues
        if mark is not None:
            mark.record(st)
        return runner.launch(tiers_, orders_, v, o, outs, use_graph=True)

    clk = []
    plain_out, plain_s, plain_launch = timed(plain, a.steps, a.warmup, clk)
    plain_copy = [x.clone() for x in plain_out]
    n_imfs_h = plain_copy[1].cpu().numpy()
    dbg_n_h, dbg_e_h = plain_copy[3].cpu().numpy(), plain_copy[4].cpu().numpy()
    flops_step = algorithmic_flops_ragged(lens_h, n_imfs_h, dbg_n_h, dbg_e_h)

    # labels for the cost model: the plain method's logged counts on the training set
    tv = torch.from_numpy(tr_vals).to(dev)
    to = torch.from_numpy(tr_offs).to(dev)
    tl0 = time.perf_counter()
    lab_runner = RaggedRunner(cfg, device=local)
    tr_out = lab_runner.run(tv, to, offsets_host=tr_offs)
    torch.cuda.synchronize(dev)
    label_s = time.perf_counter() - tl0
    labels = S.labels_from_debug(tr_out[3], tr_out[1])
    del tr_out, lab_runner
    feats_tr = S.features(tv, to)
    cm = S.CostModel(local, seed=0)
    tt0 = time.perf_counter()
    hist = cm.fit(feats_tr, labels, epochs=a.epochs, batch=4096, lr=1e-3)
    torch.cuda.synchronize(dev)
    train_s = time.perf_counter() - tt0
    del tv, to, feats_tr, labels
    torch.cuda.empty_cache()

    # learned: features + BF16 inference + per-tier order + the launches, every step

    def learned(outs, mark=None, split=not a.no_split):
        # features + BF16 inference on the device; the model orders each
        # tier's queue and (split) sends predicted-heavy traces to the wide
        # instance, which needs the per-trace prediction on the host
        tiers_, orders_ = runner.prepare_learned(v, o, cm, offsets_host=ev_offs, split_heavy=split)
        if mark is not None:
            mark.record(st)
        return runner.launch(tiers_, orders_, v, o, outs, use_graph=True)

    def learned_order_only(outs, mark=None):
        return learned(outs, mark, split=False)

    k_side = min(a.steps, 5)
    _, order_s, _ = timed(learned_order_only, k_side, 1)
    learned_out, learned_s, learned_launch = timed(learned, a.steps, a.warmup, clk)
    same = all(torch.equal(x, y) for x, y in zip(plain_copy, learned_out))
    # ceiling: the queue ordered by the TRUE cost (N x logged passes, known only afterwards)
    true_cost = torch.from_numpy(lens_h * np.maximum(np.where(dbg_n_h > 0, dbg_n_h, 0).sum(1), 1)
                                 ).to(dev, torch.float32)

    def oracle_order(outs, mark=None):
        tiers_, orders_ = runner.prepare(v, o, true_cost, offsets_host=ev_offs)
        if mark is not None:
            mark.record(st)
        return runner.launch(tiers_, orders_, v, o, outs, use_graph=True)

    k_true = k_side
    _, true_s, _ = timed(oracle_order, k_true, 1)
    feats = S.features(v, o)
    truth = S.labels_from_debug(plain_copy[3], plain_copy[1])
    pred = cm.predict(feats)
    mae_log2_passes = float((pred[:, 0] - truth[:, 0]).abs().mean())
    passes_true = torch.exp2(truth[:, 0]) - 1
    passes_pred = (torch.exp2(pred[:, 0]) - 1).clamp(min=0)
    mae_passes = float((passes_pred - passes_true).abs().mean())
    mae_nimfs = float((pred[:, 1] - truth[:, 1]).abs().mean())

    # per-tier anatomy (each tier alone, learned order)
    tiers = {}
    for t in runner._tiers.values():
        t.plan.counters(reset=True)
    runner.run_learned(v, o, cm, use_graph=False, offsets_host=ev_offs, split_heavy=not a.no_split)
    torch.cuda.synchronize(dev)
    for t in runner._prep[1]:
        ps, sp = t.plan.counters(reset=True)
        sub = torch.from_numpy(t.idx.astype(np.int32)).to(dev)
        outs = runner._alloc_out(v, o)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        runner._launch_tier(t, v, o, sub, outs)
        e1.record()
        e1.synchronize()
        name = str(t.edge) + ("-heavy" if t in runner._heavy_tiers.values() else "")
        tiers[name] = {"traces": int(t.idx.size), "arena": t.arena, "variant": t.variant,
                              "passes": ps, "spilled_frac": round(sp / max(ps, 1), 4),
                              "alone_ms": round(e0.elapsed_time(e1), 2)}
        del outs

    # end to end through the public API: pinned host CSR in, host results out
    e2e = None
    if not a.no_e2e:
        vals_pin = torch.from_numpy(ev_vals).pin_memory()
        offs_pin = torch.from_numpy(ev_offs).pin_memory()
        for _ in range(max(1, min(a.warmup, 2))):
            runner.run_host(vals_pin, offs_pin, model=cm, split_heavy=not a.no_split)
        torch.cuda.synchronize(dev)
        R.barrier(world)
        t_0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(a.steps):
            res = runner.run_host(vals_pin, offs_pin, model=cm, split_heavy=not a.no_split)
        e1.record(st)
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t_0
        te = R.max_over_ranks(max(e0.elapsed_time(e1) * 1e-3, wall), world, dev)
        h2d, d2h = runner.last_host_bytes
        ok = bool(np.array_equal(res.n_imfs.numpy(), n_imfs_h))
        e2e = {"value": round(R.whole_job_rate(B, a.steps, world, te), 2), "unit": "signals/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "d2h_dense_bytes_per_step": int(8 * cfg.max_imfs * ev_offs[-1]),
               "api": "cuda_emd.ragged.RaggedRunner.run_host(pinned values, offsets, model=cost model)",
               "note": "per step: H2D of the CSR traces, features + BF16 inference + learned order, "
                       "the tier launches, a gather of the rows that may hold data (0..n_imfs), "
                       "D2H of those rows, counts and debug rows",
               "n_imfs_equal_device_run": ok}
        del res

    # roofline of the sift kernel: algorithmic FP64 of one step over the tier launches' time
    roofline = None
    if rank == 0:
        fp64 = dgemm_tflops(dev)
        achieved = flops_step / learned_launch / 1e12
        samples = float(ev_offs[-1])
        hbm_bytes = 8.0 * samples + 8.0 * cfg.max_imfs * samples
        hbm_peak, hbm_src = hbm_peak_gbs()
        per_sample = NCU_DRAM_BYTES_PER_SAMPLE_RAGGED
        roofline = {"bound": "fp64", "achieved": round(achieved, 3), "peak": round(fp64, 3),
                    "unit": "TFLOP/s", "frac": round(achieved / fp64, 4),
                    "traffic": round(per_sample * samples) if per_sample else None,
                    "traffic_source": NCU_RAGGED_SOURCE if per_sample else None,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                    "kernel": "emd_sift_kernel (all tier launches of one step)",
                    "algorithmic_flop_per_launch": flops_step,
                    "launch_ms": round(learned_launch * 1e3, 3),
                    "hbm": {"achieved": round(hbm_bytes / learned_launch / 1e9, 1), "peak": hbm_peak,
                            "unit": "GB/s", "frac": round(hbm_bytes / learned_launch / 1e9 / hbm_peak, 5),
                            "bytes_per_launch": hbm_bytes, "peak_source": hbm_src}}
    serve = None
    if serve_traces:
        del plain_out, learned_out, plain_copy
        torch.cuda.empty_cache()
        serve = serve_sweep(cfg, local, cm, serve_traces,
                            [float(x) for x in a.serve_loads.split(",")], slots=a.slots,
                            short_slots=a.short_slots)
    value = R.whole_job_rate(B, 1, world, learned_s)
    c = next((x for x in clk if x), None)
    if c and len(clk) > 1 and clk[1]:
        c = {"sm_mhz": statistics.median([x["sm_mhz"] for x in clk if x]),
             "sm_max_mhz": max(x["sm_max_mhz"] for x in clk if x),
             "reasons": sorted(set(r for x in clk if x for r in x["reasons"])),
             "samples": sum(x["samples"] for x in clk if x)}
    if rank == 0:
        line = {
            "metric": METRIC_HEADLINE, "value": round(value, 2), "unit": "signals/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(learned_s * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, see cuda_emd/workloads.py)",
            "config": {"workload": "ragged64k", "desc": w["desc"], "batch_per_gpu": B,
                       "samples": int(ev_offs[-1]), "max_imfs": cfg.max_imfs,
                       "max_extrema": cfg.max_extrema, "max_iteration": cfg.max_iteration,
                       "queue": "persistent, learned longest-predicted-first per length tier",
                       "l2": "inputs (1.2 GB) and outputs (19 GB) larger than L2",
                       "graph": True, "tiers": tiers, "parallelism": f"replicas x{world}"},
            "plain": {"value": round(R.whole_job_rate(B, 1, world, plain_s), 2),
                      "ms_per_step": round(plain_s * 1e3, 3),
                      "launch_ms": round(plain_launch * 1e3, 3), "queue": "FIFO per length tier"},
            "learned": {"value": round(value, 2), "ms_per_step": round(learned_s * 1e3, 3),
                        "launch_ms": round(learned_launch * 1e3, 3),
                        "speedup_vs_plain": round(plain_s / learned_s, 4),
                        "bit_identical_to_fifo": bool(same),
                        "tier_choice": ("predicted-heavy traces (>= %g passes) of tiers >= %d "
                                        "samples on the wide instance" % (runner.heavy_passes,
                                                                          4096))
                                       if not a.no_split else "by length only",
                        "order_only_ms_per_step": round(order_s * 1e3, 3),
                        "speedup_order_only": round(plain_s / order_s, 4),
                        "speedup_true_cost": round(plain_s / true_s, 4),
                        "true_cost_ms_per_step": round(true_s * 1e3, 3),
                        "true_cost_note": "queue ordered by N x the trace's logged sift passes "
                                          "(known only after decomposing it): the ceiling of any "
                                          f"ordering on this batch ({k_true} steps)",
                        "mae_log2_passes": round(mae_log2_passes, 4),
                        "mae_passes": round(mae_passes, 2), "mae_n_imfs": round(mae_nimfs, 4)},
            "cost_model": {"train_traces": a.train_traces, "epochs": a.epochs, "batch": 4096,
                           "lr": 1e-3, "loss_first": round(hist[0], 5), "loss_last": round(hist[-1], 5),
                           "train_s": round(train_s, 3), "label_s": round(label_s, 3)},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": c, "serve": serve,
            "gen_s": round(gen_s, 1),
            "gpu_launches": a.steps * (len(tiers) + 2),
            "gpu_launches_note": "per learned step: one emd_sift_kernel launch per length tier, "
                                 "features_kernel, the BF16 MLP inference kernel",
        }
        print(json.dumps(line), flush=True)
    R.finish(world)


# ---------------------------------------------------------------------------
# Serving: continuous batching under Poisson load
# ---------------------------------------------------------------------------

def _gen_requests_chunk(args):
    n, lo, hi, mt, seed = args
    sys.path.insert(0, os.path.join(ROOT, "emd-cuda_b200"))
    from cuda_emd.serving import make_requests
    rng = np.random.default_rng(seed)
    return [r.traces for r in make_requests(n, rng, lo=lo, hi=hi, max_traces=mt)]


def gen_requests(pool, nreq: int, seed0: int = 4000):
    """The serving workload's requests (trace lists), generated in 8 seeded chunks."""
    w = WORKLOADS["serve"]
    parts = [(max(1, -(-nreq // 8)), w["lo"], w["hi"], w["max_traces"], seed0 + k) for k in range(8)]
    res = pool.map(_gen_requests_chunk, parts) if pool is not None else [_gen_requests_chunk(p) for p in parts]
    return [t for chunk in res for t in chunk][:nreq]


def serve_sweep(cfg, local: int, cm, traces: list, loads: list, slots: int = 4,
                short_slots: int = 2) -> dict:
    """Continuous-batching server under Poisson arrivals: closed-loop
    saturation (every request at t=0), then each offered load as a fraction of
    it; p50/p99/p99.9 latency (delivery - arrival) per level."""
    from cuda_emd.serving import EMDServer, Request, run_open_loop, poisson_arrivals
    nreq = len(traces)
    mk = lambda: [Request(i, trs) for i, trs in enumerate(traces)]
    # warm-up (plans, kernels) and saturation
    srv = lambda: EMDServer(cfg, local, slots=slots, short_slots=short_slots, cost_model=cm)
    run_open_loop(srv(), mk()[:8], np.zeros(8))
    sat = run_open_loop(srv(), mk(), np.zeros(nreq))
    sat_tps = sat["traces_per_s"]
    mean_tr = sum(len(t) for t in traces) / nreq
    rng = np.random.default_rng(77)
    levels = []
    for load in loads:
        rate = load * sat_tps / mean_tr
        arr = poisson_arrivals(rate, nreq, rng)
        arr -= arr[0]
        rep = run_open_loop(srv(), mk(), arr, timeout_s=900)
        rep.update({"offered_load": load, "offered_traces_per_s": round(load * sat_tps, 1)})
        levels.append({k: (round(v, 3) if isinstance(v, float) else v) for k, v in rep.items()})
    return {"desc": WORKLOADS["serve"]["desc"], "requests_per_level": nreq,
            "mean_traces_per_request": round(mean_tr, 2), "slots": slots,
            "short_slots": short_slots,
            "order": "learned longest-predicted-first inside each admitted batch",
            "saturation": {"traces_per_s": round(sat_tps, 1), "p50_ms": round(sat["p50_ms"], 2),
                           "p99_ms": round(sat["p99_ms"], 2)},
            "levels": levels}


def run_serve(a, rank, world, pool, cores):
    import torch
    from cuda_emd import EMDKernelConfig
    from cuda_emd import scheduler as S
    w = WORKLOADS["serve"]
    t0 = time.perf_counter()
    traces = gen_requests(pool, a.requests)
    gen_s = time.perf_counter() - t0
    if pool is not None:
        pool.close()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    cfg = EMDKernelConfig.for_device(local)
    # cost model for the in-batch order, trained on the plain method's counts of a small set
    from cuda_emd.workloads import ragged_mix
    tv, to, _ = ragged_mix(4096, lo=w["lo"], hi=4096, seed=4999)
    tvd, tod = torch.from_numpy(tv).cuda(), torch.from_numpy(to).cuda()
    L = cfg.build()
    out = L.run_ragged(tvd, tod)
    cm = S.CostModel(local, seed=0)
    cm.fit(S.features(tvd, tod), S.labels_from_debug(out[3], out[1]), epochs=a.epochs, batch=1024)
    del out, tvd, tod
    sv = serve_sweep(cfg, local, cm, traces, [float(x) for x in a.loads.split(",")],
                     slots=a.slots, short_slots=a.short_slots)
    levels = sv["levels"]
    p99_90 = next((l["p99_ms"] for l in levels if abs(l["offered_load"] - 0.9) < 1e-6), None)
    line = {
        "metric": "EMD serve latency (FP64)", "value": p99_90, "unit": "ms p99 at 90% load",
        "n_gpus": world, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": "serve", "desc": w["desc"], "requests_per_level": sv["requests_per_level"],
                   "mean_traces_per_request": sv["mean_traces_per_request"], "slots": sv["slots"],
                   "order": sv["order"]},
        "saturation": sv["saturation"], "levels": levels, "gen_s": round(gen_s, 1),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
