"""Replica runs on several GPUs (bench.py --gpus N): each rank decomposes its
own seeded batch, timing is the maximum over ranks, the reported rate is the
whole job's.  Tested here with two gloo ranks on the host: distinct per-rank
data, the max-over-ranks agreement, the whole-job rate, and each rank's
decomposition (through the oracle, standing in for the GPU path) independent
of the other rank."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "emd-cuda_b200"))
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist
    from cuda_emd import replicas as R, workloads as W
    from oracle import emd_oracle as O
    r, w, lr = R.rank_env()
    R.init(w, "gloo", timeout_s=60)
    X = W.sinusoid_batch(3, 256, seed=R.workload_seed(0, r))
    T = np.arange(256, dtype=np.float64)
    n_imfs = [O.emd_signal(x, T).n_imfs for x in X]
    R.barrier(w)
    own = 1.0 + 0.5 * r                       # a rank's own "device time"
    tmax = R.max_over_ranks(own, w)
    rate = R.whole_job_rate(X.shape[0], 2, w, tmax)
    digest = torch.tensor([float(X.sum())], dtype=torch.float64)
    all_d = [torch.zeros(1, dtype=torch.float64) for _ in range(w)]
    dist.all_gather(all_d, digest)
    q.put((r, tmax, rate, [float(d.item()) for d in all_d], n_imfs, X.tolist()))
    R.finish(w)


@pytest.mark.timeout(180)
def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=150) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, t0, rate0, d0, n0, x0), (r1, t1, rate1, d1, n1, x1) = res
    assert (r0, r1) == (0, 1)
    assert t0 == t1 == 1.5                     # the slower rank's time, on both
    assert rate0 == rate1 == 3 * 2 * 2 / 1.5   # all ranks' traces / max time
    assert d0 == d1 and d0[0] != d0[1]         # distinct per-rank batches
    # each rank's results depend only on its own traces
    sys.path.insert(0, ROOT)
    from oracle import emd_oracle as O
    T = np.arange(256, dtype=np.float64)
    assert n1 == [O.emd_signal(np.asarray(x), T).n_imfs for x in x1]
    assert n0 == [O.emd_signal(np.asarray(x), T).n_imfs for x in x0]
