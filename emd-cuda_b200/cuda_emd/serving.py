"""Continuous-batching server for EMD requests.

A request is a list of float64 traces (any lengths).  The server keeps a
pool of launch slots; each slot owns a CUDA stream and one plan per
shared-memory tier (work-queue ticket, status word, spill slab), so several
launches run on the GPU at once.  Requests that arrive while others are on
the GPU are admitted into the next free slot as soon as the device-memory
budget allows (inputs + dense outputs + counts of everything in flight), and
because the sift kernel is persistent, SMs freed by a finishing launch pick up
the CTAs of newly admitted ones: the work of old and new requests overlaps on
the device.  Inside an admitted batch the queue order is longest-predicted-
first when a cost model is attached (order never changes a result).

Each trace of a launch raises a completion flag in page-locked host memory
when its outputs are written (``emdb_run_ragged_notify``); as soon as all of
a request's traces are flagged, that request's rows are copied back on a copy
stream and the request is delivered -- it does not wait for the other
requests of its launch.

Each tier launch takes the largest shared-memory arena that still lets every
trace in flight be resident: on a lightly loaded GPU a long trace gets an SM
to itself with its knots on-chip (a sift that is latency-bound runs fastest
there), and once the traces in flight need 3 or more CTAs per SM the plan's
own throughput rule applies.  The arena never changes a result.

Per request the server records arrival, admission, device completion and
host delivery times; ``latency = delivered - arrival``.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native
from .kernels import EMDKernelConfig
from .ragged import tier_of


@dataclass
class Request:
    rid: int
    traces: list                      # list of 1-D float64 numpy arrays
    arrival: float = 0.0              # seconds (server clock)
    admitted: float = 0.0
    done: float = 0.0
    delivered: float = 0.0
    result: tuple | None = None       # (imfs list of [n_imfs, N] arrays, n_imfs, overflow)
    deadline: float | None = None     # server clock; past it the request is dropped as timed out
    status: str = "new"               # pending, running, delivered, cancelled, timeout

    @property
    def nbytes(self) -> int:
        return int(sum(t.shape[0] for t in self.traces)) * 8

    @property
    def max_len(self) -> int:
        return max((int(t.shape[0]) for t in self.traces), default=0)

    @property
    def latency(self) -> float:
        return self.delivered - self.arrival


def cost_bytes(n_samples: int, n_traces: int, max_imfs: int) -> int:
    """Device memory one launch holds: input + dense CSR output + per-trace
    counts (and the offsets / order)."""
    return n_samples * 8 * (1 + max_imfs) + n_traces * (4 * 3 * max_imfs + 24)


class Admission:
    """Which pending requests start next -- host logic only, no GPU.

    Requests wait in one FIFO queue per lane: "short" (every trace at most
    `short_max` samples) and "long".  Each lane has its own launch slots, so
    requests whose sift runs for seconds (long traces past max_extrema run to
    the iteration cap) never hold the slots short requests need.  All lanes
    share one device-memory budget.  A batch takes requests from the head of
    its lane's queue while they fit the budget and `max_batch` traces; a
    request larger than the whole budget is admitted alone once nothing else
    is in flight.  cancel() and expire() drop waiting requests (cancelled /
    past their deadline) before they reach the device."""

    LANES = ("short", "long")

    def __init__(self, short_slots: int, long_slots: int, budget: int, max_batch: int,
                 short_max: int, max_imfs: int):
        self.max_batch = int(max_batch)
        self.budget = int(budget)
        self.short_max = int(short_max)
        self.max_imfs = int(max_imfs)
        self.queues = {lane: collections.deque() for lane in self.LANES}
        # slot ids: short lane first
        self.free = {"short": collections.deque(range(short_slots)),
                     "long": collections.deque(range(short_slots, short_slots + long_slots))}
        self.in_use = 0
        self.running = 0                  # batches in flight
        self.n_short = int(short_slots)

    @property
    def nslots(self) -> int:
        return sum(len(q) for q in self.free.values()) + self.running

    def lane_of(self, req: Request) -> str:
        if not self.n_short:
            return "long"                 # no short lane: one queue for everything
        return "short" if req.max_len <= self.short_max else "long"

    def submit(self, req: Request) -> None:
        req.status = "pending"
        self.queues[self.lane_of(req)].append(req)

    def pending(self) -> int:
        return sum(len(q) for q in self.queues.values())

    def cancel(self, rid: int) -> Request | None:
        """Drop a waiting request; None if it is not waiting (running or done)."""
        for q in self.queues.values():
            for r in q:
                if r.rid == rid:
                    q.remove(r)
                    r.status = "cancelled"
                    return r
        return None

    def expire(self, now: float) -> list:
        """Drop the waiting requests whose deadline has passed."""
        out = []
        for q in self.queues.values():
            for r in [r for r in q if r.deadline is not None and now > r.deadline]:
                q.remove(r)
                r.status = "timeout"
                out.append(r)
        return out

    def next_batches(self, any_in_flight: bool) -> list:
        """(slot, lane, requests, bytes) for every batch that can start now;
        takes the slots and the budget."""
        out = []
        for lane in self.LANES:
            q, free = self.queues[lane], self.free[lane]
            while q and free:
                batch, ntr, nsamp = [], 0, 0
                while q:
                    r = q[0]
                    rs = sum(int(t.shape[0]) for t in r.traces)
                    cost = cost_bytes(nsamp + rs, ntr + len(r.traces), self.max_imfs)
                    if batch and (ntr + len(r.traces) > self.max_batch or self.in_use + cost > self.budget):
                        break
                    if not batch and self.in_use + cost > self.budget and (any_in_flight or out):
                        break                   # wait for memory to free up
                    batch.append(q.popleft())
                    ntr += len(r.traces)
                    nsamp += rs
                if not batch:
                    break
                b = cost_bytes(nsamp, ntr, self.max_imfs)
                self.in_use += b
                self.running += 1
                for r in batch:
                    r.status = "running"
                out.append((free.popleft(), lane, batch, b))
        return out

    def release(self, slot: int, lane: str, nbytes: int) -> None:
        self.in_use -= nbytes
        self.running -= 1
        self.free[lane].append(slot)


@dataclass
class _Flight:
    slot: int
    reqs: list
    event: object                     # after every kernel of the launch
    outs: tuple                       # host (imfs, n_imfs, overflow), page-locked
    dev: tuple                        # device (imfs, n_imfs, overflow)
    offsets_h: np.ndarray
    budget: int
    first: list                       # first trace index of each request
    state: list                       # per request: 0 running, 1 copying, 2 delivered, 3 dropped
    copies: list                      # per request: event of its copy-back
    keep: tuple = field(default_factory=tuple)
    lane: str = "long"
    start: object = None              # timing event before the launch's kernels


class EMDServer:
    """Continuous-batching server.  `slots` launch slots serve requests with a
    trace longer than `short_max` samples, `short_slots` more serve the
    others (Admission)."""

    def __init__(self, config: EMDKernelConfig | None = None, device: int | None = None,
                 slots: int = 4, hbm_budget_bytes: int = 32 << 30, max_batch_traces: int = 4096,
                 cost_model=None, adaptive_arena: bool = True, short_slots: int = 2,
                 short_max: int = 4096):
        import torch
        self.cfg = config or EMDKernelConfig()
        self.device = torch.cuda.current_device() if device is None else int(device)
        props = torch.cuda.get_device_properties(self.device)
        self.num_sms = props.multi_processor_count
        self.smem_sm = props.shared_memory_per_multiprocessor
        self.smem_optin = props.shared_memory_per_block_optin
        self.adaptive_arena = adaptive_arena
        self.wide_from = 4096           # tiers this long may take the wide instances
        self.min_arena: dict[int, int] = {}
        self.nslots = slots + short_slots
        self.budget = int(hbm_budget_bytes)
        self.max_batch = max_batch_traces
        self.cost_model = cost_model
        self.adm = Admission(short_slots, slots, hbm_budget_bytes, max_batch_traces, short_max,
                             self.cfg.max_imfs)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(self.nslots)]
        self.copy_stream = torch.cuda.Stream(self.device)
        self.notify = [_native.Notify(max_batch_traces, self.device) for _ in range(self.nslots)]
        self.plans: dict[tuple[int, int], _native.Plan] = {}
        self.tier_streams: dict = {}
        self.flights: list[_Flight] = []
        self.t0 = time.perf_counter()
        self.completed: list[Request] = []
        self.dropped: list[Request] = []
        # device clock origin for the launches' start / end events
        self.ev0 = torch.cuda.Event(enable_timing=True)
        self.ev0.record(torch.cuda.current_stream(self.device))
        self.intervals: list = []         # (lane, start event, end event) per launch

    def now(self) -> float:
        return time.perf_counter() - self.t0

    # -- admission ------------------------------------------------------------
    def submit(self, req: Request) -> None:
        if not req.arrival:
            req.arrival = self.now()
        self.adm.submit(req)

    @property
    def pending(self) -> int:
        return self.adm.pending()

    @property
    def in_use(self) -> int:
        return self.adm.in_use

    def cancel(self, rid: int) -> bool:
        """Cancel a request: a waiting one never reaches the device; a running
        one keeps its launch going (the kernel is not interrupted) but is not
        copied back or delivered.  False if it is unknown or already done."""
        r = self.adm.cancel(rid)
        if r is not None:
            self.dropped.append(r)
            return True
        for f in self.flights:
            for q, r in enumerate(f.reqs):
                if r.rid == rid and f.state[q] in (0, 1):
                    f.state[q] = 3
                    r.status = "cancelled"
                    self.dropped.append(r)
                    return True
        return False

    def _expire(self) -> None:
        now = self.now()
        self.dropped.extend(self.adm.expire(now))
        for f in self.flights:
            for q, r in enumerate(f.reqs):
                if f.state[q] == 0 and r.deadline is not None and now > r.deadline:
                    f.state[q] = 3
                    r.status = "timeout"
                    self.dropped.append(r)

    _cost_bytes = staticmethod(cost_bytes)

    def device_intervals(self) -> list:
        """(lane, start ms, end ms) on the device clock of every finished launch."""
        return [(lane, self.ev0.elapsed_time(a), self.ev0.elapsed_time(b))
                for lane, a, b in self.intervals if b.query()]

    def _tier_stream(self, slot: int, edge: int):
        import torch
        key = (slot, edge)
        t = self.tier_streams.get(key)
        if t is None:
            t = torch.cuda.Stream(self.device)
            self.tier_streams[key] = t
        return t

    def _plan(self, slot: int, edge: int) -> _native.Plan:
        key = (slot, edge)
        p = self.plans.get(key)
        if p is None:
            p = _native.Plan(self.cfg.to_c(), self.device)
            self.plans[key] = p
        return p

    def _tier_arena(self, edge: int, in_flight: int) -> int:
        """Arena for a tier launch of traces up to `edge` samples while
        `in_flight` traces (this launch's included) are on the GPU: the largest
        one that still lets them all be resident when that takes 1 or 2 CTAs
        per SM, else 0 (the plan's rule)."""
        if not self.adaptive_arena:
            return 0
        per_sm = max(1, -(-in_flight // self.num_sms))
        if per_sm > 2:
            return 0
        # the driver reserves 1 KB per CTA; allocation is in 128-byte units
        arena = min(self.smem_sm // per_sm - 1024, self.smem_optin) & ~127
        m = self.min_arena.get(edge)
        if m is None:
            m = self.min_arena[edge] = self._plan(0, edge).min_arena(edge)
        return arena if arena >= m else 0

    def _tier_instance(self, edge: int, in_flight: int) -> tuple[int, int]:
        """(kernel variant, arena) of a tier launch.  A lightly loaded server
        is latency-bound, so long traces get a whole SM each (the 512-thread
        wide instance, 16 warps per trace, knots on-chip) while the traces in
        flight fit one per SM, half an SM (two 256-thread CTAs) while they
        fit two per SM; otherwise the 128-thread instance with the load-sized
        arena of _tier_arena.  Results are the same bits whichever runs."""
        if self.adaptive_arena and edge >= self.wide_from:
            if in_flight <= self.num_sms:
                return 1, 0
            if in_flight <= 2 * self.num_sms:
                return 2, 0
        return 4, self._tier_arena(edge, in_flight)

    def _admit(self) -> int:
        """Admit pending requests into free slots of their lanes while the budget allows."""
        admitted = 0
        for slot, lane, batch, nbytes in self.adm.next_batches(bool(self.flights)):
            ntr = sum(len(r.traces) for r in batch)
            nsamp = sum(int(t.shape[0]) for r in batch for t in r.traces)
            self._launch(slot, batch, ntr, nsamp, lane, nbytes)
            admitted += len(batch)
        return admitted

    def _launch(self, slot: int, reqs: list, ntr: int, nsamp: int, lane: str = "long",
                budget: int = 0) -> None:
        import torch
        st = self.streams[slot]
        lens = np.array([t.shape[0] for r in reqs for t in r.traces], dtype=np.int64)
        off_h = np.zeros(ntr + 1, dtype=np.int64)
        np.cumsum(lens, out=off_h[1:])
        vals_h = np.concatenate([t for r in reqs for t in r.traces]) if ntr else np.zeros(0)
        now = self.now()
        for r in reqs:
            r.admitted = now
        mi = self.cfg.max_imfs
        dev = torch.device("cuda", self.device)
        nt = self.notify[slot]
        nt.reset(ntr, st.cuda_stream)          # the slot's previous launch has finished
        with torch.cuda.stream(st):
            vals = torch.from_numpy(vals_h).pin_memory().to(dev, non_blocking=True)
            offs = torch.from_numpy(off_h).pin_memory().to(dev, non_blocking=True)
            imfs = torch.empty(mi * nsamp, dtype=torch.float64, device=dev)
            n_imfs = torch.empty(ntr, dtype=torch.int32, device=dev)
            ovf = torch.empty(ntr, dtype=torch.int32, device=dev)
            dn = torch.empty((ntr, mi), dtype=torch.int32, device=dev)
            de = torch.empty((ntr, mi), dtype=torch.int32, device=dev)
            dz = torch.empty((ntr, mi), dtype=torch.int32, device=dev)
            cost = None
            if self.cost_model is not None and ntr > 1:
                from .scheduler import features, predicted_cost
                f = features(vals, offs)
                cost = predicted_cost(self.cost_model, f, offs[1:] - offs[:-1])
            edges = np.array([tier_of(int(n)) for n in lens])
            keep = [vals, offs]
            tiers = []
            for e in sorted(set(edges.tolist()), reverse=True):
                idx = np.flatnonzero(edges == e)
                order = torch.from_numpy(idx.astype(np.int32)).to(dev, non_blocking=True)
                if cost is not None:
                    sub = cost[order.long()]
                    order = order[torch.argsort(sub, descending=True, stable=True)]
                keep.append(order)
                tiers.append((e, idx.size, order))
            ready = torch.cuda.Event(enable_timing=True)
            ready.record(st)
        # each tier on its own stream of the slot, so a short tier's traces
        # (and the requests they finish) need not wait for a long tier
        in_flight = ntr + sum(f.first[-1] for f in self.flights)
        for e, cnt, order in tiers:
            ts = self._tier_stream(slot, e)
            ts.wait_event(ready)
            p = self._plan(slot, e)
            variant, arena = self._tier_instance(e, in_flight)
            p.set_variant(variant)
            p.set_arena(arena)
            # the plan's tail migration stays on: a serving launch is small,
            # so its traces move to whole SMs once its queue is empty -- the
            # measured sweeps favour it at 70 % load and above
            _native.check(p.L.emdb_run_ragged_notify(
                p.handle, vals.data_ptr(), offs.data_ptr(), int(cnt), int(e), None, 1,
                order.data_ptr(), imfs.data_ptr(), n_imfs.data_ptr(), ovf.data_ptr(),
                dn.data_ptr(), de.data_ptr(), dz.data_ptr(), nt.handle, ntr, ts.cuda_stream),
                "emdb_run_ragged_notify")
            done_t = torch.cuda.Event()
            done_t.record(ts)
            st.wait_event(done_t)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(st)
        self.intervals.append((lane, ready, ev))
        h_imfs = torch.empty(mi * nsamp, dtype=torch.float64).pin_memory()
        h_n = torch.empty(ntr, dtype=torch.int32).pin_memory()
        h_o = torch.empty(ntr, dtype=torch.int32).pin_memory()
        first, k = [], 0
        for r in reqs:
            first.append(k)
            k += len(r.traces)
        first.append(k)
        keep.extend([dn, de, dz])
        self.flights.append(_Flight(slot, reqs, ev, (h_imfs, h_n, h_o), (imfs, n_imfs, ovf), off_h,
                                    budget, first, [0] * len(reqs), [None] * len(reqs), tuple(keep),
                                    lane, ready))

    # -- completion -------------------------------------------------------------
    def _copy_request(self, f: _Flight, q: int, flags: np.ndarray) -> None:
        """Copy request q's rows (only those that may hold data) and counts back."""
        import torch
        h_imfs, h_n, h_o = f.outs
        d_imfs, d_n, d_o = f.dev
        mi = self.cfg.max_imfs
        k0, k1 = f.first[q], f.first[q + 1]
        with torch.cuda.stream(self.copy_stream):
            for k in range(k0, k1):
                a, b = int(f.offsets_h[k]), int(f.offsets_h[k + 1])
                # a flag still 0 here means the launch ended without it: copy all rows
                rows = mi if int(flags[k]) == 0 else min(int(flags[k]) - 1, mi)
                if rows > 0:
                    h_imfs[mi * a: mi * a + rows * (b - a)].copy_(
                        d_imfs[mi * a: mi * a + rows * (b - a)], non_blocking=True)
            h_n[k0:k1].copy_(d_n[k0:k1], non_blocking=True)
            h_o[k0:k1].copy_(d_o[k0:k1], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.copy_stream)
        f.copies[q] = ev
        f.state[q] = 1

    def _deliver(self, f: _Flight, q: int) -> None:
        h_imfs, h_n, h_o = (x.numpy() for x in f.outs)
        mi = self.cfg.max_imfs
        r = f.reqs[q]
        rows, nims, ovfs = [], [], []
        for k in range(f.first[q], f.first[q + 1]):
            a, b = int(f.offsets_h[k]), int(f.offsets_h[k + 1])
            blk = h_imfs[mi * a: mi * b].reshape(mi, b - a)
            rows.append(blk[:int(h_n[k])].copy())
            nims.append(int(h_n[k]))
            ovfs.append(int(h_o[k]))
        r.done = self.now()
        r.result = (rows, np.array(nims, dtype=np.int32), np.array(ovfs, dtype=np.int32))
        r.delivered = self.now()
        r.status = "delivered"
        self.completed.append(r)
        f.state[q] = 2

    def _reap(self) -> int:
        """Deliver every request whose traces are all done; release a slot once
        its launch has finished and all its requests are delivered."""
        done = 0
        still = []
        for f in self.flights:
            flags = self.notify[f.slot].flags
            kernels_done = f.event.query()
            for q in range(len(f.reqs)):
                if f.state[q] == 0:
                    k0, k1 = f.first[q], f.first[q + 1]
                    if kernels_done or (flags[k0:k1] != 0).all():
                        self._copy_request(f, q, flags)
                if f.state[q] == 1 and f.copies[q].query():
                    self._deliver(f, q)
                    done += 1
            if kernels_done and all(st in (2, 3) for st in f.state):
                self.adm.release(f.slot, f.lane, f.budget)
            else:
                still.append(f)
        self.flights = still
        return done

    def step(self) -> tuple[int, int]:
        """One scheduler tick: reap finished launches, admit pending requests."""
        import torch
        with torch.cuda.nvtx.range("serve reap"):
            self._expire()
            d = self._reap()
        with torch.cuda.nvtx.range("serve admit"):
            a = self._admit()
        return a, d

    def drain(self, timeout_s: float = 600.0) -> None:
        t_end = self.now() + timeout_s
        while (self.pending or self.flights) and self.now() < t_end:
            a, d = self.step()
            if not a and not d:
                time.sleep(0.0002)
        if self.pending or self.flights:
            raise TimeoutError("server did not drain in time")

    def check_status(self) -> None:
        import torch
        for p in self.plans.values():
            st = p.status(torch.cuda.current_stream(self.device).cuda_stream)
            if st:
                raise RuntimeError(f"kernel status bits {st}")


def poisson_arrivals(rate: float, n: int, rng: np.random.Generator) -> np.ndarray:
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def make_requests(n: int, rng: np.random.Generator, lo: int = 512, hi: int = 16384,
                  max_traces: int = 64) -> list[Request]:
    """Requests of 1..max_traces traces, lengths log-uniform in [lo, hi], drawn
    from the ragged mix (60 % seismic, 38 % three-tone, 2 % chirp)."""
    from . import workloads as W
    reqs = []
    for i in range(n):
        k = int(rng.integers(1, max_traces + 1))
        lens = W.ragged_lengths(rng, k, lo, hi)
        trs = []
        for N in lens:
            u = rng.uniform()
            if u < 0.60:
                trs.append(W.seismic_trace(rng, int(N)))
            elif u < 0.98:
                trs.append(W.sinusoid_trace(rng, int(N)))
            else:
                trs.append(W.chirp_trace(rng, int(N)))
        reqs.append(Request(i, trs))
    return reqs


def run_open_loop(server: EMDServer, reqs: list[Request], arrivals: np.ndarray,
                  timeout_s: float = 600.0) -> dict:
    """Feed requests at their arrival times (seconds from start), serve
    continuously, and report latency percentiles and throughput."""
    server.t0 = time.perf_counter()
    i = 0
    n = len(reqs)
    t_end = timeout_s
    while i < n or server.pending or server.flights:
        now = server.now()
        if now > t_end:
            raise TimeoutError("open-loop run exceeded its time limit")
        while i < n and arrivals[i] <= now:
            reqs[i].arrival = float(arrivals[i])
            server.submit(reqs[i])
            i += 1
        a, d = server.step()
        if not a and not d:
            nxt = arrivals[i] - server.now() if i < n else 0.0002
            time.sleep(max(0.0, min(nxt, 0.0005)))
    lat = np.array([r.latency for r in reqs])
    ntr = sum(len(r.traces) for r in reqs)
    span = max(r.delivered for r in reqs) - float(arrivals[0])
    return {"requests": n, "traces": ntr, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "p999_ms": float(np.percentile(lat, 99.9) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "traces_per_s": ntr / span, "span_s": span}
