"""Ragged (CSR) batches: shared-memory tiers, an autotuner for each tier's
arena, and a CUDA-graph-captured multi-tier launch.

Traces are grouped by length into tiers (N <= 1024, 2048, 4096, 8192, 16384,
...).  Each tier is one persistent launch of the sift kernel over that tier's
traces, with its own plan (work-queue ticket, status word, spill slab) and
its own shared-memory arena: short traces get small arenas and more resident
CTAs per SM, long traces get room for their proto-IMF and knots.  The tier
launches are issued longest tier first on forked streams, so when a tier's
queue drains, its SMs pick up the next tier's CTAs.  The whole sequence can
be captured once into a CUDA graph and replayed.

Queue order inside a tier is FIFO (trace index) or, given per-trace costs,
longest-predicted-first.  Order never changes a result.

The autotuner times every candidate (register-budget variant, arena) pair --
the largest arena that keeps k = 6..1 CTAs per SM resident, with the kernel
build compiled for max(k, 4) CTAs -- on a sample of each tier large enough to
measure throughput (about 16 traces per CTA, or the whole tier) and caches
the winner in a JSON file keyed by device, config and tier.
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import _native
from .kernels import EMDKernelConfig

TIER_EDGES = (1024, 2048, 4096, 8192, 16384, 32768)
WIDE = 1                  # plan variant of the wide instance (one 512-thread CTA per SM)
HALF_WIDE = 2             # plan variant of two 256-thread CTAs per SM
WIDE_FROM = 4096          # tiers at least this long also try the wide instance
HALF_WIDE_FROM = 2048     # ... and this long the half-wide one
SMEM_PER_SM = 233472      # B200: 228 KB per SM
CTA_RESERVED = 1024       # shared memory the runtime reserves per CTA
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "emd_b200_autotune.json")


def tier_of(n: int) -> int:
    """Length tier of a trace: the listed edges, then powers of two (traces
    past what a CTA's shared memory holds run on the wide instance with the
    proto-IMF in global memory)."""
    for e in TIER_EDGES:
        if n <= e:
            return e
    e = TIER_EDGES[-1]
    while e < n:
        e *= 2
    return e


def candidates(plan: _native.Plan, max_n: int) -> list[tuple[int, int]]:
    """(register variant, arena) pairs worth trying for traces up to max_n:
    the largest arena that keeps k CTAs per SM resident, k = 6..1, with the
    register-budget build for max(k, 4) CTAs, if the arena holds the trace
    (even with every knot spilled: more resident CTAs can beat on-chip knots,
    e.g. 3 CTAs/SM for 8192-sample seismic traces)."""
    plan.set_variant(4)
    plan.set_arena(0)
    floor = plan.min_arena(max_n)
    out = []
    for k in (6, 5, 4, 3, 2, 1):
        # 128-byte units: shared memory is allocated in those, so a 16-byte
        # rounded share can round up past the SM and lose a CTA
        a = min((SMEM_PER_SM // k - CTA_RESERVED) & ~127, 232448)
        if a >= floor:
            out.append((max(k, 4), a))
    if max_n >= HALF_WIDE_FROM and min((SMEM_PER_SM // 2 - CTA_RESERVED) & ~127, 232448) >= floor + 1024:
        # two 256-thread CTAs per SM, at the automatic (half-SM) arena
        out.append((HALF_WIDE, 0))
    if max_n >= WIDE_FROM:
        # one 512-thread CTA per SM on one trace, at the automatic (full) arena;
        # for traces too long for shared memory the only candidate
        out.append((WIDE, 0))
    return out


class Tier:
    def __init__(self, edge: int, idx: np.ndarray, cfg: EMDKernelConfig, device: int):
        self.edge = edge
        self.idx = idx                      # trace indices (host, int64)
        self.max_n = 0
        self.plan = _native.Plan(cfg.to_c(), device)
        # the tier launches share the GPU (forked streams, the learned split's
        # capped wide launch beside the light one): no tail migration, whose
        # whole-SM resume launch assumes a launch that owns the GPU (measured:
        # the learned step fell from 2.07 to 2.64 s with it on)
        self.plan.set_tail(0)
        self.arena = 0
        self.variant = 4

    def set_tuning(self, variant: int, arena: int) -> None:
        self.variant = int(variant)
        self.arena = int(arena)
        self.plan.set_variant(self.variant)
        self.plan.set_arena(self.arena)


class RaggedRunner:
    """Decompose CSR batches with per-tier launches (optionally graph-captured)."""

    def __init__(self, config: EMDKernelConfig | None = None, device: int | None = None,
                 cache_path: str | None = DEFAULT_CACHE, autotune: bool = True,
                 heavy_passes: float = 600.0, heavy_boost: float = 1.0):
        import torch
        self.cfg = config or EMDKernelConfig()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.cache_path = cache_path
        self.autotune = autotune
        # learned tier choice: traces of a long tier predicted to need at least
        # heavy_passes sift passes run in their own wide launch, on a share of
        # the SMs (their predicted share of the work, times heavy_boost)
        self.heavy_passes = float(heavy_passes)
        self.heavy_boost = float(heavy_boost)
        self._tiers: dict[int, Tier] = {}
        self._heavy_tiers: dict[int, Tier] = {}
        self._graph = None
        self._graph_key = None
        self._cache = self._load_cache()

    # -- autotune cache ----------------------------------------------------------
    def _key(self, edge: int) -> str:
        import torch
        name = torch.cuda.get_device_name(self.device)
        c = self.cfg
        # "t3": entries timed on throughput-sized samples with the wide instance
        # among the candidates (older ones are ignored)
        return f"t3|{name}|{c.max_extrema},{c.nbsym},{c.max_iteration},{c.max_imfs}|{edge}"

    def _load_cache(self) -> dict:
        if self.cache_path and os.path.isfile(self.cache_path):
            try:
                return json.load(open(self.cache_path))
            except Exception:
                return {}
        return {}

    def _save_cache(self) -> None:
        if not self.cache_path:
            return
        os.makedirs(os.path.dirname(self.cache_path), exist_ok=True)
        tmp = self.cache_path + ".tmp"
        json.dump(self._cache, open(tmp, "w"), indent=1)
        os.replace(tmp, self.cache_path)

    # -- planning ----------------------------------------------------------------
    def tiers_for(self, lengths: np.ndarray) -> list[Tier]:
        edges = np.array([tier_of(int(n)) for n in lengths]) if lengths.size else np.zeros(0)
        out = []
        for e in sorted(set(edges.tolist()), reverse=True):   # longest tier first
            idx = np.flatnonzero(edges == e)
            t = self._tiers.get(e)
            if t is None:
                t = Tier(e, idx, self.cfg, self.device)
                self._tiers[e] = t
            t.idx = idx
            t.max_n = int(lengths[idx].max())
            out.append(t)
        return out

    def tune(self, values, offsets, lengths: np.ndarray, tiers: list[Tier], sample: int = 0) -> dict:
        """Pick each tier's arena by timing the candidates on a sample of its traces."""
        import torch
        chosen = {}
        for t in tiers:
            key = self._key(t.edge)
            sms = torch.cuda.get_device_properties(self.device).multi_processor_count
            want = sample or min(t.idx.size, 16 * 6 * sms)
            c = self._cache.get(key)
            # a tuning measured on a much smaller batch than this tier's sample
            # is redone (small samples time their longest trace, not throughput)
            if c is not None and 2 * int(c.get("sample", 0)) >= want:
                t.set_tuning(c.get("variant", 4), c["arena"])
                chosen[t.edge] = c
                continue
            cands = candidates(t.plan, t.edge)
            if not cands:
                raise ValueError(f"tier {t.edge} does not fit this device")
            if len(cands) == 1 or not self.autotune:
                v4 = [c for c in cands if c[0] == 4]
                t.set_tuning(*(v4[0] if v4 else cands[0]))
                continue
            # Throughput, not a small sample's makespan: with per-trace costs
            # spread over two orders of magnitude, a sample of a few traces per
            # CTA finishes with its single longest trace, which favours fewer,
            # faster CTAs.  So the sample fills the densest candidate's CTAs
            # ~16 times over (or is the whole tier).
            n_s = want
            sub = torch.from_numpy(t.idx[:n_s].astype(np.int32)).to(values.device)
            warm = sub[:64]
            res = {}
            outs = self._alloc_out(values, offsets)
            for v, a in cands:
                t.set_tuning(v, a)
                self._launch_tier(t, values, offsets, warm, outs)      # first-launch set-up
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                self._launch_tier(t, values, offsets, sub, outs)
                e1.record()
                e1.synchronize()
                res[(v, a)] = e0.elapsed_time(e1)
            del outs
            best = min(res, key=res.get)
            t.set_tuning(*best)
            self._cache[key] = {"variant": best[0], "arena": best[1], "ms": res[best],
                                "tried": {f"{v}/{a}": ms for (v, a), ms in res.items()},
                                "sample": int(n_s)}
            chosen[t.edge] = self._cache[key]
        self._save_cache()
        return chosen

    # -- launches ------------------------------------------------------------------
    def _alloc_out(self, values, offsets):
        import torch
        B = offsets.shape[0] - 1
        mi = self.cfg.max_imfs
        dev = values.device
        return (torch.empty(mi * values.shape[0], dtype=torch.float64, device=dev),
                torch.empty(B, dtype=torch.int32, device=dev), torch.empty(B, dtype=torch.int32, device=dev),
                torch.empty((B, mi), dtype=torch.int32, device=dev),
                torch.empty((B, mi), dtype=torch.int32, device=dev),
                torch.empty((B, mi), dtype=torch.int32, device=dev))

    def _launch_tier(self, t: Tier, values, offsets, order_dev, outs, stream=None):
        import torch
        imfs, n_imfs, ovf, dn, de, dz = outs
        st = (stream or torch.cuda.current_stream(values.device)).cuda_stream
        _native.check(t.plan.L.emdb_run_ragged(
            t.plan.handle, values.data_ptr(), offsets.data_ptr(), int(order_dev.shape[0]), int(t.edge),
            None, 1, order_dev.data_ptr(), imfs.data_ptr(), n_imfs.data_ptr(), ovf.data_ptr(),
            dn.data_ptr(), de.data_ptr(), dz.data_ptr(), st), "emdb_run_ragged")

    def prepare(self, values, offsets, cost=None, offsets_host=None, heavy=None, cost_host=None):
        """Host-side plan: tiers and per-tier queue orders (device int32).

        The tiers, their tuning and one persistent order buffer per tier are
        cached for repeated calls on the same values / offsets tensors (a
        captured graph reads those buffers); each call refills the buffers on
        the current stream: FIFO, or longest `cost` first (cost: per-trace
        work estimates, device tensor or host array).  ``offsets_host`` (the
        same offsets in host memory) spares the device read-back.  ``heavy``
        (host bool per trace, with ``cost_host``): those traces of each long
        tier run in their own launch of the wide instance (split_heavy)."""
        import hashlib
        hkey = None if heavy is None else hashlib.sha1(np.packbits(heavy).tobytes()).hexdigest()
        key = (offsets.data_ptr(), int(offsets.shape[0]), values.data_ptr(), hkey)
        cached = getattr(self, "_prep", None)
        if cached is None or cached[0] != key:
            tiers, idx = self._prepare(values, offsets, offsets_host, heavy, cost_host)
            orders = [x.clone() for x in idx]
            self._prep = cached = (key, tiers, idx, orders)
        _, tiers, idx, orders = cached
        self._fill_orders(idx, orders, cost, values.device)
        return tiers, orders

    def _prepare(self, values, offsets, offsets_host=None, heavy=None, cost_host=None):
        import torch
        if offsets_host is not None:
            off_h = np.asarray(offsets_host)
        else:
            off_h = offsets.cpu().numpy() if hasattr(offsets, "cpu") else np.asarray(offsets)
        lengths = np.diff(off_h)
        tiers = self.tiers_for(lengths)
        self.tune(values, offsets, lengths, tiers)
        if heavy is not None:
            tiers = self.split_heavy(tiers, np.asarray(heavy, dtype=bool), cost_host)
        idx = [torch.from_numpy(t.idx.astype(np.int32)).to(values.device) for t in tiers]
        return tiers, idx

    def split_heavy(self, tiers: list, heavy: np.ndarray, cost: np.ndarray | None) -> list:
        """The learned tier choice: the heavy traces of each long tier that
        runs the 128-thread instance move to a launch of the wide instance
        (one 512-thread CTA per SM, knots on-chip) capped at their share of
        the SMs; the rest stay in the tuned launch.  Launched first, so their
        CTAs take their SMs before the light launch fills the others."""
        import torch
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        c = np.ones(heavy.shape[0]) if cost is None else np.asarray(cost, dtype=np.float64)
        total = float(c.sum()) or 1.0
        out = []
        for t in tiers:
            if t.edge < WIDE_FROM or t.variant == WIDE:
                out.append(t)
                continue
            h = t.idx[heavy[t.idx]]
            if h.size == 0:
                out.append(t)
                continue
            ht = self._heavy_tiers.get(t.edge)
            if ht is None:
                ht = Tier(t.edge, h, self.cfg, self.device)
                ht.set_tuning(WIDE, 0)
                self._heavy_tiers[t.edge] = ht
            ht.idx = h
            ht.max_n = t.max_n
            share = float(c[h].sum()) / total * self.heavy_boost
            ht.plan.set_max_ctas(int(min(max(1, round(share * sms)), h.size, sms)))
            out.append(ht)
            light = t.idx[~heavy[t.idx]]
            if light.size:
                t.idx = light
                out.append(t)
        return out

    @staticmethod
    def _fill_orders(idx, orders, cost, device) -> None:
        """Each tier's queue: its traces in index order (FIFO), or sorted by
        decreasing cost (stable, so equal costs keep index order)."""
        import torch
        if cost is None:
            for i, o in zip(idx, orders):
                o.copy_(i)
            return
        c = cost if isinstance(cost, torch.Tensor) else torch.from_numpy(np.asarray(cost))
        c = c.to(device=device, dtype=torch.float32)
        for i, o in zip(idx, orders):
            perm = torch.argsort(c[i.long()], descending=True, stable=True)
            o.copy_(i[perm])

    def run(self, values, offsets, cost=None, outs=None, use_graph: bool = False,
            offsets_host=None):
        """Decompose; returns (imfs_csr, n_imfs, overflow, debug_n, debug_extno, debug_nzm)."""
        import torch
        with torch.cuda.nvtx.range("ragged plan"):
            tiers, orders = self.prepare(values, offsets, cost, offsets_host)
        with torch.cuda.nvtx.range("ragged launch"):
            return self.launch(tiers, orders, values, offsets, outs, use_graph)

    def launch(self, tiers, orders, values, offsets, outs=None, use_graph: bool = False):
        """The tier launches for a prepare()d batch, with the queue orders its
        buffers hold now (graph-captured once per batch if use_graph)."""
        import torch
        if outs is None:
            outs = self._alloc_out(values, offsets)
        main = torch.cuda.current_stream(values.device)
        if use_graph:
            key = (values.data_ptr(), offsets.data_ptr(), outs[0].data_ptr(),
                   tuple(int(o.data_ptr()) for o in orders), tuple(t.arena for t in tiers),
                   tuple(t.variant for t in tiers))
            if self._graph is None or self._graph_key != key:
                self._issue(tiers, orders, values, offsets, outs, main)   # warm: allocs outside capture
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._issue(tiers, orders, values, offsets, outs, torch.cuda.current_stream())
                self._graph, self._graph_key = g, key
                self._graph_keep = (orders, outs, values, offsets)
            self._graph.replay()
        else:
            self._issue(tiers, orders, values, offsets, outs, main)
        return outs

    def run_learned(self, values, offsets, model, outs=None, use_graph: bool = False,
                    offsets_host=None, split_heavy: bool = False):
        """run() with the queue ordered longest-predicted-first by a cost model
        (cuda_emd.scheduler.CostModel): features and BF16 inference on the
        device, per-tier order on the device, then the launches.  With
        split_heavy the model also picks the tier: traces it predicts to need
        at least `heavy_passes` sift passes run on the wide instance
        (split_heavy()).  Same results as FIFO, bit for bit."""
        import torch
        tiers, orders = self.prepare_learned(values, offsets, model, offsets_host, split_heavy)
        with torch.cuda.nvtx.range("ragged launch"):
            return self.launch(tiers, orders, values, offsets, outs, use_graph)

    def prepare_learned(self, values, offsets, model, offsets_host=None, split_heavy=False):
        """The learned step's planning: predicted cost per trace on the device,
        and with split_heavy the heavy set on the host (one small read-back)."""
        import torch
        from . import scheduler as S
        with torch.cuda.nvtx.range("ragged learned plan"):
            feats = S.features(values, offsets)
            lens = offsets[1:] - offsets[:-1]
            pred = model.predict(feats)
            cost = S.cost_from_prediction(pred, lens)
            heavy = cost_h = None
            if split_heavy:
                passes = S.passes_from_prediction(pred)
                both = torch.stack([passes, cost]).cpu().numpy()
                heavy, cost_h = both[0] >= self.heavy_passes, both[1]
            return self.prepare(values, offsets, cost, offsets_host, heavy, cost_h)

    def run_host(self, values, offsets, model=None, use_graph: bool = True,
                 split_heavy: bool = False):
        """Host CSR batch in, host results out (the end-to-end path): copy the
        traces up (page-locked inputs keep the copy asynchronous), order the
        queue by `model` if given (else FIFO), decompose, gather the rows that
        may hold data (rows 0..n_imfs of each trace; every later row is zero)
        into one buffer, and copy that buffer and the counts back.  Returns a
        HostRagged; its rows() gives trace b's [n_rows, N_b] block."""
        import torch
        dev = torch.device("cuda", self.device)
        vals_h = values if isinstance(values, torch.Tensor) else torch.from_numpy(np.asarray(values))
        offs_h = offsets if isinstance(offsets, torch.Tensor) else torch.from_numpy(np.asarray(offsets))
        total, B = int(vals_h.shape[0]), int(offs_h.shape[0]) - 1
        mi = self.cfg.max_imfs
        st = getattr(self, "_host_state", None)
        if st is None or st["total"] != total or st["B"] != B:
            st = {"total": total, "B": B,
                  "v": torch.empty(total, dtype=torch.float64, device=dev),
                  "o": torch.empty(B + 1, dtype=torch.int64, device=dev),
                  "packed": torch.empty(mi * total, dtype=torch.float64, device=dev),
                  "host_rows": torch.empty(0, dtype=torch.float64).pin_memory(),
                  "counts_h": torch.empty((5, B), dtype=torch.int32).pin_memory(),
                  "dbg_h": torch.empty((3, B, mi), dtype=torch.int32).pin_memory(),
                  "rowoff_h": torch.empty(B + 1, dtype=torch.int64).pin_memory(),
                  "outs": None}
            self._host_state = st
            self._prep = None
            self._graph = self._graph_key = None
        v, o = st["v"], st["o"]
        off_np = offs_h.numpy()
        if st.get("off_np") is None or not np.array_equal(st["off_np"], off_np):
            # new batch layout in the same buffers: plan (tiers, orders, graph) again
            st["off_np"] = off_np.copy()
            self._prep = None
            self._graph = self._graph_key = None
        v.copy_(vals_h, non_blocking=True)
        o.copy_(offs_h, non_blocking=True)
        if st["outs"] is None:
            st["outs"] = self._alloc_out(v, o)
        if model is not None:
            outs = self.run_learned(v, o, model, outs=st["outs"], use_graph=use_graph,
                                    offsets_host=off_np, split_heavy=split_heavy)
        else:
            outs = self.run(v, o, outs=st["outs"], use_graph=use_graph, offsets_host=off_np)
        imfs, n_imfs, ovf, dn, de, dz = outs
        torch.cuda.nvtx.range_push("ragged copy-back")
        lens = o[1:] - o[:-1]
        n_rows = torch.clamp(n_imfs + 1, max=mi).to(torch.int32)
        row_off = torch.zeros(B + 1, dtype=torch.int64, device=dev)
        torch.cumsum(n_rows.to(torch.int64) * lens, 0, out=row_off[1:])
        _native.check(_native.load().emdb_pack_rows(
            imfs.data_ptr(), o.data_ptr(), n_rows.data_ptr(), row_off.data_ptr(), B, mi,
            st["packed"].data_ptr(), torch.cuda.current_stream(dev).cuda_stream), "emdb_pack_rows")
        st["rowoff_h"].copy_(row_off, non_blocking=True)
        counts = st["counts_h"]
        counts[0].copy_(n_imfs, non_blocking=True)
        counts[1].copy_(ovf, non_blocking=True)
        counts[2].copy_(n_rows, non_blocking=True)
        for k, x in enumerate((dn, de, dz)):
            st["dbg_h"][k].copy_(x, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        need = int(st["rowoff_h"][-1])
        if st["host_rows"].shape[0] < need:
            st["host_rows"] = torch.empty(need, dtype=torch.float64).pin_memory()
        rows_h = st["host_rows"][:need]
        rows_h.copy_(st["packed"][:need], non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        torch.cuda.nvtx.range_pop()
        self.last_host_bytes = (int(vals_h.numel()) * 8 + (B + 1) * 8,
                                need * 8 + (B + 1) * 8 + 3 * B * 4 + 3 * B * mi * 4)
        return HostRagged(rows_h, st["rowoff_h"], off_np, counts[2], counts[0], counts[1],
                          st["dbg_h"])

    def _issue(self, tiers, orders, values, offsets, outs, main):
        import torch
        streams = getattr(self, "_streams", None)
        if streams is None or len(streams) < len(tiers):
            self._streams = streams = [torch.cuda.Stream(values.device) for _ in range(max(len(tiers), 1))]
        for t, o, s in zip(tiers, orders, streams):
            s.wait_stream(main)
            with torch.cuda.stream(s):
                self._launch_tier(t, values, offsets, o, outs, stream=s)
        for s in streams[:len(tiers)]:
            main.wait_stream(s)

    def check_status(self) -> None:
        import torch
        for t in self._tiers.values():
            st = t.plan.status(torch.cuda.current_stream(self.device).cuda_stream)
            if st & _native.STATUS_TOO_LONG:
                raise ValueError("a trace did not fit its tier's shared-memory arena")
            if st & _native.STATUS_STALE_ENVELOPE:
                raise RuntimeError("a sample fell outside the envelope knot span")


class HostRagged:
    """Results of RaggedRunner.run_host, in host memory (views of page-locked
    buffers that the runner's next run_host call overwrites)."""

    def __init__(self, rows, row_off, offsets, n_rows, n_imfs, overflow, dbg):
        self.packed = rows              # f64: the rows of every trace, back to back
        self.row_off = row_off          # int64 [B+1]: trace b's rows start at packed[row_off[b]]
        self.offsets = np.asarray(offsets)
        self.n_rows = n_rows            # int32 [B]: rows copied for trace b (later rows are zero)
        self.n_imfs = n_imfs
        self.overflow = overflow
        self.debug = dbg                # int32 [3, B, max_imfs]: debug_n, debug_extno, debug_nzm

    def rows(self, b: int) -> np.ndarray:
        """Trace b's copied rows as a [n_rows, N_b] array."""
        n = int(self.offsets[b + 1] - self.offsets[b])
        k = int(self.n_rows[b])
        s = int(self.row_off[b])
        return self.packed[s:s + k * n].numpy().reshape(k, n)
