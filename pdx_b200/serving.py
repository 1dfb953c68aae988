"""Continuous-batching search server over one GPU-resident index.

Requests (query, k, nprobe, optional filter) arrive over time. The index stays resident, and so
do the filters registered with PDXIndex.register_filter; several contexts (pdxg_context: a
workspace and a CUDA stream each) stay busy. As soon as a context is free it takes the requests
that have arrived -- up to the batch cap and within its share of the device-memory budget -- and
launches them as one batch (pdxg_search_requests: per-query k, nprobe and filter inside one
launch). Requests that arrive while other batches run are admitted into the next free context,
so batches overlap on the device. Latency is measured per request from its arrival to the moment
the host sees its batch complete.

A request's result does not depend on the batch it ran in: the kernels search every query
independently with the reference's per-query semantics (Search / FilteredSearch).
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import compiled


@dataclass
class Workload:
    """Requests as arrays, sorted by arrival time (seconds from the start of the run)."""
    arrival: np.ndarray                   # f64 [n]
    queries: np.ndarray                   # f32 [n, d]
    k: np.ndarray                         # u32 [n]
    nprobe: np.ndarray                    # u32 [n] (0 = all clusters)
    filter_id: np.ndarray                 # i32 [n]: registered filter, -1 = none
    rows: Optional[List[Optional[np.ndarray]]] = None  # per-request row-id lists (or None)

    def __len__(self):
        return len(self.arrival)


@dataclass
class Served:
    ids: np.ndarray         # u32 [n, k_max], row i holds counts[i] results
    distances: np.ndarray   # f32 [n, k_max]
    counts: np.ndarray      # u32 [n]
    latency: np.ndarray     # f64 [n] seconds, arrival -> completion seen by the host
    batch: np.ndarray       # i32 [n] sequence number of the batch each request ran in
    wall: float             # seconds from the first arrival to the last completion

    def result(self, i):
        c = int(self.counts[i])
        return self.ids[i, :c], self.distances[i, :c]


class _Slot:
    """One context with its device and pinned host buffers."""

    def __init__(self, index: compiled.PDXIndex, max_batch: int, k_max: int, d: int):
        import torch
        self.ctx = compiled.Context(index)
        self.stream = torch.cuda.ExternalStream(self.ctx.stream)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.q_dev = torch.empty((max_batch, d), dtype=torch.float32, device=dev)
        self.ids_dev = torch.empty((max_batch, k_max), dtype=torch.int32, device=dev)
        self.d_dev = torch.empty((max_batch, k_max), dtype=torch.float32, device=dev)
        self.c_dev = torch.empty(max_batch, dtype=torch.int32, device=dev)
        self.q_pin = torch.empty((max_batch, d), dtype=torch.float32).pin_memory()
        self.ids_pin = torch.empty((max_batch, k_max), dtype=torch.int32).pin_memory()
        self.d_pin = torch.empty((max_batch, k_max), dtype=torch.float32).pin_memory()
        self.c_pin = torch.empty(max_batch, dtype=torch.int32).pin_memory()
        self.q_np = self.q_pin.numpy()
        self.event = torch.cuda.Event()
        self.begin = self.end = 0  # request range in flight (begin == end: idle)
        self.batch_no = -1

    def close(self):
        # torch's pinned-memory allocator records an event on every stream a pinned block was
        # copied on when the block is freed: free the buffers while the stream still exists
        if self.ctx is None:
            return
        self.event.synchronize()
        for name in ("q_dev", "ids_dev", "d_dev", "c_dev", "q_pin", "ids_pin", "d_pin", "c_pin", "q_np"):
            setattr(self, name, None)
        self.stream = None
        self.ctx.close()
        self.ctx = None


class Server:
    """Continuous batching over `n_contexts` concurrent contexts of one index."""

    def __init__(self, index: compiled.PDXIndex, max_batch: int = 2048, n_contexts: int = 3,
                 k_max: int = 100, memory_budget: Optional[int] = None):
        self.index = index
        self.max_batch = max_batch
        self.k_max = k_max
        self.d = index.get_num_dimensions()
        n_rows = index.get_num_embeddings()
        n_cl = index.get_num_clusters()
        self.slots = [_Slot(index, max_batch, k_max, self.d) for _ in range(n_contexts)]
        # device bytes one request adds to a batch: raw + rotated query, results, parameters;
        # a row-id list adds its rows, a selection bitmap and passing counts
        self.bytes_request = 8 * self.d + 8 * k_max + 4 + 16
        self.bytes_list = 4 * (n_rows // 32 + 32 * n_cl) + 4 * n_cl + 8
        if memory_budget is None:
            import torch
            free, _ = torch.cuda.mem_get_info()
            memory_budget = int(free * 0.25)
        self.budget_per_slot = max(memory_budget // n_contexts, self.bytes_request + self.bytes_list)

    def _admit(self, w: Workload, head: int, avail: int) -> int:
        """Number of requests from `head` that fit one batch (cap and memory budget)."""
        m = min(avail - head, self.max_batch)
        if w.rows is None:
            return max(1, min(m, self.budget_per_slot // self.bytes_request))
        used, n = 0, 0
        for i in range(head, head + m):
            r = w.rows[i]
            b = self.bytes_request + (0 if r is None else self.bytes_list + 4 * len(r))
            if n and used + b > self.budget_per_slot:
                break
            used += b
            n += 1
        return n

    def _launch(self, slot: _Slot, w: Workload, a: int, b: int, batch_no: int):
        import torch
        m = b - a
        slot.q_np[:m] = w.queries[a:b]
        table = compiled.request_table(m)
        table["k"] = w.k[a:b]
        table["nprobe"] = w.nprobe[a:b]
        table["filter_id"] = w.filter_id[a:b]
        rows = None
        if w.rows is not None:
            parts, pos = [], 0
            for j in range(m):
                r = w.rows[a + j]
                if r is not None and table[j]["filter_id"] < 0:
                    table[j]["filter_begin"] = pos
                    table[j]["filter_end"] = pos + len(r)
                    parts.append(np.asarray(r, dtype=np.uint32))
                    pos += len(r)
            if parts:
                rows = np.concatenate(parts)
        with torch.cuda.stream(slot.stream):
            slot.q_dev[:m].copy_(slot.q_pin[:m], non_blocking=True)
            slot.ctx.search_requests(slot.q_dev.data_ptr(), m, table, rows, self.k_max,
                                     slot.ids_dev.data_ptr(), slot.d_dev.data_ptr(), slot.c_dev.data_ptr())
            slot.ids_pin[:m].copy_(slot.ids_dev[:m], non_blocking=True)
            slot.d_pin[:m].copy_(slot.d_dev[:m], non_blocking=True)
            slot.c_pin[:m].copy_(slot.c_dev[:m], non_blocking=True)
            slot.event.record(slot.stream)
        slot.begin, slot.end, slot.batch_no = a, b, batch_no

    def run(self, w: Workload, realtime: bool = True) -> Served:
        """Serves all requests of `w`; with `realtime` each request is admitted only once the
        clock has reached its arrival time, else all are queued at time 0."""
        n = len(w)
        assert np.all(np.diff(w.arrival) >= 0), "requests must be sorted by arrival"
        arrival = w.arrival if realtime else np.zeros(n)
        ids = np.empty((n, self.k_max), np.uint32)
        ds = np.empty((n, self.k_max), np.float32)
        cnt = np.empty(n, np.uint32)
        lat = np.empty(n, np.float64)
        bno = np.empty(n, np.int32)
        head = done = batch_no = 0
        t0 = time.perf_counter()
        while done < n:
            now = time.perf_counter() - t0
            avail = int(np.searchsorted(arrival, now, side="right")) if realtime else n
            for s in self.slots:
                if s.end > s.begin and s.event.query():
                    t_done = time.perf_counter() - t0
                    a, b = s.begin, s.end
                    ids[a:b] = s.ids_pin.numpy()[:b - a].view(np.uint32)
                    ds[a:b] = s.d_pin.numpy()[:b - a]
                    cnt[a:b] = s.c_pin.numpy()[:b - a].view(np.uint32)
                    lat[a:b] = t_done - arrival[a:b]
                    bno[a:b] = s.batch_no
                    done += b - a
                    s.begin = s.end = 0
            for s in self.slots:
                if s.end == s.begin and head < avail:
                    m = self._admit(w, head, avail)
                    self._launch(s, w, head, head + m, batch_no)
                    head += m
                    batch_no += 1
            if realtime and head == avail and head < n and all(s.end == s.begin for s in self.slots):
                wait = arrival[head] - (time.perf_counter() - t0)
                if wait > 2e-4:
                    time.sleep(wait - 1e-4)
        wall = time.perf_counter() - t0 - (float(arrival[0]) if n else 0.0)
        return Served(ids, ds, cnt, lat, bno, wall)

    def close(self):
        for s in self.slots:
            s.close()


def make_filters(index: compiled.PDXIndex, n_filters: int, seed: int = 5,
                 selectivity=(0.001, 0.5)) -> List[int]:
    """Registers `n_filters` random row-id filters of log-uniform selectivity."""
    rng = np.random.default_rng([seed, 7])
    n_rows = index.get_num_embeddings()
    ids = []
    for _ in range(n_filters):
        sel = float(np.exp(rng.uniform(np.log(selectivity[0]), np.log(selectivity[1]))))
        m = max(1, int(sel * n_rows))
        rows = np.sort(rng.choice(n_rows, size=m, replace=False)).astype(np.uint64)
        ids.append(index.register_filter(rows))
    return ids


def poisson_mix(queries: np.ndarray, rate: float, filters: List[int], seed: int = 5,
                ks=(10, 20, 100), nprobes=(8, 32, 64), filtered: float = 0.5) -> Workload:
    """The serving mix: Poisson arrivals at `rate` requests/s; k and nprobe uniform over the
    given sets; a share `filtered` of requests carries one of the registered `filters`."""
    rng = np.random.default_rng(seed)
    n = len(queries)
    arrival = np.cumsum(rng.exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    k = rng.choice(np.asarray(ks, np.uint32), n)
    npb = rng.choice(np.asarray(nprobes, np.uint32), n)
    fid = np.full(n, -1, np.int32)
    if filters:
        has = rng.random(n) < filtered
        fid[has] = rng.choice(np.asarray(filters, np.int32), int(has.sum()))
    return Workload(arrival, np.ascontiguousarray(queries, np.float32), k.astype(np.uint32),
                    npb.astype(np.uint32), fid)
