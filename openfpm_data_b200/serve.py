"""Continuous-batching request server for heat and Gray-Scott sparse-grid solves.

Requests (workloads.Request: kind, domain edge, balls, steps) arrive over
time.  Each arrived request is admitted when its device footprint fits the
HBM budget: its block map is built on the device (sgb_build_balls) in a
pooled staging grid, copied into the resident batch of its kind and
advanced together with every other admitted request by one persistent
launch per step (sgb_batch_step).  Between quanta of steps, finished
requests are read back (their final fields: the response), removed from
the batch and their memory returned to the budget.  Latency is measured
from the request's arrival time to the end of its read-back.

No reference counterpart: the reference has no request or batching layer.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import _lib as L
from . import workloads as W
from .grid import Batch, SparseGridGpu

HEAT_PARAMS = [W.HEAT_DT]
GS_PARAMS = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
KIND = {"heat": L.HEAT7, "gs": L.GS7}
NFIELDS = {"heat": 1, "gs": 2}


# Device bytes the batches may hold per byte of live solve state: the live
# buffers grow by half their capacity at a time (old and new both held while
# the contents are copied), and removals are compacted into a second buffer
# set, so the peak is about 3.5 times the live state.
BATCH_OVERHEAD = 3.5


def bytes_per_chunk(kind: str, bs: int = 512) -> int:
    """Device bytes charged to the budget per chunk of a request: two
    ping-pong copies of each field, the mask, the neighbour row, the key and
    the slot id, times the batches' buffer overhead."""
    return int((bs * (2 * 4 * NFIELDS[kind] + 1) + 8 * 4 + 8 + 4) * BATCH_OVERHEAD)


def balls_of(req: W.Request) -> np.ndarray:
    return np.concatenate([req.centres, req.radii[:, None]], axis=1).astype(np.float32)


@dataclass
class Done:
    rid: int
    kind: str
    t_arrival: float
    t_admit: float
    t_done: float
    points: int
    steps: int

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


@dataclass
class ServeStats:
    done: List[Done] = field(default_factory=list)
    wall: float = 0.0
    peak_bytes: int = 0
    rejected: int = 0

    def summary(self) -> dict:
        lat = np.array([d.latency for d in self.done]) if self.done else np.zeros(1)
        pts = sum(d.points * d.steps for d in self.done)
        return {"completed": len(self.done), "wall_s": round(self.wall, 3),
                "solves_per_s": round(len(self.done) / max(self.wall, 1e-9), 2),
                "p50_latency_ms": round(float(np.percentile(lat, 50)) * 1e3, 2),
                "p99_latency_ms": round(float(np.percentile(lat, 99)) * 1e3, 2),
                "gpts_per_s": round(pts / max(self.wall, 1e-9) / 1e9, 3),
                "peak_resident_bytes": int(self.peak_bytes), "rejected": self.rejected}


class Server:
    """Admission by HBM budget + continuous batching over two resident batches."""

    def __init__(self, budget_bytes: float = 150e9, quantum: int = 25, device: int = 0, use_graph: bool = True,
                 ctas_per_sm: int = 0, stages: int = 0, keep_results: bool = False):
        self.budget = int(budget_bytes)
        self.quantum = quantum
        self.device = device
        self.use_graph = use_graph
        self.keep_results = keep_results
        self.batches: Dict[str, Batch] = {k: Batch(device) for k in KIND}
        if ctas_per_sm or stages:
            for b in self.batches.values():
                b.set_launch_config(ctas_per_sm, stages)
        self.pool: Dict[tuple, SparseGridGpu] = {}
        self.used = 0
        self.active: Dict[tuple, tuple] = {}
        self.results: Dict[int, list] = {}

    def _staging(self, kind: str, edge: int) -> SparseGridGpu:
        key = (kind, edge)
        g = self.pool.get(key)
        if g is None:
            nf = NFIELDS[kind]
            g = SparseGridGpu((edge,) * 3, ["f32"] * (2 * nf), edge=8, device=self.device)
            if kind == "gs":
                for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
                    g.setBackgroundValue(p, b)
            self.pool[key] = g
        return g

    @staticmethod
    def estimate_bytes(req: W.Request) -> int:
        """Upper bound of a request's resident bytes from its balls' bounding boxes."""
        chunks = 0
        for c, r in zip(req.centres, req.radii):
            lo = np.maximum(np.floor((c - r) / 8), 0)
            hi = np.minimum(np.floor((c + r) / 8), (req.edge - 1) // 8)
            chunks += int(np.prod(np.maximum(hi - lo + 1, 0)))
        chunks = min(chunks, (req.edge // 8) ** 3)
        return chunks * bytes_per_chunk(req.kind)

    def admit(self, req: W.Request, now: float) -> bool:
        est = self.estimate_bytes(req)
        if self.used + est > self.budget:
            return False
        g = self._staging(req.kind, req.edge)
        nf = NFIELDS[req.kind]
        init = 0 if req.kind == "heat" else 1
        g.build_balls(balls_of(req), init, req.vseed, list(range(nf)))
        src, dst = list(range(nf)), list(range(nf, 2 * nf))
        prm = HEAT_PARAMS if req.kind == "heat" else GS_PARAMS
        b = self.batches[req.kind]
        try:
            slot = b.add(g, KIND[req.kind], src, dst, prm, req.steps)
        except L.SgbError as e:
            if e.status != L.ENOMEM:
                raise
            return False  # the device is fuller than the budget says: retry once memory is returned
        n = g.nchunks
        used = n * bytes_per_chunk(req.kind)
        self.used += used
        self.active[(req.kind, slot)] = (req, now, used, n, g.countExistingElements())
        return True

    def retire(self, now_fn, stats: ServeStats) -> None:
        for key in list(self.active):
            kind, slot = key
            req, t_admit, used, n, points = self.active[key]
            b = self.batches[kind]
            if b.slot_steps(slot) < req.steps:
                continue
            # the response: the request's block map and final fields, read into pinned host memory
            keys, mask, fields = b.read(slot, NFIELDS[kind], staged=not self.keep_results)
            if self.keep_results:
                self.results[req.rid] = [keys, mask, fields]
            b.remove(slot)
            self.used -= used
            del self.active[key]
            stats.done.append(Done(req.rid, kind, req.t_arrival, t_admit, now_fn(), points, req.steps))

    def run(self, reqs: List[W.Request], realtime: bool = True, time_limit: Optional[float] = None) -> ServeStats:
        """Serve a request list.  realtime=True releases requests at their
        arrival times (open loop); otherwise all are available at t = 0."""
        stats = ServeStats()
        pending = deque(sorted(reqs, key=lambda r: r.t_arrival))
        t0 = time.perf_counter()
        now_fn = lambda: time.perf_counter() - t0  # noqa: E731
        while pending or self.active:
            now = now_fn()
            if time_limit is not None and now > time_limit:
                break
            while pending and (not realtime or pending[0].t_arrival <= now):
                if not self.admit(pending[0], now):
                    if not self.active:  # cannot ever fit
                        stats.rejected += 1
                        pending.popleft()
                        continue
                    break
                pending.popleft()
            stats.peak_bytes = max(stats.peak_bytes, self.used)
            if not self.active:
                if pending:
                    time.sleep(max(0.0, min(pending[0].t_arrival - now_fn(), 0.002)))
                continue
            for kind, b in self.batches.items():
                if any(k == kind for k, _ in self.active):
                    b.step(self.quantum, use_graph=self.use_graph)
            self.retire(now_fn, stats)
        stats.wall = now_fn()
        return stats

    def close(self):
        for g in self.pool.values():
            g.close()
        for b in self.batches.values():
            b.close()


def solve_alone(req: W.Request, device: int = 0, use_graph: bool = False):
    """One request on its own grid with plain per-grid launches (the
    non-batched baseline); returns (keys, mask, fields)."""
    nf = NFIELDS[req.kind]
    g = SparseGridGpu((req.edge,) * 3, ["f32"] * (2 * nf), edge=8, device=device)
    if req.kind == "gs":
        for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
            g.setBackgroundValue(p, b)
    g.build_balls(balls_of(req), 0 if req.kind == "heat" else 1, req.vseed, list(range(nf)))
    prm = HEAT_PARAMS if req.kind == "heat" else GS_PARAMS
    a, b = list(range(nf)), list(range(nf, 2 * nf))
    if use_graph:
        fin = g.run_steps(KIND[req.kind], a, b, prm, req.steps, use_graph=True)
    else:  # one applyStencils launch per step
        for k in range(req.steps):
            g.applyStencils(KIND[req.kind], a if k % 2 == 0 else b, b if k % 2 == 0 else a, prm)
        fin = req.steps % 2 == 1
    keys, data, mask = g.deviceToHost()
    n = len(keys)
    off = nf if fin else 0
    fields = [data[off + j][: n * 512] for j in range(nf)]
    g.close()
    return keys, mask[: n * 512], fields
