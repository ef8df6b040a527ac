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
    """Admission by HBM budget + continuous batching over two resident batches.

    The loop never waits for a quantum it has just launched: each kind's batch
    steps on its own stream (heat and Gray-Scott quanta run concurrently), new
    requests are built on a third stream and joined to their batch by a stream
    dependency, and finished requests are read back asynchronously into pinned
    memory behind the quantum that finished them; the host collects them by
    polling their completion events.  At most `depth` quanta per kind are
    queued ahead of the GPU, so a newly admitted request waits for at most
    that many quanta before its first step."""

    def __init__(self, budget_bytes: float = 150e9, quantum: int = 25, device: int = 0, use_graph: bool = True,
                 ctas_per_sm: int = 0, stages: int = 0, keep_results: bool = False, depth: int = 2):
        import torch
        self.budget = int(budget_bytes)
        self.quantum = quantum
        self.device = device
        self.use_graph = use_graph
        self.keep_results = keep_results
        self.depth = max(1, int(depth))
        self.batches: Dict[str, Batch] = {k: Batch(device) for k in KIND}
        if ctas_per_sm or stages:
            for b in self.batches.values():
                b.set_launch_config(ctas_per_sm, stages)
        self.streams = {k: torch.cuda.Stream(device=device) for k in KIND}
        self.admit_stream = torch.cuda.Stream(device=device)
        # staging grids per (kind, edge): [grid, event after the batch copied it (None: free)]
        self.pool: Dict[tuple, list] = {}
        self.used = 0
        self.active: Dict[tuple, tuple] = {}
        self.reading: list = []
        self.results: Dict[int, list] = {}

    def _staging(self, kind: str, edge: int) -> list:
        entries = self.pool.setdefault((kind, edge), [])
        for ent in entries:
            if ent[1] is None or ent[1].query():
                return ent
        nf = NFIELDS[kind]
        g = SparseGridGpu((edge,) * 3, ["f32"] * (2 * nf), edge=8, device=self.device)
        if kind == "gs":
            for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
                g.setBackgroundValue(p, b)
        ent = [g, None]
        entries.append(ent)
        return ent

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
        import torch
        est = self.estimate_bytes(req)
        if self.used + est > self.budget:
            return False
        ent = self._staging(req.kind, req.edge)
        g = ent[0]
        nf = NFIELDS[req.kind]
        init = 0 if req.kind == "heat" else 1
        # the scene is built on the admission stream (its chunk count is read back there, without
        # waiting for the quanta in flight); the batch copies it on its own stream after that
        g.build_balls(balls_of(req), init, req.vseed, list(range(nf)), stream=self.admit_stream)
        cs = self.streams[req.kind]
        cs.wait_stream(self.admit_stream)
        src, dst = list(range(nf)), list(range(nf, 2 * nf))
        prm = HEAT_PARAMS if req.kind == "heat" else GS_PARAMS
        b = self.batches[req.kind]
        try:
            slot = b.add(g, KIND[req.kind], src, dst, prm, req.steps, stream=cs)
        except L.SgbError as e:
            if e.status != L.ENOMEM:
                raise
            return False  # the device is fuller than the budget says: retry once memory is returned
        ev = torch.cuda.Event()
        ev.record(cs)
        ent[1] = ev  # the staging grid may be rebuilt once the batch has copied it
        n = g.nchunks
        used = n * bytes_per_chunk(req.kind)
        self.used += used
        self.active[(req.kind, slot)] = (req, now, used, n)
        return True

    def _start_reads(self) -> None:
        """Queue the read-back of every request whose steps are all launched, behind those steps."""
        for key in list(self.active):
            kind, slot = key
            req, t_admit, used, n = self.active[key]
            b = self.batches[kind]
            if b.slot_steps(slot) < req.steps:
                continue
            data = b.read_async(slot, NFIELDS[kind], stream=self.streams[kind])
            self.reading.append((req, kind, slot, used, t_admit, data))
            del self.active[key]

    def _collect(self, now_fn, stats: ServeStats) -> None:
        """Finish the requests whose read-back has completed: the response is in host memory."""
        still = []
        for item in self.reading:
            req, kind, slot, used, t_admit, (keys, mask, fields, ev) = item
            if not ev.query():
                still.append(item)
                continue
            t_done = now_fn()
            if self.keep_results:
                self.results[req.rid] = [keys.copy(), mask.copy(), [f.copy() for f in fields]]
            points = int(np.count_nonzero(mask & 1))
            self.batches[kind].remove(slot)
            self.used -= used
            stats.done.append(Done(req.rid, kind, req.t_arrival, t_admit, t_done, points, req.steps))
        self.reading = still

    def run(self, reqs: List[W.Request], realtime: bool = True, time_limit: Optional[float] = None) -> ServeStats:
        """Serve a request list.  realtime=True releases requests at their
        arrival times (open loop); otherwise all are available at t = 0."""
        import torch
        stats = ServeStats()
        pending = deque(sorted(reqs, key=lambda r: r.t_arrival))
        queued = {k: deque() for k in KIND}  # events after each kind's quanta in flight
        t0 = time.perf_counter()
        now_fn = lambda: time.perf_counter() - t0  # noqa: E731
        while pending or self.active or self.reading:
            now = now_fn()
            if time_limit is not None and now > time_limit:
                break
            self._collect(now_fn, stats)
            while pending and (not realtime or pending[0].t_arrival <= now):
                if not self.admit(pending[0], now):
                    if not self.active and not self.reading:  # cannot ever fit
                        stats.rejected += 1
                        pending.popleft()
                        continue
                    break
                pending.popleft()
            stats.peak_bytes = max(stats.peak_bytes, self.used)
            launched = False
            for kind, b in self.batches.items():
                if not any(k == kind for k, _ in self.active):
                    continue
                q = queued[kind]
                while len(q) >= self.depth:  # keep at most `depth` quanta queued ahead of the GPU
                    q.popleft().synchronize()
                b.step(self.quantum, use_graph=self.use_graph, stream=self.streams[kind])
                ev = torch.cuda.Event()
                ev.record(self.streams[kind])
                q.append(ev)
                launched = True
            self._start_reads()
            if not launched:
                if self.reading:
                    time.sleep(0.0002)
                elif pending:
                    time.sleep(max(0.0, min(pending[0].t_arrival - now_fn(), 0.002)))
        for q in queued.values():
            for ev in q:
                ev.synchronize()
        stats.wall = now_fn()
        return stats

    def close(self):
        import torch
        torch.cuda.synchronize(self.device)
        for entries in self.pool.values():
            for g, _ in entries:
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
