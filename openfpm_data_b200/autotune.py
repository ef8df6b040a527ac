"""Launch autotuner for the batched stencil step.

Candidates: chunk edge 8 (pipelined kernel: one 32-thread warp per
512-point chunk, each warp with its own staging ring, 2-6 CTAs of two warps
per SM or the automatic choice -1, ring depth 3, 4 or the automatic depth
-1) and chunk edge 4
(one-chunk-per-CTA tile kernel: 256 threads per 64-point chunk).  Each
candidate runs a few timed batch steps (CUDA events) on a sample of the
grids, rebuilt with its chunk edge; the fastest per active point wins.
"""
from __future__ import annotations

import itertools
import time
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np
import torch

from . import _lib as L
from .grid import Batch, SparseGridGpu


@dataclass
class Spec:
    edge: int                 # domain edge (cubic domain)
    balls: np.ndarray         # [k, 4] cx, cy, cz, r
    init: int                 # 0 heat-style uniform, 1 Gray-Scott
    seed: int


@dataclass
class TuneResult:
    chunk_edge: int
    ctas_per_sm: int
    stages: int
    threads_per_chunk: int
    ns_per_point_step: float
    table: list


def build_batch(specs: Sequence[Spec], kind: int, params, nsteps: int, chunk_edge: int, device: int = 0):
    nf = 2 if kind == L.GS7 else 1
    b = Batch(device)
    pts = 0
    staging = {}
    for sp in specs:
        g = staging.get(sp.edge)
        if g is None:
            g = SparseGridGpu((sp.edge,) * 3, ["f32"] * (2 * nf), edge=chunk_edge, device=device)
            if kind == L.GS7:
                for p, v in enumerate([1.0, 0.0, 1.0, 0.0]):
                    g.setBackgroundValue(p, v)
            staging[sp.edge] = g
        g.build_balls(sp.balls, sp.init, sp.seed, list(range(nf)))
        pts += g.countExistingElements()
        b.add(g, kind, list(range(nf)), list(range(nf, 2 * nf)), params, nsteps)
    for g in staging.values():
        g.close()
    return b, pts


def _time_steps(b: Batch, steps: int) -> float:
    b.step(2, use_graph=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.step(steps, use_graph=False)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3


def autotune(specs: Sequence[Spec], kind: int, params, steps: int = 10, device: int = 0,
             ctas=(-1, 4, 6, 8), stages=(-1, 3, 4), edges=(8, 4)) -> TuneResult:
    table = []
    best = None
    for ce in edges:
        b, pts = build_batch(specs, kind, params, 10 ** 9, ce, device)
        cands = list(itertools.product(ctas, stages)) if ce == 8 else [(0, 0)]
        for c, s in cands:
            if c:
                b.set_launch_config(c, s)
            t = _time_steps(b, steps)
            nsps = t / steps / max(pts, 1) * 1e9
            # 8^3: one consumer warp per chunk in the pipelined kernel; 4^3: one 256-thread CTA per chunk
            row = {"chunk_edge": ce, "ctas_per_sm": c, "stages": s, "threads_per_chunk": 32 if ce == 8 else 256,
                   "ns_per_point_step": round(nsps, 5)}
            table.append(row)
            if best is None or nsps < best["ns_per_point_step"]:
                best = row
        b.close()
    return TuneResult(best["chunk_edge"], best["ctas_per_sm"], best["stages"], best["threads_per_chunk"],
                      best["ns_per_point_step"], table)
