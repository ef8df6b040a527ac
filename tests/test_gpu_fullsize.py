"""Parity at full size and of the batched / served forms against the CPU oracle.

* The headline workload itself (Gray-Scott, 512^3 domain, 8^3 chunks, 40
  balls, seed 1: what bench.py times) through sgb_run_steps, checked after 1,
  2, 100 and 1000 steps against the oracle's digests cached in
  tests/golden/gs512_oracle.json (made by tests/golden/make_gs512_golden.py).
  Equal digests mean bit-identical u and v at every existing point.  Should a
  digest differ at 1, 2 or 100 steps, the oracle is run here to that step and
  the fields must agree within RTOL = 1e-6 relative.
* Batches of heat and Gray-Scott grids (8^3 and 4^3 chunks) and a served mix
  of requests: every grid's result against the oracle run on the same initial
  state for the same number of steps (the fixed-function FP32 arithmetic is
  restated exactly, so the comparison is bit for bit).
* The autotuner: its choice is one of its candidates and the batch it builds
  gives the oracle's results.
"""
import hashlib
import json
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from openfpm_data_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL = 1e-6
HERE = os.path.dirname(os.path.abspath(__file__))
GS_PRM = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]


@pytest.fixture(scope="module")
def sgb():
    import openfpm_data_b200 as m
    assert torch.cuda.is_available(), "these tests need a CUDA device"
    m.load()
    return m


def _digest(u, v, mask, n, bs=512):
    ex = (mask[: n * bs] & 1).astype(bool)
    uu = np.ascontiguousarray(u[: n * bs][ex], dtype=np.float32)
    vv = np.ascontiguousarray(v[: n * bs][ex], dtype=np.float32)
    return hashlib.sha256(uu.tobytes()).hexdigest(), hashlib.sha256(vv.tobytes()).hexdigest(), uu, vv


def _close(a, b, what):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    err = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
    err[a == b] = 0
    assert np.all(err <= RTOL), f"{what}: max rel err {err.max():.3e}"


def test_gray_scott_512_headline_matches_oracle(sgb):
    with open(os.path.join(HERE, "golden", "gs512_oracle.json")) as f:
        gold = json.load(f)
    ps = W.gray_scott()
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    n = len(keys)
    assert n == gold["chunks"]
    g = sgb.SparseGridGpu(ps.size, ["f32"] * 4, edge=8)
    for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
        g.setBackgroundValue(p, b)
    g.load_map(keys, data + [d.copy() for d in data], mask)
    done = 0
    for cp in (1, 2, 100, 1000):
        src, dst = ([0, 1], [2, 3]) if done % 2 == 0 else ([2, 3], [0, 1])
        g.run_steps(sgb.GS7, src, dst, GS_PRM, cp - done, use_graph=False)
        done = cp
        _, d, m = g.deviceToHost()
        fu, fv = (2, 3) if done % 2 == 1 else (0, 1)
        hu, hv, uu, vv = _digest(d[fu], d[fv], m, n)
        ref = gold["checkpoints"][str(cp)]
        assert int(uu.size) == ref["points"] == len(ps.coords)
        if (hu, hv) == (ref["u_sha256"], ref["v_sha256"]):
            continue  # bit-identical to the oracle
        assert cp != 1000, f"step 1000 differs from the oracle's digest (u sum {uu.sum()} vs {ref['u_sum']})"
        o = O.OracleGrid(ps.size, edge=8, ptypes=[O.T_F32] * 4)
        for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
            o.set_background(p, b)
        o.load_map(keys, data + [x.copy() for x in data], mask)
        o.gs7_steps(0, 1, 2, 3, *GS_PRM, steps=cp)
        _, od, om = o.export()
        _, _, ou, ov = _digest(od[fu], od[fv], om, n)
        _close(uu, ou, f"u after {cp} steps")
        _close(vv, ov, f"v after {cp} steps")
    g.check_device_errors()
    g.close()


# ------------------------------------------------------------------ batches against the oracle
def _oracle_solve(keys, data, mask, size, edge, kind, nsteps, bcks):
    """The oracle run of one grid: data holds the src fields (1 heat, 2 Gray-Scott) of n chunks."""
    nf = len(data)
    o = O.OracleGrid(size, edge=edge, ptypes=[O.T_F32] * (2 * nf))
    for p, b in enumerate(bcks + bcks):
        o.set_background(p, b)
    o.load_map(keys, list(data) + [d.copy() for d in data], mask)
    if kind == "heat":
        o.heat7_steps(0, 1, W.HEAT_DT, nsteps)
    else:
        o.gs7_steps(0, 1, 2, 3, *GS_PRM, steps=nsteps)
    _, od, om = o.export()
    off = nf if nsteps % 2 == 1 else 0
    n = len(keys)
    bs = edge ** 3
    return [od[off + j][: n * bs] for j in range(nf)], om[: n * bs]


def _grid_from_balls(sgb, kind, edge_dom, balls, seed, chunk_edge):
    nf = 1 if kind == "heat" else 2
    g = sgb.SparseGridGpu((edge_dom,) * 3, ["f32"] * (2 * nf), edge=chunk_edge)
    bcks = [0.0] if kind == "heat" else [1.0, 0.0]
    for p, b in enumerate(bcks + bcks):
        g.setBackgroundValue(p, b)
    g.build_balls(balls, 0 if kind == "heat" else 1, seed, list(range(nf)))
    return g, bcks


@pytest.mark.parametrize("chunk_edge", [8, 4])
def test_batch_matches_oracle(sgb, chunk_edge):
    """Heat and Gray-Scott grids of different sizes and step counts in one batch each: every
    grid's final fields equal the oracle's for its own step count."""
    rng = np.random.default_rng(23)
    cases = []
    for kind in ("heat", "gs"):
        b = sgb.Batch()
        grids = []
        for j, (dom, nsteps) in enumerate([(40, 9), (64, 14), (24, 5), (88, 14)]):
            nb = 1 + j % 3
            balls = np.concatenate([rng.uniform(0, dom, (nb, 3)), rng.uniform(0.15, 0.4, (nb, 1)) * dom], 1)
            g, bcks = _grid_from_balls(sgb, kind, dom, balls.astype(np.float32), 100 + j, chunk_edge)
            keys, data, mask = g.deviceToHost()
            nf = len(bcks)
            n = len(keys)
            bs = chunk_edge ** 3
            init = ([d[: n * bs].copy() for d in data[:nf]], mask[: n * bs].copy(), keys.copy())
            prm = [W.HEAT_DT] if kind == "heat" else GS_PRM
            kk = sgb.HEAT7 if kind == "heat" else sgb.GS7
            slot = b.add(g, kk, list(range(nf)), list(range(nf, 2 * nf)), prm, nsteps)
            grids.append((slot, dom, nsteps, init, bcks, g))
        b.step(14)
        for slot, dom, nsteps, (d0, m0, k0), bcks, g in grids:
            assert b.slot_steps(slot) == nsteps
            keys, mask, fields = b.read(slot, len(bcks), bs=chunk_edge ** 3)
            assert np.array_equal(keys, k0) and np.array_equal(mask, m0)
            ref, om = _oracle_solve(k0, d0, m0, (dom,) * 3, chunk_edge, kind, nsteps, bcks)
            ex = (m0 & 1).astype(bool)
            for a, r in zip(fields, ref):
                assert np.array_equal(a[ex].view(np.uint32), r[ex].view(np.uint32)), \
                    f"{kind} grid {dom}^3 ({nsteps} steps, edge {chunk_edge}) differs from the oracle"
            cases.append((kind, dom))
            g.close()
        b.close()
    assert len(cases) == 8


def test_served_mix_matches_oracle(sgb):
    """Requests served in a continuous-batching mix (arrivals interleaved with steps): each
    response equals the oracle's solve of the same request alone."""
    from openfpm_data_b200 import serve
    reqs = W.requests(rate=2000.0, duration=0.01, seed=41, emin=32, emax=64, steps=(6, 40))
    assert len(reqs) >= 6 and {r.kind for r in reqs} == {"heat", "gs"}
    srv = serve.Server(budget_bytes=48e6, quantum=5, keep_results=True)
    st = srv.run(reqs, realtime=False)
    assert len(st.done) == len(reqs)
    for r in reqs:
        keys, mask, fields = srv.results[r.rid]
        g, bcks = _grid_from_balls(sgb, r.kind, r.edge, serve.balls_of(r), r.vseed, 8)
        k0, d0, m0 = g.deviceToHost()
        n = len(k0)
        nf = len(bcks)
        g.close()
        assert np.array_equal(keys, k0) and np.array_equal(mask, m0[: n * 512])
        ref, _ = _oracle_solve(k0, [d[: n * 512] for d in d0[:nf]], m0[: n * 512], (r.edge,) * 3, 8, r.kind,
                               r.steps, bcks)
        ex = (mask & 1).astype(bool)
        for a, c in zip(fields, ref):
            assert np.array_equal(a[ex].view(np.uint32), c[ex].view(np.uint32)), \
                f"request {r.rid} ({r.kind}, {r.steps} steps) differs from the oracle"
    srv.close()


def test_autotune_choice_runs_and_matches_oracle(sgb):
    from openfpm_data_b200 import autotune as A
    edges, radii, seeds = W.batch_grids(6, emin=32, emax=96, seed=3)
    specs = [A.Spec(int(e), np.array([[e / 2.0, e / 2.0, e / 2.0, r]], np.float32), 0, int(s))
             for e, r, s in zip(edges, radii, seeds)]
    tune = A.autotune(specs, sgb.HEAT7, [W.HEAT_DT], steps=3, ctas=(-1, 4), stages=(-1, 3))
    assert tune.chunk_edge in (4, 8)
    assert {r["chunk_edge"] for r in tune.table} == {4, 8}
    assert any(r["chunk_edge"] == tune.chunk_edge and r["ctas_per_sm"] == tune.ctas_per_sm and
               r["stages"] == tune.stages for r in tune.table)
    b, pts = A.build_batch(specs[:3], sgb.HEAT7, [W.HEAT_DT], 6, tune.chunk_edge, 0)
    if tune.ctas_per_sm:
        b.set_launch_config(tune.ctas_per_sm, tune.stages)
    b.step(6)
    bs = tune.chunk_edge ** 3
    for slot, sp in enumerate(specs[:3]):
        g, bcks = _grid_from_balls(sgb, "heat", sp.edge, sp.balls, sp.seed, tune.chunk_edge)
        k0, d0, m0 = g.deviceToHost()
        n = len(k0)
        g.close()
        keys, mask, fields = b.read(slot, 1, bs=bs)
        assert np.array_equal(keys, k0)
        ref, _ = _oracle_solve(k0, [d0[0][: n * bs]], m0[: n * bs], (sp.edge,) * 3, tune.chunk_edge, "heat", 6, bcks)
        ex = (mask & 1).astype(bool)
        assert np.array_equal(fields[0][ex].view(np.uint32), ref[0][ex].view(np.uint32))
    b.close()
