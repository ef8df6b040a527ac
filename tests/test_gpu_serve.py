"""Scene builder, batched form and served form on the GPU."""
import numpy as np
import pytest
import torch

from openfpm_data_b200 import workloads as W

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def _splitmix(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def _hash_unit(seed, lin, stream):
    """Host restatement of the builder's counter-based generator."""
    base = _splitmix((seed ^ ((stream * 0xD1B54A32D192ED03) & M64)) & M64)
    return np.array([(_splitmix(base ^ int(l)) >> 40) / 16777216.0 for l in lin], dtype=np.float32)


@pytest.fixture(scope="module")
def sgb():
    import openfpm_data_b200 as m
    assert torch.cuda.is_available()
    m.load()
    return m


@pytest.mark.parametrize("edge", [8, 4])
def test_build_balls_matches_host_geometry(sgb, edge):
    size = 56
    cen = np.array([[10.3, 20.7, 30.1], [40.0, 40.0, 12.5], [0.0, 55.0, 28.0]])
    rad = np.array([9.5, 12.25, 7.0])
    g = sgb.SparseGridGpu((size,) * 3, ["f32", "f32"], edge=edge)
    g.setBackgroundValue(1, -3.0)
    g.build_balls(np.concatenate([cen, rad[:, None]], 1), 0, 1234, [0])
    occ = W.ball_mask((size,) * 3, cen, rad)
    pts = W.occupancy_points(occ)
    keys, data, mask = g.deviceToHost()
    ek, ed, em = W.build_block_map(pts, [np.zeros(len(pts), np.float32)], (size,) * 3, edge)
    assert np.array_equal(keys, ek) and np.array_equal(mask[: len(keys) * edge ** 3], em)
    bs = edge ** 3
    ex = em.astype(bool)
    slot = np.nonzero(ex)[0]
    lin = keys[slot // bs] * bs + slot % bs  # linear point id of every existing slot
    assert np.array_equal(data[0][: len(keys) * bs][ex], _hash_unit(1234, lin, 0))
    assert np.all(data[0][: len(keys) * bs][~ex] == 0.0)  # empty points hold the background
    assert np.all(data[1] == -3.0)  # other properties hold their background
    assert int(ex.sum()) == len(pts)


def test_batch_of_balls_matches_alone(sgb):
    from openfpm_data_b200.serve import solve_alone
    reqs = W.requests(rate=1000.0, duration=0.02, seed=7, emin=32, emax=64, steps=(5, 30))
    assert len(reqs) >= 8
    b = {"heat": sgb.Batch(), "gs": sgb.Batch()}
    slots = []
    from openfpm_data_b200 import serve
    for r in reqs:
        nf = serve.NFIELDS[r.kind]
        g = sgb.SparseGridGpu((r.edge,) * 3, ["f32"] * (2 * nf), edge=8)
        if r.kind == "gs":
            for p, v in enumerate([1.0, 0.0, 1.0, 0.0]):
                g.setBackgroundValue(p, v)
        g.build_balls(serve.balls_of(r), 0 if r.kind == "heat" else 1, r.vseed, list(range(nf)))
        prm = serve.HEAT_PARAMS if r.kind == "heat" else serve.GS_PARAMS
        slots.append((r, b[r.kind].add(g, serve.KIND[r.kind], list(range(nf)), list(range(nf, 2 * nf)), prm,
                                       r.steps)))
    for bb in b.values():
        bb.step(max(r.steps for r in reqs))
    for r, slot in slots:
        keys, mask, fields = b[r.kind].read(slot, serve.NFIELDS[r.kind])
        k2, m2, f2 = solve_alone(r)
        assert np.array_equal(keys, k2) and np.array_equal(mask, m2)
        for a, c in zip(fields, f2):
            assert np.array_equal(a, c), f"request {r.rid} ({r.kind}) differs in the batch"


def test_server_results_same_alone_and_in_mix(sgb):
    from openfpm_data_b200.serve import Server, solve_alone
    reqs = W.requests(rate=2000.0, duration=0.012, seed=4, emin=32, emax=72, steps=(10, 60))
    srv = Server(budget_bytes=64e6, quantum=7, keep_results=True)
    st = srv.run(reqs, realtime=False)
    assert len(st.done) == len(reqs)
    assert st.peak_bytes <= 64e6
    for r in reqs:
        keys, mask, fields = srv.results[r.rid]
        k2, m2, f2 = solve_alone(r)
        assert np.array_equal(keys, k2) and np.array_equal(mask, m2)
        for a, c in zip(fields, f2):
            assert np.array_equal(a, c), f"request {r.rid} ({r.kind}) differs alone / in the mix"
    s = st.summary()
    assert s["completed"] == len(reqs) and s["p99_latency_ms"] >= s["p50_latency_ms"]
    srv.close()


def test_server_budget_rejects_oversized(sgb):
    from openfpm_data_b200.serve import Server
    reqs = W.requests(rate=500.0, duration=0.01, seed=9, emin=32, emax=40, steps=(5, 6))
    srv = Server(budget_bytes=1e3, quantum=5)
    st = srv.run(reqs, realtime=False)
    assert st.rejected == len(reqs) and not st.done
    srv.close()
