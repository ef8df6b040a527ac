"""CPU-only consistency checks of the oracle, the CPU baseline and the
workload generators (no GPU)."""
import numpy as np

from oracle import oracle as O
from openfpm_data_b200 import workloads as W


def _random_points(rng, n, size):
    return rng.integers(0, size, size=(n, 3)).astype(np.int64)


def test_flush_points_equals_chunk_slot_flush():
    """The point-level flush equals the reference's chunk-slot flush
    (every insert<p> owns one chunk slot with one mask bit set)."""
    rng = np.random.default_rng(3)
    size = (32, 32, 32)
    for op in (O.OP_ADD, O.OP_RIGHT, O.OP_LEFT, O.OP_MAX):
        a = O.OracleGrid(size, edge=4, ptypes=[O.T_F32])
        b = O.OracleGrid(size, edge=4, ptypes=[O.T_F32])
        for it in range(3):
            pts = _random_points(rng, 400, size)
            pts = np.concatenate([pts, pts[:100]])
            v = rng.random(len(pts)).astype(np.float32)
            lin = a.lin_ids(pts)
            a.flush_points(lin, [v], [op])
            sd = np.zeros(len(pts) * 64, np.float32)
            sm = np.zeros(len(pts) * 64, np.uint8)
            sd[np.arange(len(pts)) * 64 + lin % 64] = v
            sm[np.arange(len(pts)) * 64 + lin % 64] = 1
            b.flush_chunks(lin // 64, [sd], sm, [op])
            ka, (da,), ma = a.export()
            kb, (db,), mb = b.export()
            assert np.array_equal(ka, kb) and np.array_equal(ma, mb)
            ex = (ma & 1).astype(bool)
            assert np.array_equal(da[ex], db[ex])


def test_sright_keeps_existing_value():
    """sRight_ reduces op(new, old) = old for a point that already exists."""
    g = O.OracleGrid((16, 16, 16), edge=8, ptypes=[O.T_F32])
    p = np.array([[1, 2, 3], [4, 5, 6]])
    g.insert_flush(p, [np.array([1.0, 2.0], np.float32)], [O.OP_RIGHT])
    g.insert_flush(np.array([[1, 2, 3], [1, 2, 3], [7, 7, 7]]), [np.array([5.0, 6.0, 9.0], np.float32)], [O.OP_RIGHT])
    assert list(g.get(0, np.array([[1, 2, 3], [4, 5, 6], [7, 7, 7]]))) == [1.0, 2.0, 9.0]
    g2 = O.OracleGrid((16, 16, 16), edge=8, ptypes=[O.T_F32])
    g2.insert_flush(np.array([[1, 2, 3], [1, 2, 3]]), [np.array([5.0, 6.0], np.float32)], [O.OP_RIGHT])
    assert g2.get(0, np.array([[1, 2, 3]]))[0] == 6.0  # last insert wins inside one flush


def test_nnfull_low_face_wrap():
    """grid_smb::BlockLinId checks only the upper bound: the NNFull -x
    neighbour of a chunk at block x = 0 is the last chunk of the previous row."""
    g = O.OracleGrid((32, 32, 32), edge=8, ptypes=[O.T_F32])
    g.insert_flush(np.array([[0, 8, 0], [31, 0, 0]]), [np.ones(2, np.float32)], [O.OP_MAX])
    nn = g.find_neighbours(O.NN_FULL)
    keys = g.export()[0]
    i = int(np.searchsorted(keys, 4))      # block (0,1,0) -> id 4
    j = int(np.searchsorted(keys, 3))      # block (3,0,0) -> id 3
    assert nn[i, 0 + 3 * 1 + 9 * 1] == j    # dx=-1, dy=0, dz=0 wraps to (3,0,0)
    assert g.find_neighbours(O.NN_STAR)[i, 0] == len(keys)  # NNStar checks dpos < 0


def test_cpu_baseline_matches_oracle():
    ps = W.gray_scott(size=48, nballs=3, rmin=5.0, rmax=10.0, seed=2)
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    o = O.OracleGrid(ps.size, edge=8, ptypes=[O.T_F32] * 4)
    for p in range(4):
        o.set_background(p, ps.bck[p % 2])
    o.load_map(keys, data + [d.copy() for d in data], mask)
    c = O.CpuSgrid(ps.size, 4, [1.0, 0.0, 1.0, 0.0])
    c.insert(ps.coords, ps.values + ps.values)
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    for k in range(6):
        a, b = ([0, 1], [2, 3]) if k % 2 == 0 else ([2, 3], [0, 1])
        o.gs7(a[0], a[1], b[0], b[1], *prm)
    c.gs(0, 1, 2, 3, *prm, steps=6, threads=2)
    got = c.get(0, ps.coords)
    ref = o.get(0, ps.coords)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-6)


def test_f64_oracle_close_to_f32():
    ps = W.heat_shell(size=64, r_in=10, r_out=16)
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    o = O.OracleGrid(ps.size, edge=8, ptypes=[O.T_F32, O.T_F32])
    o.load_map(keys, data + [data[0].copy()], mask)
    for k in range(20):
        o.heat7(k % 2, 1 - k % 2, 0.1)
    f = np.concatenate([data[0], np.zeros(512, np.float32)]).astype(np.float64)
    f64 = o.heat7_f64(f, 0.1, 0.0, 20)
    _, (d0, _), m = o.export()
    ex = (m & 1).astype(bool)
    assert np.max(np.abs(d0[ex] - f64[ex])) < 1e-5


def test_workloads_deterministic():
    a = W.heat_shell()
    b = W.heat_shell()
    assert len(a.coords) == 103694 and np.array_equal(a.values[0], b.values[0])
    keys, _, _ = W.build_block_map(a.coords, a.values, a.size, 8)
    assert len(keys) == 379
    p1, f1, i1 = W.insert_batch(0, npts=10000)
    p2, f2, i2 = W.insert_batch(0, npts=10000)
    assert np.array_equal(p1, p2) and np.array_equal(f1, f2) and np.array_equal(i1, i2)
    assert len(np.unique(p1, axis=0)) < len(p1)  # exact duplicates present
    e, r, s = W.batch_grids()
    assert len(e) == 256 and e.min() >= 32 and e.max() <= 384 and np.all(e % 8 == 0)
    reqs = W.requests(duration=0.05)
    assert all(q.kind in ("heat", "gs") and 32 <= q.edge <= 256 for q in reqs)


def test_threaded_oracle_steps_equal_serial_calls():
    """gs7_steps / heat7_steps share each step's chunks over threads: same bits as the serial calls."""
    ps = W.gray_scott(size=64, nballs=4, rmin=6.0, rmax=14.0, seed=3)
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]

    def grid():
        o = O.OracleGrid(ps.size, edge=8, ptypes=[O.T_F32] * 4)
        for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
            o.set_background(p, b)
        o.load_map(keys, data + [d.copy() for d in data], mask)
        return o

    a, b = grid(), grid()
    for k in range(5):
        s, d = ((0, 1), (2, 3)) if k % 2 == 0 else ((2, 3), (0, 1))
        a.gs7(s[0], s[1], d[0], d[1], *prm)
    b.gs7_steps(0, 1, 2, 3, *prm, steps=5, threads=3)
    for x, y in zip(a.export()[1], b.export()[1]):
        assert np.array_equal(x, y)
    a.heat7(0, 2, 0.1)
    a.heat7(2, 0, 0.1)
    b.heat7_steps(0, 2, 0.1, 2, threads=4)
    assert np.array_equal(a.export()[1][0], b.export()[1][0])


def test_oracle_reproduces_headline_golden_digests():
    """The oracle run here gives the digests cached in tests/golden/gs512_oracle.json for the
    first two steps of the headline Gray-Scott workload (pins the cached fixture)."""
    import json
    import os
    import sys
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    import make_gs512_golden as G
    with open(os.path.join(here, "gs512_oracle.json")) as f:
        gold = json.load(f)
    o, keys = G.oracle_grid()
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    o.gs7_steps(0, 1, 2, 3, *prm, steps=1)
    _, d, m = o.export()
    got = G.field_digest(d[2], d[3], m, len(keys))
    assert got == gold["checkpoints"]["1"]
    o.gs7_steps(2, 3, 0, 1, *prm, steps=1)
    _, d, m = o.export()
    assert G.field_digest(d[0], d[1], m, len(keys)) == gold["checkpoints"]["2"]


def test_heat_config0_fp32_within_1e5_of_fp64():
    """Config 0 (heat 128^3 shell, 100 steps): the FP32 oracle, which the GPU matches bit for bit,
    stays within 1e-5 relative of the same update in double precision at every active point."""
    ps = W.heat_shell()
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    o = O.OracleGrid(ps.size, edge=8, ptypes=[O.T_F32] * 2)
    o.load_map(keys, data + [data[0].copy()], mask)
    f64 = o.heat7_f64(data[0], W.HEAT_DT, 0.0, 100)
    o.heat7_steps(0, 1, W.HEAT_DT, 100)
    _, d, m = o.export()
    n = len(keys)
    ex = (m[: n * 512] & 1).astype(bool)
    a = d[0][: n * 512][ex].astype(np.float64)
    b = f64[: n * 512][ex]
    assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)) < 1e-5
