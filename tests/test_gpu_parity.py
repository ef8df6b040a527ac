"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Integer / byte / index results (block map keys, masks, neighbour tables,
flushed values) must be bit-exact.  FP32 stencil fields are compared with a
relative tolerance of 1e-6 per step (the reference's arithmetic is restated
exactly, so in practice they are bit-identical too; the tolerance covers
flush-to-zero corner cases of the host FPU).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from openfpm_data_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL = 1e-6


@pytest.fixture(scope="module")
def sgb():
    import openfpm_data_b200 as m
    assert torch.cuda.is_available(), "these tests need a CUDA device"
    m.load()
    return m


def _npt(t):
    return {O.T_F32: "f32", O.T_I32: "i32", O.T_F64: "f64", O.T_U8: "u8"}[t]


def _assert_fields_close(a, b, rtol=RTOL):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    err = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
    err[(a == b)] = 0
    assert np.all(err <= rtol), f"max rel err {err.max():.3e} at {np.argmax(err)}"


def _compare_maps(g, o, props=None, exact=True):
    keys, data, mask = g.deviceToHost()
    okeys, odata, omask = o.export()
    n = len(okeys)
    assert np.array_equal(keys, okeys)
    assert np.array_equal(mask[: n * g.bs], omask[: n * g.bs])
    ex = (mask[: n * g.bs] & 1).astype(bool)
    for p in props if props is not None else range(len(data)):
        a, b = data[p][: n * g.bs][ex], odata[p][: n * g.bs][ex]
        if exact:
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"property {p} differs"
        else:
            _assert_fields_close(a, b)


def _random_points(rng, n, size, lowface=False):
    pts = rng.integers(0, size, size=(n, 3))
    if lowface:
        pts[: n // 4, rng.integers(0, 3)] = rng.integers(0, 2, size=n // 4)
    return pts.astype(np.int64)


# ------------------------------------------------------------------ flush
@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("op", ["sRight_", "sLeft_", "sadd_", "smax_", "smin_"])
def test_flush_matches_oracle(sgb, edge, op):
    rng = np.random.default_rng(11)
    size = (64, 48, 40)
    ptypes = [O.T_F32, O.T_I32, O.T_F64, O.T_U8]
    g = sgb.SparseGridGpu(size, [_npt(t) for t in ptypes], edge=edge)
    o = O.OracleGrid(size, edge=edge, ptypes=ptypes)
    for p, b in enumerate([1.5, -7, 2.25, 3]):
        g.setBackgroundValue(p, b)
        o.set_background(p, b)
    iop = O.__dict__[{"sRight_": "OP_RIGHT", "sLeft_": "OP_LEFT", "sadd_": "OP_ADD", "smax_": "OP_MAX",
                      "smin_": "OP_MIN"}[op]]
    ops = [iop, iop, iop, iop]
    for it in range(3):
        n = 5000 * (it + 1)
        pts = _random_points(rng, n, size)
        pts = np.concatenate([pts, pts[rng.integers(0, n, n // 3)]])  # exact duplicates
        vals = [rng.standard_normal(len(pts)).astype(np.float32),
                rng.integers(-1000, 1000, len(pts)).astype(np.int32),
                rng.standard_normal(len(pts)),
                rng.integers(0, 255, len(pts)).astype(np.uint8)]
        g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda() for v in vals])
        g.flush(ops)
        o.insert_flush(pts, vals, ops)
        _compare_maps(g, o)
    g.check_device_errors()


def test_flush_bitwise_or_and_unlisted(sgb):
    rng = np.random.default_rng(5)
    size = (32, 32, 32)
    g = sgb.SparseGridGpu(size, ["i32", "f32"], edge=8)
    o = O.OracleGrid(size, edge=8, ptypes=[O.T_I32, O.T_F32])
    for it in range(3):
        pts = _random_points(rng, 3000, size)
        vals = [rng.integers(0, 1 << 20, len(pts)).astype(np.int32), rng.random(len(pts)).astype(np.float32)]
        g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda() for v in vals])
        g.flush(["sBitwiseOr_", "smax_"])
        o.insert_flush(pts, vals, [O.OP_OR, O.OP_MAX])
        _compare_maps(g, o)


@pytest.mark.parametrize("mode", ["insert", "half"])
def test_blockmap_insert_golden_on_gpu(sgb, mode):
    """BlockMapGpu_tests.cu:126-216 through the device flush (4^3 chunks = DataBlock<float,64>)."""
    g = sgb.SparseGridGpu((64, 64, 64), ["f32"], edge=4)
    g.setBackgroundValue(0, 666.0)
    pos = np.arange(384)
    if mode == "half":
        pos = pos[(pos % 128) % 64 < 32]
    g.insert_lin(torch.from_numpy(pos).cuda(), [torch.from_numpy(pos.astype(np.float32)).cuda()])
    g.flush(["smax_"])
    keys, (d,), m = g.deviceToHost()
    read = np.arange(512)
    p = np.searchsorted(keys, read // 64)
    found = (p < len(keys)) & (keys[np.minimum(p, len(keys) - 1)] == read // 64)
    idx = np.where(found, p, len(keys)) * 64 + read % 64
    got = np.where(m[idx] & 1, d[idx], d[len(keys) * 64])
    exp = np.where(read < 384, read, 666).astype(np.float32)
    if mode == "half":
        exp = np.where(read % 64 < 32, exp, 666)
    assert np.array_equal(got, exp)


def test_out_of_domain_insert_is_rejected(sgb):
    g = sgb.SparseGridGpu((16, 16, 16), ["f32"], edge=8)
    pts = torch.tensor([[1, 2, 3], [16, 0, 0]], dtype=torch.int32).cuda()
    g.insert(pts, [torch.ones(2).cuda()])
    with pytest.raises(sgb.SgbError, match="outside"):
        g.flush(["smax_"])
    assert g.nchunks == 0


# ------------------------------------------------------------------ neighbours / tag
def _sparse_grid(sgb, rng, size, edge, npts, lowface=True, ptypes=(O.T_F32,)):
    pts = np.unique(_random_points(rng, npts, size, lowface=lowface), axis=0)
    vals = [rng.random(len(pts)).astype(np.float32) for _ in ptypes]
    g = sgb.SparseGridGpu(size, [_npt(t) for t in ptypes], edge=edge)
    o = O.OracleGrid(size, edge=edge, ptypes=list(ptypes))
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda() for v in vals])
    g.flush(["smax_"] * len(ptypes))
    o.insert_flush(pts, vals, [O.OP_MAX] * len(ptypes))
    return g, o, pts


@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("nn", [O.NN_STAR, O.NN_FULL])
def test_neighbour_table_matches_oracle(sgb, edge, nn):
    rng = np.random.default_rng(21)
    g, o, _ = _sparse_grid(sgb, rng, (40, 48, 56), edge, 3000)
    assert np.array_equal(g.neighbour_table(nn), o.find_neighbours(nn))


@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("nn", [O.NN_STAR, O.NN_FULL])
@pytest.mark.parametrize("density", [800, 20000])
def test_tag_boundaries_matches_oracle(sgb, edge, nn, density):
    rng = np.random.default_rng(7 + density)
    g, o, _ = _sparse_grid(sgb, rng, (48, 40, 64), edge, density)
    g.tagBoundaries(nn)
    o.tag_boundaries(nn)
    _compare_maps(g, o)
    # a second tag over already tagged masks clears / keeps bits the same way
    g.tagBoundaries(nn)
    o.tag_boundaries(nn)
    _compare_maps(g, o)


def test_tag_boundaries_2d_golden_as_slab(sgb):
    """testTagBoundaries point sets in a z-slab: NNStar in 3-D also flags z faces."""
    g = sgb.SparseGridGpu((16, 16, 8), ["f32"], edge=8)
    o = O.OracleGrid((16, 16, 8), edge=8, ptypes=[O.T_F32])
    pts = np.array([(x, y, z) for z in range(3, 6) for (x, y) in [(0, 0), (6, 6), (7, 6), (8, 6)] +
                    [(x, y) for y in range(9, 12) for x in (6, 7, 8, 9)]], dtype=np.int64)
    v = np.ones(len(pts), np.float32)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda()])
    g.flush(["smax_"])
    o.insert_flush(pts, [v], [O.OP_MAX])
    g.tagBoundaries(O.NN_STAR)
    o.tag_boundaries(O.NN_STAR)
    _compare_maps(g, o)
    assert g.countBoundaryElements() < g.countExistingElements()


# ------------------------------------------------------------------ stencils
def _load_pointset(sgb, ps, edge, nprop_extra=1, bcks=None):
    """Grid with the point set's fields followed by as many ping-pong copies
    (backgrounds `bcks` per property, default the point set's)."""
    nf = len(ps.values)
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, edge, ps.bck)
    ptypes = [O.T_F32] * (nf * 2)
    g = sgb.SparseGridGpu(ps.size, ["f32"] * (nf * 2), edge=edge)
    o = O.OracleGrid(ps.size, edge=edge, ptypes=ptypes)
    for p in range(nf * 2):
        b = ps.bck[p % nf] if bcks is None else bcks[p]
        g.setBackgroundValue(p, b)
        o.set_background(p, b)
    full = data + [d.copy() for d in data]
    g.load_map(keys, full, mask)
    o.load_map(keys, full, mask)
    return g, o


@pytest.mark.parametrize("edge", [8, 4])
def test_heat_config0_matches_oracle(sgb, edge):
    ps = W.heat_shell()
    g, o = _load_pointset(sgb, ps, edge)
    fin = g.run_steps(sgb.HEAT7, [0], [1], [W.HEAT_DT], 100, use_graph=True)
    for k in range(100):
        o.heat7(k % 2, 1 - k % 2, W.HEAT_DT)
    assert fin is False  # 100 steps end in property 0
    _compare_maps(g, o, props=[0, 1], exact=False)
    g.check_device_errors()


def test_heat_pipelined_equals_tiled(sgb):
    rng = np.random.default_rng(1)
    g1, _, pts = _sparse_grid(sgb, rng, (96, 80, 72), 8, 60000, ptypes=(O.T_F32, O.T_F32))
    keys, data, mask = g1.deviceToHost()
    g2 = sgb.SparseGridGpu((96, 80, 72), ["f32", "f32"], edge=8)
    n = len(keys)
    g2.load_map(keys, [d[: n * 512] for d in data], mask[: n * 512])
    g1.tagBoundaries()
    g2.tagBoundaries()
    for k in range(6):
        s, d = k % 2, 1 - k % 2
        g1.applyStencils(sgb.HEAT7, [s], [d], [0.1])
        g2.applyStencils(sgb.HEAT7, [s], [d], [0.1], tiled=True)
    a, b = g1.deviceToHost(), g2.deviceToHost()
    assert np.array_equal(a[1][0], b[1][0]) and np.array_equal(a[1][1], b[1][1])


@pytest.mark.parametrize("box", [None, ((5, 9, 13), (60, 70, 50))])
def test_gray_scott_pipelined_equals_tiled(sgb, box):
    """The pipelined 8^3 kernel and the one-chunk-per-CTA kernel give the same
    bits everywhere, existing points and the background-filled rest alike,
    with padding points (tagBoundaries) and a box leaving existing points
    untouched."""
    rng = np.random.default_rng(5)
    g1, _, _ = _sparse_grid(sgb, rng, (96, 80, 72), 8, 60000, ptypes=(O.T_F32,) * 4)
    keys, data, mask = g1.deviceToHost()
    g2 = sgb.SparseGridGpu((96, 80, 72), ["f32"] * 4, edge=8)
    for g in (g1, g2):
        for p, b in enumerate([1.0, 0.0, 0.5, 0.25]):
            g.setBackgroundValue(p, b)
    n = len(keys)
    g1.load_map(keys, [d[: n * 512] for d in data], mask[: n * 512])
    g2.load_map(keys, [d[: n * 512] for d in data], mask[: n * 512])
    g1.tagBoundaries()
    g2.tagBoundaries()
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    for k in range(5):
        a, b = ([0, 1], [2, 3]) if k % 2 == 0 else ([2, 3], [0, 1])
        g1.applyStencils(sgb.GS7, a, b, prm, box=box)
        g2.applyStencils(sgb.GS7, a, b, prm, box=box, tiled=True)
    x, y = g1.deviceToHost(), g2.deviceToHost()
    for p in range(4):
        assert np.array_equal(x[1][p].view(np.uint32), y[1][p].view(np.uint32)), f"property {p}"
    g1.check_device_errors()


def _small_gs(size=96, nballs=6, seed=9):
    return W.gray_scott(size=size, nballs=nballs, rmin=8.0, rmax=20.0, seed=seed)


@pytest.mark.parametrize("edge", [8, 4])
def test_gray_scott_matches_oracle(sgb, edge):
    ps = _small_gs()
    g, o = _load_pointset(sgb, ps, edge)
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    steps = 40
    for k in range(steps):
        a, b = ([0, 1], [2, 3]) if k % 2 == 0 else ([2, 3], [0, 1])
        g.applyStencils(sgb.GS7, a, b, prm)
        o.gs7(a[0], a[1], b[0], b[1], *prm)
        if k in (0, 1, steps - 1):
            _compare_maps(g, o, props=[0, 1, 2, 3], exact=False)
    g.check_device_errors()


@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("kind", ["heat", "gs"])
def test_pingpong_with_distinct_backgrounds(sgb, edge, kind):
    """Source and destination properties with different backgrounds: every
    ping-pong step must substitute the background of the buffer it reads
    (HeatStencil's storeBlock copies the source background into the
    destination's non-existing points; reads there give the destination's)."""
    if kind == "heat":
        ps = W.heat_shell()
        g, o = _load_pointset(sgb, ps, edge, bcks=[0.3, 0.9])
        fin = g.run_steps(sgb.HEAT7, [0], [1], [W.HEAT_DT], 7, use_graph=True)
        for k in range(7):
            o.heat7(k % 2, 1 - k % 2, W.HEAT_DT)
        assert fin is True
        props = [0, 1]
    else:
        ps = _small_gs(size=64, nballs=4, seed=5)
        g, o = _load_pointset(sgb, ps, edge, bcks=[1.0, 0.0, 0.75, 0.125])
        prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
        g.run_steps(sgb.GS7, [0, 1], [2, 3], prm, 7, use_graph=True)
        for k in range(7):
            a, b = ([0, 1], [2, 3]) if k % 2 == 0 else ([2, 3], [0, 1])
            o.gs7(a[0], a[1], b[0], b[1], *prm)
        props = [0, 1, 2, 3]
    _compare_maps(g, o, props=props, exact=False)
    # reads of non-existing points see each property's own background
    keys, data, mask = g.deviceToHost()
    n = len(keys)
    off = (mask[: n * g.bs] & 1) == 0
    bcks = [0.3, 0.9] if kind == "heat" else [1.0, 0.0, 0.75, 0.125]
    for p in props:
        assert np.all(data[p][: n * g.bs][off] == np.float32(bcks[p]))
    g.check_device_errors()


def test_gray_scott_launch_configs_agree(sgb):
    ps = _small_gs(size=80, nballs=5, seed=4)
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    outs = []
    for ctas, stages in [(1, 3), (2, 6), (3, 8), (4, 4), (2, 12), (8, 16)]:
        g, _ = _load_pointset(sgb, ps, 8)
        g.setLaunchConfig(ctas, stages)
        g.run_steps(sgb.GS7, [0, 1], [2, 3], prm, 9)
        outs.append(g.deviceToHost()[1])
        g.check_device_errors()
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert np.array_equal(a, b)


def test_box_restricted_stencil(sgb):
    rng = np.random.default_rng(2)
    g, o, _ = _sparse_grid(sgb, rng, (64, 64, 64), 8, 100000, ptypes=(O.T_F32, O.T_F32))
    box = ((5, 9, 13), (40, 50, 33))
    g.applyStencils(sgb.HEAT7, [0], [1], [0.05], box=box)
    o.heat7(0, 1, 0.05, box=box)
    _compare_maps(g, o, props=[1], exact=False)
    g.applyStencils(sgb.HEAT7, [1], [0], [0.05], box=box, tiled=True)
    o.heat7(1, 0, 0.05, box=box)
    _compare_maps(g, o, props=[0], exact=False)


@pytest.mark.parametrize("edge", [8, 4])
def test_box27_matches_oracle(sgb, edge):
    rng = np.random.default_rng(31)
    g, o, _ = _sparse_grid(sgb, rng, (48, 56, 64), edge, 40000, lowface=True, ptypes=(O.T_F32, O.T_F32))
    g.tagBoundaries(O.NN_FULL)
    o.tag_boundaries(O.NN_FULL)
    coeff = (np.ones(27, np.float32) / np.float32(27)).tolist()
    g.applyStencils(sgb.BOX27, [0], [1], coeff)
    o.box27(0, 1, coeff)
    _compare_maps(g, o, exact=False)


def test_conv3x3x3_golden_on_gpu(sgb):
    """test3x3x3convolution (SparseGridGpu_tests.cu:1012-1141): out == 27*in at mask == 1."""
    r = np.arange(256, 384)
    X, Y, Z = np.meshgrid(r, r, r, indexing="ij")
    x, y, z = (X - 320).ravel(), (Y - 320).ravel(), (Z - 320).ravel()
    rad = np.sqrt((x * x + y * y + z * z).astype(np.float32))
    act = (rad < 64) & (rad > 56)
    pts = np.stack([X.ravel()[act], Y.ravel()[act], Z.ravel()[act]], -1)
    v = (x + y + z)[act].astype(np.float32)
    g = sgb.SparseGridGpu((1000, 1000, 1000), ["f32", "f32"], edge=4)
    g.setBackgroundValue(0, 0.0)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda(), None])
    g.flush(["smax_", None])
    g.tagBoundaries(O.NN_FULL)
    g.applyStencils(sgb.BOX27, [0], [1], [1.0] * 27)
    _, (d0, d1), m = g.deviceToHost()
    sel = m == 1
    assert sel.sum() > 10000
    assert np.array_equal(d1[sel], d0[sel] * 27)


# ------------------------------------------------------------------ batches
def test_batch_matches_single_grids(sgb):
    edges, radii, vseeds = W.batch_grids(ngrids=6, emin=16, emax=64, seed=3)
    singles, batch, slots = [], sgb.Batch(), []
    steps = [7, 12, 3, 12, 9, 12]
    for e, r, vs, st in zip(edges, radii, vseeds, steps):
        ps = W.single_ball_grid(int(e), float(r), int(vs))
        g, _ = _load_pointset(sgb, ps, 8)
        gb, _ = _load_pointset(sgb, ps, 8)
        g.run_steps(sgb.HEAT7, [0], [1], [0.1], st, use_graph=False)
        singles.append(g)
        slots.append((batch.add(gb, sgb.HEAT7, [0], [1], [0.1], st), gb))
    batch.step(12, use_graph=True)
    for (slot, gb), g, st in zip(slots, singles, steps):
        assert batch.slot_steps(slot) == st
        batch.extract(slot, gb)
        a, b = g.deviceToHost()[1], gb.deviceToHost()[1]
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_batch_continuous_add_remove(sgb):
    """Grids joining mid-run give the same result as alone."""
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    specs = [(48, 3, 11), (40, 2, 6), (56, 4, 9)]
    alone = []
    for e, nb, st in specs:
        ps = W.gray_scott(size=e, nballs=nb, rmin=5.0, rmax=12.0, seed=e)
        g, _ = _load_pointset(sgb, ps, 8)
        g.run_steps(sgb.GS7, [0, 1], [2, 3], prm, st)
        alone.append(g.deviceToHost()[1])
    batch = sgb.Batch()
    grids = []
    for j, (e, nb, st) in enumerate(specs):
        ps = W.gray_scott(size=e, nballs=nb, rmin=5.0, rmax=12.0, seed=e)
        gb, _ = _load_pointset(sgb, ps, 8)
        grids.append((batch.add(gb, sgb.GS7, [0, 1], [2, 3], prm, st), gb))
        batch.step(4)
        if j == 0:
            batch.remove(batch.add(gb, sgb.GS7, [0, 1], [2, 3], prm, 5))  # a request that is cancelled
    batch.step(12)
    for (slot, gb), ref in zip(grids, alone):
        batch.extract(slot, gb)
        got = gb.deviceToHost()[1]
        for a, b in zip(ref, got):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("edge", [8, 4])
def test_existing_offsets_and_counts(sgb, edge):
    rng = np.random.default_rng(17)
    g, o, pts = _sparse_grid(sgb, rng, (64, 56, 72), edge, 30000, ptypes=(O.T_F32,))
    g.tagBoundaries(O.NN_STAR)
    o.tag_boundaries(O.NN_STAR)
    _, _, m = o.export()
    n = g.nchunks
    per = (m[: n * g.bs] & 1).reshape(n, g.bs).sum(1)
    exp = np.concatenate([[0], np.cumsum(per)])
    assert np.array_equal(g.existing_offsets().cpu().numpy(), exp)
    assert g.countExistingElements() == int(exp[-1]) == len(pts)
    assert g.countBoundaryElements() == int(((m & 3) == 3).sum())


@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("kind", ["heat", "gs"])
@pytest.mark.parametrize("nsteps", [2, 7, 64])
def test_run_steps_small_grid_one_launch(sgb, edge, kind, nsteps):
    """A small grid runs all steps in one cooperative launch: the result equals the
    step-by-step applyStencils path bit for bit (ping-pong, distinct backgrounds)."""
    rng = np.random.default_rng(100 + edge + nsteps)
    size = (40, 36, 44) if edge == 8 else (24, 20, 28)
    pts = np.unique(rng.integers(0, size, size=(9000 if edge == 8 else 3000, 3)), axis=0).astype(np.int64)
    bck = [0.3, -0.2, 0.7, 0.1]
    grids = []
    for _ in range(2):
        g = sgb.SparseGridGpu(size, ["f32"] * 4, edge=edge)
        for p, b in enumerate(bck):
            g.setBackgroundValue(p, b)
        vals = [np.random.default_rng(7).random(len(pts)).astype(np.float32) for _ in range(4)]
        g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda() for v in vals])
        g.flush(["sRight_"] * 4)
        g.tagBoundaries(sgb.NN_STAR)
        grids.append(g)
    a, b = grids
    assert a.nchunks <= 4 * torch.cuda.get_device_properties(0).multi_processor_count
    if kind == "heat":
        src, dst, prm, k = [0], [1], [0.1], sgb.HEAT7
    else:
        src, dst, prm, k = [0, 1], [2, 3], [0.16, 0.08, 0.035, 0.065, 1.0], sgb.GS7
    fin = a.run_steps(k, src, dst, prm, nsteps, use_graph=False)
    for s in range(nsteps):
        b.applyStencils(k, src if s % 2 == 0 else dst, dst if s % 2 == 0 else src, prm)
    assert fin == (nsteps % 2 == 1)
    ka, da, ma = a.deviceToHost()
    kb, db, mb = b.deviceToHost()
    assert np.array_equal(ka, kb) and np.array_equal(ma, mb)
    for p in range(4):
        assert np.array_equal(da[p].view(np.uint32), db[p].view(np.uint32)), f"property {p}"
    a.check_device_errors()


@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("boxed", [False, True])
def test_box27_sparse_chunks_point_path(sgb, edge, boxed):
    """Conv3x3x3 on sparse chunks (fewer than an eighth of their points exist) runs over
    the existing-point list; the result equals the shared-tile kernel's bit for bit and
    the oracle's."""
    rng = np.random.default_rng(200 + edge)
    size = (96, 80, 88)
    pts = np.unique(rng.integers(0, size, size=(12000, 3)), axis=0).astype(np.int64)
    v = (rng.random(len(pts)).astype(np.float32) - 0.5) * 3
    coeff = (rng.random(27).astype(np.float32) - 0.4).tolist()
    box = ((4, 3, 5), (80, 70, 77)) if boxed else None
    out = []
    for tiled in (False, True):
        g = sgb.SparseGridGpu(size, ["f32", "f32"], edge=edge)
        g.setBackgroundValue(0, 0.4)
        g.setBackgroundValue(1, -0.6)
        g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda(), None])
        g.flush(["sRight_", None])
        g.tagBoundaries(sgb.NN_FULL)
        assert g.countExistingElements() * 8 < g.nchunks * g.bs  # sparse: the point path is taken
        g.applyStencils(sgb.BOX27, [0], [1], coeff, box=box, tiled=tiled)
        out.append(g.deviceToHost())
        g.check_device_errors()
    (ka, da, ma), (kb, db, mb) = out
    assert np.array_equal(ka, kb) and np.array_equal(ma, mb)
    act = (ma[: len(ka) * (edge ** 3)] & 3) == 1
    n = len(ka) * edge ** 3
    assert np.array_equal(da[1][:n][act].view(np.uint32), db[1][:n][act].view(np.uint32))
    o = O.OracleGrid(size, edge=edge, ptypes=[O.T_F32, O.T_F32])
    o.set_background(0, 0.4)
    o.set_background(1, -0.6)
    o.insert_flush(pts, [v, np.zeros(len(v), np.float32)], [O.OP_RIGHT, O.OP_NONE])
    o.tag_boundaries(O.NN_FULL)
    o.box27(0, 1, np.asarray(coeff, np.float32), box)
    ok_, od, om = o.export()
    assert np.array_equal(da[1][:n][act].view(np.uint32), od[1][:n][act].view(np.uint32))
