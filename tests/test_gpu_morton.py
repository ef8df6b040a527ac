"""Grids with Morton chunk ids (SparseGridGpu_z: grid_zmb linearizer) against
the oracle run with the same linearizer, bit for bit: the block map after
inserts, the neighbour tables, tagBoundaries, every stencil, pack / unpack,
removal, iteration order and links; plus the reference's 27-point all-ones
known answer on the Morton grid (SparseGridGpu_tests.cu:1145-1180)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests import sphere_kat as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sgb():
    import openfpm_data_b200 as m
    assert torch.cuda.is_available(), "these tests need a CUDA device"
    m.load()
    return m


def _pair(sgb, size, npts, seed, edge=8, zorder=True, nprop=2):
    rng = np.random.default_rng(seed)
    pts = np.unique(rng.integers(0, size, size=(npts, 3)), axis=0).astype(np.int64)
    vals = [rng.random(len(pts)).astype(np.float32) for _ in range(nprop)]
    g = sgb.SparseGridGpu(size, ["f32"] * nprop, edge=edge, linearizer="zmb" if zorder else "smb")
    o = O.OracleGrid(size, edge=edge, ptypes=[O.T_F32] * nprop, zorder=zorder)
    for p in range(nprop):
        g.setBackgroundValue(p, 0.25 * (p + 1))
        o.set_background(p, 0.25 * (p + 1))
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda() for v in vals])
    g.flush(["smax_"] * nprop)
    o.insert_flush(pts, vals, [O.OP_MAX] * nprop)
    return g, o, pts, rng


def _same_map(g, o, props):
    keys, data, mask = g.deviceToHost()
    okeys, odata, omask = o.export()
    n = len(okeys)
    assert np.array_equal(keys, okeys)
    assert np.array_equal(mask[: n * g.bs], omask[: n * g.bs])
    act = (mask[: n * g.bs] & 1).astype(bool)
    for p in props:
        assert np.array_equal(data[p][: n * g.bs][act].view(np.uint32), odata[p][: n * g.bs][act].view(np.uint32))


@pytest.mark.parametrize("edge", [8, 4])
def test_morton_block_map_and_tables(sgb, edge):
    g, o, pts, _ = _pair(sgb, (70, 90, 60), 40000, 3, edge)
    _same_map(g, o, [0, 1])
    keys = g.private_get_index_array().cpu().numpy()
    # the ids are Morton codes of the chunks' block coordinates, and sorted
    assert np.all(np.diff(keys) > 0)
    bc = o.block_coords(keys)
    assert np.array_equal(o.block_key(bc), keys)
    assert np.array_equal(np.unique(pts // edge, axis=0), np.unique(bc, axis=0))
    for nn, onn in ((sgb.NN_STAR, O.NN_STAR), (sgb.NN_FULL, O.NN_FULL)):
        t = g.neighbour_table(nn)
        ot = o.find_neighbours(onn)
        if nn == sgb.NN_STAR:
            t, ot = t[:, :6], ot[:, :6]
        assert np.array_equal(t, ot)
    g.tagBoundaries(sgb.NN_FULL)
    o.tag_boundaries(O.NN_FULL)
    _same_map(g, o, [0, 1])


@pytest.mark.parametrize("kind", ["heat", "gs", "box27", "box27ns"])
def test_morton_stencils(sgb, kind):
    g, o, pts, rng = _pair(sgb, (64, 72, 56), 45000, 9, 8, nprop=4)
    g.tagBoundaries(sgb.NN_STAR)
    o.tag_boundaries(O.NN_STAR)
    box = ((3, 2, 1), (60, 66, 50))
    if kind == "heat":
        g.applyStencils(sgb.HEAT7, [0], [1], [0.1], box=box)
        o.heat7(0, 1, 0.1, box)
    elif kind == "gs":
        prm = [0.16, 0.08, 0.035, 0.065, 1.0]
        g.applyStencils(sgb.GS7, [0, 1], [2, 3], prm, box=box)
        o.gs7(0, 1, 2, 3, *prm, box=box)
    else:
        c = (rng.random(27).astype(np.float32) - 0.5)
        g.applyStencils(sgb.BOX27 if kind == "box27" else sgb.BOX27_NS, [0], [1], c.tolist(), box=box)
        (o.box27 if kind == "box27" else o.box27_noshared)(0, 1, c, box)
    _same_map(g, o, [0, 1, 2, 3] if kind == "gs" else [0, 1])
    g.check_device_errors()


def test_morton_equals_row_major_by_coordinate(sgb):
    # the same points in a grid_smb grid and a grid_zmb grid: the same values at every point
    gz, _, pts, _ = _pair(sgb, (48, 40, 56), 20000, 21, 8, zorder=True)
    gs, _, _, _ = _pair(sgb, (48, 40, 56), 20000, 21, 8, zorder=False)
    for g in (gz, gs):
        g.applyStencils(sgb.HEAT7, [0], [1], [0.2])
    c = torch.from_numpy(pts.astype(np.int32)).cuda()
    assert torch.equal(gz.get(1, c), gs.get(1, c))
    ez, es = gz.existing_points().cpu().numpy(), gs.existing_points().cpu().numpy()
    assert np.array_equal(np.unique(ez, axis=0), np.unique(es, axis=0))
    assert gz.countExistingElements() == gs.countExistingElements()


def test_morton_conv_all_ones_kat(sgb):
    g = sgb.SparseGridGpu(K.SIZE, ["f32", "f32"], edge=K.EDGE, linearizer="zmb")
    c, rel = K.sphere()
    g.insert(torch.from_numpy(c).cuda(), [torch.from_numpy(K.sphere_values(rel)[0]).cuda(), None])
    g.flush(["smax_", None])
    g.tagBoundaries(sgb.NN_FULL, calculate_existing_points=True)
    for kind in (sgb.BOX27, sgb.BOX27_NS):
        g.applyStencils(kind, [0], [1], [1.0] * 27)
        keys, data, mask = g.deviceToHost()
        n = len(keys) * g.bs
        act = mask[:n] == 1
        assert act.sum() > 100000
        assert np.array_equal(data[1][:n][act], data[0][:n][act] * 27)


def test_morton_pack_remove_iterate_links(sgb):
    g, o, pts, _ = _pair(sgb, (64, 64, 64), 30000, 33, 8)
    boxes = np.array([[5, 6, 7, 40, 50, 30], [0, 0, 0, 63, 63, 63]], dtype=np.int64)
    buf = g.pack_boxes(boxes, [1, 0])
    ref = o.pack(boxes, [1, 0])
    assert bytes(buf.cpu().numpy()) == ref
    dst = sgb.SparseGridGpu((64, 64, 64), ["f32"] * 2, edge=8, linearizer="zmb")
    odst = O.OracleGrid((64, 64, 64), edge=8, ptypes=[O.T_F32] * 2, zorder=True)
    for p in range(2):
        dst.setBackgroundValue(p, 0.25 * (p + 1))
        odst.set_background(p, 0.25 * (p + 1))
    off = dst.unpack(buf, [1, 0], (10, 3, 20))
    dst.removeAddUnpackFinalize([1, 0])
    coords, vals = odst.unpack(ref[: off], [1, 0], [(10, 3, 20)])[0]
    odst.insert_flush(coords, [vals[1], vals[0]], [O.OP_RIGHT, O.OP_RIGHT])
    _same_map(dst, odst, [0, 1])
    # removal and iteration order (chunk positions follow the Morton ids)
    g.remove(((10, 10, 10), (30, 50, 60)))
    g.removePoints()
    o.remove_boxes([[10, 10, 10, 30, 50, 60]])
    assert np.array_equal(g.existing_points().cpu().numpy(), o.existing_points())
    # links between two Morton levels
    g.tagBoundaries(sgb.NN_STAR)
    o.tag_boundaries(O.NN_STAR)
    fine, ofine, _, _ = _pair(sgb, (128, 128, 128), 200000, 35, 8)
    box = ((0, 0, 0), (63, 63, 63))
    g.construct_link_dw(fine, box, (1, 0, 0))
    ref_links = o.construct_links(ofine, box, (1, 0, 0), up=False)
    got = g.getDownLinks()
    for k in ("pad_pos", "pad_off", "offsets", "link_pos", "link_off"):
        assert np.array_equal(got[k].cpu().numpy(), ref_links[k]), k


def test_morton_rejected_where_unsupported(sgb):
    from openfpm_data_b200 import _lib as L
    g, _, _, _ = _pair(sgb, (32, 32, 32), 100, 1, 8)
    with pytest.raises(sgb.SgbError):  # the linearizer is chosen while the grid is empty
        L.check(g._lib.sgb_set_linearizer(g._h, L.LIN_SMB), "sgb_set_linearizer")
    b = sgb.Batch()
    with pytest.raises(sgb.SgbError):  # batches hold x-fastest grids
        b.add(g, sgb.HEAT7, [0], [1], [0.1], 10)
