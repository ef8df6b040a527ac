"""pack / unpack for ghost exchange against the oracle: packed buffers
byte-identical to the oracle's restatement of the reference's packed-box
format, the reference's own known answers on its sphere case
(SparseGridGpu_tests.cu:1382-1447, 1533-1937), unpacks into grids that
already hold points, and the error paths."""
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


def _sphere_pair(sgb, odd_only=False):
    g = sgb.SparseGridGpu(K.SIZE, ["f32"] * 4, edge=K.EDGE)
    o = O.OracleGrid(K.SIZE, edge=K.EDGE, ptypes=(O.T_F32,) * 4)
    c, rel = K.sphere(odd_only)
    vals = K.sphere_values(rel)
    g.insert(torch.from_numpy(c).cuda(), [torch.from_numpy(v).cuda() for v in vals])
    g.flush(["smax_"] * 4)
    o.insert_flush(c, vals, [O.OP_MAX] * 4)
    return g, o


def _same_map(g, o):
    keys, data, mask = g.deviceToHost()
    okeys, odata, omask = o.export()
    n = len(okeys)
    assert np.array_equal(keys, okeys)
    assert np.array_equal(mask[: n * g.bs], omask[: n * g.bs])
    ex = (mask[: n * g.bs] & 1).astype(bool)
    for p in range(len(data)):
        a, b = data[p][: (n + 1) * g.bs], odata[p]
        assert np.array_equal(a[: n * g.bs][ex].view(np.uint8), b[: n * g.bs][ex].view(np.uint8)), f"property {p}"
        assert np.array_equal(a[n * g.bs:].view(np.uint8), b[n * g.bs:].view(np.uint8)), f"background {p}"


def test_pack_request_kat(sgb):
    g, o = _sphere_pair(sgb)
    sizes = g.pack_sizes(K.box_rows(K.HALF_BOXES), [0])
    assert sizes == [K.packed_size(c, p, 4) for c, p in zip(K.HALF_NCNK, K.HALF_NPNT)]
    g.packReset()
    for b in [((0, 0, 0), (999, 999, 999))] * 2:
        g.packRequest(b)
    cnt = g.countExistingElements()
    assert g.packCalculate([0]) == 2 * K.packed_size(g.nchunks, cnt, 4)


def test_pack_unpack_kat(sgb):
    src, osrc = _sphere_pair(sgb)
    props = [0, 1, 2, 3]
    buf = src.pack_boxes(K.box_rows(K.SRC_BOXES), props)
    ref = osrc.pack(K.box_rows(K.SRC_BOXES), props)
    assert buf.numel() == len(ref) == sum(K.packed_size(c, p, 16) for c, p in zip(K.PACK_NCNK, K.PACK_NPNT))
    assert bytes(buf.cpu().numpy()) == ref

    dst = sgb.SparseGridGpu(K.SIZE, ["f32"] * 4, edge=K.EDGE)
    odst = O.OracleGrid(K.SIZE, edge=K.EDGE, ptypes=(O.T_F32,) * 4)
    starts = [lo for lo, _ in K.DST_BOXES]
    for odd, expect in ((False, K.UNPACK_CNT_ALL), (True, K.UNPACK_CNT_ODD)):
        if odd:
            src, osrc = _sphere_pair(sgb, odd_only=True)
            buf = src.pack_boxes(K.box_rows(K.SRC_BOXES), props)
            ref = osrc.pack(K.box_rows(K.SRC_BOXES), props)
            assert bytes(buf.cpu().numpy()) == ref
        dst.removeAddUnpackReset()
        off = 0
        for b, st in zip(K.DST_BOXES, starts):
            dst.remove(b)
            off = dst.unpack(buf, props, st, off)
        assert off == buf.numel()
        dst.removeAddUnpackFinalize(props)
        odst.remove_boxes(K.box_rows(K.DST_BOXES))
        parts = odst.unpack(ref, props, starts)
        odst.insert_flush(np.concatenate([c for c, _ in parts]),
                          [np.concatenate([v[p] for _, v in parts]) for p in range(4)], [O.OP_RIGHT] * 4)
        _same_map(dst, odst)
        for b, n in zip(K.DST_BOXES, expect):
            assert dst.existing_points(b).shape[0] == n
    dst.check_device_errors()


TYPES = (["f32", "i32", "u8", "f64"], [O.T_F32, O.T_I32, O.T_U8, O.T_F64])
BCK = [0.25, -3, 7, 1.5]


def _random_pair(sgb, size, npts, seed, edge=8, bck=BCK):
    rng = np.random.default_rng(seed)
    pts = np.unique(rng.integers(0, size, size=(npts, 3)), axis=0).astype(np.int64)
    vals = [rng.random(len(pts)).astype(np.float32), rng.integers(-1000, 1000, len(pts)).astype(np.int32),
            rng.integers(0, 255, len(pts)).astype(np.uint8), rng.random(len(pts))]
    g = sgb.SparseGridGpu(size, TYPES[0], edge=edge)
    o = O.OracleGrid(size, edge=edge, ptypes=TYPES[1])
    for p, b in enumerate(bck):
        g.setBackgroundValue(p, b)
        o.set_background(p, b)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda() for v in vals])
    g.flush(["smax_"] * 4)
    o.insert_flush(pts, vals, [O.OP_MAX] * 4)
    return g, o


RBOXES = [((10, 12, 5), (40, 30, 60)),     # ordinary
          ((35, 0, 0), (50, 70, 20)),      # overlaps the first
          ((0, 0, 0), (95, 95, 95)),       # the whole domain
          ((200, 200, 200), (300, 300, 300)),  # outside: an empty box
          ((7, 7, 7), (7, 7, 7)),          # one point
          ((40, 40, 40), (30, 30, 30))]    # inverted: empty


@pytest.mark.parametrize("props", [[0, 1, 2, 3], [3, 0], [2], []])
@pytest.mark.parametrize("edge", [8, 4])
def test_pack_random_bytes(sgb, props, edge):
    g, o = _random_pair(sgb, (96, 96, 96), 80000, 3 + edge, edge)
    buf = g.pack_boxes(K.box_rows(RBOXES), props)
    ref = o.pack(K.box_rows(RBOXES), props)
    assert bytes(buf.cpu().numpy()) == ref
    # the request matches what pack wrote; the empty boxes are 40-byte headers
    sizes = g.pack_sizes(K.box_rows(RBOXES), props)
    assert sum(sizes) == len(ref) and sizes[3] == sizes[5] == 40
    # the bytes_written form into a larger buffer
    big = torch.full((len(ref) + 64,), 0xAB, dtype=torch.uint8, device="cuda")
    g.packReset()
    for b in RBOXES:
        g.packRequest(b)
    assert g.packFinalize(big, props) == len(ref)
    assert bytes(big[: len(ref)].cpu().numpy()) == ref


@pytest.mark.parametrize("shift", [(0, 0, 0), (3, -5, 17), (-9, 2, 0)])
def test_unpack_into_populated_grid(sgb, shift):
    src, osrc = _random_pair(sgb, (96, 96, 96), 60000, 11)
    dst, odst = _random_pair(sgb, (128, 128, 128), 40000, 12, bck=[-1.0, 9, 3, 2.5])
    boxes = [((10, 12, 5), (40, 30, 60)), ((50, 50, 50), (80, 90, 70))]
    props = [3, 0, 2]  # property 1 is not unpacked: existing points keep it, new ones read the background
    buf = src.pack_boxes(K.box_rows(boxes), props)
    ref = osrc.pack(K.box_rows(boxes), props)
    assert bytes(buf.cpu().numpy()) == ref
    starts = [tuple(np.add(lo, shift) + 20) for lo, _ in boxes]
    off = 0
    for st in starts:
        off = dst.unpack(buf, props, st, off)
    dst.removeAddUnpackFinalize(props)
    parts = odst.unpack(ref, props, starts)
    coords = np.concatenate([c for c, _ in parts])
    vals = [None] * 4
    for k, p in enumerate(props):
        vals[p] = np.concatenate([v[k] for _, v in parts])
    vals[1] = np.zeros(len(coords), dtype=np.int32)
    odst.insert_flush(coords, vals, [O.OP_RIGHT, O.OP_NONE, O.OP_RIGHT, O.OP_RIGHT])
    _same_map(dst, odst)
    dst.check_device_errors()


def test_unpack_in_place_roundtrip(sgb):
    # pack the whole grid, unpack into an empty grid of the same size: the same block map
    src, osrc = _random_pair(sgb, (96, 96, 96), 50000, 21)
    buf = src.pack_boxes(K.box_rows([((0, 0, 0), (95, 95, 95))]), [0, 1, 2, 3])
    dst = sgb.SparseGridGpu((96, 96, 96), TYPES[0], edge=8)
    for p, b in enumerate(BCK):
        dst.setBackgroundValue(p, b)
    assert dst.unpack(buf, [0, 1, 2, 3]) == buf.numel()
    dst.removeAddUnpackFinalize([0, 1, 2, 3])
    _same_map(dst, osrc)


def test_pack_errors(sgb):
    g, _ = _random_pair(sgb, (64, 64, 64), 5000, 31)
    rows = K.box_rows([((0, 0, 0), (63, 63, 63))])
    need = g.pack_sizes(rows, [0])[0]
    small = torch.empty(need - 8, dtype=torch.uint8, device="cuda")
    with pytest.raises(sgb.SgbError):
        g.pack_boxes(rows, [0], small)
    buf = torch.empty(need + 8, dtype=torch.uint8, device="cuda")
    with pytest.raises(sgb.SgbError):  # misaligned destination
        g.pack_boxes(rows, [0], buf[4:])
    with pytest.raises(sgb.SgbError):  # property out of range
        g.pack_boxes(rows, [7])
    packed = g.pack_boxes(rows, [0])
    with pytest.raises(sgb.SgbError):  # truncated
        g.unpack(packed[:-8], [0])
    with pytest.raises(sgb.SgbError):  # packed with other properties: sizes do not add up
        g.unpack(packed, [0, 3])
    # points that land outside the domain fail the flush, like out-of-domain inserts
    g.unpack(packed, [0], (10, 10, 10))
    with pytest.raises(sgb.SgbError):
        g.removeAddUnpackFinalize([0])
    g.check_device_errors()


@pytest.mark.parametrize("with_starts", [True, False])
def test_unpack_boxes_equals_box_by_box(sgb, with_starts):
    src, osrc = _random_pair(sgb, (96, 96, 96), 60000, 51)
    boxes = RBOXES  # includes empty and inverted boxes
    props = [0, 3, 1]
    buf = src.pack_boxes(K.box_rows(boxes), props)
    starts = [tuple(np.add(lo, 7)) for lo, _ in boxes] if with_starts else None
    a, _ = _random_pair(sgb, (128, 128, 128), 20000, 52)
    b, _ = _random_pair(sgb, (128, 128, 128), 20000, 52)
    off = 0
    for k in range(len(boxes)):
        off = a.unpack(buf, props, None if starts is None else starts[k], off)
    assert b.unpack_boxes(buf, props, starts, nboxes=len(boxes)) == off == buf.numel()
    a.removeAddUnpackFinalize(props)
    b.removeAddUnpackFinalize(props)
    ka, da, ma = a.deviceToHost()
    kb, db, mb = b.deviceToHost()
    assert np.array_equal(ka, kb) and np.array_equal(ma, mb)
    for p in range(4):
        assert np.array_equal(da[p].view(np.uint8), db[p].view(np.uint8))
    # a truncated buffer is refused before anything is staged
    n_before = b.countExistingElements()
    with pytest.raises(sgb.SgbError):
        b.unpack_boxes(buf[: buf.numel() - 8], props, starts, nboxes=len(boxes))
    b.removeAddUnpackFinalize(props)
    assert b.countExistingElements() == n_before
    b.check_device_errors()
