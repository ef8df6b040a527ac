"""The oracle's pack / unpack against the reference's known answers
(src/SparseGridGpu/tests/SparseGridGpu_tests.cu:1382-1447 test_pack_request_with_iterator,
1533-1937 sparsegridgpu_pack_unpack)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import sphere_kat as K


def _sphere_grid(nprop, odd_only=False):
    g = O.OracleGrid(K.SIZE, edge=K.EDGE, ptypes=(O.T_F32,) * nprop)
    c, rel = K.sphere(odd_only)
    g.insert_flush(c, K.sphere_values(rel)[:nprop], [O.OP_MAX] * nprop)
    return g


def _headers(buf, point_size):
    out, pos = [], 0
    while pos < len(buf):
        n_cnk = int(np.frombuffer(buf, "<u8", 1, pos)[0])
        n_pnt = int(np.frombuffer(buf, "<u4", 1, pos + 32 + 12 * n_cnk)[0])
        out.append((n_cnk, n_pnt))
        pos += K.packed_size(n_cnk, n_pnt, point_size)
    assert pos == len(buf)
    return out


def test_pack_request_halves():
    g = _sphere_grid(1)
    buf = g.pack(K.box_rows(K.HALF_BOXES), [0])
    assert _headers(buf, 4) == list(zip(K.HALF_NCNK, K.HALF_NPNT))
    # packing the whole domain twice: every chunk and every point, twice
    whole = g.pack(K.box_rows([((0, 0, 0), (999, 999, 999))] * 2), [0])
    cnt = len(g.existing_points())
    assert _headers(whole, 4) == [(g.nchunks, cnt)] * 2


def test_pack_unpack_sphere():
    src = _sphere_grid(4)
    props = [0, 1, 2, 3]  # float + float[3]: 16 bytes per point
    buf = src.pack(K.box_rows(K.SRC_BOXES), props)
    assert _headers(buf, 16) == list(zip(K.PACK_NCNK, K.PACK_NPNT))
    # the first box's header: start = box corner, size = grid size
    assert list(np.frombuffer(buf, "<i4", 6, 8)) == [256, 256, 256, 1000, 1000, 1000]

    dst = O.OracleGrid(K.SIZE, edge=K.EDGE, ptypes=(O.T_F32,) * 4)
    for odd, expect in ((False, K.UNPACK_CNT_ALL), (True, K.UNPACK_CNT_ODD)):
        if odd:
            src = _sphere_grid(4, odd_only=True)
            buf = src.pack(K.box_rows(K.SRC_BOXES), props)
        dst.remove_boxes(K.box_rows(K.DST_BOXES))
        starts = [lo for lo, _ in K.DST_BOXES]
        parts = dst.unpack(buf, props, starts)
        coords = np.concatenate([c for c, _ in parts])
        vals = [np.concatenate([v[p] for _, v in parts]) for p in range(4)]
        dst.insert_flush(coords, vals, [O.OP_RIGHT] * 4)
        pts = dst.existing_points()
        for (lo, hi), n in zip(K.DST_BOXES, expect):
            inside = np.all((pts >= lo) & (pts <= hi), axis=1)
            assert inside.sum() == n
        # every unpacked point carries its source point's values
        for (lo, hi), (slo, _) in zip(K.DST_BOXES, K.SRC_BOXES):
            p = dst.existing_points((lo, hi))
            rel = p - np.asarray(lo) + np.asarray(slo) - K.CENTRE
            np.testing.assert_array_equal(dst.get(0, p), rel.sum(axis=1).astype(np.float32))
            np.testing.assert_array_equal(dst.get(3, p), rel[:, 2].astype(np.float32))


def test_conv3x3x3_noshared_all_ones():
    """SparseGridGpu_tests.cu:1073-1141 test3x3x3convolution_no_shared: the
    hollow sphere (edge 4), NNFull, every coefficient 1: out = 27 * in at the
    active points (mask byte 1)."""
    g = O.OracleGrid(K.SIZE, edge=K.EDGE, ptypes=(O.T_F32, O.T_F32))
    c, rel = K.sphere()
    g.insert_flush(c, [K.sphere_values(rel)[0], np.zeros(len(c), np.float32)], [O.OP_MAX, O.OP_NONE])
    g.tag_boundaries(O.NN_FULL)
    g.box27_noshared(0, 1, np.ones(27, np.float32))
    keys, data, mask = g.export()
    n = len(keys) * g.bs
    act = mask[:n] == 1
    assert act.sum() > 100000
    np.testing.assert_array_equal(data[1][:n][act], data[0][:n][act] * 27)


@pytest.mark.parametrize("noshared", [False, True])
def test_conv3x3x3_all_ones_morton(noshared):
    """SparseGridGpu_tests.cu:1145-1180: the same all-ones known answers on
    SparseGridGpu_z (chunk ids by Morton code)."""
    g = O.OracleGrid(K.SIZE, edge=K.EDGE, ptypes=(O.T_F32, O.T_F32), zorder=True)
    c, rel = K.sphere()
    g.insert_flush(c, [K.sphere_values(rel)[0], np.zeros(len(c), np.float32)], [O.OP_MAX, O.OP_NONE])
    keys, _, _ = g.export()
    # the ids are the Morton codes of the chunk coordinates, in order
    bc = np.unique(c // K.EDGE, axis=0)
    morton = np.zeros(len(bc), np.int64)
    for i in range(10):
        for d in range(3):
            morton |= ((bc[:, d] >> i) & 1) << (3 * i + d)
    assert np.array_equal(keys, np.sort(morton))
    g.tag_boundaries(O.NN_FULL)
    (g.box27_noshared if noshared else g.box27)(0, 1, np.ones(27, np.float32))
    keys, data, mask = g.export()
    n = len(keys) * g.bs
    act = mask[:n] == 1
    np.testing.assert_array_equal(data[1][:n][act], data[0][:n][act] * 27)
