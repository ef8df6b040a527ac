"""Pin the CPU oracle against the reference's own known-answer tests.

Each case restates one test of openfpm_data (cited by file:line, paths inside
the reference project) end to end: the reference's inputs, the reference's
expected outputs.  The oracle is what the GPU parity tests compare against,
so these cases are what make those comparisons mean "same as the reference".
"""
import numpy as np
import pytest

from oracle import oracle as O


def _grid(size, edge, ptypes=(O.T_F32,), dim=None):
    return O.OracleGrid(size, edge=edge, ptypes=ptypes, dim=dim)


# ---------------------------------------------------------------------------
# BlockMapGpu_kernels_tests.cu:16-190  testSegreduce_total
# 7 new segments of sizes 4,1,2,1,3,6,1; segments 1, 3, 4 also have an old
# chunk.  New chunks: value i+1 (mask 1) for i < 32, 666 (mask 0) above; old
# chunks: 100+i+1 (mask 1) for i < 32, slot 33 = 665 (mask 1), 666 (mask 0)
# elsewhere.  Reduction: plus.  Expected: with old, out[i] = 100+(i+1)(m+1)
# and out[33] = 665; without old, out[i] = (i+1) m.
# ---------------------------------------------------------------------------
def test_segreduce_total():
    g = _grid((64, 64, 64), 4)  # 4^3 chunks: 64 points, like DataBlock<float,64>
    sizes = [4, 1, 2, 1, 3, 6, 1]
    keys = [10, 20, 30, 40, 50, 60, 70]
    has_old = [False, True, False, True, True, False, False]
    blk = np.where(np.arange(64) < 32, np.arange(64) + 1, 666).astype(np.float32)
    msk = (np.arange(64) < 32).astype(np.uint8)
    old = np.where(np.arange(64) < 32, 100 + np.arange(64) + 1, 666).astype(np.float32)
    old_m = msk.copy()
    old[33], old_m[33] = 665, 1
    old_keys = [k for k, h in zip(keys, has_old) if h]
    g.load_map(old_keys, [np.tile(old, len(old_keys))], np.tile(old_m, len(old_keys)))
    slot_keys = np.repeat(keys, sizes)
    n = len(slot_keys)
    g.flush_chunks(slot_keys, [np.tile(blk, n)], np.tile(msk, n), [O.OP_ADD])
    k, (d,), m = g.export()
    assert list(k) == keys
    for j, (mult, h) in enumerate(zip(sizes, has_old)):
        out = d[j * 64:(j + 1) * 64]
        om = m[j * 64:(j + 1) * 64]
        i = np.arange(32)
        assert np.all(om[:32] == 1)
        if h:
            assert np.all(out[:32] == 100 + (i + 1) * (mult + 1))
            assert out[33] == 665 and om[33] == 1
        else:
            assert np.all(out[:32] == (i + 1) * mult)


# ---------------------------------------------------------------------------
# BlockMapGpu_kernels_tests.cu:344-495  testSolve_conflicts  (sadd_)
# Old chunks 0..3 at keys 1, 4, 8, 10 hold value i (slot 0 = 1); new chunks
# 0..9 at keys 0,2,4,5,6,7,9,11,13,13 hold value ii+5 (slot 0 = 1).
# ---------------------------------------------------------------------------
def test_solve_conflicts():
    g = _grid((64, 64, 64), 4)
    old_keys = [1, 4, 8, 10]
    old = np.concatenate([np.full(64, i, np.float32) for i in range(4)])
    old[::64] = 1
    g.load_map(old_keys, [old], np.ones(4 * 64, np.uint8))
    new_keys = [0, 2, 4, 5, 6, 7, 9, 11, 13, 13]
    new = np.concatenate([np.full(64, ii + 5, np.float32) for ii in range(10)])
    new[::64] = 1
    g.flush_chunks(new_keys, [new], np.ones(10 * 64, np.uint8), [O.OP_ADD])
    k, (d,), m = g.export()
    assert list(k) == [0, 1, 2, 4, 5, 6, 7, 8, 9, 10, 11, 13]
    assert list(d[0:12 * 64:64]) == [1, 1, 1, 2, 1, 1, 1, 1, 1, 1, 1, 2]
    assert list(d[1:12 * 64:64]) == [5, 0, 6, 8, 8, 9, 10, 2, 11, 3, 12, 27]


# ---------------------------------------------------------------------------
# BlockMapGpu_kernels_tests.cu:193-342  test_maps_create
# 9 old keys merged with 7 new keys: new segments land at 0,1,8,9,12,13,14;
# key 56 reduces with old chunk 6; old chunks 0..5 move to 2..7, 7 and 8 to
# 10 and 11.
# ---------------------------------------------------------------------------
def test_maps_create_layout():
    g = _grid((64, 64, 64), 4)
    old_keys = [33, 34, 36, 37, 43, 45, 56, 60, 61]
    old = np.concatenate([np.full(64, 1000 + j, np.float32) for j in range(9)])
    g.load_map(old_keys, [old], np.ones(9 * 64, np.uint8))
    new_keys = [22, 23, 46, 56, 63, 64, 65]
    new = np.concatenate([np.full(64, 2000 + j, np.float32) for j in range(7)])
    g.flush_chunks(new_keys, [new], np.ones(7 * 64, np.uint8), [O.OP_MAX])
    k, (d,), _ = g.export()
    assert len(k) == 15
    out_map = [0, 1, 8, 9, 12, 13, 14]
    for j, pos in enumerate(out_map):
        assert k[pos] == new_keys[j]
    copy_src = [0, 1, 2, 3, 4, 5, 7, 8]
    copy_dst = [2, 3, 4, 5, 6, 7, 10, 11]
    for s, t in zip(copy_src, copy_dst):
        assert k[t] == old_keys[s] and d[t * 64] == 1000 + s
    assert d[9 * 64] == 2003  # max(new 2003, old 1006)


# ---------------------------------------------------------------------------
# BlockMapGpu_tests.cu:126-267  testInsert / testInsert_halfBlock /
# testInsert_blocked: value = linear id, background 666, smax_.
# DataBlock<float,64> chunks == 4^3 chunks of a 3-D grid addressed by lin id.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("mode", ["insert", "half", "blocked"])
def test_blockmap_insert(mode):
    g = _grid((64, 64, 64), 4)
    g.set_background(0, 666.0)
    n = 3 * 128
    pos = np.arange(n)
    if mode == "half":
        pos = pos[(pos % 128) % 64 < 32]
    if mode == "blocked":
        slot_keys = np.arange(6)
        g.flush_chunks(slot_keys, [np.arange(n, dtype=np.float32)], np.ones(n, np.uint8), [O.OP_MAX])
    else:
        g.flush_points(pos, [pos.astype(np.float32)], [O.OP_MAX])
    k, (d,), m = g.export()
    read = np.arange(4 * 128)
    bkey, off = read // 64, read % 64
    p = np.searchsorted(k, bkey)
    found = (p < len(k)) & (k[np.minimum(p, len(k) - 1)] == bkey)
    idx = np.where(found, p, len(k)) * 64 + off
    got = np.where(m[idx] & 1, d[idx], d[len(k) * 64])
    exp = np.where(read < n, read, 666).astype(np.float32)
    if mode == "half":
        exp = np.where(read % 64 < 32, exp, 666)
    assert np.array_equal(got, exp)


# ---------------------------------------------------------------------------
# SparseGridGpu_tests.cu:209-282  testInsert (2-D, 8x8 chunks, 2x2 blocks)
# and testInsert3D (4^3 chunks, 2x2x2 blocks): value = x coordinate.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dim,edge", [(2, 8), (3, 4)])
def test_sparsegrid_insert(dim, edge):
    size = (2 * edge,) * dim
    g = _grid(size, edge, dim=dim)
    g.set_background(0, 666.0)
    coords = np.stack(np.meshgrid(*[np.arange(s) for s in size], indexing="ij"), -1).reshape(-1, dim)
    g.insert_flush(coords, [coords[:, 0].astype(np.float32)], [O.OP_MAX])
    lin = np.arange(int(np.prod(size)))
    c = g.inv_lin(lin)
    assert np.array_equal(g.lin_ids(c), lin)
    assert np.array_equal(g.get(0, c), c[:, 0].astype(np.float32))


# ---------------------------------------------------------------------------
# SparseGridGpu_tests.cu:284-470  testTagBoundaries / testTagBoundaries2:
# exact sets of padding linear ids on a 16x16 2-D grid of 8x8 chunks.
# ---------------------------------------------------------------------------
def _tag_case(batches):
    g = _grid((16, 16), 8, dim=2)
    g.set_background(0, 666.0)
    for pts in batches:
        pts = np.array(pts, dtype=np.int64)
        g.insert_flush(pts, [np.ones(len(pts), np.float32)], [O.OP_MAX])
    g.tag_boundaries(O.NN_STAR)
    lin = np.arange(256)
    m = g.mask_at(g.inv_lin(lin))
    return set(lin[(m & 1).astype(bool) & (m & 2).astype(bool)].tolist())


def test_tag_boundaries():
    b = [[(0, 0), (6, 6), (7, 6)], [(8, 6)],
         [(x, y) for y in range(9, 12) for x in (6, 7)],
         [(x, y) for y in range(9, 12) for x in (8, 9)]]
    assert _tag_case(b) == {0, 54, 55, 112, 142, 143, 200, 201, 150, 209, 158, 159, 216, 217}


def test_tag_boundaries2():
    b = [[(6, 6), (6, 7), (7, 6), (7, 7)], [(8, 6), (9, 6), (8, 7), (9, 7)],
         [(6, 8), (7, 8), (6, 9), (7, 9)], [(8, 8), (8, 9), (9, 8), (9, 9)]]
    assert _tag_case(b) == {54, 55, 62, 134, 142, 143, 112, 113, 121, 200, 193, 201}


# ---------------------------------------------------------------------------
# SparseGridGpu_tests.cu:472-530  testStencilHeat: 16x16 grid, padding set
# to 10*x/15 by BoundaryStencilSetXRescaled (tests/utils/
# SparseGridGpu_testKernels.cuh:38-79), then 1000 x (heat 0->1 dt 0.1, heat
# 1->0 dt 0.01): property 1 converges to the linear profile within 1e-2.
# ---------------------------------------------------------------------------
def test_stencil_heat_linear_profile():
    g = _grid((16, 16), 8, ptypes=(O.T_F32, O.T_F32), dim=2)
    g.set_background(0, 0.0)
    coords = np.stack(np.meshgrid(np.arange(16), np.arange(16), indexing="ij"), -1).reshape(-1, 2)
    z = np.zeros(len(coords), np.float32)
    g.insert_flush(coords, [z, z], [O.OP_MAX, O.OP_NONE])
    g.tag_boundaries(O.NN_STAR)
    keys, (d0, d1), m = g.export()
    c = g.inv_lin(keys.repeat(64) * 64 + np.tile(np.arange(64), len(keys)))
    pad = m[: len(keys) * 64] == 3
    x = c[:, 0].astype(np.float32)
    val = np.float32(10.0) * (x - np.float32(0.0)) / (np.float32(16.0) - np.float32(0.0) - np.float32(1.0))
    d0[: len(keys) * 64] = np.where(pad, val, d0[: len(keys) * 64])
    g.load_map(keys, [d0[: len(keys) * 64], d1[: len(keys) * 64]], m[: len(keys) * 64])
    for _ in range(1000):
        g.heat7(0, 1, 0.1)
        g.heat7(1, 0, 0.01)
    got = g.get(1, coords)
    assert np.all(np.abs(got - 10.0 * coords[:, 0] / 15.0) < 1e-2)


# ---------------------------------------------------------------------------
# SparseGridGpu_tests.cu:1012-1141  test3x3x3convolution: 1000^3 grid of 4^3
# chunks, shell 56 < r < 64 about (320,320,320) with value x+y+z (relative
# coordinates, insertSphere3D_radius, tests/utils/SparseGridGpu_testKernels.cuh:
# 203-259), NNFull tagBoundaries, all-ones Conv3x3x3: out == 27*in wherever
# mask == 1.
# ---------------------------------------------------------------------------
def test_conv3x3x3_all_ones():
    g = _grid((1000, 1000, 1000), 4, ptypes=(O.T_F32, O.T_F32))
    g.set_background(0, 0.0)
    r = np.arange(256, 384)
    X, Y, Z = np.meshgrid(r, r, r, indexing="ij")
    x, y, z = (X - 320).ravel(), (Y - 320).ravel(), (Z - 320).ravel()
    rad = np.sqrt((x * x + y * y + z * z).astype(np.float32))
    act = (rad < 64) & (rad > 56)
    coords = np.stack([X.ravel()[act], Y.ravel()[act], Z.ravel()[act]], -1)
    v = (x + y + z)[act].astype(np.float32)
    g.insert_flush(coords, [v, np.zeros_like(v)], [O.OP_MAX, O.OP_NONE])
    g.tag_boundaries(O.NN_FULL)
    g.box27(0, 1, np.ones(27, np.float32))
    keys, (d0, d1), m = g.export()
    sel = m == 1
    assert sel.sum() > 10000
    assert np.array_equal(d1[sel], d0[sel] * 27)
