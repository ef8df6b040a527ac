"""A block map that grows past the size at which its arrays grow in place (256 MB).

Five flushes each add 60,000 chunks (one point per new chunk) to a 2048^3 grid with a
float32 and an int32 property, so the property arrays pass 256 MB on the third flush
and then grow by mapping more memory behind their end, in both buffer sets the flush
alternates between.  After every flush the chunk count is checked; after the last one
the whole map (keys, masks and both properties at every point) is compared with what
was inserted, so values from the first flush must have survived every growth."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

EDGE = 8
NB = 256  # chunks per dimension of the 2048^3 grid
PER_FLUSH = 60_000
FLUSHES = 5


@pytest.fixture(scope="module")
def sgb():
    import openfpm_data_b200 as m
    assert torch.cuda.is_available(), "these tests need a CUDA device"
    m.load()
    return m


def test_map_grows_in_place_and_keeps_its_contents(sgb):
    rng = np.random.default_rng(11)
    keys_all = rng.choice(NB ** 3, size=PER_FLUSH * FLUSHES, replace=False).astype(np.int64)
    g = sgb.SparseGridGpu((NB * EDGE,) * 3, ["f32", "i32"], edge=EDGE)
    g.setBackgroundValue(0, 0)
    g.setBackgroundValue(1, 0)

    def point_of(keys):
        bx, by, bz = keys % NB, (keys // NB) % NB, keys // (NB * NB)
        off = keys % 512  # the point inside the chunk
        ox, oy, oz = off % 8, (off // 8) % 8, off // 64
        return np.stack([bx * 8 + ox, by * 8 + oy, bz * 8 + oz], axis=1).astype(np.int32), off

    def values_of(keys):
        return (keys % 1_000_003).astype(np.float32) * np.float32(0.5), (keys * 7 + 1).astype(np.int32)

    for f in range(FLUSHES):
        ks = keys_all[f * PER_FLUSH:(f + 1) * PER_FLUSH]
        pts, _ = point_of(ks)
        fv, iv = values_of(ks)
        g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(fv).cuda(), torch.from_numpy(iv).cuda()])
        g.flush(["sRight_", "sRight_"])
        assert g.nchunks == PER_FLUSH * (f + 1), f"flush {f}: chunk count"
    g.check_device_errors()

    keys, data, mask = g.deviceToHost()
    want = np.sort(keys_all)
    n = len(want)
    assert np.array_equal(keys[:n], want), "block map keys"
    _, off = point_of(want)
    fv, iv = values_of(want)
    rows = np.arange(n, dtype=np.int64) * 512
    m = mask[: n * 512].reshape(n, 512)
    assert np.all(m[np.arange(n), off] & 1), "inserted points exist"
    assert int((m & 1).sum()) == n, "no other point exists"
    d0 = data[0][: n * 512]
    d1 = data[1][: n * 512]
    assert np.array_equal(d0[rows + off].view(np.uint32), fv.view(np.uint32)), "float32 property"
    assert np.array_equal(d1[rows + off], iv), "int32 property"
    others = np.ones(n * 512, bool)
    others[rows + off] = False
    assert not np.any(d0[others]) and not np.any(d1[others]), "points that do not exist hold the background"
