"""remove(box) + removePoints and the existing-point iteration against the
oracle: masks bit-exact after removal (points in any box, the reference's
unsigned box test included), stencils after a removal, and the iteration
order of all points and of a sub-box."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sgb():
    import openfpm_data_b200 as m
    assert torch.cuda.is_available(), "these tests need a CUDA device"
    m.load()
    return m


def _grid_pair(sgb, size, npts, seed, edge=8):
    rng = np.random.default_rng(seed)
    pts = np.unique(rng.integers(0, size, size=(npts, 3)), axis=0).astype(np.int64)
    vals = [rng.random(len(pts)).astype(np.float32) for _ in range(2)]
    g = sgb.SparseGridGpu(size, ["f32", "f32"], edge=edge)
    o = O.OracleGrid(size, edge=edge, ptypes=[O.T_F32, O.T_F32])
    for p, b in enumerate([0.25, 0.5]):
        g.setBackgroundValue(p, b)
        o.set_background(p, b)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda() for v in vals])
    g.flush(["smax_", "smax_"])
    o.insert_flush(pts, vals, [O.OP_MAX, O.OP_MAX])
    return g, o


BOXES = [((10, 12, 5), (40, 30, 60)),     # ordinary
         ((35, 0, 0), (50, 70, 20)),      # overlaps the first
         ((-1, 0, 0), (70, 70, 70)),      # negative lower corner: removes nothing (unsigned test)
         ((0, 0, 64), (70, 70, 71))]      # the top slab


@pytest.mark.parametrize("edge", [8, 4])
def test_remove_points_matches_oracle(sgb, edge):
    g, o = _grid_pair(sgb, (72, 72, 72), 60000, 1, edge)
    n_before = g.countExistingElements()
    for b in BOXES:
        g.remove(b)
    g.removePoints()
    o.remove_boxes([list(lo) + list(hi) for lo, hi in BOXES])
    keys, data, mask = g.deviceToHost()
    okeys, odata, omask = o.export()
    n = len(okeys)
    assert np.array_equal(keys, okeys) and n == g.nchunks  # chunks stay
    assert np.array_equal(mask[: n * g.bs], omask[: n * g.bs])
    ex = (mask[: n * g.bs] & 1).astype(bool)
    for p, b in enumerate([0.25, 0.5]):
        assert np.array_equal(data[p][: n * g.bs][ex], odata[p][: n * g.bs][ex])
        assert np.all(data[p][: n * g.bs][~ex] == np.float32(b))  # removed points read the background
    assert 0 < g.countExistingElements() < n_before
    # a stencil after the removal sees the background where points went away
    g.applyStencils(sgb.HEAT7, [0], [1], [0.1])
    o.heat7(0, 1, 0.1)
    keys, data, mask = g.deviceToHost()
    okeys, odata, omask = o.export()
    a, b = data[1][: n * g.bs][ex].astype(np.float64), odata[1][: n * g.bs][ex].astype(np.float64)
    err = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
    err[a == b] = 0
    assert err.max(initial=0) <= 1e-6
    g.check_device_errors()


def test_remove_nothing_queued_or_empty_grid(sgb):
    g = sgb.SparseGridGpu((16, 16, 16), ["f32"], edge=8)
    g.removePoints()
    g.remove(((0, 0, 0), (15, 15, 15)))
    g.removePoints()  # empty grid
    assert g.nchunks == 0 and g.existing_points().shape == (0, 3)


@pytest.mark.parametrize("edge", [8, 4])
def test_existing_points_order_matches_oracle(sgb, edge):
    g, o = _grid_pair(sgb, (64, 40, 48), 20000, 2, edge)
    pts = g.existing_points().cpu().numpy().astype(np.int64)
    assert np.array_equal(pts, o.existing_points())
    box = ((5, 7, 9), (33, 30, 40))
    sub = g.existing_points(box).cpu().numpy().astype(np.int64)
    assert np.array_equal(sub, o.existing_points(box))
    assert len(list(g.getIterator((5, 7, 9), (33, 30, 40)))) == len(sub)
