"""The point-list stencil mode (applyStencils in STENCIL_MODE_INPLACE_NO_SHARED
with Conv3x3x3_noshared) and the existing-point list against the oracle,
bit for bit, plus the reference's all-ones known answer
(SparseGridGpu_tests.cu:1073-1141)."""
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


def _pair(sgb, size, npts, seed, edge):
    rng = np.random.default_rng(seed)
    pts = np.unique(rng.integers(0, size, size=(npts, 3)), axis=0).astype(np.int64)
    v = (rng.random(len(pts)).astype(np.float32) - 0.5) * 4
    g = sgb.SparseGridGpu(size, ["f32", "f32"], edge=edge)
    o = O.OracleGrid(size, edge=edge, ptypes=[O.T_F32, O.T_F32])
    for p, b in enumerate([0.75, -1.25]):
        g.setBackgroundValue(p, b)
        o.set_background(p, b)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda(), None])
    g.flush(["smax_", None])
    o.insert_flush(pts, [v, np.zeros(len(v), np.float32)], [O.OP_MAX, O.OP_NONE])
    return g, o, rng


def _check(g, o):
    keys, data, mask = g.deviceToHost()
    okeys, odata, omask = o.export()
    n = len(okeys) * g.bs
    assert np.array_equal(keys, okeys) and np.array_equal(mask[:n], omask[:n])
    act = (mask[:n] & 3) == 1
    assert np.array_equal(data[1][:n][act].view(np.uint32), odata[1][:n][act].view(np.uint32))


def test_noshared_all_ones_kat(sgb):
    g = sgb.SparseGridGpu(K.SIZE, ["f32", "f32"], edge=K.EDGE)
    c, rel = K.sphere()
    g.insert(torch.from_numpy(c).cuda(), [torch.from_numpy(K.sphere_values(rel)[0]).cuda(), None])
    g.flush(["smax_", None])
    g.findNeighbours(sgb.NN_FULL)
    g.tagBoundaries(sgb.NN_FULL, calculate_existing_points=True)
    g.applyStencils(sgb.BOX27_NS, [0], [1], [1.0] * 27)
    keys, data, mask = g.deviceToHost()
    n = len(keys) * g.bs
    act = mask[:n] == 1
    assert act.sum() > 100000
    assert np.array_equal(data[1][:n][act], data[0][:n][act] * 27)


@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("boxed", [False, True])
def test_noshared_matches_oracle(sgb, edge, boxed):
    g, o, rng = _pair(sgb, (72, 80, 64), 70000, 5 + edge, edge)
    g.tagBoundaries(sgb.NN_FULL)
    o.tag_boundaries(O.NN_FULL)
    coeff = (rng.random(27).astype(np.float32) - 0.3)
    box = ((5, 9, 2), (60, 70, 50)) if boxed else None
    g.applyStencils(sgb.BOX27_NS, [0], [1], coeff.tolist(), box=box)
    o.box27_noshared(0, 1, coeff, box)
    _check(g, o)
    # the transposed coefficients through Conv3x3x3 give the same sums in another order:
    # equal to within rounding, not bit for bit
    t = coeff.reshape(3, 3, 3).transpose(2, 1, 0).ravel()
    g.applyStencils(sgb.BOX27, [0], [1], t.tolist(), box=box)
    keys, data, mask = g.deviceToHost()
    okeys, odata, _ = o.export()
    n = len(okeys) * g.bs
    act = (mask[:n] & 3) == 1
    np.testing.assert_allclose(data[1][:n][act], odata[1][:n][act], rtol=1e-5, atol=1e-5)
    g.check_device_errors()


def test_point_list_and_rebuild(sgb):
    g, o, rng = _pair(sgb, (64, 64, 64), 20000, 41, 8)
    ids = g.existing_point_list().cpu().numpy()
    keys, _, mask = g.deviceToHost()
    expect = np.nonzero(mask[: len(keys) * g.bs] & 1)[0]
    assert np.array_equal(ids, expect) and len(ids) == g.countExistingElements()
    # new points: the list is rebuilt and the stencil covers them
    pts = rng.integers(0, 64, size=(5000, 3)).astype(np.int64)
    v = rng.random(len(pts)).astype(np.float32)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda(), None])
    g.flush(["sadd_", None])
    o.insert_flush(pts, [v, np.zeros(len(v), np.float32)], [O.OP_ADD, O.OP_NONE])
    assert g.calc_existing_points() == g.countExistingElements()
    coeff = rng.random(27).astype(np.float32)
    g.applyStencils(sgb.BOX27_NS, [0], [1], coeff.tolist())
    o.box27_noshared(0, 1, coeff)
    _check(g, o)
    # removal changes existence: the list follows
    g.remove(((0, 0, 0), (31, 63, 63)))
    g.removePoints()
    assert len(g.existing_point_list()) == g.countExistingElements()
    g.check_device_errors()


def test_noshared_steps_graph(sgb):
    # many ping-pong steps in one graph: the list is built before the capture
    g, o, rng = _pair(sgb, (48, 48, 48), 15000, 43, 8)
    coeff = (rng.random(27).astype(np.float32) / 27.0)
    fin = g.run_steps(sgb.BOX27_NS, [0], [1], coeff.tolist(), 4, use_graph=True)
    for k in range(4):
        if k % 2 == 0:
            o.box27_noshared(0, 1, coeff)
        else:
            o.box27_noshared(1, 0, coeff)
    assert fin is False
    keys, data, mask = g.deviceToHost()
    okeys, odata, _ = o.export()
    n = len(okeys) * g.bs
    act = (mask[:n] & 3) == 1
    assert np.array_equal(data[0][:n][act].view(np.uint32), odata[0][:n][act].view(np.uint32))
