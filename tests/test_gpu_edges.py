"""Edge cases of the CUDA path against the oracle: empty grids and empty
inserts, single-chunk and ragged domains (sizes that are not multiples of
the chunk edge), points on the domain's upper faces, every point of a chunk
duplicated many times, and a stencil on a grid whose chunks have no
neighbours at all."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from openfpm_data_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sgb():
    import openfpm_data_b200 as m
    assert torch.cuda.is_available(), "these tests need a CUDA device"
    m.load()
    return m


def _same_map(g, o, props, rtol=None):
    """Keys and masks bit-exact; fields bit-exact, or within rtol relative (stencil results)."""
    keys, data, mask = g.deviceToHost()
    okeys, odata, omask = o.export()
    n = len(okeys)
    assert np.array_equal(keys, okeys)
    assert np.array_equal(mask[: n * g.bs], omask[: n * g.bs])
    ex = (mask[: n * g.bs] & 1).astype(bool)
    for p in props:
        a, b = data[p][: n * g.bs][ex], odata[p][: n * g.bs][ex]
        if rtol is None:
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
        else:
            a, b = a.astype(np.float64), b.astype(np.float64)
            err = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
            err[a == b] = 0
            assert err.max(initial=0) <= rtol


def test_empty_grid_operations(sgb):
    g = sgb.SparseGridGpu((40, 24, 16), ["f32", "f32"], edge=8)
    g.flush(["smax_", "smax_"])  # nothing staged
    g.insert(torch.zeros((0, 3), dtype=torch.int32).cuda(), [torch.zeros(0).cuda(), None])
    g.flush(["smax_", "smax_"])  # an empty insert
    assert g.nchunks == 0 and g.countExistingElements() == 0 and g.countBoundaryElements() == 0
    g.findNeighbours()
    g.tagBoundaries()
    g.applyStencils(sgb.HEAT7, [0], [1], [0.1])
    g.applyStencils(sgb.HEAT7, [0], [1], [0.1], tiled=True)
    assert g.run_steps(sgb.HEAT7, [0], [1], [0.1], 5) is True
    keys, data, mask = g.deviceToHost()
    assert len(keys) == 0 and len(mask) == 512  # the background chunk only
    g.check_device_errors()


@pytest.mark.parametrize("size", [(8, 8, 8), (13, 7, 29), (1, 1, 1), (64, 9, 3)])
def test_ragged_domains_flush_tag_heat(sgb, size):
    """Domain sizes that are not multiples of 8 (the last chunk row is partial);
    every point of the domain inserted, the upper faces included."""
    pts = np.stack(np.meshgrid(*[np.arange(s) for s in size], indexing="ij"), -1).reshape(-1, 3).astype(np.int64)
    rng = np.random.default_rng(3)
    v = rng.random(len(pts)).astype(np.float32)
    g = sgb.SparseGridGpu(size, ["f32", "f32"], edge=8)
    o = O.OracleGrid(size, edge=8, ptypes=[O.T_F32, O.T_F32])
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda(), torch.from_numpy(v).cuda()])
    g.flush(["smax_", "smax_"])
    o.insert_flush(pts, [v, v], [O.OP_MAX, O.OP_MAX])
    g.tagBoundaries(O.NN_STAR)
    o.tag_boundaries(O.NN_STAR)
    for k in range(3):
        g.applyStencils(sgb.HEAT7, [k % 2], [1 - k % 2], [0.1])
        o.heat7(k % 2, 1 - k % 2, 0.1)
    _same_map(g, o, [0, 1], rtol=1e-6)
    assert g.countExistingElements() == int(np.prod(size))
    g.check_device_errors()


def test_one_point_many_duplicates(sgb):
    """10^5 copies of one point in insertion order: sRight_ keeps the last,
    sLeft_ the first, sadd_ the sum in insertion order."""
    n = 100000
    pts = np.tile(np.array([[5, 6, 7]], np.int64), (n, 1))
    v = (np.arange(n, dtype=np.float32) * np.float32(0.001)).astype(np.float32)
    for op, oop in (("sRight_", O.OP_RIGHT), ("sLeft_", O.OP_LEFT), ("sadd_", O.OP_ADD)):
        g = sgb.SparseGridGpu((16, 16, 16), ["f32"], edge=8)
        o = O.OracleGrid((16, 16, 16), edge=8, ptypes=[O.T_F32])
        g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda()])
        g.flush([op])
        o.insert_flush(pts, [v], [oop])
        _same_map(g, o, [0])
        val = g.get(0, torch.tensor([[5, 6, 7]]))[0].item()
        if op == "sRight_":
            assert val == v[-1]
        elif op == "sLeft_":
            assert val == v[0]


def test_isolated_chunks_stencils(sgb):
    """Chunks with no neighbour chunk at all: every halo read is the background."""
    size = (256, 256, 256)
    cen = np.array([[20, 20, 20], [100, 180, 60], [230, 40, 200]], np.int64)
    pts = np.concatenate([c + np.stack(np.meshgrid(*[np.arange(8)] * 3, indexing="ij"), -1).reshape(-1, 3) -
                          (c % 8) for c in cen])  # three whole, isolated 8^3 chunks
    rng = np.random.default_rng(4)
    vals = [rng.random(len(pts)).astype(np.float32) for _ in range(4)]
    g = sgb.SparseGridGpu(size, ["f32"] * 4, edge=8)
    o = O.OracleGrid(size, edge=8, ptypes=[O.T_F32] * 4)
    for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
        g.setBackgroundValue(p, b)
        o.set_background(p, b)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(x).cuda() for x in vals])
    g.flush(["smax_"] * 4)
    o.insert_flush(pts, vals, [O.OP_MAX] * 4)
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    for k in range(4):
        a, b = ([0, 1], [2, 3]) if k % 2 == 0 else ([2, 3], [0, 1])
        g.applyStencils(sgb.GS7, a, b, prm)
        o.gs7(a[0], a[1], b[0], b[1], *prm)
    keys, data, mask = g.deviceToHost()
    okeys, odata, omask = o.export()
    n = len(okeys)
    assert np.array_equal(keys, okeys) and n == 3
    for p in range(4):
        a, b = data[p][: n * 512].astype(np.float64), odata[p][: n * 512].astype(np.float64)
        err = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
        err[a == b] = 0
        assert err.max() <= 1e-6
    g.check_device_errors()


def test_occupancy_and_release(sgb):
    rng = np.random.default_rng(8)
    size = (40, 40, 40)
    pts = np.unique(rng.integers(0, size, size=(9000, 3)), axis=0).astype(np.int64)
    g = sgb.SparseGridGpu(size, ["f32", "f32"], edge=8)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(rng.random(len(pts)).astype(np.float32)).cuda(), None])
    g.flush(["sRight_", None])
    g.tagBoundaries(sgb.NN_STAR)
    keys, _, mask = g.deviceToHost()
    n = len(keys)
    mean, dev = g.measureBlockOccupancy()
    assert abs(mean * n * 512 - ((mask[: n * 512] & 3) == 1).sum()) < 1e-6 and dev > 0
    mem_mean, _ = g.measureBlockOccupancy(memory=True)
    assert abs(mem_mean * n * 512 - len(pts)) < 1e-6
    g.removeUnusedBuffers()
    g.applyStencils(sgb.HEAT7, [0], [1], [0.1])
    more = rng.integers(0, size, size=(500, 3)).astype(np.int64)
    g.insert(torch.from_numpy(more).cuda(), [torch.from_numpy(rng.random(500).astype(np.float32)).cuda(), None])
    g.flush(["sRight_", None])
    assert g.countExistingElements() == len(np.unique(np.concatenate([pts, more]), axis=0))
    g.check_device_errors()


def test_bounded_waits_give_up_and_the_device_stays_usable(sgb):
    """Failure detection without a GPU fault: a wait on an mbarrier phase nobody completes
    and one on a counter nobody increments each give up after 20 ms; the host reads
    SGB_ETIMEOUT and the device keeps working."""
    from openfpm_data_b200 import _lib as L
    lib = L.load()
    st = lib.sgb_probe_bounded_waits(20_000_000, 0, None)
    assert st == 6  # SGB_ETIMEOUT
    g = sgb.SparseGridGpu((32, 32, 32), ["f32", "f32"], edge=8)
    pts = np.array([[1, 2, 3], [4, 5, 6], [30, 30, 30]], dtype=np.int64)
    g.insert(torch.from_numpy(pts).cuda(), [torch.ones(3, device="cuda"), None])
    g.flush(["sRight_", None])
    g.applyStencils(sgb.HEAT7, [0], [1], [0.1])
    g.check_device_errors()
    assert g.countExistingElements() == 3
