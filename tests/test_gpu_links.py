"""Multi-resolution links (construct_link_dw / construct_link_up) against the
oracle's restatement of the reference kernels: padding points, per-point
offsets and links, exact.  No reference test covers the links, so parity is
pinned by the restated kernels only."""
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


def _level(sgb, size, pts, edge):
    g = sgb.SparseGridGpu(size, ["f32"], edge=edge)
    o = O.OracleGrid(size, edge=edge, ptypes=[O.T_F32])
    v = np.ones(len(pts), np.float32)
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v).cuda()])
    g.flush(["sRight_"])
    o.insert_flush(pts, [v], [O.OP_RIGHT])
    g.tagBoundaries(sgb.NN_STAR)
    o.tag_boundaries(O.NN_STAR)
    return g, o


def _ball(c, r, size):
    lo = np.maximum(np.floor(np.array(c) - r).astype(int), 0)
    hi = np.minimum(np.ceil(np.array(c) + r).astype(int), np.array(size) - 1)
    ax = [np.arange(a, b + 1) for a, b in zip(lo, hi)]
    g = np.stack(np.meshgrid(*ax, indexing="ij"), axis=-1).reshape(-1, 3)
    return g[((g - np.array(c)) ** 2).sum(axis=1) <= r * r].astype(np.int64)


def _same(a, b):
    for k in ("pad_pos", "pad_off", "offsets", "link_pos", "link_off"):
        assert np.array_equal(a[k].cpu().numpy(), b[k]), k


@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("shift", [(0, 0, 0), (1, -1, 0), (-2, 3, 1)])
def test_links_match_oracle(sgb, edge, shift):
    # a coarse level (a ball) and a finer level (a ball twice as large, slightly off), both
    # tagged so their surfaces are padding points
    coarse_size, fine_size = (60, 52, 56), (120, 104, 112)
    gc, oc = _level(sgb, coarse_size, _ball((28, 25, 27), 17, coarse_size), edge)
    gf, of = _level(sgb, fine_size, _ball((57, 51, 55), 33, fine_size), edge)
    box = ((3, 0, 2), (50, 48, 51))
    gc.construct_link_dw(gf, box, shift)
    _same(gc.getDownLinks(), oc.construct_links(of, box, shift, up=False))
    fbox = ((0, 0, 0), (119, 103, 111))
    gf.construct_link_up(gc, fbox, shift)
    _same(gf.getUpLinks(), of.construct_links(oc, fbox, shift, up=True))
    d = gc.getDownLinks()
    assert d["pad_pos"].numel() > 1000 and d["link_pos"].numel() > 0
    # the reference's loop bound: at most 6 links per padding point
    assert int((d["offsets"][1:] - d["offsets"][:-1]).max()) <= 6


def test_links_out_of_domain_and_empty(sgb):
    # children past the fine grid's last chunk wrap through the unchecked linearisation,
    # like the reference's; an empty box gives no padding point
    gc, oc = _level(sgb, (32, 32, 32), _ball((25, 16, 16), 7, (32, 32, 32)), 8)
    gf, of = _level(sgb, (40, 64, 64), _ball((30, 32, 32), 9, (40, 64, 64)), 8)
    box = ((0, 0, 0), (31, 31, 31))
    gc.construct_link_dw(gf, box, (0, 0, 0))
    _same(gc.getDownLinks(), oc.construct_links(of, box, (0, 0, 0), up=False))
    gc.construct_link_dw(gf, ((40, 40, 40), (30, 30, 30)), (0, 0, 0))
    d = gc.getDownLinks()
    assert d["pad_pos"].numel() == 0 and d["link_pos"].numel() == 0 and int(d["offsets"][0]) == 0
