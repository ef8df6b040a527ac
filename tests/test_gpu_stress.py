"""The insert / flush / tag / 27-point stress workload at its full size: a
1024^3 grid of 8^3 chunks with float32 + int32 properties and a float32
destination; each iteration inserts 2M clustered points (64 Gaussian
clusters, sigma 24, 30% exact duplicates, seed 2), flushes with sRight_ on
both properties, tags boundaries (NNStar) and applies one 27-point box
average (coefficients 1/27, NNFull).  Everything integer / byte / index is
compared bit for bit with the oracle after every iteration; the box average
within 1e-6 relative."""
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


def test_insert_flush_tag_box27_stress(sgb):
    size = (1024, 1024, 1024)
    ptypes = [O.T_F32, O.T_I32, O.T_F32]
    g = sgb.SparseGridGpu(size, ["f32", "i32", "f32"], edge=8)
    o = O.OracleGrid(size, edge=8, ptypes=ptypes)
    for p in range(3):
        g.setBackgroundValue(p, 0)
        o.set_background(p, 0)
    coeff = np.full(27, np.float32(1.0 / 27.0), dtype=np.float32)
    for it in range(3):
        pts, fv, iv = W.insert_batch(it)
        g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(fv).cuda(), torch.from_numpy(iv).cuda(), None])
        g.flush(["sRight_", "sRight_"])
        o.insert_flush(pts, [fv, iv, np.zeros(len(pts), np.float32)], [O.OP_RIGHT, O.OP_RIGHT, O.OP_NONE])
        g.tagBoundaries(O.NN_STAR)
        o.tag_boundaries(O.NN_STAR)
        g.applyStencils(sgb.BOX27, [0], [2], coeff)
        o.box27(0, 2, coeff)
        keys, data, mask = g.deviceToHost()
        okeys, odata, omask = o.export()
        n = len(okeys)
        assert np.array_equal(keys, okeys), f"iteration {it}: block map"
        assert np.array_equal(mask[: n * 512], omask[: n * 512]), f"iteration {it}: masks"
        ex = (mask[: n * 512] & 1).astype(bool)
        for p in (0, 1):
            assert np.array_equal(data[p][: n * 512][ex].view(np.uint8), odata[p][: n * 512][ex].view(np.uint8))
        act = (mask[: n * 512] & 3) == 1
        a = data[2][: n * 512][act].astype(np.float64)
        b = odata[2][: n * 512][act].astype(np.float64)
        err = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
        err[a == b] = 0
        assert err.max(initial=0) <= RTOL
        # size-independent checks: every inserted point exists, the duplicates collapsed
        assert g.countExistingElements() == int(ex.sum())
    g.check_device_errors()
