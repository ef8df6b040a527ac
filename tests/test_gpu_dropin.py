"""The drop-in surfaces above the C ABI on the GPU: the C++ header
include/openfpm_b200/SparseGridGpu.hpp (compiled user code with device insert
pools and conv lambdas, tests/cpp/test_dropin.cu) and the pool / view entry
points it is built on (sgb_insert_pools, sgb_get_view)."""
import subprocess

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


def test_cpp_dropin_header():
    from openfpm_data_b200.build import build_dropin_test
    exe = build_dropin_test()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASSED" in r.stdout and "FAIL " not in r.stdout


@pytest.mark.parametrize("op", ["sRight_", "sLeft_", "sadd_", "smax_", "smin_"])
def test_insert_pools_equals_insert_in_pool_order(sgb, op):
    """Pools are staged pool after pool, slot order inside a pool (the
    reference's make_continuos), so a pool flush equals a staged insert of
    the concatenated pool contents, order-dependent reductions included."""
    rng = np.random.default_rng(3)
    size = (40, 56, 48)
    npools, nslot = 37, 300
    counts = rng.integers(0, nslot + 1, npools).astype(np.int32)
    counts[5] = 0
    counts[6] = nslot
    pts = rng.integers(0, size, size=(npools, nslot, 3))
    pts[:, nslot // 2:] = pts[:, : nslot - nslot // 2]  # duplicates inside pools
    pts[1::2, :40] = pts[::2, :40][: len(pts[1::2])]    # and across pools
    lin = np.empty((npools, nslot), np.int64)
    bsz = [(s + 7) // 8 for s in size]
    bid = ((pts[..., 2] // 8) * bsz[1] + pts[..., 1] // 8) * bsz[0] + pts[..., 0] // 8
    loc = ((pts[..., 2] % 8) * 8 + pts[..., 1] % 8) * 8 + pts[..., 0] % 8
    lin[:] = bid * 512 + loc
    v0 = rng.random((npools, nslot)).astype(np.float32)
    v1 = rng.integers(-1000, 1000, (npools, nslot)).astype(np.int32)
    ops = [op, op]

    a = sgb.SparseGridGpu(size, ["f32", "i32"], edge=8)
    a.insert_pools(torch.from_numpy(counts), torch.from_numpy(lin), [torch.from_numpy(v0), torch.from_numpy(v1)])
    a.flush(ops)

    sel = np.concatenate([np.arange(c) + i * nslot for i, c in enumerate(counts)])
    b = sgb.SparseGridGpu(size, ["f32", "i32"], edge=8)
    b.insert_lin(torch.from_numpy(lin.reshape(-1)[sel]),
                 [torch.from_numpy(v0.reshape(-1)[sel]), torch.from_numpy(v1.reshape(-1)[sel])])
    b.flush(ops)

    ka, da, ma = a.deviceToHost()
    kb, db, mb = b.deviceToHost()
    assert np.array_equal(ka, kb) and np.array_equal(ma, mb)
    ex = (ma & 1).astype(bool)
    for p in range(2):
        assert np.array_equal(da[p][ex].view(np.uint8), db[p][ex].view(np.uint8))
    a.check_device_errors()
    b.check_device_errors()


def test_insert_pools_overflow_is_reported(sgb):
    g = sgb.SparseGridGpu((16, 16, 16), ["f32"], edge=8)
    counts = torch.tensor([3, 9], dtype=torch.int32)  # 9 > nslot
    lin = torch.zeros((2, 4), dtype=torch.int64)
    g.insert_pools(counts, lin, [torch.ones((2, 4))])
    with pytest.raises(sgb.SgbError, match="insert pool"):
        g.flush(["smax_"])
    assert g.nchunks == 0  # the staged inserts were dropped
    g.check_device_errors()  # and the error word cleared


def test_view_describes_the_block_map(sgb):
    rng = np.random.default_rng(8)
    size = (64, 32, 40)
    pts = np.unique(rng.integers(0, size, size=(4000, 3)), axis=0)
    g = sgb.SparseGridGpu(size, ["f32", "f64"], edge=4)
    g.insert(torch.from_numpy(pts).cuda(), [torch.ones(len(pts)).cuda(), torch.ones(len(pts)).cuda()])
    g.flush(["smax_", "smax_"])
    for nn in (O.NN_STAR, O.NN_FULL):
        v = g.view(nn)
        assert v["n"] == g.nchunks and v["edge"] == 4 and v["bs"] == 64 and v["nprop"] == 2
        assert v["size"] == size and v["bsz"] == (16, 8, 10) and v["nn_kind"] == nn
        assert v["keys"] == g.private_get_index_array().data_ptr()
        k = 8 if nn == O.NN_STAR else 27
        # the view's int32 table (-1 absent) is the reference-format table with n -> -1
        from openfpm_data_b200.grid import _DevView
        t = torch.as_tensor(_DevView(v["nn"], (v["n"] * k,), "<i4"), device="cuda").cpu().numpy()
        t = t.reshape(v["n"], k).astype(np.int64)
        ref = g.neighbour_table(nn)
        exp = ref.copy()
        exp[exp == v["n"]] = -1
        used = ref != -1 if nn == O.NN_STAR else np.ones_like(ref, bool)
        assert np.array_equal(t[used], exp[used])


@pytest.mark.parametrize("edge", [8, 4])
@pytest.mark.parametrize("op", ["sRight_", "sadd_", "smax_"])
def test_insert_blocks_matches_chunk_slot_flush(sgb, edge, op):
    """Chunk slots written through insertBlock (BlockMapGpu_ker.cuh:199-227), flushed onto a map
    that already holds points: bit-exact against the oracle's chunk-slot flush
    (segreduce_total / solve_conflicts restated), duplicates across slots and pools included."""
    rng = np.random.default_rng(31 + edge)
    size = (48, 40, 56)
    bs = edge ** 3
    bsz = [(s + edge - 1) // edge for s in size]
    nkeys = bsz[0] * bsz[1] * bsz[2]
    npools, nslot = 13, 5
    counts = rng.integers(1, nslot + 1, npools).astype(np.int32)
    keys = rng.integers(0, nkeys, (npools, nslot)).astype(np.int64)
    keys[3:6, :2] = keys[0, 0]  # the same chunk in several slots and pools
    masks = (rng.random((npools, nslot, bs)) < 0.3).astype(np.uint8)
    masks[..., 0] = 1  # every slot holds at least one point
    v0 = rng.random((npools, nslot, bs)).astype(np.float32)
    v1 = rng.integers(-500, 500, (npools, nslot, bs)).astype(np.int32)
    ops = [op, op]
    oops = [getattr(O, {"sRight_": "OP_RIGHT", "sadd_": "OP_ADD", "smax_": "OP_MAX"}[op])] * 2

    g = sgb.SparseGridGpu(size, ["f32", "i32"], edge=edge)
    o = O.OracleGrid(size, edge=edge, ptypes=[O.T_F32, O.T_I32])
    # points already in the map, so that slots merge with old chunks
    pts = rng.integers(0, size, size=(3000, 3)).astype(np.int64)
    pv = [rng.random(3000).astype(np.float32), rng.integers(-9, 9, 3000).astype(np.int32)]
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(x).cuda() for x in pv])
    g.flush(["smax_", "smax_"])
    o.insert_flush(pts, pv, [O.OP_MAX, O.OP_MAX])

    g.insert_blocks(torch.from_numpy(counts), torch.from_numpy(keys), [torch.from_numpy(v0), torch.from_numpy(v1)],
                    torch.from_numpy(masks))
    g.flush(ops)
    sel = np.concatenate([np.arange(c) + i * nslot for i, c in enumerate(counts)])
    o.flush_chunks(keys.reshape(-1)[sel], [v0.reshape(-1, bs)[sel].reshape(-1), v1.reshape(-1, bs)[sel].reshape(-1)],
                   masks.reshape(-1, bs)[sel].reshape(-1), oops)
    kg, dg, mg = g.deviceToHost()
    ko, do, mo = o.export()
    n = len(ko)
    assert np.array_equal(kg, ko) and np.array_equal(mg[: n * bs], mo[: n * bs])
    ex = (mo[: n * bs] & 1).astype(bool)
    for p in range(2):
        assert np.array_equal(dg[p][: n * bs][ex].view(np.uint8), do[p][: n * bs][ex].view(np.uint8)), f"prop {p}"
    g.check_device_errors()


def test_insert_blocks_overflow_is_reported(sgb):
    g = sgb.SparseGridGpu((16, 16, 16), ["f32"], edge=8)
    masks = torch.ones((1, 2, 512), dtype=torch.uint8)
    g.insert_blocks(torch.tensor([3], dtype=torch.int32), torch.zeros((1, 2), dtype=torch.int64),
                    [torch.ones((1, 2, 512))], masks)
    with pytest.raises(sgb.SgbError, match="insert pool"):
        g.flush(["smax_"])
    g.check_device_errors()
