"""A batch whose field arrays pass the size at which device arrays grow in place (256 MB).

Four heat grids of 384^3 (a ball of radius 0.45 edge, about 45,000 chunks each) join a
batch; one is removed, so the next add compacts the batch into arrays that hold the
remaining 135,000 chunks, and a small 256^3 grid joins without the batch growing again.
Every grid that finishes is compared bit for bit with the same grid stepped alone."""
import numpy as np
import pytest
import torch

from openfpm_data_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sgb():
    import openfpm_data_b200 as m
    assert torch.cuda.is_available(), "these tests need a CUDA device"
    m.load()
    return m


def _maps(edge, vseed):
    ps = W.single_ball_grid(edge, 0.45 * edge, vseed)
    return ps.size, W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)


def _grid(sgb, size, m):
    keys, data, mask = m
    g = sgb.SparseGridGpu(size, ["f32", "f32"], edge=8)
    g.setBackgroundValue(0, 0.0)
    g.setBackgroundValue(1, 0.0)
    g.load_map(keys, data + [data[0].copy()], mask)
    return g


def test_large_batch_with_holes_matches_single_grids(sgb):
    big_size, big = _maps(384, 5)
    small_size, small = _maps(256, 6)
    assert 3 * len(big[0]) * 512 * 4 > (256 << 20), "the compacted field arrays pass 256 MB"
    # name: (grid, steps)
    plan = {"a": ("big", 5), "b": ("big", 8), "c": ("big", 8), "e": ("big", 5), "d": ("small", 6)}
    maps = {"big": (big_size, big), "small": (small_size, small)}
    alone = {}
    for kind, st in {(k, s) for k, s in plan.values()}:
        g = _grid(sgb, *maps[kind])
        g.run_steps(sgb.HEAT7, [0], [1], [0.1], st, use_graph=False)
        alone[(kind, st)] = g.deviceToHost()[1]
        del g
    batch = sgb.Batch()
    slots = {}
    for name in ("a", "b", "c", "e"):
        kind, st = plan[name]
        gb = _grid(sgb, *maps[kind])
        slots[name] = (batch.add(gb, sgb.HEAT7, [0], [1], [0.1], st), gb)
    batch.step(2)
    batch.remove(slots.pop("b")[0])
    kind, st = plan["d"]
    gb = _grid(sgb, *maps[kind])
    slots["d"] = (batch.add(gb, sgb.HEAT7, [0], [1], [0.1], st), gb)  # compaction first, then the add
    batch.step(8)
    for name, (slot, gb) in slots.items():
        kind, st = plan[name]
        assert batch.slot_steps(slot) == st
        batch.extract(slot, gb)
        got = gb.deviceToHost()[1]
        for a, b in zip(alone[(kind, st)], got):
            assert np.array_equal(a, b), f"grid {name}"
    batch.close()
