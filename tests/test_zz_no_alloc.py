"""sgb_existing_offsets_noalloc: the allocation-free variant of
sgb_existing_offsets, for callers that may not allocate device memory (their
memory belongs to their own pool allocator, or a cudaMalloc that can
synchronise the device is not allowed where they call).  Its result must
equal the allocating entry point's on consecutive calls (the scratch array is
shared and keeps the previous call's contents), and grids above its stated
maximum of 1,048,576 chunks must be refused.  This file is collected last."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _offsets(lib, g, noalloc):
    out = torch.full((g.nchunks + 1,), -7, dtype=torch.int64, device="cuda")
    fn = lib.sgb_existing_offsets_noalloc if noalloc else lib.sgb_existing_offsets
    st = fn(g.handle, C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return st, out.cpu().numpy()


def test_noalloc_offsets_match_allocating_entry_point():
    import openfpm_data_b200 as sgb
    from openfpm_data_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(12)
    grids = []
    for edge, size, npts in [(8, (96, 80, 72), 60000), (4, (64, 64, 64), 90000)]:
        g = sgb.SparseGridGpu(size, ["f32"], edge=edge)
        pts = rng.integers(0, size, size=(npts, 3)).astype(np.int64)
        g.insert(torch.from_numpy(pts).cuda(), [torch.ones(npts, device="cuda")])
        g.flush(["smax_"])
        grids.append(g)
    # two calls in a row (different grids, then the first again): the shared
    # scratch must not carry anything from one call into the next
    for g in grids + grids[:1]:
        st_a, ref = _offsets(lib, g, noalloc=False)
        st_b, got = _offsets(lib, g, noalloc=True)
        assert st_a == 0 and st_b == 0
        assert np.array_equal(got, ref)
        assert got[-1] == g.countExistingElements()


def test_noalloc_rejects_grids_above_its_maximum():
    import openfpm_data_b200 as sgb
    from openfpm_data_b200 import _lib
    lib = _lib.load()
    n = 1_048_577  # one chunk more than the stated maximum
    g = sgb.SparseGridGpu((1024, 1024, 1024), ["u8"], edge=4)
    keys = torch.arange(n, dtype=torch.int64, device="cuda")
    g.load_map_dev(keys, [torch.zeros(n * 64, dtype=torch.uint8, device="cuda")],
                   torch.ones(n * 64, dtype=torch.uint8, device="cuda"))
    st, _ = _offsets(lib, g, noalloc=True)
    assert st == _lib.ERANGE
    assert b"1048576" in lib.sgb_last_error_string()
    st, ref = _offsets(lib, g, noalloc=False)  # the allocating entry point has no such limit
    assert st == 0 and ref[-1] == n * 64


def test_noalloc_offsets_at_the_maximum_size():
    """Exactly 1,048,576 chunks: all 512 scan tiles and the full one-CTA scan of
    the tile sums run; the result must equal the allocating entry point's."""
    import openfpm_data_b200 as sgb
    from openfpm_data_b200 import _lib
    lib = _lib.load()
    n = 1_048_576
    g = sgb.SparseGridGpu((1024, 1024, 1024), ["u8"], edge=4)
    keys = torch.arange(n, dtype=torch.int64, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(5)
    mask = (torch.rand(n * 64, device="cuda", generator=gen) < 0.37).to(torch.uint8)
    g.load_map_dev(keys, [torch.zeros(n * 64, dtype=torch.uint8, device="cuda")], mask)
    for _ in range(2):  # two calls in a row on the shared scratch
        st_a, ref = _offsets(lib, g, noalloc=False)
        st_b, got = _offsets(lib, g, noalloc=True)
        assert st_a == 0 and st_b == 0
        assert np.array_equal(got, ref)
    assert got[-1] == int(mask.sum().item())
