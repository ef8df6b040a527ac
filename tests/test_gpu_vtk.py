"""write(): the points whose mask byte is not 0, their properties and mask
bytes, read back from the VTK file and compared with the oracle's points."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _read_vtk(path):
    b = open(path, "rb").read()
    i = b.index(b"POINTS ")
    j = b.index(b"\n", i)
    m = int(b[i:j].split()[1])
    pos = np.frombuffer(b, ">f4", 3 * m, j + 1).reshape(m, 3)
    data = {}
    k = j
    while True:
        k = b.find(b"SCALARS ", k)
        if k < 0:
            break
        e = b.index(b"\n", k)
        name, vt = b[k:e].split()[1:3]
        s = b.index(b"\n", e + 1) + 1  # LOOKUP_TABLE line
        dt = {b"float": ">f4", b"int": ">i4", b"double": ">f8", b"unsigned_char": "u1"}[vt]
        data[name.decode()] = np.frombuffer(b, dt, m, s)
        k = s + m * np.dtype(dt).itemsize
    return pos, data


@pytest.mark.parametrize("lin", ["smb", "zmb"])
def test_write_vtk(tmp_path, lin):
    import openfpm_data_b200 as sgb
    rng = np.random.default_rng(5)
    size = (40, 48, 36)
    pts = np.unique(rng.integers(0, size, size=(6000, 3)), axis=0).astype(np.int64)
    v0 = rng.random(len(pts)).astype(np.float32)
    v1 = rng.integers(-50, 50, len(pts)).astype(np.int32)
    g = sgb.SparseGridGpu(size, ["f32", "i32"], edge=8, linearizer=lin)
    o = O.OracleGrid(size, edge=8, ptypes=[O.T_F32, O.T_I32], zorder=lin == "zmb")
    g.insert(torch.from_numpy(pts).cuda(), [torch.from_numpy(v0).cuda(), torch.from_numpy(v1).cuda()])
    g.flush(["sRight_", "sRight_"])
    o.insert_flush(pts, [v0, v1], [O.OP_RIGHT, O.OP_RIGHT])
    g.tagBoundaries(sgb.NN_STAR)
    o.tag_boundaries(O.NN_STAR)
    f = tmp_path / "sg.vtk"
    assert g.write(str(f), spacing=(0.5, 0.5, 0.5), offset=(1.0, 2.0, 3.0))
    pos, data = _read_vtk(str(f))
    ex = o.existing_points()  # every existing point (mask bytes 1 or 3), in chunk then offset order
    assert np.array_equal(pos, ((ex + np.array([1.0, 2.0, 3.0])) * 0.5).astype(np.float32))
    assert np.array_equal(data["attr0"], o.get(0, ex)) and np.array_equal(data["attr1"], o.get(1, ex))
    assert np.array_equal(data["mask"], o.mask_at(ex))
