"""Inputs of the reference's pack / unpack known-answer tests.

The hollow sphere of insertSphere3D_radius / insertSphere3D_radiusV
(src/SparseGridGpu/tests/utils/SparseGridGpu_testKernels.cuh:202-316): 32^3
chunks of edge 4 from (256, 256, 256), centre (320, 320, 320); a point exists
when 56 < sqrtf(x^2 + y^2 + z^2) < 64 (x, y, z relative to the centre, the
square root in float); values x+y+z and, for the V variant, the float[3]
(x, y, z).  The pack / unpack boxes of SparseGridGpu_tests.cu:1382-1420 and
1533-1730 and their expected counts.
"""
import numpy as np

SIZE = (1000, 1000, 1000)
EDGE = 4
START = 256
CENTRE = START + 32 // 2 * EDGE

# SparseGridGpu_tests.cu:1536-1541 source boxes, 1705-1709 destination boxes (inclusive)
SRC_BOXES = [((256, 256, 256), (273, 390, 390)), ((320, 256, 256), (337, 390, 390)),
             ((256, 256, 256), (273, 320, 390)), ((320, 256, 256), (337, 320, 390))]
DST_BOXES = [((256, 256, 256), (273, 390, 390)), ((274, 256, 256), (291, 390, 390)),
             ((300, 256, 256), (317, 320, 390)), ((320, 256, 256), (337, 320, 390))]
# 1633-1672: chunks and points of each packed box; 1817-1820 and 1933-1936: points per
# destination box after unpacking, all points and odd points (x+y+z odd) only
PACK_NCNK = [1107, 1420, 610, 739]
PACK_NPNT = [41003, 54276, 20828, 27283]
UNPACK_CNT_ALL = [41003, 54276, 20828, 27283]
UNPACK_CNT_ODD = [20520, 27152, 10423, 13649]
# 1410-1432: packRequest of the x < 322 and x >= 322 halves of the one-property sphere
HALF_BOXES = [((0, 0, 0), (321, 999, 999)), ((322, 0, 0), (999, 999, 999))]
HALF_NCNK = [4685, 4475]
HALF_NPNT = [185807, 176787]


def sphere(odd_only=False):
    """(coords [n, 3] int64, rel [n, 3] int64) of the sphere's points, chunk-major."""
    r = np.arange(START, START + 32 * EDGE, dtype=np.int64)
    x, y, z = np.meshgrid(r, r, r, indexing="ij")
    c = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    rel = c - CENTRE
    d2 = (rel * rel).sum(axis=1).astype(np.float32)
    rad = np.sqrt(d2)
    keep = (rad < np.float32(64)) & (rad > np.float32(56))
    if odd_only:
        keep &= c.sum(axis=1) % 2 == 1
    return c[keep], rel[keep]


def sphere_values(rel):
    """[x+y+z, x, y, z] as float32 arrays."""
    return [rel.sum(axis=1).astype(np.float32)] + [rel[:, d].astype(np.float32) for d in range(3)]


def box_rows(boxes):
    return np.array([list(lo) + list(hi) for lo, hi in boxes], dtype=np.int64)


def packed_size(n_cnk, n_pnt, point_size):
    """SparseGridGpu.hpp:3192-3200."""
    a8 = lambda b: (b + 7) & ~7
    return 8 + 2 * 3 * 4 + 8 * n_cnk + a8(4 * (n_cnk + 1)) + a8(n_pnt * point_size) + a8(2 * n_pnt) + a8(n_pnt)
