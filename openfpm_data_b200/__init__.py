"""B200-native SparseGridGpu hot path (insert / flush / tagBoundaries / stencils).

The compute lives in ``libsgb200.so`` (CUDA, sm_100a) behind the C ABI of
``include/sgb200.h``; this package is the Python host mirror used by tests,
benchmarks and the serving loop.  The C++ drop-in front-end is
``include/openfpm_b200/SparseGridGpu.hpp``.
"""
from ._lib import (BOX27, BOX27_NS, F32, F64, GS7, HEAT7, I32, NN_FULL, NN_STAR, OP_ADD, OP_LEFT, OP_MAX, OP_MIN, OP_NONE,
                   OP_OR, OP_RIGHT, U8, SgbError, load)
from .grid import OPS, Batch, SparseGridGpu

__all__ = ["SparseGridGpu", "Batch", "OPS", "SgbError", "load", "F32", "I32", "F64", "U8", "OP_NONE", "OP_RIGHT",
           "OP_LEFT", "OP_ADD", "OP_MAX", "OP_MIN", "OP_OR", "NN_STAR", "NN_FULL", "HEAT7", "GS7", "BOX27", "BOX27_NS"]
