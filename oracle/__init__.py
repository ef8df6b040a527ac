"""CPU oracle and CPU baseline for the SparseGridGpu hot path (test infrastructure only)."""
