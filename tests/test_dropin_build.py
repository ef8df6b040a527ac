"""The C++ drop-in header compiles as user code (nvcc cross-compiles for
sm_100a without a GPU); running it is tests/test_gpu_dropin.py."""
import os
import shutil

import pytest


@pytest.mark.skipif(shutil.which(os.environ.get("NVCC", "nvcc")) is None, reason="nvcc not found")
def test_dropin_header_compiles():
    from openfpm_data_b200.build import build_dropin_test
    exe = build_dropin_test()
    assert os.path.exists(exe) and os.access(exe, os.X_OK)
