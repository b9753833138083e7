"""The allocation-free 2D filter entry point against the context entry point.

fbp2d_filter_sinogram_noalloc serves callers that cannot allocate device
memory while they run (memory owned by the host application's pool, real-time
loops where an allocation would synchronise the device). It keeps its tables
in a fixed device array instead of context scratch, so its result must equal
fbp2d_filter_sinogram's, call after call, on the same input. This file is
collected last so that a failure here cannot hide any other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import relative_rmse

pytestmark = pytest.mark.gpu

TOL = 1e-6  # filtered rows, FP32 (same tolerance as the other row-filter tests)


def test_noalloc_filter_matches_context_filter_twice():
    import torch

    import fbp_b200 as F

    lib = F.library()
    ctx = F.Context(0)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(2024)
    # two calls in a row with different sizes, filters and weighting: the
    # second call must not see anything the first left in the shared array
    cases = [(360, 367, F.FilterType.RAM_LAK, 0.0, 0.0), (720, 768, F.FilterType.SHEPP_LOGAN, 1000.0, 768.0)]
    for views, bins, filt, sdd, width in cases:
        sino = (rng.standard_normal((views, bins)) + 1.0).astype(np.float32)
        ref = torch.tensor(sino, device="cuda")
        out = ref.clone()
        ctx.call("fbp2d_filter_sinogram", C.c_void_p(ref.data_ptr()), bins, views, int(filt), sdd, width)
        ctx.call("fbp_synchronize")
        rc = lib.fbp2d_filter_sinogram_noalloc(C.c_void_p(out.data_ptr()), bins, views, int(filt), sdd, width, 0,
                                               C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.fbp_last_error(None)
        stream.synchronize()
        assert relative_rmse(out.cpu().numpy(), ref.cpu().numpy()) < TOL
    ctx.close()


def test_noalloc_filter_rejects_rows_beyond_its_capacity():
    import fbp_b200 as F

    lib = F.library()
    # 5000 bins pad to 8192 samples, above the 4096-sample maximum: rejected
    # before any device work
    rc = lib.fbp2d_filter_sinogram_noalloc(C.c_void_p(16), 5000, 2, 0, 0.0, 0.0, 0, None)
    assert rc == -6
    assert b"4096" in lib.fbp_last_error(None)
