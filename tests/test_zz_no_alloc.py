"""The allocation-free 2D filter entry point.

fbp2d_filter_sinogram_noalloc serves callers that cannot allocate device
memory while they run: hosts that own all GPU memory through their own pool,
real-time read-out loops where an allocation would synchronise the device and
stall the detector, plugin hosts that forbid allocations after start-up. It
keeps its tables in one fixed device array instead of context scratch, so its
result must equal fbp2d_filter_sinogram's bit for bit, call after call, on
the same input, and agree with the FP64 oracle. This file is collected last
so that a failure here cannot hide any other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import relative_rmse

pytestmark = pytest.mark.gpu

TOL_ROWS = 1e-6  # filtered rows, FP32 (the tolerance of the other row-filter tests)

# Consecutive calls share the array: the sizes go up, then down (a large
# table followed by a smaller one leaves stale entries past the new length),
# with different filters and weighting, and end with a one-bin row.
CASES = [
    (360, 367, 0, 0.0, 0.0),         # RAM_LAK, n 512
    (720, 768, 1, 1000.0, 768.0),    # SHEPP_LOGAN, fan weight, n 1024
    (301, 200, 2, 0.0, 0.0),         # COSINE, n 256
    (64, 1, 3, 0.0, 0.0),            # HANN, one bin, n 1
]


def _oracle_rows(oracle, sino, filt, sdd, width):
    x = sino.astype(np.float64)
    if sdd > 0.0:
        bins = x.shape[1]
        x = oracle.fdk_weight(x[:, None, :], sdd, width / bins, 1.0)[:, 0, :]
    return oracle.filter_rows(x, filt)


def test_noalloc_filter_matches_context_filter_and_oracle(oracle):
    import torch

    import fbp_b200 as F

    lib = F.library()
    ctx = F.Context(0)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(2024)
    for views, bins, filt, sdd, width in CASES:
        sino = (rng.standard_normal((views, bins)) + 1.0).astype(np.float32)
        ref = torch.tensor(sino, device="cuda")
        out = ref.clone()
        ctx.call("fbp2d_filter_sinogram", C.c_void_p(ref.data_ptr()), bins, views, filt, sdd, width)
        ctx.call("fbp_synchronize")
        rc = lib.fbp2d_filter_sinogram_noalloc(C.c_void_p(out.data_ptr()), bins, views, filt, sdd, width, 0,
                                               C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.fbp_last_error(None)
        stream.synchronize()
        # same kernels, same tables, same arguments: identical bits
        assert torch.equal(out, ref), (views, bins, filt)
        err = relative_rmse(out.cpu().numpy(), _oracle_rows(oracle, sino, filt, sdd, width))
        assert err < TOL_ROWS, (views, bins, filt, err)
    ctx.close()


def test_noalloc_filter_repeats_bit_for_bit():
    """Two calls in a row on the same input give the same bits (nothing the
    first call leaves in the shared array changes the second)."""
    import torch

    import fbp_b200 as F

    lib = F.library()
    stream = torch.cuda.current_stream()
    sino = torch.tensor(np.random.default_rng(5).standard_normal((128, 500)).astype(np.float32), device="cuda")
    outs = []
    for _ in range(2):
        x = sino.clone()
        rc = lib.fbp2d_filter_sinogram_noalloc(C.c_void_p(x.data_ptr()), 500, 128, 0, 0.0, 0.0, 0,
                                               C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.fbp_last_error(None)
        outs.append(x)
    stream.synchronize()
    assert torch.equal(outs[0], outs[1])


def test_noalloc_filter_rejects_rows_beyond_its_capacity():
    import fbp_b200 as F

    lib = F.library()
    # 5000 bins pad to 8192 samples, above the 4096-sample maximum: rejected
    # before any device work
    rc = lib.fbp2d_filter_sinogram_noalloc(C.c_void_p(16), 5000, 2, 0, 0.0, 0.0, 0, None)
    assert rc == -6
    assert b"4096" in lib.fbp_last_error(None)
