"""FP32 arithmetic of the symmetric backprojector's voxel step, restated in
numpy (CPU only).

The staged path of the interleaved-quad kernel steps the detector row
coordinate v of the 8 voxels of a column as pairs: (vl, vl + dvv), then
+ (2 dvv, 2 dvv) per pair, each a single-rounded FP32 add. The unstaged path
(and the form the staged path replaced) computes v_j = fma(j, dvv, vl). The
two may differ by the rounding of the repeated additions; bilinear
interpolation is continuous in v, so a difference of a few ulps of v moves a
tap by a few ulps of the detector sample spacing."""
from __future__ import annotations

import numpy as np

NY = 8  # voxels per thread column


def _f32(x):
    return np.asarray(x, np.float64).astype(np.float32)


def v_fma(vl, dvv):
    # fma(j, dvv, vl): exact j * dvv + vl (all products exact in FP64), one rounding
    j = np.arange(NY, dtype=np.float64)[:, None]
    return _f32(j * dvv.astype(np.float64) + vl.astype(np.float64))


def v_stepped(vl, dvv):
    out = np.empty((NY,) + vl.shape, np.float32)
    v0, v1 = vl.copy(), _f32(vl.astype(np.float64) + dvv.astype(np.float64))
    step = _f32(2.0 * dvv.astype(np.float64))  # exact: a power-of-two scaling
    for j in range(0, NY, 2):
        if j:
            v0 = _f32(v0.astype(np.float64) + step.astype(np.float64))
            v1 = _f32(v1.astype(np.float64) + step.astype(np.float64))
        out[j], out[j + 1] = v0, v1
    return out


def test_stepped_v_stays_within_a_few_ulps_of_the_fma_form():
    rng = np.random.default_rng(3)
    n = 200_000
    # window-local v of the first voxel and the per-voxel row step: windows are
    # at most a few hundred rows high, cone magnification keeps dvv below ~4
    vl = _f32(rng.uniform(0.0, 256.0, n))
    dvv = _f32(rng.uniform(0.05, 4.0, n))
    a, b = v_fma(vl, dvv), v_stepped(vl, dvv)
    ulp = np.spacing(np.maximum(np.abs(a), np.abs(b)).astype(np.float32))
    d = np.abs(a.astype(np.float64) - b.astype(np.float64)) / ulp
    # three rounded adds (voxels 6, 7) and the FMA's own rounding: at most 2 ulps
    assert d.max() <= 2.0, d.max()
    # voxels 0 and 1 are formed exactly as in the FMA form
    assert np.array_equal(a[:2], b[:2])
    # most taps land on the same row with the same fraction
    assert (d == 0).mean() > 0.5
