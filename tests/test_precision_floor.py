"""Storage-precision floor of 16-bit filtered views on the large noisy cone
workload (1440^3-class, 1536^2 detector at 0.254 mm, Poisson I0 = 5e4, Hann
ramp). Each 16-bit format below is emulated on two filtered views of that
workload at 2e5 random bilinear taps: none gets its per-tap relative error
under 1e-4 (FP16 has an 11-bit significand; int16 loses ~4.5 bits to the
max/RMS ratio of ~22 of ramp-filtered views), while a 24-bit (FP32 with the
low byte dropped) format stays near 1e-5. The reconstructed volume's error is
smaller than the per-tap error (tap errors are independent across the 1440
views, the signal adds coherently). The FP16 gradient quads take each
difference against the corner values as they will be read back (error
feedback), which halves their per-tap error against independently rounded
differences."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def taps(oracle, phantoms):
    c = phantoms.config_cone1440()
    p = oracle.project_ellipsoids_cone(phantoms.ellipsoids_for(c), c, views=[0, 400])
    rng = np.random.default_rng(5)
    p = phantoms.poisson_log(p, c["i0"], rng)
    w = oracle.fdk_weight(p, c["sdd"], c["du"], c["dv"])
    f = oracle.filter_rows(w.reshape(-1, c["nu"]), c["filter"]).reshape(w.shape).astype(np.float32).astype(np.float64)
    n = 200_000
    k = rng.integers(0, f.shape[0], n)
    v = rng.integers(0, c["nv"] - 1, n)
    u = rng.integers(0, c["nu"] - 1, n)
    fu, fv = rng.random(n), rng.random(n)
    corners = [f[k, v, u], f[k, v, u + 1], f[k, v + 1, u], f[k, v + 1, u + 1]]
    wts = [(1 - fu) * (1 - fv), fu * (1 - fv), (1 - fu) * fv, fu * fv]
    exact = sum(w_ * x for w_, x in zip(wts, corners))
    return dict(f=f, k=k, fu=fu, fv=fv, corners=corners, wts=wts, exact=exact)


def _rel(t, val):
    return float(np.sqrt(np.mean((val - t["exact"]) ** 2) / np.mean(t["exact"] ** 2)))


def test_sixteen_bit_formats_exceed_1e4(taps):
    t = taps
    h = lambda x: x.astype(np.float16).astype(np.float64)
    a, c_, b, d = t["corners"]
    mx = np.abs(t["f"]).max(axis=(1, 2))[t["k"]]
    # FP16 gradient form with per-view scale (the MIXED layout: pack_quadg16_kernel),
    # u fraction in FP16; differences against the read-back values
    sc = 8192.0 / mx
    fuh = h(t["fu"])
    ar = h(a * sc)
    c1 = h(c_ * sc - ar)
    g0 = h(b * sc - ar)
    g1 = h(d * sc - (ar + c1 + g0))
    errs = {"fp16 gradient": _rel(t, (ar + fuh * c1 + t["fv"] * (g0 + fuh * g1)) / sc)}
    # the same with each difference rounded on its own
    A = h(a * sc) + fuh * h((c_ - a) * sc)
    G = h((b - a) * sc) + fuh * h((d - c_ - b + a) * sc)
    independent = _rel(t, (A + t["fv"] * G) / sc)
    assert errs["fp16 gradient"] < 0.6 * independent
    # FP16 raw corners, FP32 weights
    sc = 32768.0 / mx
    errs["fp16 corners"] = _rel(t, sum(w * h(x * sc) for w, x in zip(t["wts"], t["corners"])) / sc)
    # int16 raw corners with a per-view scale
    q = 32767.0 / mx
    errs["int16 corners"] = _rel(t, sum(w * np.round(x * q) for w, x in zip(t["wts"], t["corners"])) / q)
    print(errs)
    assert min(errs.values()) > 1e-4


def test_twentyfour_bit_format_meets_1e4(taps):
    t = taps

    def f24(x):  # FP32 rounded to a 15-bit stored significand
        b = x.astype(np.float32).view(np.uint32).astype(np.uint64)
        b = ((b + 0x80) & ~np.uint64(0xFF)).astype(np.uint32)
        return b.view(np.float32).astype(np.float64)

    err = _rel(t, sum(w * f24(x) for w, x in zip(t["wts"], t["corners"])))
    print("24-bit corners", err)
    assert err < 2e-5


def test_24bit_store_rule_picks_the_nearest_value():
    """The 24-bit view format stores the top three bytes S of an FP32 and reads
    back the float with bits (S << 8) | (S & 0xff); the pack keeps the best of
    the candidates t - 1, t, t + 1 around the truncation t = bits >> 8. A
    brute-force search over t - 3 .. t + 3 finds nothing nearer, and the
    rebuilt values err like rounding to 16 significant bits (|err| <= 2^-15
    relative, mean ~0)."""
    rng = np.random.default_rng(11)
    x = (rng.standard_normal(400_000) * np.exp(rng.uniform(-20, 20, 400_000))).astype(np.float32)
    mag = x.view(np.uint32).astype(np.int64) & 0x7FFFFFFF
    t = mag >> 8

    def back(s):
        return (s << 8) | (s & 0xFF)

    def pick(lo, hi):
        cand = np.stack([t + d for d in range(lo, hi + 1)])
        ok = (cand >= 0) & (cand <= 0x7FFFFF)
        err = np.where(ok, np.abs(back(np.clip(cand, 0, 0x7FFFFF)) - mag), np.iinfo(np.int64).max)
        return np.take_along_axis(cand, np.argmin(err, axis=0)[None], 0)[0], err.min(axis=0)

    s1, e1 = pick(-1, 1)
    s3, e3 = pick(-3, 3)
    assert np.array_equal(e1, e3)
    sign = x.view(np.uint32).astype(np.int64) & 0x80000000
    got = (sign | back(s1)).astype(np.uint32).view(np.float32).astype(np.float64)
    rel = (got - x) / np.abs(x.astype(np.float64))
    assert np.abs(rel).max() <= 2.0 ** -15
    assert abs(rel.mean()) < 1e-7
