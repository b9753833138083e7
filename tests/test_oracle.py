"""The FP64 oracle against the reference's golden vectors and known answers."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import relative_rmse

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_fft.npz"


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def test_repo_pi_constant(oracle, golden):
    # FastFourierTransform.h:9 stores the float literal 3.14154965f in a double
    assert oracle.lib().orc_pi(oracle.PI_REPO) == float(golden["pi_repo"])
    assert oracle.lib().orc_pi(oracle.PI_EXACT) == np.pi


@pytest.mark.parametrize("n", [2, 8, 64, 512, 2048])
def test_fft_matches_reference_bit_for_bit(oracle, golden, n):
    z = golden[f"fft_in_{n}"]
    assert np.array_equal(oracle.fft(z, pi_mode=oracle.PI_REPO), golden[f"fft_out_{n}"])
    assert np.array_equal(oracle.fft(z, inverse=True, pi_mode=oracle.PI_REPO), golden[f"ifft_out_{n}"])


def test_fft_known_answer_ramp8(oracle, golden):
    out = oracle.fft(np.arange(8.0), pi_mode=oracle.PI_REPO)
    assert np.array_equal(out, golden["fft_ramp8_out"])
    # the reference's wrong pi shows in the 5th digit
    assert abs(out[1] - (-4.000208 + 9.656915j)) < 1e-6
    exact = oracle.fft(np.arange(8.0))
    assert abs(exact[1] - (-4 + 9.656854249492381j)) < 1e-12


@pytest.mark.parametrize("n", [2, 16, 512, 4096])
def test_exact_fft_against_numpy(oracle, n):
    rng = np.random.default_rng(n)
    z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert np.abs(oracle.fft(z) - np.fft.fft(z)).max() < 1e-12 * n
    assert np.abs(oracle.fft(z, inverse=True) - np.fft.ifft(z)).max() < 1e-12


@pytest.mark.parametrize("key", ["367_0", "768_1", "384_3"])
def test_filter_path_matches_reference_fft(oracle, golden, key):
    """Rows filtered along the reference's path with its own FFT equal the
    oracle's repo-pi restatement up to the FP32 output rounding."""
    m, filt = map(int, key.split("_"))
    rows = golden[f"filter_in_{key}"]
    ref = golden[f"filter_out_{key}"].astype(np.float64)
    ours = oracle.filter_rows(rows.astype(np.float64), filt, pi_mode=oracle.PI_REPO)
    assert np.abs(ours - ref).max() <= 2e-7 * np.abs(ref).max()
    # the exact-pi oracle differs from the reference FFT by the pi typo only
    exact = oracle.filter_rows(rows.astype(np.float64), filt)
    dev = relative_rmse(ref, exact)
    assert 1e-6 < dev < 1e-2


def test_padded_length_rule(oracle):
    # 1 << ceil_log2(m), ceil_log2(m) = floor_log2(2m - 1): no padding for powers of two
    for m, n in [(1, 1), (2, 2), (3, 4), (367, 512), (384, 512), (512, 512), (768, 1024), (1536, 2048)]:
        assert oracle.padded_length(m) == n


@pytest.mark.parametrize("filt", [0, 1, 2, 3])
def test_fft_filter_equals_circular_convolution(oracle, filt):
    rng = np.random.default_rng(filt)
    rows = rng.standard_normal((3, 367))
    a = oracle.filter_rows(rows, filt)
    b = oracle.filter_rows(rows, filt, direct=True)
    assert np.abs(a - b).max() < 1e-12 * np.abs(b).max()


def test_ramp_kernel_known_answers(oracle):
    n = 512
    g = oracle.filter_kernel(n, oracle.RAM_LAK)
    # the circular spatial kernel is the band-limited ramp h(0)=1/4,
    # h(odd k) = -1/(pi k)^2, h(even k) = 0 (Kak & Slaney eq. 3.61)
    assert abs(g[0] - 0.25) < 1e-12
    assert abs(g[1] + 1 / np.pi ** 2) < 1e-12
    assert abs(g[3] + 1 / (9 * np.pi ** 2)) < 1e-12
    assert abs(g[2]) < 1e-12 and abs(g[4]) < 1e-12
    H = oracle.filter_response(n, oracle.RAM_LAK)
    assert abs(H[n // 2] - 0.5) < 2e-3  # ~|f| at Nyquist
    # filtering a delta returns the kernel
    row = np.zeros((1, 300))
    row[0, 100] = 1.0
    out = oracle.filter_rows(row, oracle.RAM_LAK, n=n)[0]
    assert abs(out[100] - 0.25) < 1e-12 and abs(out[101] + 1 / np.pi ** 2) < 1e-12
    # windows taper the high frequencies
    for f in (oracle.SHEPP_LOGAN, oracle.COSINE, oracle.HANN):
        Hw = oracle.filter_response(n, f)
        assert Hw[n // 2] < H[n // 2] and abs(Hw[1] - H[1]) < 1e-3


def test_parallel2d_reconstructs_shepp_logan(oracle, phantoms):
    c = phantoms.config_parallel2d()
    E = phantoms.ellipses_for(c)
    s = oracle.project_ellipses_parallel2d(E, c["nu"], c["nviews"], c["du"], c["span"])
    img = oracle.fbp_parallel2d(s, c, oracle.RAM_LAK)
    ref = oracle.rasterize_ellipses(E, c["nx"], c["nz"], c["vox"])
    yy, xx = np.mgrid[:256, :256]
    disc = (xx - 127.5) ** 2 + (yy - 127.5) ** 2 < 100 ** 2
    assert np.median(np.abs(img - ref)[disc]) < 5e-3


def test_cone_reconstructs_ellipsoids(oracle, phantoms):
    c = phantoms.scaled_cone(phantoms.config_cone256(), 4)
    E = phantoms.ellipsoids_for(c)
    proj = oracle.project_ellipsoids_cone(E, c)
    vol = oracle.fdk(proj, c, oracle.RAM_LAK)
    ref = oracle.rasterize_ellipsoids(E, c["nx"], c["ny"], c["nz"], c["vox"])
    mid = c["ny"] // 2
    assert np.median(np.abs(vol[:, mid, :] - ref[:, mid, :])) < 2e-2


def test_uniform_disc_parallel_level(oracle):
    """A disc of density 1: the reconstruction is ~1 well inside it."""
    E = np.array([[1.0, 60.0, 60.0, 0.0, 0.0, 0.0]])
    s = oracle.project_ellipses_parallel2d(E, 256, 180, 1.0, np.pi)
    img = oracle.fbp_parallel2d(s, dict(nx=128, nz=128, vox=1.0, du=1.0, span=np.pi, offset=0.0))
    assert abs(img[64, 64] - 1.0) < 5e-3


def test_fan_rebinning_matches_parallel_projection(oracle):
    E = np.array([[1.0, 40.0, 25.0, 10.0, -5.0, 0.3]])
    sod, sdd = 500.0, 1000.0
    fan = oracle.project_ellipses_fan2d(E, 512, 720, sod, sdd, 0.5, 2 * np.pi)
    par = oracle.rebin_fan_to_parallel(fan, dict(sod=sod, sdd=sdd, du=0.5, span=2 * np.pi, offset=0.0), 256, 0.5)
    exact = oracle.project_ellipses_parallel2d(E, 256, 720, 0.5, 2 * np.pi)
    assert relative_rmse(par, exact) < 2e-2


def test_cone_points_match_full_volume(oracle, phantoms):
    c = phantoms.scaled_cone(phantoms.config_cone256(), 8)
    rng = np.random.default_rng(5)
    q = rng.standard_normal((c["nviews"], c["nv"], c["nu"]))
    vol = oracle.bp_cone(q, c)
    ijk = np.stack([rng.integers(0, c["nx"], 50), rng.integers(0, c["ny"], 50), rng.integers(0, c["nz"], 50)], 1)
    pts = oracle.bp_cone_points(q, c, ijk)
    assert np.allclose(pts, vol[ijk[:, 2], ijk[:, 1], ijk[:, 0]], rtol=0, atol=1e-12)


def test_cpu_f32_backprojector_matches_oracle(oracle, phantoms):
    c = phantoms.scaled_cone(phantoms.config_cone256(), 8)
    rng = np.random.default_rng(7)
    q = rng.standard_normal((c["nviews"], c["nv"], c["nu"])).astype(np.float32)
    ref = oracle.bp_cone(q.astype(np.float64), c)
    out = np.zeros((c["nz"], c["ny"], c["nx"]), np.float32)
    oracle.cpu_bp_cone_f32(q, np.arange(c["nviews"]), c, 0, c["ny"], out)
    assert relative_rmse(out, ref) < 1e-5
    # a slab of a subset of views is the matching slice of the subset's sum
    sub = np.arange(3, c["nviews"], 5)
    slab = np.zeros((c["nz"], 6, c["nx"]), np.float32)
    oracle.cpu_bp_cone_f32(q[sub], sub, c, 10, 16, slab)
    qz = np.zeros_like(q, dtype=np.float64)
    qz[sub] = q[sub]
    ref_sub = oracle.bp_cone(qz, c)[:, 10:16, :]
    assert relative_rmse(slab, ref_sub) < 1e-5


def test_forward_projection_known_answers(oracle):
    """Ray-driven forward projection (the library's definition of the
    reference's absent radon shaders): a parallel projection conserves mass
    (detector sum x pixel area = volume integral) and the central ray through
    a voxelised ball has the chord length of the ball."""
    import math
    n, r = 40, 14.0
    ax = np.arange(n) + 0.5 - n / 2
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    ball = ((X ** 2 + Y ** 2 + Z ** 2) <= r * r).astype(np.float64)
    c = dict(vox=1.0, nu=64, nv=64, nviews=3, du=1.0, dv=1.0, span=math.pi, offset=0.3)
    p = oracle.forward_project(ball, c, cone=False)
    for k in range(3):
        assert abs(p[k].sum() - ball.sum()) < 2e-3 * ball.sum()
    centre = p[:, 31:33, 31:33].mean()
    assert abs(centre - 2 * r) < 1.0
    cc = dict(c, sod=80.0, sdd=160.0, du=2.0, dv=2.0, span=2 * math.pi)
    q = oracle.forward_project(ball, cc, cone=True)
    assert abs(q[:, 31:33, 31:33].mean() - 2 * r) < 1.0  # central ray passes the centre
