"""ctypes bindings for the FP64 CPU oracle (oracle/_build/liboracle.so) and
for the reference's own CPU FFT compiled from its sources
(oracle/_ref/libreffft.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke entry point and the
bench's CPU-baseline legs, as the checker. The product library never uses it.
See fbp_oracle.cpp for what each routine restates and its parity status.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
REF_PATH = HERE / "_ref" / "libreffft.so"

PI_EXACT, PI_REPO = 0, 1
RAM_LAK, SHEPP_LOGAN, COSINE, HANN, RAMP_SAMPLED = 0, 1, 2, 3, 4

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)

_lib = None
_ref = None


def build(with_ref: bool = True) -> None:
    target = "all" if with_ref else "oracle"
    subprocess.run(["make", "-s", "-C", str(HERE), target], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build(with_ref=False)
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def ref_available() -> bool:
    return REF_PATH.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_PATH.exists():
            raise FileNotFoundError(f"{REF_PATH} not built (needs the reference sources)")
        _ref = C.CDLL(str(REF_PATH))
        _ref.ref_pi.restype = C.c_double
        _ref.ref_fft.argtypes = [_D, _D, C.c_int, C.c_int]
        _ref.ref_fft_shift.argtypes = [_D, _D, C.c_int, C.c_int]
        _ref.ref_filter_rows.argtypes = [_F, _F, C.c_long, C.c_int, C.c_int, _D, C.c_int]
    return _ref


def _declare(L: C.CDLL) -> None:
    i, d, lng = C.c_int, C.c_double, C.c_long
    L.orc_padded_length.argtypes = [i]
    L.orc_pi.argtypes = [i]
    L.orc_pi.restype = d
    L.orc_fft.argtypes = [_D, _D, i, i, i]
    L.orc_fft_shift.argtypes = [_D, _D, i, i]
    L.orc_filter_response.argtypes = [_D, i, i]
    L.orc_filter_kernel.argtypes = [_D, i, i]
    L.orc_filter_rows.argtypes = [_D, _D, lng, i, i, i, i]
    L.orc_filter_rows_direct.argtypes = [_D, _D, lng, i, i, i]
    L.orc_fdk_weight.argtypes = [_D, i, i, i, d, d, d]
    L.orc_log_normalize.argtypes = [_D, lng, d]
    L.orc_bp_cone.argtypes = [_D, i, i, i, d, d, d, d, d, d, i, i, i, d, _D]
    L.orc_bp_cone_points.argtypes = [_D, i, i, i, d, d, d, d, d, d, i, i, i, d, _I, lng, _D]
    L.orc_bp_parallel3d.argtypes = [_D, i, i, i, d, d, d, d, i, i, i, d, _D]
    L.orc_bp_parallel2d.argtypes = [_D, i, i, d, d, d, i, i, d, _D]
    L.orc_bp_fan2d.argtypes = [_D, i, i, d, d, d, d, d, i, i, d, _D]
    L.orc_rebin_fan_to_parallel.argtypes = [_D, i, i, d, d, d, d, d, i, d, _D]
    L.orc_clip_negatives.argtypes = [_D, i, i, i, i]
    L.orc_fdk.argtypes = [_F, i, i, i, d, d, d, d, d, d, i, i, i, d, i, i, i, i, _D]
    L.orc_project_ellipses_parallel2d.argtypes = [_D, i, i, i, d, d, d, _F]
    L.orc_project_ellipses_fan2d.argtypes = [_D, i, i, i, d, d, d, d, d, _F]
    L.orc_project_ellipsoids_cone.argtypes = [_D, i, i, i, i, d, d, d, d, d, d, _I, i, _F]
    L.orc_rasterize_ellipses.argtypes = [_D, i, i, i, d, _D]
    L.orc_rasterize_ellipsoids.argtypes = [_D, i, i, i, i, d, _D]
    L.orc_bp_cone_f32.argtypes = [_F, _I, i, i, i, i, d, d, d, d, d, d, i, i, i, d, i, i, _F]
    L.orc_forward_project.argtypes = [_D, i, i, i, d, i, d, d, d, d, i, i, i, d, d, _D]
    L.orc_num_threads.restype = i
    L.orc_set_num_threads.argtypes = [i]


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _f(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with status {rc}")


# ----------------------------------------------------------------- FFT / filter
def padded_length(m: int) -> int:
    return lib().orc_padded_length(m)


def fft(x: np.ndarray, inverse: bool = False, pi_mode: int = PI_EXACT) -> np.ndarray:
    x = np.asarray(x, dtype=np.complex128)
    re, im = np.ascontiguousarray(x.real), np.ascontiguousarray(x.imag)
    _check(lib().orc_fft(_d(re), _d(im), len(x), int(inverse), pi_mode), "fft")
    return re + 1j * im


def fft_shift(x: np.ndarray, shift: int) -> np.ndarray:
    x = np.asarray(x, dtype=np.complex128)
    re, im = np.ascontiguousarray(x.real), np.ascontiguousarray(x.imag)
    _check(lib().orc_fft_shift(_d(re), _d(im), len(x), shift), "fft_shift")
    return re + 1j * im


def filter_response(n: int, filt: int) -> np.ndarray:
    H = np.zeros(n, np.float64)
    _check(lib().orc_filter_response(_d(H), n, filt), "filter_response")
    return H


def filter_kernel(n: int, filt: int) -> np.ndarray:
    g = np.zeros(n, np.float64)
    _check(lib().orc_filter_kernel(_d(g), n, filt), "filter_kernel")
    return g


def filter_rows(rows: np.ndarray, filt: int, n: int | None = None, pi_mode: int = PI_EXACT,
                direct: bool = False) -> np.ndarray:
    x = np.ascontiguousarray(rows, dtype=np.float64)
    m = x.shape[-1]
    nrows = x.size // m
    n = n or padded_length(m)
    out = np.zeros_like(x)
    if direct:
        rc = lib().orc_filter_rows_direct(_d(x), _d(out), nrows, m, n, filt)
    else:
        rc = lib().orc_filter_rows(_d(x), _d(out), nrows, m, n, filt, pi_mode)
    _check(rc, "filter_rows")
    return out


def fdk_weight(p: np.ndarray, sdd: float, du: float, dv: float) -> np.ndarray:
    p = np.array(p, dtype=np.float64, order="C", copy=True)
    nviews, nv, nu = p.shape
    lib().orc_fdk_weight(_d(p), nu, nv, nviews, sdd, du, dv)
    return p


def log_normalize(p: np.ndarray, base: float) -> np.ndarray:
    p = np.array(p, dtype=np.float64, order="C", copy=True)
    lib().orc_log_normalize(_d(p), p.size, base)
    return p


# ---------------------------------------------------------------- backprojection
def bp_cone(q: np.ndarray, g: dict) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64)
    nviews, nv, nu = q.shape
    vol = np.zeros((g["nz"], g["ny"], g["nx"]), np.float64)
    lib().orc_bp_cone(_d(q), nu, nv, nviews, g["sod"], g["sdd"], g["du"], g["dv"], g["span"],
                      g["offset"], g["nx"], g["ny"], g["nz"], g["vox"], _d(vol))
    return vol


def bp_cone_points(q: np.ndarray, g: dict, ijk: np.ndarray) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64)
    nviews, nv, nu = q.shape
    ijk = np.ascontiguousarray(ijk, dtype=np.int32)
    out = np.zeros(len(ijk), np.float64)
    lib().orc_bp_cone_points(_d(q), nu, nv, nviews, g["sod"], g["sdd"], g["du"], g["dv"],
                             g["span"], g["offset"], g["nx"], g["ny"], g["nz"], g["vox"],
                             ijk.ctypes.data_as(_I), len(ijk), _d(out))
    return out


def bp_parallel3d(q: np.ndarray, g: dict) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64)
    nviews, nv, nu = q.shape
    vol = np.zeros((g["nz"], g["ny"], g["nx"]), np.float64)
    lib().orc_bp_parallel3d(_d(q), nu, nv, nviews, g["du"], g["dv"], g["span"], g["offset"],
                            g["nx"], g["ny"], g["nz"], g["vox"], _d(vol))
    return vol


def bp_parallel2d(q: np.ndarray, g: dict) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64)
    nviews, nbins = q.shape
    img = np.zeros((g["nz"], g["nx"]), np.float64)
    lib().orc_bp_parallel2d(_d(q), nbins, nviews, g["du"], g["span"], g["offset"], g["nx"],
                            g["nz"], g["vox"], _d(img))
    return img


def bp_fan2d(q: np.ndarray, g: dict) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64)
    nviews, nbins = q.shape
    img = np.zeros((g["nz"], g["nx"]), np.float64)
    lib().orc_bp_fan2d(_d(q), nbins, nviews, g["sod"], g["sdd"], g["du"], g["span"], g["offset"],
                       g["nx"], g["nz"], g["vox"], _d(img))
    return img


def rebin_fan_to_parallel(fan: np.ndarray, g: dict, n_out: int, du_out: float) -> np.ndarray:
    fan = np.ascontiguousarray(fan, dtype=np.float64)
    nviews, nbins = fan.shape
    out = np.zeros((nviews, n_out), np.float64)
    lib().orc_rebin_fan_to_parallel(_d(fan), nbins, nviews, g["sod"], g["sdd"], g["du"],
                                    g["span"], g["offset"], n_out, du_out, _d(out))
    return out


def decode_projection_file(raw: bytes, width: int, height: int, channels: int, byte_per_channel: int) -> np.ndarray:
    """One raw projection file as FBP3D::read_projections loads it
    (Source/FilteredBackProjection/FBP3D.cpp:110-117): channel 0, normalised
    like an UNSIGNED_SHORT / UNSIGNED_BYTE texture upload (v / 65535, v / 255)."""
    dt = np.dtype("<u2") if byte_per_channel == 2 else np.dtype("u1")
    a = np.frombuffer(raw, dtype=dt, count=width * height * channels).reshape(height, width, channels)[:, :, 0]
    return (a.astype(np.float32) / np.float32(65535 if byte_per_channel == 2 else 255)).astype(np.float32)


def resample_bilinear(img: np.ndarray, tw: int, th: int) -> np.ndarray:
    """The library's resize for read_projections (the reference's Image::resize
    lives in its absent GraphicsCortex library): pixel centres aligned, edges
    clamped, FP32 in the library's operation order."""
    img = np.asarray(img, dtype=np.float32)
    fh, fw = img.shape
    if (fw, fh) == (tw, th):
        return img.copy()
    f32 = np.float32
    rx, ry = f32(fw) / f32(tw), f32(fh) / f32(th)
    sx = np.clip((np.arange(tw, dtype=f32) + f32(0.5)) * rx - f32(0.5), f32(0), f32(fw - 1)).astype(f32)
    sy = np.clip((np.arange(th, dtype=f32) + f32(0.5)) * ry - f32(0.5), f32(0), f32(fh - 1)).astype(f32)
    x0 = sx.astype(np.int64); y0 = sy.astype(np.int64)
    x1 = np.minimum(x0 + 1, fw - 1); y1 = np.minimum(y0 + 1, fh - 1)
    ax = (sx - x0.astype(f32)).astype(f32)[None, :]; ay = (sy - y0.astype(f32)).astype(f32)[:, None]
    one = f32(1)
    top = ((one - ax) * img[y0][:, x0] + ax * img[y0][:, x1]).astype(f32)
    bot = ((one - ax) * img[y1][:, x0] + ax * img[y1][:, x1]).astype(f32)
    return ((one - ay) * top + ay * bot).astype(f32)


def volume_slices_u16(vol: np.ndarray) -> np.ndarray:
    """FBP3D::write_volume's slice conversion (FBP3D.cpp:178-195): y-slices
    [y][z][x] as round(clamp(v, 0, 1) * 65535), GL's float -> normalised
    unsigned short rule (round half to even)."""
    v = np.clip(np.asarray(vol, dtype=np.float32), 0, 1).astype(np.float32)
    return np.rint(v * np.float32(65535)).astype(np.uint16).transpose(1, 0, 2).copy()


def forward_project(vol: np.ndarray, c: dict, cone: bool = True) -> np.ndarray:
    """Ray-driven forward projection of a [z][y][x] volume in FP64 (see
    orc_forward_project): c gives vox, nu, nv, nviews, du, dv, span, offset and,
    for cone beam, sod and sdd. Returns [view][v][u]."""
    v = np.ascontiguousarray(vol, dtype=np.float64)
    nz, ny, nx = v.shape
    out = np.zeros((c["nviews"], c["nv"], c["nu"]), np.float64)
    _check(lib().orc_forward_project(_d(v), nx, ny, nz, c["vox"], int(cone), c.get("sod", 0.0), c.get("sdd", 0.0),
                                     c["du"], c["dv"], c["nu"], c["nv"], c["nviews"], c["span"], c["offset"], _d(out)),
           "forward_project")
    return out


def normalize_histogram(vol: np.ndarray, min_value: float | None = None, max_value: float | None = None) -> np.ndarray:
    """FBP3D::normalize_histogram (Source/FilteredBackProjection/FBP3D.cpp:780-826)
    restated in FP32 with the library's operation order: d = v - min, r = max - min,
    d / r (IEEE division), 0 everywhere when max <= min; the extremes ignore NaN."""
    v = np.asarray(vol, dtype=np.float32)
    if min_value is None:
        finite = v[~np.isnan(v)]
        min_value, max_value = (float(finite.min()), float(finite.max())) if finite.size else (0.0, 0.0)
    mn, mx = np.float32(min_value), np.float32(max_value)
    r = np.float32(mx - mn)
    if not r > 0:
        return np.zeros_like(v)
    return ((v - mn) / r).astype(np.float32)


def clip_negatives(vol: np.ndarray, y_limit: int | None = None) -> np.ndarray:
    vol = np.array(vol, dtype=np.float64, order="C", copy=True)
    nz, ny, nx = vol.shape
    lib().orc_clip_negatives(_d(vol), nx, ny, nz, nz if y_limit is None else y_limit)
    return vol


# ------------------------------------------------------------------ pipelines
def fdk(proj: np.ndarray, g: dict, filt: int = RAM_LAK, n_pad: int | None = None,
        pi_mode: int = PI_EXACT, clip: bool = False) -> np.ndarray:
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    nviews, nv, nu = proj.shape
    n_pad = n_pad or padded_length(nu)
    vol = np.zeros((g["nz"], g["ny"], g["nx"]), np.float64)
    _check(lib().orc_fdk(_f(proj), nu, nv, nviews, g["sod"], g["sdd"], g["du"], g["dv"], g["span"],
                         g["offset"], g["nx"], g["ny"], g["nz"], g["vox"], filt, n_pad, pi_mode,
                         int(clip), _d(vol)), "fdk")
    return vol


def fbp_parallel2d(sino: np.ndarray, g: dict, filt: int = RAM_LAK, n_pad: int | None = None,
                   pi_mode: int = PI_EXACT) -> np.ndarray:
    q = filter_rows(np.asarray(sino, np.float64), filt, n_pad, pi_mode)
    return bp_parallel2d(q, g)


def fbp_fan2d(sino: np.ndarray, g: dict, filt: int = RAM_LAK, n_pad: int | None = None,
              pi_mode: int = PI_EXACT) -> np.ndarray:
    s = np.asarray(sino, np.float64)[:, None, :]
    w = fdk_weight(s, g["sdd"], g["du"], 0.0)[:, 0, :]
    q = filter_rows(w, filt, n_pad, pi_mode)
    return bp_fan2d(q, g)


# --------------------------------------------------------------------- phantoms
def project_ellipses_parallel2d(E: np.ndarray, nbins: int, nviews: int, du: float, span: float,
                                offset: float = 0.0) -> np.ndarray:
    E = np.ascontiguousarray(E, dtype=np.float64)
    out = np.zeros((nviews, nbins), np.float32)
    lib().orc_project_ellipses_parallel2d(_d(E), len(E), nbins, nviews, du, span, offset, _f(out))
    return out


def project_ellipses_fan2d(E: np.ndarray, nbins: int, nviews: int, sod: float, sdd: float,
                           du: float, span: float, offset: float = 0.0) -> np.ndarray:
    E = np.ascontiguousarray(E, dtype=np.float64)
    out = np.zeros((nviews, nbins), np.float32)
    lib().orc_project_ellipses_fan2d(_d(E), len(E), nbins, nviews, sod, sdd, du, span, offset,
                                     _f(out))
    return out


def project_ellipsoids_cone(E: np.ndarray, g: dict, views=None) -> np.ndarray:
    E = np.ascontiguousarray(E, dtype=np.float64)
    nsel = g["nviews"] if views is None else len(views)
    out = np.zeros((nsel, g["nv"], g["nu"]), np.float32)
    vptr = None
    if views is not None:
        views = np.ascontiguousarray(views, dtype=np.int32)
        vptr = views.ctypes.data_as(_I)
    lib().orc_project_ellipsoids_cone(_d(E), len(E), g["nu"], g["nv"], g["nviews"], g["sod"],
                                      g["sdd"], g["du"], g["dv"], g["span"], g["offset"], vptr,
                                      nsel, _f(out))
    return out


def rasterize_ellipses(E: np.ndarray, nx: int, nz: int, pix: float) -> np.ndarray:
    E = np.ascontiguousarray(E, dtype=np.float64)
    img = np.zeros((nz, nx), np.float64)
    lib().orc_rasterize_ellipses(_d(E), len(E), nx, nz, pix, _d(img))
    return img


def rasterize_ellipsoids(E: np.ndarray, nx: int, ny: int, nz: int, vox: float) -> np.ndarray:
    E = np.ascontiguousarray(E, dtype=np.float64)
    vol = np.zeros((nz, ny, nx), np.float64)
    lib().orc_rasterize_ellipsoids(_d(E), len(E), nx, ny, nz, vox, _d(vol))
    return vol


# ----------------------------------------------------------- CPU baseline legs
def cpu_bp_cone_f32(q: np.ndarray, views, g: dict, y0: int, y1: int, vol: np.ndarray) -> None:
    """FP32 CPU backprojection of the listed views (q[s] = view views[s]) over
    the y-slab [y0, y1), added into vol[z][y - y0][x]."""
    q = np.ascontiguousarray(q, dtype=np.float32)
    nsel, nv, nu = q.shape
    views = np.ascontiguousarray(views, dtype=np.int32)
    assert len(views) == nsel and vol.shape == (g["nz"], y1 - y0, g["nx"]) and vol.dtype == np.float32
    lib().orc_bp_cone_f32(_f(q), views.ctypes.data_as(_I), nsel, nu, nv, g["nviews"], g["sod"], g["sdd"], g["du"],
                          g["dv"], g["span"], g["offset"], g["nx"], g["ny"], g["nz"], g["vox"], y0, y1, _f(vol))


def ref_filter_rows(rows: np.ndarray, filt: int, n: int | None = None,
                    threads: int = 0) -> np.ndarray:
    """Filter float32 rows with the reference's own FFT (compiled from its
    sources) along the reference's path: pad, fft, shift, multiply, unshift,
    inverse fft, real part."""
    x = np.ascontiguousarray(rows, dtype=np.float32)
    m = x.shape[-1]
    n = n or padded_length(m)
    H = filter_response(n, filt)
    Hs = np.ascontiguousarray(np.roll(H, -(n // 2)))  # shifted[i] = H[(i + n/2) % n]
    out = np.zeros_like(x)
    rc = ref().ref_filter_rows(_f(x), _f(out), x.size // m, m, n, _d(Hs), threads)
    _check(rc, "ref_filter_rows")
    return out


def ref_fft(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    x = np.asarray(x, dtype=np.complex128)
    re, im = np.ascontiguousarray(x.real), np.ascontiguousarray(x.imag)
    _check(ref().ref_fft(_d(re), _d(im), len(x), int(inverse)), "ref_fft")
    return re + 1j * im


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))
