"""Seeded analytic phantoms and the benchmark geometries.

Shared by the tests and bench.py to build synthetic inputs with the shapes,
sizes and value distributions of the five workloads (2D parallel, 2D fan,
cone 256^3, cone 1440x1470x1440, mixed serving stream). Parameters only: line
integrals come from the FP64 oracle (small cases) or the library's FP64
ellipsoid projector (large cases).

Ellipse rows: [density, a, b, cx, cz, phi]. Ellipsoid rows: [density, a, b,
c, cx, cy, cz, R00..R22], R row-major with the ellipsoid axes as columns.
"""
from __future__ import annotations

import math

import numpy as np

# Modified Shepp-Logan head phantom (Shepp & Logan 1974, with the higher
# contrast intensities of Toft 1996): density, semi-axes, centre in units of
# the phantom radius, rotation in degrees.
_MODIFIED_SHEPP_LOGAN = [
    (1.0, 0.69, 0.92, 0.0, 0.0, 0.0),
    (-0.8, 0.6624, 0.8740, 0.0, -0.0184, 0.0),
    (-0.2, 0.1100, 0.3100, 0.22, 0.0, -18.0),
    (-0.2, 0.1600, 0.4100, -0.22, 0.0, 18.0),
    (0.1, 0.2100, 0.2500, 0.0, 0.35, 0.0),
    (0.1, 0.0460, 0.0460, 0.0, 0.1, 0.0),
    (0.1, 0.0460, 0.0460, 0.0, -0.1, 0.0),
    (0.1, 0.0460, 0.0230, -0.08, -0.605, 0.0),
    (0.1, 0.0230, 0.0230, 0.0, -0.606, 0.0),
    (0.1, 0.0230, 0.0460, 0.06, -0.605, 0.0),
]


def shepp_logan_2d(radius: float) -> np.ndarray:
    rows = []
    for rho, a, b, x, z, deg in _MODIFIED_SHEPP_LOGAN:
        rows.append([rho, a * radius, b * radius, x * radius, z * radius, math.radians(deg)])
    return np.array(rows, np.float64)


def random_ellipses(rng: np.random.Generator, count: int, radius: float) -> np.ndarray:
    """Centres uniform in a disc of 0.8 R, semi-axes U(0.03, 0.3) R, angle
    U(0, pi), density U(-0.2, 0.8)."""
    r = 0.8 * radius * np.sqrt(rng.random(count))
    t = 2 * np.pi * rng.random(count)
    a = rng.uniform(0.03, 0.3, count) * radius
    b = rng.uniform(0.03, 0.3, count) * radius
    phi = rng.uniform(0, np.pi, count)
    rho = rng.uniform(-0.2, 0.8, count)
    return np.stack([rho, a, b, r * np.cos(t), r * np.sin(t), phi], axis=1)


def haar_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniformly distributed rotation: QR of a Gaussian matrix with the signs
    of R's diagonal folded into Q (Mezzadri 2007), determinant forced to +1."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def random_ellipsoids(rng: np.random.Generator, count: int, radius: float) -> np.ndarray:
    """Centres uniform in a ball of 0.7 R, semi-axes U(0.05, 0.35) R, uniform
    random rotation, density U(-0.2, 1.0)."""
    out = np.zeros((count, 16), np.float64)
    for i in range(count):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        c = d * 0.7 * radius * rng.random() ** (1.0 / 3.0)
        axes = rng.uniform(0.05, 0.35, 3) * radius
        rho = rng.uniform(-0.2, 1.0)
        out[i, 0] = rho
        out[i, 1:4] = axes
        out[i, 4:7] = c
        out[i, 7:16] = haar_rotation(rng).reshape(-1)
    return out


def poisson_log(p: np.ndarray, i0: float, rng: np.random.Generator) -> np.ndarray:
    """Counts ~ Poisson(I0 exp(-p)), then -log(max(counts, 1) / I0)."""
    counts = rng.poisson(i0 * np.exp(-p.astype(np.float64)))
    return (-np.log(np.maximum(counts, 1) / i0)).astype(np.float32)


# --------------------------------------------------------------------- configs
# Geometry dictionaries use the oracle's keys: sod, sdd, du, dv, span, offset,
# nu, nv, nviews, nx, ny, nz, vox.

def config_parallel2d() -> dict:
    """256x256 modified Shepp-Logan, 360 views over [0, pi), 367 bins at pixel
    pitch, Ram-Lak, rows padded to 512."""
    return dict(name="parallel2d_256", kind="parallel2d", nx=256, ny=1, nz=256, vox=1.0, nu=367, nv=1,
                nviews=360, du=1.0, dv=1.0, span=math.pi, offset=0.0, sod=0.0, sdd=0.0, filter=0,
                seed=1000)


def config_fan2d() -> dict:
    """512x512 over a 256 mm FOV, 720 views over 2 pi, 768 bins x 1.0 mm, SOD
    500, SDD 1000, Shepp-Logan + 12 random ellipses, Poisson I0 = 1e5,
    Shepp-Logan-windowed ramp, rows padded to 1024."""
    return dict(name="fan2d_512", kind="fan2d", nx=512, ny=1, nz=512, vox=0.5, nu=768, nv=1, nviews=720,
                du=1.0, dv=1.0, span=2 * math.pi, offset=0.0, sod=500.0, sdd=1000.0, filter=1, i0=1e5,
                seed=1001)


def config_cone256() -> dict:
    """256^3 at 1 mm, 360 views over 2 pi, 384x384 detector at 1.6 mm, SOD 750,
    SDD 1200, 20 random ellipsoids, Ram-Lak, rows padded to 512."""
    return dict(name="cone_256", kind="cone", nx=256, ny=256, nz=256, vox=1.0, nu=384, nv=384, nviews=360,
                du=1.6, dv=1.6, span=2 * math.pi, offset=0.0, sod=750.0, sdd=1200.0, filter=0,
                n_ellipsoids=20, seed=1002)


def config_cone1440() -> dict:
    """1440x1470x1440 (x, y, z; y is the rotation axis) at 0.2 mm, 1440 views
    over 2 pi, 1536x1536 detector at 0.254 mm, SOD 400, SDD 800, 40 random
    ellipsoids, Poisson I0 = 5e4, Hann-windowed ramp, rows padded to 2048."""
    return dict(name="cone_1440x1470x1440", kind="cone", nx=1440, ny=1470, nz=1440, vox=0.2, nu=1536,
                nv=1536, nviews=1440, du=0.254, dv=0.254, span=2 * math.pi, offset=0.0, sod=400.0,
                sdd=800.0, filter=3, n_ellipsoids=40, i0=5e4, seed=1003)


def scaled_cone(cfg: dict, factor: int) -> dict:
    """The same cone geometry with volume, detector and views divided by
    `factor` (pitches multiplied), for checks that must finish quickly."""
    out = dict(cfg)
    for k in ("nx", "ny", "nz", "nu", "nv", "nviews"):
        out[k] = max(1, cfg[k] // factor)
    out["vox"] = cfg["vox"] * cfg["nx"] / out["nx"]
    out["du"] = cfg["du"] * cfg["nu"] / out["nu"]
    out["dv"] = out["du"]
    out["name"] = f"{cfg['name']}_div{factor}"
    return out


def phantom_radius(cfg: dict) -> float:
    return 0.5 * cfg["nx"] * cfg["vox"]


def ellipsoids_for(cfg: dict) -> np.ndarray:
    rng = np.random.default_rng(cfg["seed"])
    return random_ellipsoids(rng, cfg.get("n_ellipsoids", 20), phantom_radius(cfg))


def ellipses_for(cfg: dict) -> np.ndarray:
    r = phantom_radius(cfg)
    if cfg["kind"] == "parallel2d":
        return shepp_logan_2d(r)
    rng = np.random.default_rng(cfg["seed"])
    return np.concatenate([shepp_logan_2d(r), random_ellipses(rng, 12, r)])


def geometry_args(cfg: dict) -> dict:
    """Reference-API arguments of a cone config: (xray_source_distance,
    detector_panel_distance, detector_width, volume_width)."""
    return dict(sod=cfg["sod"], odd=cfg["sdd"] - cfg["sod"], detector_width=cfg["nu"] * cfg["du"],
                volume_width=cfg["nx"] * cfg["vox"], full_rotation_count=cfg["span"] / (2 * math.pi),
                offset=cfg["offset"])
