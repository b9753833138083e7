"""The bench's sampled FP64-oracle accuracy check (large cone workloads):
the view-chunked weight/filter/backprojection of the sampled voxels must
give the same values as the whole-volume oracle FDK, and the bands must
cover the whole rotation axis, the reference's unclipped band included."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def test_oracle_sample_equals_whole_volume_fdk(oracle, phantoms):
    sys.path.insert(0, str(ROOT))
    import bench

    c = phantoms.scaled_cone(phantoms.config_cone1440(), 16)  # 90 x 91 x 90, 90 views, 96^2 detector
    rng = np.random.default_rng(3)
    raw = rng.random((c["nviews"], c["nv"], c["nu"])).astype(np.float32)
    chk = bench.oracle_sample(c, lambda k0, k1: raw[k0:k1], 3000, slice_vox=500, chunk=7)
    whole = oracle.fdk(raw, c, c["filter"], clip=True)
    ijk = chk["ijk"]
    ref = whole[ijk[:, 2], ijk[:, 1], ijk[:, 0]]
    assert np.max(np.abs(chk["ref"] - ref)) <= 1e-12 * np.max(np.abs(ref))
    ys = sorted({int(ijk[a, 1]) for name, (a, b) in chk["bands"].items() if name.startswith("y=")})
    assert ys[0] <= 1 and ys[-1] >= c["ny"] - 2 and len(ys) == 6
    assert any(y >= c["nz"] for y in ys)  # y >= z_size: left unclipped by the reference's loop
    a, b = chk["bands"]["random voxels"]
    assert b - a == 3000
    # bands are disjoint and cover the sample
    spans = sorted(chk["bands"].values())
    assert spans[0][0] == 0 and spans[-1][1] == len(ijk)
    assert all(spans[i][1] == spans[i + 1][0] for i in range(len(spans) - 1))


def test_field_of_view_mask_against_every_view(phantoms):
    """The closed-form field-of-view mask of the bench's accuracy bands: a
    voxel it keeps projects inside the detector's sample grid in every view
    (checked view by view), and the voxels it drops that do stay inside in
    every listed view lie at the boundary (the closed form takes the
    continuous orbit's extreme, which the discrete views may just miss)."""
    sys.path.insert(0, str(ROOT))
    import bench

    c = phantoms.scaled_cone(phantoms.config_cone1440(), 8)  # 180 x 183 x 180, 180 views, 192^2 detector
    rng = np.random.default_rng(11)
    n = 20000
    ijk = np.stack([rng.integers(0, c["nx"], n), rng.integers(0, c["ny"], n), rng.integers(0, c["nz"], n)], 1)
    mask = bench.in_field_of_view(c, ijk)
    X = (ijk[:, 0] + 0.5 - c["nx"] / 2.0) * c["vox"]
    Y = (ijk[:, 1] + 0.5 - c["ny"] / 2.0) * c["vox"]
    Z = (ijk[:, 2] + 0.5 - c["nz"] / 2.0) * c["vox"]
    th = c["offset"] + c["span"] * np.arange(c["nviews"]) / c["nviews"]
    t = X[:, None] * np.cos(th) + Z[:, None] * np.sin(th)
    s = -X[:, None] * np.sin(th) + Z[:, None] * np.cos(th)
    L = c["sod"] + t
    ui = c["sdd"] * s / L / c["du"] + c["nu"] / 2.0 - 0.5
    vi = c["sdd"] * Y[:, None] / L / c["dv"] + c["nv"] / 2.0 - 0.5
    inside = ((L > 0) & (ui >= 0) & (ui <= c["nu"] - 1) & (vi >= 0) & (vi <= c["nv"] - 1)).all(axis=1)
    assert 0.05 < mask.mean() < 0.95
    assert not (mask & ~inside).any()
    # dropped although every discrete view is inside: within 2% of the limits
    near = inside & ~mask
    r = np.hypot(X, Z)[near]
    u_max = c["sdd"] * r / np.sqrt(c["sod"] ** 2 - r ** 2)
    v_max = c["sdd"] * np.abs(Y[near]) / (c["sod"] - r)
    lim_u, lim_v = (c["nu"] - 1) / 2.0 * c["du"], (c["nv"] - 1) / 2.0 * c["dv"]
    assert np.all((u_max <= 1.02 * lim_u) & (v_max <= 1.02 * lim_v))
    assert near.mean() < 0.02


def test_sample_error_reports_bands_over_the_field_of_view():
    """Per band: the relative RMSE over the band, over its voxels inside the
    field of view (None when it has none), and the share of such voxels."""
    sys.path.insert(0, str(ROOT))
    import bench

    rng = np.random.default_rng(5)
    ref = rng.uniform(1.0, 2.0, 300)
    got = ref + rng.normal(0.0, 1e-3, 300)
    got[200:] = ref[200:] + 0.5  # a band with large errors, all outside the field of view
    in_fov = np.zeros(300, bool)
    in_fov[:150] = True
    out = bench.sample_error(got, ref, {"a": (0, 100), "b": (100, 200), "c": (200, 300)}, in_fov)
    a, b, c = out["bands"]["a"], out["bands"]["b"], out["bands"]["c"]
    assert a["in_fov_share"] == 1.0 and b["in_fov_share"] == 0.5 and c["in_fov_share"] == 0.0
    assert c["rel_rmse_in_fov"] is None
    d = got - ref
    assert np.isclose(b["rel_rmse_in_fov"], np.linalg.norm(d[100:150]) / np.linalg.norm(ref[100:150]))
    assert np.isclose(out["rel_rmse_in_fov"], np.linalg.norm(d[:150]) / np.linalg.norm(ref[:150]))
    assert out["rel_rmse_in_fov"] < 1e-2 < out["rel_rmse"]
    # without a mask the bands carry no field-of-view keys
    assert "in_fov_share" not in bench.sample_error(got, ref, {"a": (0, 100)})["bands"]["a"]
