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
