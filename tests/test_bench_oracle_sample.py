"""The bench's sampled FP64-oracle accuracy check (large cone workloads):
the band-limited weight/filter/backprojection of the sampled voxels must give
the same values as the whole-detector oracle FDK."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def test_oracle_sample_equals_whole_detector_fdk(oracle, phantoms):
    sys.path.insert(0, str(ROOT))
    import bench

    c = phantoms.scaled_cone(phantoms.config_cone1440(), 16)  # 90 x 91 x 90, 90 views, 96^2 detector
    rng = np.random.default_rng(3)
    raw = rng.random((c["nviews"], c["nv"], c["nu"])).astype(np.float32)
    chk = bench.oracle_sample(c, lambda r0, r1: raw[:, r0:r1, :], 3000)
    assert chk and chk["rows"][1] - chk["rows"][0] < c["nv"]  # a strict band
    whole = oracle.fdk(raw, c, c["filter"], clip=True)
    ijk = chk["ijk"]
    ref = whole[ijk[:, 2], ijk[:, 1], ijk[:, 0]]
    assert np.max(np.abs(chk["ref"] - ref)) <= 1e-12 * np.max(np.abs(ref))
