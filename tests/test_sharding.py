"""y-slab sharding of one volume (no collective on the data path): the host
planner and the gather, on CPU with gloo ranks. The GPU side of a rank is the
same library call sequence the single-GPU tests cover (test_gpu_parity.py
runs the ranks of a plan one after another on one GPU)."""
from __future__ import annotations

import math
import socket

import numpy as np
import pytest


def _config():
    # small cone: source 120 mm, detector 80 mm further, 40 x 36 detector at 1 mm
    return dict(sod=120.0, sdd=200.0, du=1.0, dv=1.0, span=2 * math.pi, offset=0.05, nu=40, nv=36, nviews=48,
                nx=32, ny=30, nz=32, vox=1.0)


def _geometry(F, c):
    return F.Geometry.cone(c["sod"], c["sdd"] - c["sod"], c["nu"] * c["du"], c["nx"] * c["vox"],
                           c["span"] / (2 * math.pi), c["offset"])


def test_plan_slabs_cover_every_projected_row(fbp):
    """Brute force over every voxel centre of each slab and every view: each
    row a bilinear tap can touch lies inside the slab's band."""
    c = _config()
    plan = fbp.plan_slabs(_geometry(fbp, c), c["nu"], c["nv"], c["nx"], c["ny"], 3)
    assert [p[0] for p in plan] == [0, 10, 20] and [p[1] for p in plan] == [10, 20, 30]
    th = c["offset"] + c["span"] * np.arange(c["nviews"]) / c["nviews"]
    ax = (np.arange(c["nx"]) + 0.5 - c["nx"] / 2) * c["vox"]
    X, Z = np.meshgrid(ax, ax, indexing="ij")
    D = (c["sod"] + X[..., None] * np.cos(th) + Z[..., None] * np.sin(th)) / c["sod"]
    G = c["sdd"] / (c["sod"] * c["dv"])
    for y0, y1, r0, r1 in plan:
        assert 0 <= r0 < r1 <= c["nv"]
        Y = (np.arange(y0, y1) + 0.5 - c["ny"] / 2) * c["vox"]
        v = G * Y[:, None, None, None] / D[None] + (c["nv"] / 2 - 0.5)
        f = np.floor(v)
        rows = np.concatenate([f.ravel(), f.ravel() + 1])
        rows = rows[(rows >= 0) & (rows < c["nv"])]
        assert rows.min() >= r0 and rows.max() < r1, (y0, y1, r0, r1, rows.min(), rows.max())
    assert min(r1 - r0 for _, _, r0, r1 in plan) < c["nv"]  # the bands save rows


def test_plan_slabs_rejects_bad_arguments(fbp):
    g = _geometry(fbp, _config())
    with pytest.raises(fbp.FBPError):
        fbp.plan_slabs(g, 40, 36, 32, 30, 31)  # more slabs than slices
    with pytest.raises(fbp.FBPError):
        fbp.plan_slabs(g, 0, 36, 32, 30, 2)


def _rank(rank, world, port):
    import torch
    import torch.distributed as dist

    import fbp_b200 as F
    import oracle as O
    import sharding
    from phantoms import random_ellipsoids

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        c = _config()
        E = random_ellipsoids(np.random.default_rng(41), 8, 0.5 * c["nx"] * c["vox"])
        proj = O.project_ellipsoids_cone(E, c)
        plan = F.plan_slabs(_geometry(F, c), c["nu"], c["nv"], c["nx"], c["ny"], world)
        y0, y1, r0, r1 = plan[rank]
        band_only = np.zeros_like(proj)  # this rank sees its row band and nothing else
        band_only[:, r0:r1, :] = proj[:, r0:r1, :]
        slab = O.fdk(band_only, c, 0)[:, y0:y1, :]
        vol = sharding.gather_slabs(torch.from_numpy(np.ascontiguousarray(slab)), plan, rank, world)
        if rank == 0:
            ref = O.fdk(proj, c, 0)
            assert vol.shape == ref.shape
            assert np.array_equal(vol.numpy(), ref), float(np.abs(vol.numpy() - ref).max())
        else:
            assert vol is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_slab_reconstruction_gloo(fbp, oracle):
    """Two gloo ranks: each reconstructs its slab from its detector row band
    alone (the oracle stands in for the GPU); the gathered volume equals the
    whole-detector reconstruction bit for bit."""
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_rank, args=(2, port), nprocs=2, join=True)
