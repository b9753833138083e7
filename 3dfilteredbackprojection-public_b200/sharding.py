"""One FDK volume over several GPUs by y-slabs, one process per GPU.

The volume's rotation axis is y; y-slab k of the volume only needs the
detector rows its voxels project to (fbp_plan_slabs gives the band, cone
magnification over every view included), so each rank uploads, weights,
filters and backprojects its own band and slab: no collective on the data
path. Gathering the slabs onto one rank (gather_slabs) is optional and uses
torch.distributed (NCCL on GPUs, gloo on CPU).

    plan = fbp_b200.plan_slabs(geometry, nu, nv, h, v, world)
    reconstruct_slab(solver, projections, geometry, h, v, filter, plan[rank])
    volume = gather_slabs(solver.read_volume(torch_tensor), plan, rank, world)
"""
from __future__ import annotations

import numpy as np


def band_of(projections, row0: int, row1: int):
    """Rows [row0, row1) of every projection ([count][v][u] numpy or torch), contiguous."""
    b = projections[:, row0:row1, :]
    return b.contiguous() if hasattr(b, "contiguous") else np.ascontiguousarray(b)


def reconstruct_slab(solver, projections, geometry, volume_h: int, volume_v: int, filter_type: int, slab) -> None:
    """FDK of y-slices [y0, y1) of the volume on this rank's solver: uploads
    only rows [row0, row1) of `projections` ([count][rows][cols], numpy or
    torch, host or device), so the rank's context holds the band and the slab.
    geometry: fbp_b200.Geometry (cone)."""
    y0, y1, row0, row1 = slab
    solver.upload_projections(band_of(projections, row0, row1))
    solver.set_detector_rows(row0, projections.shape[1])
    solver.set_volume_slab(y0, y1 - y0)
    g = geometry
    solver.apply_fdk_weights_to_projections(g.source_distance, g.detector_distance, g.detector_width)
    solver.apply_filter_to_projections(filter_type)
    solver.project_backward_cone_fdk_from_projections(g.source_distance, g.detector_distance, g.detector_width,
                                                      g.volume_width, g.full_rotation_count, volume_h, volume_v,
                                                      g.rotation_offset_radian)


def gather_slabs(slab_volume, plan, rank: int, world: int, dst: int = 0, group=None):
    """Assemble the [z][y][x] volume on rank `dst` from every rank's [z][y1-y0][x]
    slab (torch tensors on the process group's device). Returns the volume on
    `dst`, None elsewhere."""
    import torch
    import torch.distributed as dist
    heights = [s[1] - s[0] for s in plan]
    hmax = max(heights)
    nz, h, nx = slab_volume.shape
    assert h == heights[rank], "slab height does not match the plan"
    pad = slab_volume.new_zeros((nz, hmax, nx))
    pad[:, :h, :] = slab_volume
    bufs = [torch.empty_like(pad) for _ in range(world)] if rank == dst else None
    dist.gather(pad, gather_list=bufs, dst=dst, group=group)
    if rank != dst:
        return None
    return torch.cat([b[:, :heights[k], :] for k, b in enumerate(bufs)], dim=1)
