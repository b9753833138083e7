#!/usr/bin/env python
"""FDK throughput benchmark: cone-beam 1440x1470x1440 volume (x, y, z; y the
rotation axis) at 0.2 mm, 1440 views over 360 deg, 1536x1536 detector at
0.254 mm, SOD 400 mm, SDD 800 mm, Hann-windowed ramp; 40 seeded random
ellipsoids with analytic FP64 line integrals and Poisson noise (I0 = 5e4).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one reconstruction: restore the raw projections (device-to-device,
the filter works in place), FDK weights, row filter, backprojection with the
fused clip epilogue. `value` (Gvox*view/s = 1440*1470*1440*1440 / step time)
is the chosen form (split-precision: FP16 filtered views with per-view scale,
FP32 accumulation) with inputs resident in HBM; the plain
FP32 form is reported beside it. `e2e` repeats the chosen form through the C
ABI with pinned host buffers: the projection upload and the volume readback
are inside the timed region. The K reconstructions run from two host threads
with one context and stream each, so one reconstruction's transfers overlap
the other's kernels; `e2e.serial` is the same with one context, one call
after another. Multi-GPU runs (torchrun) reconstruct one
independent volume per rank (weak scaling, no collective on the data path);
times are the max over ranks.

`--impl reference` times the reference's CPU path on the host cores: row
filtering with the reference's own FFT compiled from its sources (the
oracle's PI_MODE_REPO restatement where that build is absent) plus a CPU FP32
restatement of the backprojector (the reference ships no CPU backprojector),
on a bounded sample of the same workload, extrapolated to the full job.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "3dfilteredbackprojection-public_b200"
sys.path.insert(0, str(PKG))

METRIC = "FDK Gvox·view/s"
FILTER_NAMES = {0: "ram_lak", 1: "shepp_logan", 2: "cosine", 3: "hann", 4: "ramp_sampled"}
UNIT = "Gvox·view/s"
# bench forms: precision, bytes per stored filtered sample, storage note
FORMS = {"chosen": ("MIXED", 2, "f16 filtered views"), "chosen24": ("MIXED24", 3, "24-bit filtered views"),
         "plain": ("FP32", 4, "f32")}
# arithmetic / storage types of each form, for the line's dtype
DTYPES = {"chosen": "f32 accumulate / f16 filtered views", "chosen24": "f32 accumulate / 24-bit filtered views",
          "plain": "f32"}


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--scale", type=int, default=1,
                   help="divide volume, detector and views by this factor (profiling runs); 1 = full workload")
    p.add_argument("--workload", choices=["cone1440", "cone256", "serving"], default="cone1440",
                   help="cone1440: the headline 1440x1470x1440 case; cone256: 256^3, 360 views (profiling); "
                        "serving: the mixed request stream (reconstructions/s, p50/p99 latency)")
    p.add_argument("--requests", type=int, default=2000, help="serving: requests in the stream")
    p.add_argument("--poisson-requests", type=int, default=600,
                   help="serving: requests of the stream timed under Poisson arrivals")
    p.add_argument("--no-serving", action="store_true",
                   help="cone workloads: leave the serving block (config 5) out of the line")
    p.add_argument("--slots", type=int, default=5, help="serving: concurrent jobs of the chosen form")
    p.add_argument("--load", type=float, default=0.7,
                   help="serving: Poisson arrival rate as a fraction of the plain one-at-a-time capacity")
    p.add_argument("--forms", default="chosen,chosen24,plain", help="comma list of " + ",".join(FORMS))
    p.add_argument("--head", default="chosen", choices=list(FORMS), help="form of the headline value")
    p.add_argument("--shard", choices=["replicas", "slabs"], default="replicas",
                   help="N>1: replicas = one independent volume per rank (weak scaling); slabs = one volume "
                        "split into y-slabs, each rank holding its detector row band (strong scaling)")
    p.add_argument("--backprojector", choices=["auto", "generic", "generic_y8", "symmetric", "tuned"], default="auto",
                   help="backprojector variant of both forms (tuned: timed per geometry on first use)")
    p.add_argument("--tile-ny", type=int, default=0, choices=[0, 8, 16],
                   help="voxels per thread along y of the symmetric backprojector (0: the library default)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--oracle-voxels", type=int, default=1000000,
                   help="uniformly drawn voxels of the sampled FP64-oracle accuracy check (0: skip the check)")
    p.add_argument("--oracle-slice-voxels", type=int, default=100000,
                   help="voxels in each y-slice band of the FP64-oracle accuracy check")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the CPU-baseline sample")
    return p.parse_args()


def workload(scale: int, name: str = "cone1440") -> dict:
    import phantoms as P
    c = P.config_cone1440() if name == "cone1440" else P.config_cone256()
    return c if scale == 1 else P.scaled_cone(c, scale)


def measured_traffic(workload_name: str, form: str):
    """DRAM bytes (read + write) of one backprojector launch for this workload
    and form, read from the ncu summary committed in profiles/ (None if
    absent). The summary holds a one-pass capture of the backprojector kernel
    alone at the full workload size (the command is in its header)."""
    try:
        for line in (ROOT / "profiles" / "bp_dram_traffic.txt").read_text().splitlines():
            f = line.split()
            if len(f) == 4 and not line.startswith("#") and f[0] == workload_name and f[1] == form:
                return float(f[2]) + float(f[3])
    except OSError:
        pass
    return None


def data_note(c: dict) -> str:
    noise = f", Poisson noise I0={c['i0']:g}" if c.get("i0") else ""
    return f"synthetic: {c.get('n_ellipsoids', 20)} seeded random ellipsoids, analytic FP64 line integrals{noise}"


def updates_of(c: dict) -> int:
    return c["nx"] * c["ny"] * c["nz"] * c["nviews"]


# ------------------------------------------------------------------ CPU legs
def _oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    O.build(with_ref=False)
    return O


def oracle_sample(c: dict, raw_views, nvox: int, slice_vox: int = 100_000, chunk: int = 24) -> dict:
    """FP64 oracle values of seeded voxels spread over the whole volume, for
    the accuracy of a cone workload too large for a whole-volume oracle:
    `slice_vox` voxels in each of the y-slices near y = 0, ny/4, ny/2, 3 ny/4
    and ny - 1 and, when ny > nz, one in the band y >= nz that the reference's
    clip extent leaves unclipped (FBP3D.cpp:448), plus `nvox` voxels drawn
    uniformly over the volume (near-source tiles included). The oracle weights
    and filters the whole detector in FP64, `chunk` views at a time, and adds
    each chunk's backprojection at the sampled voxels (a chunk of views is the
    same orbit arc with its share of the pi / K scale). raw_views(k0, k1)
    returns views [k0, k1) of the raw projections as a [view][v][u] FP32 array.
    Returns the voxels (ix, iy, iz), their FP64 values and the index range of
    each band."""
    import numpy as np
    O = _oracle()
    rng = np.random.default_rng(c["seed"] + 17)
    nx, ny, nz, K = c["nx"], c["ny"], c["nz"], c["nviews"]
    ys = [1, ny // 4, ny // 2, (3 * ny) // 4, ny - 2]
    if ny > nz:
        ys.insert(4, nz + (ny - nz) // 2)
    ys = sorted({int(min(max(y, 0), ny - 1)) for y in ys})
    parts, bands, at = [], {}, 0
    for y in ys:
        parts.append(np.stack([rng.integers(0, nx, slice_vox), np.full(slice_vox, y), rng.integers(0, nz, slice_vox)], 1))
        bands[f"y={y}" + (" (unclipped band)" if y >= nz else "")] = (at, at + slice_vox)
        at += slice_vox
    if nvox > 0:
        parts.append(np.stack([rng.integers(0, nx, nvox), rng.integers(0, ny, nvox), rng.integers(0, nz, nvox)], 1))
        bands["random voxels"] = (at, at + nvox)
    ijk = np.ascontiguousarray(np.concatenate(parts).astype(np.int32))
    t0 = time.perf_counter()
    ref = np.zeros(len(ijk), np.float64)
    for k0 in range(0, K, chunk):
        k1 = min(K, k0 + chunk)
        p = O.fdk_weight(raw_views(k0, k1), c["sdd"], c["du"], c["dv"])
        q = O.filter_rows(p.reshape(-1, c["nu"]), c["filter"]).reshape(p.shape)
        del p
        arc = dict(c, span=c["span"] * (k1 - k0) / K, offset=c["offset"] + c["span"] * k0 / K)
        ref += O.bp_cone_points(q, arc, ijk) * ((k1 - k0) / K)
        del q
    clip = ijk[:, 1] < nz  # the reference's clip extent (y-slices below z_size)
    ref[clip] = np.maximum(ref[clip], 0.0)
    return {"ijk": ijk, "ref": ref, "bands": bands, "in_fov": in_field_of_view(c, ijk),
            "seconds": time.perf_counter() - t0, "threads": O.num_threads()}


def in_field_of_view(c: dict, ijk):
    """True for voxels whose projection lands inside the detector's sample
    grid in every view of a full circular orbit (so a relative error over
    them compares reconstructed signal, not the zero fill outside the
    detector). Closed form for a voxel at radius r from the rotation axis and
    height Y: its detector u over the orbit peaks at SDD r / sqrt(SOD^2 - r^2)
    (the tangent ray) and its |v| at SDD |Y| / (SOD - r) (the view with the
    voxel nearest the source)."""
    import numpy as np
    ix, iy, iz = (ijk[:, i].astype(np.float64) for i in range(3))
    X = (ix + 0.5 - c["nx"] / 2.0) * c["vox"]
    Y = (iy + 0.5 - c["ny"] / 2.0) * c["vox"]
    Z = (iz + 0.5 - c["nz"] / 2.0) * c["vox"]
    r = np.hypot(X, Z)
    sod, sdd = c["sod"], c["sdd"]
    u_half = (c["nu"] - 1) / 2.0 * c["du"]  # outermost sample centres: no zero-fill in the bilinear tap
    v_half = (c["nv"] - 1) / 2.0 * c["dv"]
    ok = r < sod
    rs = np.where(ok, r, 0.0)
    u_max = sdd * rs / np.sqrt(np.maximum(sod * sod - rs * rs, 1e-300))
    v_max = sdd * np.abs(Y) / np.maximum(sod - rs, 1e-300)
    return ok & (u_max <= u_half) & (v_max <= v_half)


def sample_error(got, ref, bands=None, in_fov=None) -> dict:
    """Relative RMSE and max abs error of `got` against the FP64 `ref`,
    overall and (bands: name -> index range) per band. With `in_fov` (a mask
    of the voxels the detector sees in every view) each band also reports
    the share of its voxels in the field of view and the relative RMSE over
    those voxels alone (None when the band has none)."""
    import numpy as np
    d = np.asarray(got, np.float64) - ref
    out = {"rel_rmse": float(np.linalg.norm(d) / np.linalg.norm(ref)), "max_abs": float(np.abs(d).max())}
    if in_fov is not None and in_fov.any():
        out["rel_rmse_in_fov"] = float(np.linalg.norm(d[in_fov]) / np.linalg.norm(ref[in_fov]))
    if bands:
        # per band: RMSE over the band's own reference RMS (ill-conditioned where
        # the band holds almost no signal, e.g. slices outside the phantom or
        # outside the detector's field of view) and over the whole sample's
        # reference RMS
        rms_all = float(np.sqrt(np.mean(ref ** 2)))
        out["bands"] = {}
        for k, (a, b) in bands.items():
            band = {"rel_rmse": float(np.linalg.norm(d[a:b]) / np.linalg.norm(ref[a:b])),
                    "rmse_over_sample_rms": float(np.sqrt(np.mean(d[a:b] ** 2)) / rms_all),
                    "ref_rms_over_sample_rms": float(np.sqrt(np.mean(ref[a:b] ** 2)) / rms_all),
                    "max_abs": float(np.abs(d[a:b]).max())}
            if in_fov is not None:
                m = in_fov[a:b]
                band["in_fov_share"] = float(m.mean())
                band["rel_rmse_in_fov"] = (float(np.linalg.norm(d[a:b][m]) / np.linalg.norm(ref[a:b][m]))
                                           if m.any() and np.linalg.norm(ref[a:b][m]) > 0 else None)
            out["bands"][k] = band
    return out


def cpu_sample(c: dict, proj_views, view_ids, target_s: float) -> dict:
    """Time the reference CPU path on a bounded sample and extrapolate.

    Filter stage: FDK weights + row filter of the sampled views with the
    reference's FFT (compiled from its sources; the oracle's repo-pi
    restatement where that build is absent), OpenMP over rows.
    Backprojection stage: the FP32 CPU restatement over four y-slabs spread
    along the rotation axis for the sampled views, sized so that this stage
    takes about 60% of `target_s`. Each stage's cost per unit (row, update)
    is scaled to the full job's units."""
    import numpy as np
    O = _oracle()
    threads = O.num_threads()
    use_ref = O.ref_available()
    n = O.padded_length(c["nu"])
    t0 = time.perf_counter()
    w = O.fdk_weight(proj_views, c["sdd"], c["du"], c["dv"]).astype(np.float32)
    rows = w.reshape(-1, c["nu"])
    if use_ref:
        filt = O.ref_filter_rows(rows, c["filter"], n)
    else:
        filt = O.filter_rows(rows.astype(np.float64), c["filter"], n, pi_mode=O.PI_REPO).astype(np.float32)
    t_filter = time.perf_counter() - t0
    per_row = t_filter / rows.shape[0]
    q = filt.reshape(len(view_ids), c["nv"], c["nu"])
    nsel = len(view_ids)

    def slabs(height: int):
        """Four slabs of `height` slices spread along y; returns updates done."""
        done = 0
        for f in (0.125, 0.375, 0.625, 0.875):
            y0 = min(c["ny"] - height, int(f * c["ny"]))
            vol = np.zeros((c["nz"], height, c["nx"]), np.float32)
            O.cpu_bp_cone_f32(q, view_ids, c, y0, y0 + height, vol)
            done += c["nx"] * c["nz"] * height * nsel
        return done

    t0 = time.perf_counter()
    probe = slabs(1)
    t_probe = time.perf_counter() - t0
    per_update = t_probe / probe
    height = max(1, min(c["ny"] // 4, int(0.6 * target_s / (per_update * 4 * c["nx"] * c["nz"] * nsel))))
    t0 = time.perf_counter()
    nup = slabs(height)
    t_bp = time.perf_counter() - t0
    per_update = t_bp / nup
    t_full = per_row * c["nviews"] * c["nv"] + per_update * updates_of(c)
    return dict(value=updates_of(c) / t_full / 1e9, cores=threads, use_ref=use_ref, per_row_s=per_row,
                per_update_s=per_update, sample_rows=int(rows.shape[0]), sample_updates=int(nup),
                sample_seconds=t_filter + t_bp, full_seconds=t_full)


def cpu_inputs(c: dict, nviews_sample: int):
    """Analytic projections of the benchmark phantom for a few views (FP64 on
    the CPU), with the workload's Poisson noise."""
    import numpy as np
    import phantoms as P
    O = _oracle()
    E = P.ellipsoids_for(c)
    views = np.linspace(0, c["nviews"] - 1, nviews_sample).round().astype(np.int32)
    proj = O.project_ellipsoids_cone(E, c, views)
    if "i0" in c:
        if c.get("i0"):
            proj = P.poisson_log(proj, c["i0"], np.random.default_rng(c["seed"]))
    return proj, views


def reference_arm(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    if args.workload == "serving":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving path (one "
                          "reconstruction per process); its CPU arm is measured on the cone workloads"}), flush=True)
        return
    c = workload(args.scale, args.workload)
    nsv = 8 if args.scale == 1 else 4
    proj, views = cpu_inputs(c, nsv)
    results = []
    for i in range(args.warmup + args.steps):
        r = cpu_sample(c, proj, views, target_s=args.cpu_seconds / 3)
        if i >= args.warmup:
            results.append(r)
    val = statistics.mean(r["value"] for r in results)
    r0 = results[-1]
    ms = updates_of(c) / (val * 1e9) * 1e3
    kind = "reference" if r0["use_ref"] else "port"
    sample = (f"{r0['sample_rows']} detector rows filtered with the reference's FFT::fft_radix2 "
              f"{'(compiled from its sources)' if r0['use_ref'] else '(oracle restatement, repo pi)'} and "
              f"{r0['sample_updates']:.3g} voxel-view updates of the CPU FP32 backprojector restatement "
              f"(the reference has no CPU backprojector), extrapolated linearly to the full job")
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 filter / f32 backprojection",
        "data": data_note(c),
        "config": {"workload": c["name"], "volume_xyz": [c["nx"], c["ny"], c["nz"]], "views": c["nviews"],
                   "detector": [c["nu"], c["nv"]], "filter": FILTER_NAMES[c["filter"]], "parallelism": "host cores"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": r0["cores"], "kind": kind, "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        # each step times a sample of the job and extrapolates: ms_per_step is
        # the full job's estimated time, not the time the step took
        "extrapolated": True,
        "sampled_fraction": {"filter_rows": r0["sample_rows"] / (c["nviews"] * c["nv"]),
                             "backprojection_updates": r0["sample_updates"] / updates_of(c)},
        "sample_seconds_per_step": statistics.mean(r["sample_seconds"] for r in results),
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples of this process's GPU."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.proc = None
        self.out = Path(os.environ.get("TMPDIR", "/tmp")) / f"fbp_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.out, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            if self.uuid and self.uuid not in parts[0]:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        self.out.unlink(missing_ok=True)
        loaded = sorted(sm)[len(sm) // 4:] if sm else []  # drop the idle quarter
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ our arm
def serving_requests(n: int, seed: int = 1004) -> list[dict]:
    """The mixed stream: 40 % 2D fan (512^2 or 1024^2 images, 720-1440 views,
    768-1536 bins), 40 % cone FDK (edge in {128, 192, 256, 384, 512}, 360-720
    views, detector 1.5 x edge), 20 % cone 768^3 with 1024 views. View and
    bin counts are drawn on a grid (multiples of 120 views, 256 bins) so that
    the inputs come from a pool of distinct shapes."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        u = rng.random()
        if u < 0.4:
            out.append(dict(kind="fan", n=int(rng.choice([512, 1024])), views=int(rng.choice([720, 960, 1200, 1440])),
                            bins=int(rng.choice([768, 1024, 1280, 1536]))))
        elif u < 0.8:
            e = int(rng.choice([128, 192, 256, 384, 512]))
            out.append(dict(kind="cone", n=e, views=int(rng.choice([360, 480, 600, 720])), det=e * 3 // 2))
        else:
            out.append(dict(kind="cone", n=768, views=1024, det=1152))
    return out


def serving_block(args, n_requests: int, n_poisson: int) -> dict:
    """Serving on one GPU: the chosen form under continuous
    batching (MIXED, `--slots` worker slots, cone backprojections through the
    persistent multi-job backprojector) against the plain FP32 form run one
    job at a time. Capacity = reconstructions/s with the whole stream
    submitted at once; latency = p50 / p99 of finish - arrival under seeded
    Poisson arrivals at `--load` x the plain capacity (the first `n_poisson`
    requests). The plain form runs one job at a time, so its stream time is
    the sum of its jobs' service times: every distinct job shape is timed
    alone through the server (one slot, upload + reconstruction + readback,
    median of 3) and the plain capacity and FIFO latencies follow from those
    times; an actual plain run of the first 200 requests checks the sum.
    Inputs: seeded random ellipsoids projected analytically on the GPU (fan
    jobs: the central detector row), held in pinned host memory."""
    import numpy as np
    import torch

    import build as B
    B.build()
    import fbp_b200 as F
    import phantoms as P

    torch.cuda.set_device(0)
    reqs = serving_requests(n_requests)

    def shape_key(r):
        return (r["kind"], r["n"], r["views"], r.get("det", r.get("bins")))

    def geometry(r):
        if r["kind"] == "cone":  # 1 mm voxels, magnification 1.5, detector 1.5 x the volume's shadow
            e = r["n"]
            return F.Geometry.cone(3.0 * e, 1.5 * e, 1.5 * r["det"], float(e), 1.0, 0.0)
        # fan: SOD 500, SDD 1000, 256 mm field of view, 768 mm detector
        return F.Geometry.cone(500.0, 500.0, 768.0, 256.0, 1.0, 0.0)

    # ---- input pool (pinned host), one seeded phantom per distinct shape
    pool, outs = {}, {}
    gen = F.FBP3D(0)
    for i, key in enumerate(sorted({shape_key(r) for r in reqs})):
        kind, n, views, cols = key
        rows = cols if kind == "cone" else 1
        g = geometry(dict(kind=kind, n=n, views=views, det=cols, bins=cols))
        radius = 0.5 * g.volume_width
        E = P.random_ellipsoids(np.random.default_rng(2000 + i), 20, radius)
        gen.generate_blank_projections(cols, rows, views)
        gen.project_ellipsoids(E, g)
        host = torch.empty((views, rows, cols), dtype=torch.float32, pin_memory=True)
        gen.download_projections(host)
        pool[key] = host
        vol_shape = (n, n, n) if kind == "cone" else (n, n)
        outs[key] = [torch.empty(vol_shape, dtype=torch.float32, pin_memory=True) for _ in range(args.slots + 1)]
    gen.ctx.close()
    del gen

    def request_struct(r, precision, out):
        key = shape_key(r)
        q = F.Request()
        q.kind = F.JobKind.CONE if r["kind"] == "cone" else F.JobKind.FAN2D
        q.precision = precision
        q.filter_type = 0 if r["kind"] == "cone" else 1
        q.clip = 1
        q.geometry = geometry(r)
        inp = pool[key]
        q.views, q.det_rows, q.det_cols = inp.shape
        q.vol_h = r["n"]
        q.vol_v = r["n"] if r["kind"] == "cone" else 1
        q.input, q.output = inp.data_ptr(), out.data_ptr()
        return q

    def server(precision, slots):
        srv = F.Server(0, 0, slots)
        srv.set_batching(precision != F.Precision.FP32)
        # warm every slot's buffers with the largest jobs (buffers only grow)
        big = max(reqs, key=lambda r: r["n"] ** 3 * r["views"] if r["kind"] == "cone" else 0)
        big2 = max(reqs, key=lambda r: r["n"] ** 2 * r["views"] if r["kind"] == "fan" else 0)
        warm = [srv.submit(request_struct(w, precision, outs[shape_key(w)][0])) for w in [big] * slots + [big2] * slots]
        for t in warm:
            assert srv.wait(t).status == 0
        return srv

    def run(precision, slots, stream, arrivals=None):
        srv = server(precision, slots)
        rr = {k: 0 for k in outs}
        tickets = []
        t0 = time.perf_counter()
        for i, r in enumerate(stream):
            if arrivals is not None:
                delay = arrivals[i] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            key = shape_key(r)
            out = outs[key][rr[key] % len(outs[key])]
            rr[key] += 1
            tickets.append(srv.submit(request_struct(r, precision, out)))
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
        srv.close()
        bad = [x.error.decode() for x in res if x.status != 0]
        assert not bad, bad[:3]
        lat = np.array([x.finished_ms - x.queued_ms for x in res])
        span = (max(x.finished_ms for x in res) - min(x.queued_ms for x in res)) * 1e-3
        return dict(requests=len(res), recon_per_s=len(res) / span, p50_ms=float(np.percentile(lat, 50)),
                    p99_ms=float(np.percentile(lat, 99)), makespan_s=span, server_stats=st)

    # ---- plain one at a time: per-shape service times
    srv = server(F.Precision.FP32, 1)
    service = {}
    for key in sorted({shape_key(r) for r in reqs}):
        r = next(x for x in reqs if shape_key(x) == key)
        ts = []
        for _ in range(3):
            res = srv.wait(srv.submit(request_struct(r, F.Precision.FP32, outs[key][0])))
            assert res.status == 0, res.error
            ts.append((res.finished_ms - res.started_ms) * 1e-3)
        service[key] = float(np.median(ts))
    srv.close()
    t_plain = np.array([service[shape_key(r)] for r in reqs])
    plain_cap = {"requests": len(reqs), "recon_per_s": len(reqs) / t_plain.sum(), "makespan_s": float(t_plain.sum()),
                 "from": "sum of per-shape service times measured alone"}
    check = run(F.Precision.FP32, 1, reqs[:200])
    plain_cap["measured_first_200"] = {"recon_per_s": check["recon_per_s"],
                                       "from_service_times": 200 / t_plain[:200].sum()}
    rate = args.load * plain_cap["recon_per_s"]
    npo = min(n_poisson, len(reqs))
    arrivals = np.cumsum(np.random.default_rng(1005).exponential(1.0 / rate, size=npo))
    # plain under Poisson arrivals: one FIFO server with those service times
    fin, lat = 0.0, []
    for a, t in zip(arrivals, t_plain[:npo]):
        fin = max(a, fin) + t
        lat.append((fin - a) * 1e3)
    plain_lat = {"requests": npo, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                 "from": "FIFO of the measured service times"}
    chosen_cap = run(F.Precision.MIXED, args.slots, reqs)
    chosen_lat = run(F.Precision.MIXED, args.slots, reqs[:npo], arrivals)
    mix = {"fan2d": sum(r["kind"] == "fan" for r in reqs), "cone_128_512": sum(r["kind"] == "cone" and r["n"] < 768
                                                                               for r in reqs),
           "cone_768": sum(r["kind"] == "cone" and r["n"] == 768 for r in reqs)}
    return {
        "metric": "mixed-stream reconstructions/s", "value": chosen_cap["recon_per_s"], "unit": "recon/s",
        "config": {"workload": "serving_mixed_stream", "requests": len(reqs), "mix": mix, "slots": args.slots,
                   "poisson_requests": npo, "arrival_rate_per_s": rate, "load_vs_plain_capacity": args.load,
                   "batching": "cone jobs of up to 1e10 voxel-view updates through the persistent multi-job "
                               "backprojector, larger ones (768^3) through their own slab pipelines"},
        "chosen": {"capacity": chosen_cap, "poisson": chosen_lat},
        "plain_one_at_a_time_fp32": {"capacity": plain_cap, "poisson": plain_lat},
        "chosen_over_plain_recon_per_s": chosen_cap["recon_per_s"] / plain_cap["recon_per_s"],
        "p50_ms": chosen_lat["p50_ms"], "p99_ms": chosen_lat["p99_ms"],
    }


def serving_main(args) -> None:
    """--workload serving: the serving block alone, as its own JSON line."""
    blk = serving_block(args, args.requests, args.poisson_requests)
    line = {"metric": blk["metric"], "value": blk["value"], "unit": blk["unit"], "n_gpus": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 accumulate / f16 filtered views (chosen)",
            "data": "synthetic: seeded random ellipsoids, analytic projections (GPU), pinned host inputs"}
    line.update({k: v for k, v in blk.items() if k not in line})
    print(json.dumps(line), flush=True)


def main() -> None:
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.workload == "serving":
        serving_main(args)
        return

    import numpy as np
    import torch

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    import build as B
    B.build()
    import fbp_b200 as F
    import phantoms as P

    c = workload(args.scale, args.workload)
    U = updates_of(c)
    ga = P.geometry_args(c)
    geom = F.Geometry.cone(ga["sod"], ga["odd"], ga["detector_width"], ga["volume_width"],
                           ga["full_rotation_count"], c["offset"])
    stream = torch.cuda.Stream(dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def sum_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- inputs: analytic projections on the device + Poisson noise
    gen = F.FBP3D(local_rank)
    gen.set_stream(stream)
    gen.generate_blank_projections(c["nu"], c["nv"], c["nviews"])
    gen.project_ellipsoids(P.ellipsoids_for(c), geom)
    pristine = torch.empty((c["nviews"], c["nv"], c["nu"]), dtype=torch.float32, device=dev)
    gen.download_projections(pristine)
    gen.synchronize()
    gen.ctx.close()
    del gen
    with torch.cuda.stream(stream):
        g = torch.Generator(device=dev)
        g.manual_seed(c["seed"] + 7919 * rank)
        for k0 in range(0, c["nviews"] if c.get("i0") else 0, 64):
            blk = pristine[k0:k0 + 64]
            counts = torch.poisson(c["i0"] * torch.exp(-blk), generator=g)
            blk.copy_(-torch.log(torch.clamp(counts, min=1.0) / c["i0"]))
            del counts
    stream.synchronize()

    # y-slab sharding: this rank keeps only its detector row band and volume slab
    slab = (0, c["ny"], 0, c["nv"])
    if args.shard == "slabs":
        slab = F.plan_slabs(geom, c["nu"], c["nv"], c["nx"], c["ny"], world)[rank]
        pristine = pristine[:, slab[2]:slab[3], :].contiguous()
        torch.cuda.empty_cache()
    slab_ny = slab[1] - slab[0]
    job_units = U if args.shard == "slabs" else world * U  # voxel-view updates of the whole job

    sod, odd, w, vw, rot = ga["sod"], ga["odd"], ga["detector_width"], ga["volume_width"], ga["full_rotation_count"]

    def make_solver(form: str, on_stream=None):
        s = F.FBP3D(local_rank)
        s.set_stream(stream if on_stream is None else on_stream)
        s.set_precision(getattr(F.Precision, FORMS[form][0]))
        s.set_clip_after_backprojection(True)
        if args.tile_ny:
            s.set_symmetric_tile(args.tile_ny)
        if args.backprojector == "tuned":
            s.set_autotune(True)
        elif args.backprojector != "auto":
            s.set_backprojector(getattr(F.Backprojector, args.backprojector.upper()))
        if args.shard == "slabs":
            s.set_detector_rows(slab[2], c["nv"])
            s.set_volume_slab(slab[0], slab_ny)
        return s

    def step(s, src, ev=None):
        s.upload_projections(src)
        s.apply_fdk_weights_to_projections(sod, odd, w)
        if ev is not None:
            ev[0].record(stream)
        s.apply_filter_to_projections(c["filter"])
        if ev is not None:
            ev[1].record(stream)
        s.project_backward_cone_fdk_from_projections(sod, odd, w, vw, rot, c["nx"], c["ny"], c["offset"])
        if ev is not None:
            ev[2].record(stream)

    def e2e_step(s, src, dst):
        # host buffers in and out through one C-ABI call; the volume readback
        # overlaps the slab-wise backprojection
        s.reconstruct_fdk_to_host(src, geom, c["filter"], c["nx"], c["ny"], out=dst, slabs=8)

    def timed(s, src, readback=None, streamed=False) -> dict:
        for _ in range(args.warmup):
            if streamed:
                e2e_step(s, src, readback)
                continue
            step(s, src)
            if readback is not None:
                s.read_volume(readback)
        s.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = s.kernel_launch_count()
        barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(str(torch.cuda.get_device_properties(dev).uuid) if hasattr(
            torch.cuda.get_device_properties(dev), "uuid") else "")
        clocks.start()
        t_wall = time.perf_counter()
        start.record(stream)
        for k in range(args.steps):
            if streamed:
                e2e_step(s, src, readback)
                continue
            step(s, src, evs[k])
            if readback is not None:
                s.read_volume(readback)
        end.record(stream)
        stream.synchronize()
        t_wall = time.perf_counter() - t_wall
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop()
        launches = s.kernel_launch_count() - launches0
        ms = max_over_ranks(start.elapsed_time(end) / args.steps)
        filt_ms = 0.0 if streamed else statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
        bp_ms = 0.0 if streamed else statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
        return dict(ms=ms, filter_ms=filt_ms, bp_ms=bp_ms, launches=launches, clocks=clk,
                    wall_ms=t_wall * 1e3 / args.steps)

    def pipelined(solvers, src, dsts) -> dict:
        """K reconstructions through e2e_step, alternating over the solvers from
        one host thread each; the second thread starts one projection upload
        later (the H2D time measured here) so the two uploads do not split the
        link. Device-timed: events on the torch stream around the whole run,
        after a device-wide synchronisation on both sides."""
        for i in range(max(args.warmup, len(solvers))):
            e2e_step(solvers[i % len(solvers)], src, dsts[i % len(solvers)])
        probe = torch.empty(1 << 28, dtype=torch.float32, device=dev)  # 1 GiB
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flat = src.view(-1)[: probe.numel()]
        h0.record()
        probe.copy_(flat, non_blocking=True)
        h1.record()
        h1.synchronize()
        delay_s = h0.elapsed_time(h1) * 1e-3 * (src.numel() / probe.numel())
        del probe, flat
        counts = [args.steps // len(solvers) + (1 if i < args.steps % len(solvers) else 0)
                  for i in range(len(solvers))]
        errors = []

        def worker(i):
            try:
                if i:
                    time.sleep(delay_s)
                for _ in range(counts[i]):
                    e2e_step(solvers[i], src, dsts[i])
            except Exception as exc:  # re-raised on the main thread
                errors.append(exc)

        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        start.record()
        threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(solvers)) if counts[i]]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        torch.cuda.synchronize()
        end.record()
        end.synchronize()
        barrier()
        if errors:
            raise errors[0]
        return dict(ms=max_over_ranks(start.elapsed_time(end) / args.steps), delay_ms=delay_s * 1e3)

    forms = [f.strip() for f in args.forms.split(",") if f.strip()]
    res, vols = {}, {}
    smem_bw = None
    for form in forms:
        s = make_solver(form)
        res[form] = timed(s, pristine)
        res[form]["kernel"] = s.last_backprojection()
        vols[form] = torch.empty((c["nz"], slab_ny, c["nx"]), dtype=torch.float32, device=dev)
        s.read_volume(vols[form])
        if smem_bw is None:
            smem_bw = s.measure_smem_bandwidth()
        s.ctx.close()
        del s
        torch.cuda.empty_cache()

    accuracy = {}
    if rank == 0 and world == 1 and args.shard != "slabs" and args.oracle_voxels > 0:
        chk = oracle_sample(c, lambda k0, k1: pristine[k0:k1].cpu().numpy(), args.oracle_voxels,
                            args.oracle_slice_voxels)
        ix, iy, iz = (torch.as_tensor(chk["ijk"][:, i], device=dev, dtype=torch.long) for i in range(3))
        for form, vol in vols.items():
            accuracy[f"{form}_vs_fp64_oracle"] = sample_error(vol[iz, iy, ix].double().cpu().numpy(), chk["ref"],
                                                              chk["bands"], chk["in_fov"])
        accuracy["oracle_sample"] = (f"{args.oracle_slice_voxels} seeded voxels in each y-slice band and "
                                     f"{args.oracle_voxels} seeded voxels uniform over the volume, each "
                                     f"backprojected in FP64 from the whole detector weighted and filtered "
                                     f"in FP64 ({chk['seconds']:.0f} s on {chk['threads']} host threads); "
                                     f"rel_rmse_in_fov: over the sampled voxels that project inside the "
                                     f"detector in every view ({float(chk['in_fov'].mean()):.2f} of the "
                                     f"sample; none in the outermost slices, which the cone never sees whole)")
    for form in [f for f in vols if f != "plain" and "plain" in vols]:
        a, b = vols[form].double(), vols["plain"].double()
        accuracy[f"{form}_vs_plain_rel_rmse"] = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        accuracy[f"{form}_vs_plain_max_abs"] = float((a - b).abs().max())
        del a, b
    vols.clear()
    torch.cuda.empty_cache()

    # ---- end to end through the C ABI with pinned host buffers (chosen form)
    e2e = None
    head = args.head if args.head in res else forms[0]
    if not args.no_e2e:
        host_proj = torch.empty(tuple(pristine.shape), dtype=torch.float32, pin_memory=True)
        host_proj.copy_(pristine)
        host_vol = torch.empty((c["nz"], slab_ny, c["nx"]), dtype=torch.float32, pin_memory=True)
        s = make_solver(head)
        r = timed(s, host_proj, readback=host_vol, streamed=args.shard != "slabs")
        e2e = {"value": job_units / (r["ms"] * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(sum_over_ranks(host_proj.numel() * 4)),
               "d2h_bytes_per_step": int(sum_over_ranks(host_vol.numel() * 4)),
               "ms_per_step": r["ms"]}
        if args.shard != "slabs":
            # the same calls from two host threads, each with its own context and
            # stream: one reconstruction's upload and readback overlap the other's
            # kernels (every step still moves its own inputs and volume)
            host_vol2 = torch.empty_like(host_vol, pin_memory=True)
            s2 = make_solver(head, torch.cuda.Stream(dev))
            p = pipelined([s, s2], host_proj, [host_vol, host_vol2])
            e2e = {"value": job_units / (p["ms"] * 1e-3) / 1e9, "unit": UNIT,
                   "h2d_bytes_per_step": e2e["h2d_bytes_per_step"], "d2h_bytes_per_step": e2e["d2h_bytes_per_step"],
                   "ms_per_step": p["ms"], "contexts": 2, "launch_delay_ms": p["delay_ms"],
                   "serial": {"value": e2e["value"], "ms_per_step": e2e["ms_per_step"]},
                   "note": "fbp_reconstruct_fdk_to_host from two host threads with one context and stream each; "
                           "serial: one context, one call after another"}
            s2.ctx.close()
            del s2, host_vol2
        s.ctx.close()
        del s
        del host_proj, host_vol

    h = res[head]
    value = job_units / (h["ms"] * 1e-3) / 1e9
    # roofline of the dominant kernel (the backprojector)
    esize = FORMS[head][1]
    bp_s = h["bp_ms"] * 1e-3
    band_rows = slab[3] - slab[2]
    local_units = c["nx"] * slab_ny * c["nz"] * c["nviews"]  # this rank's updates
    hbm_bytes = c["nviews"] * band_rows * c["nu"] * esize + 4 * c["nx"] * slab_ny * c["nz"]
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    gather_bytes = 4 * esize * local_units  # four bilinear taps per update
    traffic = measured_traffic(c["name"], head) if slab == (0, c["ny"], 0, c["nv"]) else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": h["ms"], "higher_is_better": True,
        "scaling": "strong" if args.shard == "slabs" else "weak",
        "vs_baseline": None, "dtype": DTYPES[head], "storage_dtype": FORMS[head][2],
        "data": data_note(c),
        "config": {"workload": c["name"], "volume_xyz": [c["nx"], c["ny"], c["nz"]], "voxel_mm": c["vox"],
                   "views": c["nviews"], "detector": [c["nu"], c["nv"]], "pitch_mm": c["du"],
                   "sod_mm": c["sod"], "sdd_mm": c["sdd"], "filter": FILTER_NAMES[c["filter"]], "form": head,
                   "parallelism": (f"y-slabs x{world}" if args.shard == "slabs" else f"replicas x{world}")
                   if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (projections %.1f GB)" % (c["nviews"] * c["nv"] * c["nu"] * 4 / 1e9),
                   "step": "D2D restore of raw projections + weights + filter + backprojection + clip"},
        "stages_ms": {"filter": h["filter_ms"], "backprojection": h["bp_ms"]},
        "roofline": {"bound": "hbm", "achieved": hbm_bytes / bp_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
                     "frac": hbm_bytes / bp_s / 1e9 / hbm_peak, "traffic": traffic,
                     "traffic_source": "profiles/bp_dram_traffic.txt (ncu dram__bytes_read.sum + "
                                       "dram__bytes_write.sum of one launch, not measured in this run)",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                     "note": "backprojector algorithmic HBM bytes (filtered views read once + volume written "
                             "once); the kernel is bound by shared-memory gathers, see roofline_smem"},
        "roofline_smem": {"bound": "smem", "achieved": gather_bytes / bp_s / 1e12,
                          "peak": smem_bw / 1e12, "unit": "TB/s",
                          "frac": (gather_bytes / bp_s) / smem_bw,
                          "bytes_per_update": 4 * esize},
        "gpu_launches": h["launches"],
        "clocks": h["clocks"],
        "accuracy": accuracy,
    }
    for form, r in res.items():
        line[f"form_{form}"] = {"value": job_units / (r["ms"] * 1e-3) / 1e9, "ms_per_step": r["ms"],
                                "filter_ms": r["filter_ms"], "backprojection_ms": r["bp_ms"],
                                "gpu_launches": r["launches"], "clocks": r["clocks"], "backprojector": r["kernel"]}
    for form in [f for f in res if f != "plain" and "plain" in res]:
        line[f"{form}_over_plain"] = res["plain"]["ms"] / res[form]["ms"]
    if e2e is not None:
        line["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        proj, views = cpu_inputs(c, 8 if args.scale == 1 else 4)
        r = cpu_sample(c, proj, views, target_s=args.cpu_seconds)
        line["cpu_baseline"] = {
            "value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference" if r["use_ref"] else "port",
            "sample": (f"{r['sample_rows']} detector rows filtered with the reference's own FFT "
                       f"({'compiled from its sources' if r['use_ref'] else 'oracle restatement'}), "
                       f"{r['sample_updates']:.3g} updates of the FP32 CPU backprojector restatement, "
                       f"extrapolated to the full job ({r['full_seconds']:.0f} s)")}
    if rank == 0 and world == 1 and args.workload == "cone1440" and args.scale == 1 and not args.no_serving:
        del pristine
        torch.cuda.empty_cache()
        line["serving"] = serving_block(args, args.requests, args.poisson_requests)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
