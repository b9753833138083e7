"""Python host side of the B200 CT reconstruction core.

Loads libfbp_b200.so (built in place by build.py) through ctypes and mirrors
the reference's classes (furkanunsal42/3DFilteredBackProjection-Public):

  FBP3D  Source/FilteredBackProjection/FBP3D.h:16-170
  FBP2D  Source/FilteredBackProjection/FBP2D.h:8-72
  FFFT   Source/FastFourierTransformGPU/FastFourierTransformGPU.h:10-67

with the same method names and argument order. Where the reference passes
GL textures, these take numpy arrays (host) or torch CUDA tensors (device).
Every failing call raises FBPError carrying the library's message, where the
reference printed and ASSERTed. There is no CPU fallback: without the
compiled library or a B200 every call raises.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libfbp_b200.so"

OK = 0


class FBPError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[fbp_b200 status {status}] {message}")
        self.status = status


class FilterType(enum.IntEnum):
    """FBP2D::FilterType (FBP2D.h:10-14) plus two added filters."""
    RAM_LAK = 0
    SHEPP_LOGAN = 1
    COSINE = 2
    HANN = 3
    RAMP_SAMPLED = 4


class Precision(enum.IntEnum):
    FP32 = 0
    MIXED = 1
    MIXED24 = 2


class Backprojector(enum.IntEnum):
    AUTO = 0
    GENERIC = 1
    SYMMETRIC = 2
    GENERIC_Y8 = 3


class FilterImpl(enum.IntEnum):
    AUTO = 0
    FFT = 1
    TOEPLITZ = 2


class JobKind(enum.IntEnum):
    CONE = 0
    FAN2D = 1
    PARALLEL2D = 2
    HOST_WAIT = 3


class Geometry(C.Structure):
    """fbp_geometry (include/fbp_b200.h)."""
    CONE = 0
    PARALLEL = 1
    _fields_ = [
        ("kind", C.c_int),
        ("source_distance", C.c_float),
        ("detector_distance", C.c_float),
        ("detector_width", C.c_float),
        ("volume_width", C.c_float),
        ("full_rotation_count", C.c_float),
        ("rotation_offset_radian", C.c_float),
    ]

    @classmethod
    def cone(cls, sod, odd, detector_width, volume_width, full_rotation_count=1.0, offset=0.0):
        return cls(cls.CONE, sod, odd, detector_width, volume_width, full_rotation_count, offset)

    @classmethod
    def parallel(cls, detector_width, volume_width, full_rotation_count=0.5, offset=0.0):
        return cls(cls.PARALLEL, 0.0, 0.0, detector_width, volume_width, full_rotation_count, offset)


_lib: Optional[C.CDLL] = None
_P = C.c_void_p
_F = C.c_float
_I = C.c_int

# (name, argtypes) of every entry point declared in include/fbp_b200.h
SIGNATURES = {
    "fbp_create": [C.POINTER(_P), _I],
    "fbp_destroy": [_P],
    "fbp_last_error": [_P],
    "fbp_set_stream": [_P, _P],
    "fbp_synchronize": [_P],
    "fbp_set_precision": [_P, _I],
    "fbp_set_filter_impl": [_P, _I],
    "fbp_set_filter_padding": [_P, _I],
    "fbp_set_clip_after_backprojection": [_P, _I],
    "fbp_set_backprojector": [_P, _I],
    "fbp_memory_in_use": [_P, C.POINTER(C.c_size_t)],
    "fbp_last_backprojection": [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_int)],
    "fbp_set_autotune": [_P, _I],
    "fbp_set_symmetric_tile": [_P, _I],
    "fbp_set_autotune_cache": [_P, C.c_char_p],
    "fbp_autotune_stats": [_P, C.POINTER(_I), C.POINTER(_I)],
    "fbp_set_view_ring": [_P, _I],
    "fbp_project_backward_cone_fdk_batch": [C.POINTER(C.c_void_p), C.POINTER(Geometry), C.POINTER(_I),
                                            C.POINTER(_I), _I, _P],
    "fbp_generate_blank_volume": [_P, _I, _I, _I],
    "fbp_generate_blank_projections": [_P, _I, _I, _I],
    "fbp_generate_blank_sinograms": [_P, _I, _I, _I],
    "fbp_free_volume": [_P],
    "fbp_free_projections": [_P],
    "fbp_free_sinograms": [_P],
    "fbp_get_volume_size": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)],
    "fbp_get_projections_size": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)],
    "fbp_get_sinograms_size": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)],
    "fbp_upload_projections": [_P, _P, _I, _I, _I, _I],
    "fbp_upload_sinograms": [_P, _P, _I, _I, _I, _I],
    "fbp_download_projections": [_P, _P, _I],
    "fbp_download_sinograms": [_P, _P, _I],
    "fbp_store_projection": [_P, _P, _I, _I],
    "fbp_load_projection": [_P, _I, _P, _I],
    "fbp_store_sinogram": [_P, _P, _I, _I],
    "fbp_load_sinogram": [_P, _I, _P, _I],
    "fbp_load_projection_from_sinograms": [_P, _I, _P, _I],
    "fbp_store_projection_to_sinograms": [_P, _P, _I, _I],
    "fbp_load_volume_slice_x": [_P, _I, _P, _I],
    "fbp_load_volume_slice_y": [_P, _I, _P, _I],
    "fbp_load_volume_slice_z": [_P, _I, _P, _I],
    "fbp_store_volume_slice_x": [_P, _P, _I, _I],
    "fbp_store_volume_slice_y": [_P, _P, _I, _I],
    "fbp_store_volume_slice_z": [_P, _P, _I, _I],
    "fbp_read_volume": [_P, _P, _I],
    "fbp_write_volume_data": [_P, _P, _I],
    "fbp_volume_device_ptr": [_P, C.POINTER(_P)],
    "fbp_projections_device_ptr": [_P, C.POINTER(_P), C.POINTER(_I)],
    "fbp_log_normalize_projections": [_P, _F],
    "fbp_log_normalize_sinograms": [_P, _F],
    "fbp_apply_fdk_weights_to_projections": [_P, _F, _F, _F],
    "fbp_apply_fdk_weights_to_sinograms": [_P, _F, _F, _F],
    "fbp_apply_filter_to_projections": [_P, _I],
    "fbp_apply_filter_to_sinograms": [_P, _I],
    "fbp_clip_negatives_of_volume": [_P],
    "fbp_volume_min_max": [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)],
    "fbp_read_projections": [_P, C.c_char_p, _I, _I, _I, _I, _I, _I, _I],
    "fbp_read_projections_as_sinograms": [_P, C.c_char_p, _I, _I, _I, _I, _I, _I, _I],
    "fbp_write_volume": [_P, C.c_char_p],
    "fbp_projection_file_index": [C.c_char_p],
    "fbp_plan_slabs": [C.POINTER(Geometry), _I, _I, _I, _I, _I, C.POINTER(C.c_int)],
    "fbp_reconstruct_fdk_to_host": [_P, _P, _I, _I, _I, C.POINTER(Geometry), _I, _I, _I, _P, _I],
    "fbp_project_forward_cone_to_projections": [_P, _F, _F, _F, _F, _F, _I, _F],
    "fbp_project_forward_cone_to_sinograms": [_P, _F, _F, _F, _F, _F, _I, _F],
    "fbp_project_forward_parallel_to_projections": [_P, _F, _I, _F],
    "fbp_project_forward_parallel_to_sinograms": [_P, _F, _I, _F],
    "fbp2d_project_forward": [_P, _P, _I, _I, _P, _I, _I, C.POINTER(Geometry)],
    "fbp_server_create": [C.POINTER(C.c_void_p), _I, C.c_size_t, _I],
    "fbp_server_submit": [C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong)],
    "fbp_server_set_batching": [C.c_void_p, _I, C.c_double],
    "fbp_server_set_batch_limit": [C.c_void_p, C.c_double],
    "fbp_server_stats": [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                         C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "fbp_server_wait": [C.c_void_p, C.c_longlong, C.c_void_p],
    "fbp_server_destroy": [C.c_void_p],
    "fbp_set_detector_rows": [_P, _I, _I],
    "fbp_set_volume_slab": [_P, _I, _I],
    "fbp_normalize_histogram": [_P],
    "fbp_normalize_histogram_range": [_P, C.c_float, C.c_float],
    "fbp_project_backward_cone_fdk_from_projections": [_P, _F, _F, _F, _F, _F, _I, _I, _F],
    "fbp_project_backward_cone_fdk_from_sinograms": [_P, _F, _F, _F, _F, _F, _I, _I, _F],
    "fbp_project_backward_parallel_from_projections": [_P, _F, _I, _I, _F],
    "fbp_project_backward_parallel_from_sinograms": [_P, _F, _I, _I, _F],
    "fbp_reconstruct_fdk": [_P, C.POINTER(Geometry), _I, _I, _I],
    "fbp2d_filter_sinogram": [_P, _P, _I, _I, _I, _F, _F],
    "fbp2d_filter_sinogram_noalloc": [_P, _I, _I, _I, _F, _F, _I, _P],
    "fbp2d_project_backward": [_P, _P, _I, _I, C.POINTER(Geometry), _P, _I, _I],
    "fbp2d_parallelize_fan_beam_sinogram": [_P, _P, _I, _I, C.POINTER(Geometry), _P, _I, _F],
    "fbp_fft_rows": [_P, _P, _I, _I, _I],
    "fbp_fft_shift_rows": [_P, _P, _I, _I, _I],
    "fbp_project_ellipsoids_to_projections": [_P, _P, _I, C.POINTER(Geometry)],
    "fbp_kernel_launch_count": [_P, C.POINTER(C.c_uint64)],
    "fbp_measure_smem_bandwidth": [_P, C.POINTER(C.c_double)],
}


class Request(C.Structure):
    """fbp_request (include/fbp_b200.h)."""
    _fields_ = [("kind", C.c_int), ("precision", C.c_int), ("filter_type", C.c_int), ("clip", C.c_int),
                ("geometry", Geometry), ("det_cols", C.c_int), ("det_rows", C.c_int), ("views", C.c_int),
                ("vol_h", C.c_int), ("vol_v", C.c_int), ("reserve_bytes", C.c_longlong),
                ("input", C.c_void_p), ("output", C.c_void_p)]


class JobResult(C.Structure):
    """fbp_job_result (include/fbp_b200.h)."""
    _fields_ = [("status", C.c_int), ("queued_ms", C.c_double), ("started_ms", C.c_double),
                ("finished_ms", C.c_double), ("error", C.c_char * 128)]


class Server:
    """Reconstruction server (fbp_server_*): continuous batching of independent
    jobs on one GPU over `slots` contexts. device < 0: host-only scheduler for
    FBP_JOB_HOST_WAIT jobs. Host arrays passed to submit() must stay alive
    (and should be pinned) until wait() returns."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, slots: int = 3):
        self.lib = library()
        self.handle = C.c_void_p()
        rc = self.lib.fbp_server_create(C.byref(self.handle), int(device), C.c_size_t(hbm_budget_bytes), int(slots))
        if rc != 0:
            raise FBPError(rc, self.lib.fbp_last_error(None).decode())
        self._keep = {}

    def set_batching(self, enable: bool, chunk_updates: float = 0.0) -> None:
        """Cone backprojections through the persistent multi-job backprojector
        (default on), in launches of about chunk_updates voxel-view updates."""
        rc = self.lib.fbp_server_set_batching(self.handle, 1 if enable else 0, float(chunk_updates))
        if rc != 0:
            raise FBPError(rc, "fbp_server_set_batching failed")

    def set_batch_limit(self, max_updates: float) -> None:
        """Cone jobs of at most max_updates voxel-view updates are batched
        (<= 0: 1e10); larger ones run their own slab pipelines."""
        rc = self.lib.fbp_server_set_batch_limit(self.handle, float(max_updates))
        if rc != 0:
            raise FBPError(rc, "fbp_server_set_batch_limit failed")

    def stats(self) -> dict:
        """fbp_server_stats: batched backprojection device time, upload / readback host time."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        d, e = C.c_longlong(), C.c_longlong()
        rc = self.lib.fbp_server_stats(self.handle, C.byref(a), C.byref(b), C.byref(c), C.byref(d), C.byref(e))
        if rc != 0:
            raise FBPError(rc, "fbp_server_stats failed")
        return {"batch_gpu_ms": a.value, "upload_ms": b.value, "readback_ms": c.value,
                "batch_launches": d.value, "batched_jobs": e.value}

    def submit(self, request: Request, keep=None) -> int:
        t = C.c_longlong()
        rc = self.lib.fbp_server_submit(self.handle, C.byref(request), C.byref(t))
        if rc != 0:
            raise FBPError(rc, "fbp_server_submit failed")
        self._keep[t.value] = keep  # the arrays behind input / output
        return t.value

    def wait(self, ticket: int) -> JobResult:
        r = JobResult()
        rc = self.lib.fbp_server_wait(self.handle, int(ticket), C.byref(r))
        if rc == -2:  # FBP_ERR_STATE: the job still runs for the caller already waiting on it
            raise FBPError(rc, "fbp_server_wait: another caller is waiting on this ticket")
        self._keep.pop(ticket, None)
        if rc != 0:
            raise FBPError(rc, "fbp_server_wait: unknown ticket")
        return r

    def close(self) -> None:
        if self.handle:
            self.lib.fbp_server_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def projection_file_index(path: str) -> int:
    """Projection index that read_projections takes from a file name, or -1."""
    return library().fbp_projection_file_index(str(path).encode())


def plan_slabs(geometry: "Geometry", detector_cols: int, detector_rows: int, volume_h: int, volume_v: int,
               slabs: int) -> list[tuple[int, int, int, int]]:
    """fbp_plan_slabs: per slab (y0, y1, row0, row1); host only, no device needed."""
    out = (C.c_int * (4 * slabs))()
    rc = library().fbp_plan_slabs(C.byref(geometry), detector_cols, detector_rows, volume_h, volume_v, slabs, out)
    if rc != 0:
        raise FBPError(rc, "fbp_plan_slabs: invalid arguments")
    return [tuple(out[4 * k:4 * k + 4]) for k in range(slabs)]


def project_backward_cone_fdk_batch(solvers: list, geometries: list, volume_sizes: list, launcher=None) -> None:
    """fbp_project_backward_cone_fdk_batch: each solver's FDK backprojection
    (its pending weights, filter, precision and clip setting), the jobs on the
    symmetric backprojector in one persistent launch on the launcher's stream.
    volume_sizes: (h, v) per job. Asynchronous; each solver's later calls are
    ordered after the batch."""
    n = len(solvers)
    ctxs = (C.c_void_p * n)(*[s.ctx.handle for s in solvers])
    geoms = (Geometry * n)(*geometries)
    hs = (C.c_int * n)(*[int(h) for h, _ in volume_sizes])
    vs = (C.c_int * n)(*[int(v) for _, v in volume_sizes])
    launch = (launcher or solvers[0]).ctx
    launch._check(launch.lib.fbp_project_backward_cone_fdk_batch(ctxs, geoms, hs, vs, n, launch.handle),
                  launch.handle)


def library() -> C.CDLL:
    """Load libfbp_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with "
                f"`python {HERE / 'build.py'}` (nvcc, sm_100a)")
        lib = C.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = C.c_char_p if name == "fbp_last_error" else C.c_int
        _lib = lib
    return _lib


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x):
    """(pointer, on_device) for a numpy array or a torch tensor."""
    if _is_torch(x):
        assert x.is_contiguous(), "tensor must be contiguous"
        assert x.dtype.is_floating_point and x.element_size() == 4, "float32 tensor expected"
        return C.c_void_p(x.data_ptr()), int(x.is_cuda)
    assert isinstance(x, np.ndarray) and x.dtype == np.float32 and x.flags.c_contiguous, \
        "C-contiguous float32 numpy array expected"
    return C.c_void_p(x.ctypes.data), 0


class Context:
    """Owner of one fbp_context (device buffers + stream) on one GPU."""

    def __init__(self, device: int = 0):
        self.lib = library()
        h = C.c_void_p()
        self._check(self.lib.fbp_create(C.byref(h), device), None)
        self.handle = h

    def _check(self, status: int, handle=None) -> None:
        if status != OK:
            msg = self.lib.fbp_last_error(handle if handle is not None else getattr(self, "handle", None))
            raise FBPError(status, (msg or b"").decode())

    def call(self, name: str, *args) -> None:
        self._check(getattr(self.lib, name)(self.handle, *args), self.handle)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.fbp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class FBP3D:
    """Mirror of class FBP3D (FBP3D.h:16-170) on device buffers."""

    def __init__(self, device: int = 0, context: Optional[Context] = None):
        self.ctx = context or Context(device)

    # -- options
    def set_precision(self, precision: int) -> None:
        self.ctx.call("fbp_set_precision", int(precision))

    def set_filter_impl(self, impl: int) -> None:
        self.ctx.call("fbp_set_filter_impl", int(impl))

    def set_filter_padding(self, padded_length: int) -> None:
        self.ctx.call("fbp_set_filter_padding", int(padded_length))

    def set_backprojector(self, variant: int) -> None:
        self.ctx.call("fbp_set_backprojector", int(variant))

    def set_clip_after_backprojection(self, enable: bool) -> None:
        self.ctx.call("fbp_set_clip_after_backprojection", int(bool(enable)))

    def set_stream(self, stream) -> None:
        """stream: a torch.cuda.Stream, an int handle, or None."""
        h = 0 if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        self.ctx.call("fbp_set_stream", C.c_void_p(h))

    def synchronize(self) -> None:
        self.ctx.call("fbp_synchronize")

    def kernel_launch_count(self) -> int:
        c = C.c_uint64()
        self.ctx.call("fbp_kernel_launch_count", C.byref(c))
        return c.value

    def measure_smem_bandwidth(self) -> float:
        """Shared-memory load bandwidth of the device in bytes/s."""
        b = C.c_double()
        self.ctx.call("fbp_measure_smem_bandwidth", C.byref(b))
        return b.value

    def last_backprojection(self) -> dict:
        """Kernel, staged layout and window box of the last backprojection."""
        v, l, bu, bv, ny = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self.ctx.call("fbp_last_backprojection", C.byref(v), C.byref(l), C.byref(bu), C.byref(bv), C.byref(ny))
        names = {0: "rows32", 1: "pairs32", 2: "pairs16", 3: "quads16", 4: "quads24"}
        kernels = {Backprojector.SYMMETRIC: "symmetric", Backprojector.GENERIC_Y8: "generic_y8"}
        return {"kernel": kernels.get(v.value, "generic"),
                "layout": names.get(l.value, str(l.value)), "box": (bu.value, bv.value), "tile_ny": ny.value}

    def set_symmetric_tile(self, voxels_per_thread_y: int) -> None:
        """Voxels per thread along y of the symmetric backprojector (8, 16; 0 = 16)."""
        self.ctx.call("fbp_set_symmetric_tile", int(voxels_per_thread_y))

    def set_autotune_cache(self, path) -> None:
        """File of tuning choices shared between processes (None: none)."""
        self.ctx.call("fbp_set_autotune_cache", None if path is None else str(path).encode())

    def autotune_stats(self) -> tuple[int, int]:
        """(geometries timed, geometries taken from known choices)."""
        a, b = C.c_int(), C.c_int()
        self.ctx.call("fbp_autotune_stats", C.byref(a), C.byref(b))
        return a.value, b.value

    def set_view_ring(self, stages: int) -> None:
        """View ring stages of the generic backprojector (2..8; 0 = as many as fit)."""
        self.ctx.call("fbp_set_view_ring", int(stages))

    def set_autotune(self, enable: bool) -> None:
        """Time the backprojector variants on the first backprojection of each geometry and keep the fastest."""
        self.ctx.call("fbp_set_autotune", 1 if enable else 0)

    # -- forward projection (FBP3D.cpp:212-330)
    def project_forward_cone_to_projections(self, xray_source_distance, detector_panel_distance, detector_width,
                                            volume_width, full_rotation_count, projection_count,
                                            rotation_offset_radian=0.0) -> None:
        self.ctx.call("fbp_project_forward_cone_to_projections", xray_source_distance, detector_panel_distance,
                      detector_width, volume_width, full_rotation_count, int(projection_count),
                      rotation_offset_radian)

    def project_forward_cone_to_sinogram(self, xray_source_distance, detector_panel_distance, detector_width,
                                         volume_width, full_rotation_count, projection_count,
                                         rotation_offset_radian=0.0) -> None:
        self.ctx.call("fbp_project_forward_cone_to_sinograms", xray_source_distance, detector_panel_distance,
                      detector_width, volume_width, full_rotation_count, int(projection_count),
                      rotation_offset_radian)

    def project_forward_parallel_to_projections(self, full_rotation_count, projection_count,
                                                rotation_offset_radian=0.0) -> None:
        self.ctx.call("fbp_project_forward_parallel_to_projections", full_rotation_count, int(projection_count),
                      rotation_offset_radian)

    def project_forward_parallel_to_sinogram(self, full_rotation_count, projection_count,
                                             rotation_offset_radian=0.0) -> None:
        self.ctx.call("fbp_project_forward_parallel_to_sinograms", full_rotation_count, int(projection_count),
                      rotation_offset_radian)

    def reconstruct_fdk_to_host(self, projections, geometry: "Geometry", filter_type: int, volume_h: int,
                                volume_v: int, out=None, slabs: int = 8):
        """fbp_reconstruct_fdk_to_host: host projections [count][rows][cols] in, host
        [z][y][x] volume out; the slab readback overlaps the backprojection."""
        n, rows, cols = projections.shape
        if out is None:
            out = np.empty((volume_h, volume_v, volume_h), np.float32)
        p, pdev = _ptr(projections)
        o, odev = _ptr(out)
        if pdev or odev:
            raise ValueError("reconstruct_fdk_to_host takes host buffers")
        self.ctx.call("fbp_reconstruct_fdk_to_host", p, cols, rows, n, C.byref(geometry), int(filter_type),
                      int(volume_h), int(volume_v), o, int(slabs))
        return out

    def set_detector_rows(self, row_offset: int, total_rows: int) -> None:
        """The stacks hold rows [row_offset, row_offset + v) of a total_rows-row detector (0, 0: whole)."""
        self.ctx.call("fbp_set_detector_rows", int(row_offset), int(total_rows))

    def set_volume_slab(self, y_offset: int, y_count: int) -> None:
        """project_backward_* compute only y-slices [y_offset, y_offset + y_count) (0, 0: whole)."""
        self.ctx.call("fbp_set_volume_slab", int(y_offset), int(y_count))

    def memory_in_use(self) -> int:
        b = C.c_size_t()
        self.ctx.call("fbp_memory_in_use", C.byref(b))
        return b.value

    # -- buffers (FBP3D.cpp:16-56)
    def generate_blank_volume(self, x_size: int, y_size: int, z_size: int) -> None:
        self.ctx.call("fbp_generate_blank_volume", x_size, y_size, z_size)

    def generate_blank_projections(self, x_size: int, y_size: int, projection_amount: int) -> None:
        self.ctx.call("fbp_generate_blank_projections", x_size, y_size, projection_amount)

    def generate_blank_sinograms(self, x_size: int, y_size: int, projection_amount: int) -> None:
        self.ctx.call("fbp_generate_blank_sinograms", x_size, y_size, projection_amount)

    def free_volume(self) -> None:
        self.ctx.call("fbp_free_volume")

    # -- file I/O (FBP3D.cpp:74-195)
    def read_projections(self, upper_directory: str, file_width: int, file_height: int, file_channel_count: int,
                         byte_per_channel: int, target_projection_width: int, target_projection_height: int,
                         projection_count: int) -> None:
        self.ctx.call("fbp_read_projections", str(upper_directory).encode(), file_width, file_height,
                      file_channel_count, byte_per_channel, target_projection_width, target_projection_height,
                      projection_count)

    def read_projections_as_sinograms(self, upper_directory: str, file_width: int, file_height: int,
                                      file_channel_count: int, byte_per_channel: int, target_projection_width: int,
                                      target_projection_height: int, projection_count: int) -> None:
        self.ctx.call("fbp_read_projections_as_sinograms", str(upper_directory).encode(), file_width, file_height,
                      file_channel_count, byte_per_channel, target_projection_width, target_projection_height,
                      projection_count)

    def write_volume(self, upper_directory: str) -> None:
        self.ctx.call("fbp_write_volume", str(upper_directory).encode())

    def free_projections(self) -> None:
        self.ctx.call("fbp_free_projections")

    def free_sinograms(self) -> None:
        self.ctx.call("fbp_free_sinograms")

    def volume_size(self) -> tuple[int, int, int]:
        x, y, z = C.c_int(), C.c_int(), C.c_int()
        self.ctx.call("fbp_get_volume_size", C.byref(x), C.byref(y), C.byref(z))
        return x.value, y.value, z.value

    def projections_size(self) -> tuple[int, int, int]:
        u, v, n = C.c_int(), C.c_int(), C.c_int()
        self.ctx.call("fbp_get_projections_size", C.byref(u), C.byref(v), C.byref(n))
        return u.value, v.value, n.value

    def sinograms_size(self) -> tuple[int, int, int]:
        """(detector columns, detector rows, views) of the sinogram stack."""
        u, v, n = C.c_int(), C.c_int(), C.c_int()
        self.ctx.call("fbp_get_sinograms_size", C.byref(u), C.byref(v), C.byref(n))
        return u.value, v.value, n.value

    # -- transfers
    def upload_projections(self, projections) -> None:
        """[count][v][u] float32 array / tensor (replaces read_projections' upload)."""
        n, v, u = projections.shape
        p, dev = _ptr(projections)
        self.ctx.call("fbp_upload_projections", p, u, v, n, dev)

    def upload_sinograms(self, sinograms) -> None:
        """[v][count][u] float32 array / tensor."""
        v, n, u = sinograms.shape
        p, dev = _ptr(sinograms)
        self.ctx.call("fbp_upload_sinograms", p, u, v, n, dev)

    def download_projections(self, out=None):
        u, v, n = self.projections_size()
        out = np.empty((n, v, u), np.float32) if out is None else out
        p, dev = _ptr(out)
        self.ctx.call("fbp_download_projections", p, dev)
        return out

    def download_sinograms(self, out):
        p, dev = _ptr(out)
        self.ctx.call("fbp_download_sinograms", p, dev)
        return out

    def store_projection(self, source, projection_index: int) -> None:
        p, dev = _ptr(source)
        self.ctx.call("fbp_store_projection", p, projection_index, dev)

    def load_projection(self, projection_index: int, target=None):
        u, v, _ = self.projections_size()
        target = np.empty((v, u), np.float32) if target is None else target
        p, dev = _ptr(target)
        self.ctx.call("fbp_load_projection", projection_index, p, dev)
        return target

    def store_sinogram(self, source, y_index: int) -> None:
        p, dev = _ptr(source)
        self.ctx.call("fbp_store_sinogram", p, y_index, dev)

    def load_sinogram(self, y_index: int, target):
        p, dev = _ptr(target)
        self.ctx.call("fbp_load_sinogram", y_index, p, dev)
        return target

    def load_projection_from_sinograms(self, projection_index: int, target=None):
        """FBP3D::load_projection_from_sinograms (FBP3D.cpp:755-765): view
        projection_index of the sinogram stack as a [v][u] projection."""
        u, v, _ = self.sinograms_size()
        target = np.empty((v, u), np.float32) if target is None else target
        p, dev = _ptr(target)
        self.ctx.call("fbp_load_projection_from_sinograms", projection_index, p, dev)
        return target

    def store_projection_to_sinograms(self, source, projection_index: int) -> None:
        """FBP3D::store_projection_to_sinograms (FBP3D.cpp:767-778): a [v][u]
        projection into view projection_index of the sinogram stack."""
        p, dev = _ptr(source)
        self.ctx.call("fbp_store_projection_to_sinograms", p, projection_index, dev)

    def _slice(self, axis: str, index: int, target, load: bool):
        x, y, z = self.volume_size()
        shape = {"x": (z, y), "y": (z, x), "z": (y, x)}[axis]
        if target is None:
            target = np.empty(shape, np.float32)
        p, dev = _ptr(target)
        if load:
            self.ctx.call(f"fbp_load_volume_slice_{axis}", index, p, dev)
        else:
            self.ctx.call(f"fbp_store_volume_slice_{axis}", p, index, dev)
        return target

    def load_volume_slice_x(self, x_index: int, target=None):
        return self._slice("x", x_index, target, True)

    def load_volume_slice_y(self, y_index: int, target=None):
        return self._slice("y", y_index, target, True)

    def load_volume_slice_z(self, z_index: int, target=None):
        return self._slice("z", z_index, target, True)

    def store_volume_slice_x(self, source, x_index: int) -> None:
        self._slice("x", x_index, source, False)

    def store_volume_slice_y(self, source, y_index: int) -> None:
        self._slice("y", y_index, source, False)

    def store_volume_slice_z(self, source, z_index: int) -> None:
        self._slice("z", z_index, source, False)

    def read_volume(self, out=None):
        """Whole volume [z][y][x]."""
        x, y, z = self.volume_size()
        out = np.empty((z, y, x), np.float32) if out is None else out
        p, dev = _ptr(out)
        self.ctx.call("fbp_read_volume", p, dev)
        return out

    def write_volume_data(self, data) -> None:
        p, dev = _ptr(data)
        self.ctx.call("fbp_write_volume_data", p, dev)

    def volume_device_ptr(self) -> int:
        ptr = C.c_void_p()
        self.ctx.call("fbp_volume_device_ptr", C.byref(ptr))
        return ptr.value or 0

    def projections_device_ptr(self) -> tuple[int, int]:
        ptr, pitch = C.c_void_p(), C.c_int()
        self.ctx.call("fbp_projections_device_ptr", C.byref(ptr), C.byref(pitch))
        return ptr.value or 0, pitch.value

    # -- pipeline (FBP3D.cpp:333-593)
    def log_normalize_projections(self, base_value: float) -> None:
        self.ctx.call("fbp_log_normalize_projections", base_value)

    def log_normalize_sinograms(self, base_value: float) -> None:
        self.ctx.call("fbp_log_normalize_sinograms", base_value)

    def apply_fdk_weights_to_projections(self, xray_source_distance, detector_panel_distance, detector_width):
        self.ctx.call("fbp_apply_fdk_weights_to_projections", xray_source_distance, detector_panel_distance,
                      detector_width)

    def apply_fdk_weights_to_sinograms(self, xray_source_distance, detector_panel_distance, detector_width):
        self.ctx.call("fbp_apply_fdk_weights_to_sinograms", xray_source_distance, detector_panel_distance,
                      detector_width)

    def apply_filter_to_projections(self, filter_type: int) -> None:
        self.ctx.call("fbp_apply_filter_to_projections", int(filter_type))

    def apply_filter_to_sinograms(self, filter_type: int) -> None:
        self.ctx.call("fbp_apply_filter_to_sinograms", int(filter_type))

    def clip_negatives_of_volume(self) -> None:
        self.ctx.call("fbp_clip_negatives_of_volume")

    def volume_min_max(self) -> tuple[float, float]:
        """compute_min_value_of_volume / compute_max_value_of_volume (FBP3D.cpp:780-800)."""
        lo, hi = C.c_float(), C.c_float()
        self.ctx.call("fbp_volume_min_max", C.byref(lo), C.byref(hi))
        return lo.value, hi.value

    def normalize_histogram(self, min_value=None, max_value=None) -> None:
        """FBP3D::normalize_histogram (FBP3D.cpp:802-826): the volume's own range, or a given one."""
        if min_value is None:
            self.ctx.call("fbp_normalize_histogram")
        else:
            self.ctx.call("fbp_normalize_histogram_range", float(min_value), float(max_value))

    def project_backward_cone_fdk_from_projections(self, xray_source_distance, detector_panel_distance,
                                                   detector_width, volume_width, full_rotation_count,
                                                   volume_resolution_horizontal, volume_resolution_vertical,
                                                   rotation_offset_radian=0.0):
        self.ctx.call("fbp_project_backward_cone_fdk_from_projections", xray_source_distance,
                      detector_panel_distance, detector_width, volume_width, full_rotation_count,
                      volume_resolution_horizontal, volume_resolution_vertical, rotation_offset_radian)

    def project_backward_cone_fdk_from_sinograms(self, xray_source_distance, detector_panel_distance,
                                                 detector_width, volume_width, full_rotation_count,
                                                 volume_resolution_horizontal, volume_resolution_vertical,
                                                 rotation_offset_radian=0.0):
        self.ctx.call("fbp_project_backward_cone_fdk_from_sinograms", xray_source_distance,
                      detector_panel_distance, detector_width, volume_width, full_rotation_count,
                      volume_resolution_horizontal, volume_resolution_vertical, rotation_offset_radian)

    def project_backward_parallel_from_projections(self, full_rotation_count, volume_resolution_horizontal,
                                                   volume_resolution_vertical, rotation_offset_radian=0.0):
        self.ctx.call("fbp_project_backward_parallel_from_projections", full_rotation_count,
                      volume_resolution_horizontal, volume_resolution_vertical, rotation_offset_radian)

    def project_backward_parallel_from_sinograms(self, full_rotation_count, volume_resolution_horizontal,
                                                 volume_resolution_vertical, rotation_offset_radian=0.0):
        self.ctx.call("fbp_project_backward_parallel_from_sinograms", full_rotation_count,
                      volume_resolution_horizontal, volume_resolution_vertical, rotation_offset_radian)

    def reconstruct_fdk(self, geometry: Geometry, filter_type: int, volume_resolution_horizontal: int,
                        volume_resolution_vertical: int) -> None:
        self.ctx.call("fbp_reconstruct_fdk", C.byref(geometry), int(filter_type),
                      volume_resolution_horizontal, volume_resolution_vertical)

    # -- phantom input generation
    def project_ellipsoids(self, ellipsoids: np.ndarray, geometry: Geometry) -> None:
        e = np.ascontiguousarray(ellipsoids, dtype=np.float64).reshape(-1, 16)
        self.ctx.call("fbp_project_ellipsoids_to_projections", C.c_void_p(e.ctypes.data), len(e),
                      C.byref(geometry))


class FBP2D:
    """Mirror of class FBP2D (FBP2D.h:8-72) on torch CUDA tensors.

    sinograms are [views][bins], images [rows][cols]; numpy inputs are
    copied to the device and results returned as numpy."""

    FilterType = FilterType

    def __init__(self, device: int = 0, context: Optional[Context] = None):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)
        self.ctx = context or Context(device)

    def set_precision(self, precision: int) -> None:
        """Precision form of apply_filter: FP32 (FFT) or MIXED / MIXED24
        (tcgen05 split-BF16 Toeplitz product)."""
        self.ctx.call("fbp_set_precision", int(precision))

    def set_filter_impl(self, impl: int) -> None:
        self.ctx.call("fbp_set_filter_impl", int(impl))

    def _dev(self, x):
        if _is_torch(x) and x.is_cuda:
            return x.contiguous(), False
        return self.torch.as_tensor(np.ascontiguousarray(x, np.float32), device=self.device), True

    def apply_filter(self, sinogram, filter_type: int = FilterType.RAM_LAK, fan_sdd: float = 0.0,
                     detector_width: float = 0.0):
        """Weight (fan beam when fan_sdd > 0) and filter every row in place;
        combines FBP2D::apply_filter (FBP2D.cpp:124-144) with the FFT calls
        around it. Returns the filtered sinogram."""
        d, copied = self._dev(sinogram)
        views, bins = d.shape
        self.ctx.call("fbp2d_filter_sinogram", C.c_void_p(d.data_ptr()), bins, views, int(filter_type),
                      float(fan_sdd), float(detector_width))
        return self._ret(d, copied)

    def project_backward(self, sinogram, geometry: Geometry, image_size: tuple[int, int], out=None):
        """2D backprojection (FBP2D.cpp:96-122); image_size = (cols, rows)."""
        d, copied = self._dev(sinogram)
        views, bins = d.shape
        nx, nz = image_size
        img = out if out is not None else self.torch.empty((nz, nx), dtype=self.torch.float32, device=self.device)
        self.ctx.call("fbp2d_project_backward", C.c_void_p(d.data_ptr()), bins, views, C.byref(geometry),
                      C.c_void_p(img.data_ptr()), nx, nz)
        return self._ret(img, copied)

    def project_forward(self, image, geometry: Geometry, bins: int, views: int, out=None):
        """FBP2D::project_forward (FBP2D.cpp:54-94): ray-driven sinogram [views][bins]
        of image [rows][cols] (parallel beam, or flat-detector fan for a cone geometry)."""
        d, copied = self._dev(image)
        nz, nx = d.shape
        sino = out if out is not None else self.torch.empty((views, bins), dtype=self.torch.float32,
                                                            device=self.device)
        self.ctx.call("fbp2d_project_forward", C.c_void_p(d.data_ptr()), nx, nz, C.c_void_p(sino.data_ptr()), bins,
                      views, C.byref(geometry))
        return self._ret(sino, copied)

    def parallelize_fan_beam_sinogram(self, source_sinogram, geometry: Geometry, out_bins: int,
                                      out_detector_width: float):
        d, copied = self._dev(source_sinogram)
        views, bins = d.shape
        out = self.torch.empty((views, out_bins), dtype=self.torch.float32, device=self.device)
        self.ctx.call("fbp2d_parallelize_fan_beam_sinogram", C.c_void_p(d.data_ptr()), bins, views,
                      C.byref(geometry), C.c_void_p(out.data_ptr()), out_bins, float(out_detector_width))
        return self._ret(out, copied)

    def _ret(self, t, to_host: bool):
        self.ctx.call("fbp_synchronize")
        return t.cpu().numpy() if to_host else t


class FFFT:
    """Mirror of class FFFT (FastFourierTransformGPU.h:10-67) on complex rows."""

    def __init__(self, device: int = 0, context: Optional[Context] = None):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)
        self.ctx = context or Context(device)

    def _run(self, x, name, *args):
        t = self.torch.as_tensor(np.ascontiguousarray(x, np.complex64), device=self.device) \
            if not _is_torch(x) else x.contiguous()
        rows, n = t.shape
        fr = self.torch.view_as_real(t)
        self.ctx.call(name, C.c_void_p(fr.data_ptr()), n, rows, *args)
        self.ctx.call("fbp_synchronize")
        return t if _is_torch(x) else t.cpu().numpy()

    def fft_radix2(self, complex_rows):
        return self._run(complex_rows, "fbp_fft_rows", 0)

    def inverse_fft_radix2(self, complex_rows):
        return self._run(complex_rows, "fbp_fft_rows", 1)

    def fft_shift(self, complex_rows, shift_amount: Optional[int] = None):
        n = complex_rows.shape[-1]
        return self._run(complex_rows, "fbp_fft_shift_rows", n // 2 if shift_amount is None else shift_amount)

    def inverse_fft_shift(self, complex_rows, shift_amount: Optional[int] = None):
        n = complex_rows.shape[-1]
        return self._run(complex_rows, "fbp_fft_shift_rows", -(n // 2 if shift_amount is None else shift_amount))


def padded_length(width: int) -> int:
    """The reference's padded row length: next power of two >= width
    (FastFourierTransformGPU.cpp:258-262, 269-280)."""
    return 1 << int(math.floor(math.log2(2 * width - 1)))
