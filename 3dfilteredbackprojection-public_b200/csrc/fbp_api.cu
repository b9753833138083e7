// C ABI of libfbp_b200: context, device buffers, transfers and the pipeline
// stages of class FBP3D / FBP2D (Source/FilteredBackProjection/FBP3D.h:16-170,
// FBP2D.h:8-72 in the reference). Every entry point returns a status code and
// records a message instead of the reference's `std::cout` + ASSERT(false).

#include "fbp_internal.h"

#include <cstdio>
#include <cstdlib>

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using fbp::Stack;

namespace {

thread_local std::string g_thread_error;
constexpr double kPi = 3.14159265358979323846;

int round_up(int x, int m) { return (x + m - 1) / m * m; }

int next_pow2_reference(int m) {
  // 1 << ceil_log2(m), ceil_log2(m) = floor_log2(2m - 1)
  // (FastFourierTransformGPU.cpp:258-262, 269-280)
  int l = 0;
  for (long t = 2L * m - 1; t > 1; t >>= 1) l++;
  return 1 << l;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

#define FBP_CTX(ctx)                                                                   \
  if (!(ctx)) {                                                                        \
    g_thread_error = "null context";                                                  \
    return FBP_ERR_INVALID_ARGUMENT;                                                   \
  }                                                                                    \
  DeviceGuard device_guard_((ctx)->device)

#define FBP_TRY(expr)          \
  do {                         \
    int rc_ = (expr);          \
    if (rc_ != FBP_OK) return rc_; \
  } while (0)

// Rows of `width` bytes between pitched buffers: one linear copy when both
// pitches equal the width (the rows are one contiguous block), else a 2D copy.
cudaError_t copy_rows(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t rows,
                      cudaMemcpyKind kind, cudaStream_t stream) {
  if (dpitch == width && spitch == width) return cudaMemcpyAsync(dst, src, width * rows, kind, stream);
  return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, stream);
}

cudaMemcpyKind kind_of(bool src_dev, bool dst_dev) {
  if (src_dev && dst_dev) return cudaMemcpyDeviceToDevice;
  if (src_dev) return cudaMemcpyDeviceToHost;
  if (dst_dev) return cudaMemcpyHostToDevice;
  return cudaMemcpyHostToHost;
}

// Device error word -> status (and reset).
int check_device_error(fbp_context* ctx) {
  int h = 0;
  FBP_TRY(fbp::cuda_check(ctx, cudaMemcpyAsync(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream),
                          "error word readback"));
  FBP_TRY(fbp::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"));
  if (h == fbp::kDevOk) return FBP_OK;
  cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  switch (h) {
    case fbp::kDevTimeout:
      return fbp::set_error(ctx, FBP_ERR_DEVICE_TIMEOUT, "a bounded device-side wait expired");
    case fbp::kDevFootprint:
      return fbp::set_error(ctx, FBP_ERR_DEVICE_CHECK, "detector footprint exceeded the staged window");
    case fbp::kDevGeometry:
      return fbp::set_error(ctx, FBP_ERR_DEVICE_CHECK,
                            "a voxel lies at or behind the source plane (source distance too small)");
    default:
      return fbp::set_error(ctx, FBP_ERR_DEVICE_CHECK, "device check failed");
  }
}

int sync_host(fbp_context* ctx, bool host_involved) {
  if (!host_involved) return FBP_OK;
  FBP_TRY(fbp::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"));
  return check_device_error(ctx);
}

void free_stack(Stack& s) {
  cudaFree(s.f32);
  cudaFree(s.filt);
  cudaFree(s.inv_scale);
  bool sino = s.sinogram;
  s = Stack();
  s.sinogram = sino;
}

// Size the stack for u x v x n (clearing it, as generate_blank_* do,
// FBP3D.cpp:30-56). The allocation only grows: a smaller stack reuses it, so
// a context serving jobs of varying size stops allocating (and cudaFree's
// device-wide synchronisation) once it has seen its largest job.
int alloc_stack(fbp_context* ctx, Stack& s, int u, int v, int n, bool clear = true) {
  if (u <= 0 || v <= 0 || n <= 0) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "stack sizes must be positive");
  const int pitch = round_up(u, 4);
  const size_t need = (size_t)pitch * v * n * sizeof(float);
  if (!s.f32 || s.f32_cap < need) {
    cudaFree(s.f32);
    s.f32 = nullptr;
    s.f32_cap = 0;
    if (cudaMalloc(&s.f32, need) != cudaSuccess) {
      s.f32 = nullptr;
      cudaGetLastError();
      return fbp::set_error(ctx, FBP_ERR_OUT_OF_MEMORY, "cudaMalloc of the detector stack failed");
    }
    s.f32_cap = need;
  }
  s.u = u;
  s.v = v;
  s.n = n;
  s.pitch = pitch;
  s.filtered = false;
  s.log_pending = s.weights_pending = false;
  if (!clear) return FBP_OK;
  return fbp::cuda_check(ctx, cudaMemsetAsync(s.f32, 0, s.bytes32(), ctx->stream), "clear stack");
}

fbp::RowSet rowset_of(Stack& s) {
  fbp::RowSet rs{};
  rs.data = s.f32;
  rs.pitch = s.pitch;
  rs.rows = (long long)s.rows();
  rs.m = s.u;
  rs.n_views = s.n;
  rs.n_v = s.v;
  rs.sinogram = s.sinogram;
  rs.log_norm = s.log_pending;
  rs.log_base = (float)s.log_base;
  rs.weight = s.weights_pending;
  rs.w_sdd = (float)s.w_sdd;
  rs.w_du = (float)s.w_du;
  rs.w_dv = (float)s.w_dv;
  rs.w_voff = (float)s.w_voff;
  return rs;
}

// Apply any pending log / weight to the f32 rows in place.
int flush_pending(fbp_context* ctx, Stack& s) {
  if (!s.log_pending && !s.weights_pending) return FBP_OK;
  FBP_TRY(fbp::launch_elementwise_pre(ctx, rowset_of(s)));
  s.log_pending = s.weights_pending = false;
  return FBP_OK;
}

// Bring the content back into the f32 rows (from the filtered buffer) and
// apply anything pending.
int materialize_f32(fbp_context* ctx, Stack& s) {
  if (s.filtered) {
    FBP_TRY(fbp::launch_unpack_rows(ctx, s, 0, s.rows(), s.f32, s.pitch));
    s.filtered = false;
  }
  return flush_pending(ctx, s);
}

int require_stack(fbp_context* ctx, const Stack& s, const char* what) {
  if (!s.f32) return fbp::set_error(ctx, FBP_ERR_STATE, std::string(what) + " but the buffer is not allocated");
  return FBP_OK;
}

int ensure_volume(fbp_context* ctx, int x, int y, int z, bool clear) {
  ctx->minmax_valid = false;
  if (x <= 0 || y <= 0 || z <= 0) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "volume sizes must be positive");
  const size_t need = sizeof(float) * (size_t)x * y * z;
  if (!(ctx->vol && ctx->vx == x && ctx->vy == y && ctx->vz == z)) {
    if (!ctx->vol || ctx->vol_cap < need) {  // grow only, like the stacks
      cudaFree(ctx->vol);
      ctx->vol = nullptr;
      ctx->vol_cap = 0;
      if (cudaMalloc(&ctx->vol, need) != cudaSuccess) {
        ctx->vol = nullptr;
        ctx->vx = ctx->vy = ctx->vz = 0;
        cudaGetLastError();
        return fbp::set_error(ctx, FBP_ERR_OUT_OF_MEMORY, "cudaMalloc of the volume failed");
      }
      ctx->vol_cap = need;
    }
    ctx->vx = x;
    ctx->vy = y;
    ctx->vz = z;
    clear = true;
  }
  if (clear) return fbp::cuda_check(ctx, cudaMemsetAsync(ctx->vol, 0, need, ctx->stream), "clear volume");
  return FBP_OK;
}

int upload_stack(fbp_context* ctx, Stack& s, const float* src, int u, int v, int n, int on_dev) {
  if (!src) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null source pointer");
  if (!(s.f32 && s.u == u && s.v == v && s.n == n)) FBP_TRY(alloc_stack(ctx, s, u, v, n, false));
  s.filtered = false;
  s.log_pending = s.weights_pending = false;
  FBP_TRY(fbp::cuda_check(ctx,
                          copy_rows(s.f32, (size_t)s.pitch * 4, src, (size_t)u * 4, (size_t)u * 4,
                                            s.rows(), kind_of(on_dev, true), ctx->stream),
                          "stack upload"));
  return sync_host(ctx, !on_dev);
}

// Rows row0, row0 + row_step, ... (nrows of them) to dst, packed [nrows][u].
// row_step 1 is a contiguous band; row_step = views picks one view's rows
// out of a sinogram stack [v][view][u].
int download_rows(fbp_context* ctx, Stack& s, size_t row0, size_t nrows, float* dst, int on_dev, size_t row_step = 1) {
  if (!dst) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null destination pointer");
  FBP_TRY(flush_pending(ctx, s));
  if (s.filtered) {
    // unpack just these rows into a scratch f32 block
    float* tmp = static_cast<float*>(fbp::scratch(ctx, sizeof(float) * nrows * s.pitch));
    if (!tmp) return FBP_ERR_OUT_OF_MEMORY;
    FBP_TRY(fbp::launch_unpack_rows(ctx, s, row0, nrows, tmp, s.pitch, (long long)row_step));
    FBP_TRY(fbp::cuda_check(ctx,
                            copy_rows(dst, (size_t)s.u * 4, tmp, (size_t)s.pitch * 4, (size_t)s.u * 4, nrows,
                                              kind_of(true, on_dev), ctx->stream),
                            "row download"));
  } else {
    FBP_TRY(fbp::cuda_check(ctx,
                            copy_rows(dst, (size_t)s.u * 4, s.f32 + row0 * s.pitch, (size_t)s.pitch * 4 * row_step,
                                              (size_t)s.u * 4, nrows, kind_of(true, on_dev), ctx->stream),
                            "row download"));
  }
  return sync_host(ctx, !on_dev);
}

// Rows row0, row0 + row_step, ... (nrows of them) from src, packed [nrows][u].
int upload_rows(fbp_context* ctx, Stack& s, size_t row0, size_t nrows, const float* src, int on_dev,
                size_t row_step = 1) {
  if (!src) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null source pointer");
  FBP_TRY(materialize_f32(ctx, s));
  FBP_TRY(fbp::cuda_check(ctx,
                          copy_rows(s.f32 + row0 * s.pitch, (size_t)s.pitch * 4 * row_step, src,
                                            (size_t)s.u * 4, (size_t)s.u * 4, nrows, kind_of(on_dev, true),
                                            ctx->stream),
                          "row upload"));
  return sync_host(ctx, !on_dev);
}

// Run weights / log (pending) + filter on a stack; the result goes to the
// stack's filtered buffer in the backprojector's pair layout (FP32 pairs for
// the FP32 form, FP16 pairs with a per-view scale for the MIXED form).
int filter_stack(fbp_context* ctx, Stack& s, int filter_type) {
  if (filter_type < 0 || filter_type > FBP_FILTER_RAMP_SAMPLED)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "unknown filter type");
  if (s.filtered) FBP_TRY(materialize_f32(ctx, s));  // filtering filtered data
  const int n = ctx->pad_len > 0 ? ctx->pad_len : next_pow2_reference(s.u);
  if (n < s.u || (n & (n - 1)))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "padded length must be a power of two >= the row width");
  FBP_TRY(fbp::ensure_filter_tables(ctx, n, filter_type));
  const bool mixed = ctx->precision != FBP_PRECISION_FP32;
  int impl = ctx->filter_impl;
  if (impl == FBP_FILTER_IMPL_AUTO)
    impl = (mixed && fbp::toeplitz_supported(s.u)) ? FBP_FILTER_IMPL_TOEPLITZ : FBP_FILTER_IMPL_FFT;
  fbp::RowSet rs = rowset_of(s);
  if (!mixed) {
    // FP32 form: straight into the backprojector's float2 pair layout
    const int layout = fbp::kLayoutPair32;
    const int fpitch = round_up(s.u, 4);
    const size_t need = (size_t)fpitch * s.filt_rows() * Stack::elem_bytes(layout);
    if (!s.filt || s.filt_bytes < need) {
      cudaFree(s.filt);
      s.filt = nullptr;
      s.filt_bytes = 0;
      if (fbp::cuda_check(ctx, cudaMalloc(&s.filt, need), "cudaMalloc(filtered views)")) return FBP_ERR_OUT_OF_MEMORY;
      s.filt_bytes = need;
    }
    s.filt_layout = layout;
    s.filt_pitch = fpitch;
    rs.out = s.filt;
    rs.out_layout = layout;
    rs.out_pitch = fpitch;
  }
  // MIXED form: FP32 rows in place; the backprojector packs them to FP16
  // with per-view scales in the layout of the kernel it selects
  if (impl == FBP_FILTER_IMPL_TOEPLITZ)
    FBP_TRY(fbp::launch_filter_toeplitz(ctx, rs, n, filter_type));
  else
    FBP_TRY(fbp::launch_filter_fft(ctx, rs, n));
  s.log_pending = s.weights_pending = false;
  s.filtered = !mixed;
  return FBP_OK;
}

int record_weights(fbp_context* ctx, Stack& s, float sod, float odd, float det_w, const char* what) {
  FBP_TRY(require_stack(ctx, s, what));
  if (!(sod > 0.f) || !(odd >= 0.f) || !(det_w > 0.f))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "distances and detector width must be positive");
  if (s.filtered) FBP_TRY(materialize_f32(ctx, s));
  if (s.weights_pending) FBP_TRY(flush_pending(ctx, s));
  s.weights_pending = true;
  s.w_sdd = (double)sod + (double)odd;
  s.w_du = (double)det_w / s.u;
  s.w_dv = s.w_du;  // square detector pixels
  // a row band of a taller detector: the weight needs the global row index
  s.w_voff = ctx->det_rows_total > 0 ? ctx->det_row_off + 0.5 * ((double)s.v - ctx->det_rows_total) : 0.0;
  return FBP_OK;
}

int record_log(fbp_context* ctx, Stack& s, float base, const char* what) {
  FBP_TRY(require_stack(ctx, s, what));
  if (!(base > 0.f)) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "base_value must be positive");
  if (s.filtered) FBP_TRY(materialize_f32(ctx, s));
  // log must run before weights; if weights are already pending (or a log
  // is), materialise them first so that the call order is honoured
  if (s.weights_pending || s.log_pending) FBP_TRY(flush_pending(ctx, s));
  s.log_pending = true;
  s.log_base = base;
  return FBP_OK;
}

fbp::BPGeom cone_geom(const Stack& s, float sod, float odd, float det_w, float vol_w, float rot, int h, int v,
                      float offset) {
  fbp::BPGeom g{};
  g.kind = FBP_GEOMETRY_CONE;
  g.sod = sod;
  g.sdd = (double)sod + (double)odd;
  g.du = (double)det_w / s.u;
  g.dv = g.du;
  g.vox = (double)vol_w / h;
  g.span = 2.0 * kPi * (double)rot;
  g.offset = offset;
  g.nu = s.u;
  g.nv = s.v;
  g.nviews = s.n;
  g.nx = h;
  g.ny = v;
  g.nz = h;
  return g;
}

// Autotuner: the first backprojection of a geometry (with autotuning on) times
// each applicable shape - the four-fold symmetric kernel with 16 voxels per
// thread along y (one CTA per SM) or 8 (two CTAs per SM), the generic kernel
// with 16 or 8 voxels per thread, each with its full view ring or a 4-stage
// one - on a central slab of up to 48 y-slices (written into the volume,
// which the real launch then overwrites) and keeps the fastest for that
// geometry, form, stack layout and GPU. With a cache file set, choices are
// read from it and new ones appended, so other processes skip the timing.
using TuneShape = fbp_context::TuneShape;

void tune_key(const fbp_context* ctx, const Stack& s, const fbp::BPGeom& g, double* key) {
  const double k[fbp_context::kTuneKey] = {
      (double)g.kind, g.sod, g.sdd, g.du, g.dv, g.vox, g.span, g.offset, (double)g.nu, (double)g.nv,
      (double)g.nviews, (double)g.nx, (double)g.ny, (double)g.nz, (double)ctx->precision,
      (double)(s.filtered ? s.filt_layout : -1), (double)g.row_off, (double)g.nv_total, (double)g.y_off,
      (double)g.ny_total, (double)s.sinogram, (double)ctx->num_sms, (double)ctx->device_cc};
  std::copy(k, k + fbp_context::kTuneKey, key);
}

void apply_shape(fbp_context* ctx, const TuneShape& t) {
  ctx->bp_variant = t.variant;
  ctx->quad_tile_ny = t.quad_ny;
  ctx->bp_stages = t.stages;
}

// "key... | variant quad_ny stages ms" per line
void load_tune_cache(fbp_context* ctx) {
  ctx->tune_cache_loaded = true;
  FILE* f = std::fopen(ctx->tune_cache.c_str(), "r");
  if (!f) return;
  char line[2048];
  while (std::fgets(line, sizeof line, f)) {
    fbp_context::TuneEntry t;
    char* p = line;
    bool ok = true;
    for (int i = 0; i < fbp_context::kTuneKey && ok; ++i) {
      char* end = nullptr;
      t.key[i] = std::strtod(p, &end);
      ok = end != p;
      p = end;
    }
    if (!ok || std::sscanf(p, " | %d %d %d %f", &t.shape.variant, &t.shape.quad_ny, &t.shape.stages, &t.ms) != 4)
      continue;
    ctx->tuned.push_back(t);
  }
  std::fclose(f);
}

void store_tune_cache(const fbp_context* ctx, const fbp_context::TuneEntry& t) {
  std::string line;
  char buf[64];
  for (int i = 0; i < fbp_context::kTuneKey; ++i) {
    std::snprintf(buf, sizeof buf, "%.17g ", t.key[i]);
    line += buf;
  }
  std::snprintf(buf, sizeof buf, "| %d %d %d %.4f\n", t.shape.variant, t.shape.quad_ny, t.shape.stages, t.ms);
  line += buf;
  // one short write in append mode: lines of concurrent processes do not interleave
  if (FILE* f = std::fopen(ctx->tune_cache.c_str(), "a")) {
    std::fwrite(line.data(), 1, line.size(), f);
    std::fclose(f);
  }
}

int autotune_backprojector(fbp_context* ctx, Stack& s, const fbp::BPGeom& g, bool mixed, TuneShape* best_shape) {
  double key[fbp_context::kTuneKey];
  tune_key(ctx, s, g, key);
  if (!ctx->tune_cache.empty() && !ctx->tune_cache_loaded) load_tune_cache(ctx);
  for (const auto& t : ctx->tuned)
    if (std::equal(key, key + fbp_context::kTuneKey, t.key)) {
      *best_shape = t.shape;
      ++ctx->tune_cached;
      return FBP_OK;
    }
  const int nt = std::min(g.ny, 48), y0 = (g.ny - nt) / 2;
  fbp::BPGeom gt = g;
  gt.ny_total = g.ny_total > 0 ? g.ny_total : g.ny;
  gt.y_off = g.y_off + y0;
  gt.ny = nt;
  gt.vol_ystride = g.vol_ystride > 0 ? g.vol_ystride : g.ny;
  const TuneShape cand[6] = {{FBP_BACKPROJECTOR_SYMMETRIC, 16, 0}, {FBP_BACKPROJECTOR_SYMMETRIC, 8, 0},
                             {FBP_BACKPROJECTOR_GENERIC, 0, 0},    {FBP_BACKPROJECTOR_GENERIC, 0, 4},
                             {FBP_BACKPROJECTOR_GENERIC_Y8, 0, 0}, {FBP_BACKPROJECTOR_GENERIC_Y8, 0, 4}};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FBP_TRY(fbp::cuda_check(ctx, cudaEventCreate(&e0), "event"));
  FBP_TRY(fbp::cuda_check(ctx, cudaEventCreate(&e1), "event"));
  const TuneShape saved{ctx->bp_variant, ctx->quad_tile_ny, ctx->bp_stages};
  float best = 1e30f;
  int rc = FBP_OK;
  *best_shape = TuneShape{FBP_BACKPROJECTOR_GENERIC, 0, 0};
  for (const TuneShape& c : cand) {
    apply_shape(ctx, c);
    int r = fbp::launch_backproject(ctx, gt, s, ctx->vol + (size_t)y0 * g.nx, 0, mixed);  // plan, pack: untimed
    if (r == FBP_ERR_UNSUPPORTED) continue;  // geometry not symmetric, windows too large, ...
    if (r) {
      rc = r;
      break;
    }
    s.pack_ready = mixed && !s.filtered;  // the timed launch reuses the packed views
    cudaEventRecord(e0, ctx->stream);
    r = fbp::launch_backproject(ctx, gt, s, ctx->vol + (size_t)y0 * g.nx, 0, mixed);
    cudaEventRecord(e1, ctx->stream);
    if (r || (r = sync_host(ctx, true))) {
      rc = r;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) {
      best = ms;
      *best_shape = c;
    }
  }
  apply_shape(ctx, saved);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  ++ctx->tune_timed;
  fbp_context::TuneEntry t;
  std::copy(key, key + fbp_context::kTuneKey, t.key);
  t.shape = *best_shape;
  t.ms = best;
  ctx->tuned.push_back(t);
  if (!ctx->tune_cache.empty()) store_tune_cache(ctx, t);
  return FBP_OK;
}

// Checks, sharding offsets, pending row operations and the volume buffer of
// a backprojection; *ylim = clip extent, *mixed = reduced-precision form.
int setup_backproject(fbp_context* ctx, Stack& s, fbp::BPGeom& g, int* ylim, bool* mixed) {
  if (g.nx <= 0 || g.ny <= 0 || g.nz <= 0)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "volume resolution must be positive");
  // sharding: detector row band and volume y-slab set on the context
  if (ctx->det_rows_total > 0) {
    if (ctx->det_row_off + s.v > ctx->det_rows_total)
      return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "detector row band exceeds the detector");
    g.row_off = ctx->det_row_off;
    g.nv_total = ctx->det_rows_total;
  }
  int clip_limit = g.nz;  // the reference clips y-slices below z_size (FBP3D.cpp:448)
  if (ctx->slab_ny > 0) {
    if (ctx->slab_y0 + ctx->slab_ny > g.ny)
      return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "volume slab exceeds the volume");
    g.ny_total = g.ny;
    g.y_off = ctx->slab_y0;
    g.ny = ctx->slab_ny;
    clip_limit = std::max(0, std::min(g.ny, g.nz - g.y_off));
  }
  if (g.kind == FBP_GEOMETRY_CONE && !(g.sod > 0.0 && g.sdd >= g.sod))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "source distance must be positive");
  if (!(g.du > 0.0) || !(g.vox > 0.0))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "detector and volume widths must be positive");
  FBP_TRY(flush_pending(ctx, s));
  FBP_TRY(ensure_volume(ctx, g.nx, g.ny, g.nz, false));
  *ylim = ctx->clip_after_bp ? clip_limit : 0;
  *mixed = ctx->precision != FBP_PRECISION_FP32;
  return FBP_OK;
}

int backproject(fbp_context* ctx, Stack& s, fbp::BPGeom g) {
  int ylim = 0;
  bool mixed = false;
  FBP_TRY(setup_backproject(ctx, s, g, &ylim, &mixed));
  if (ctx->autotune && ctx->bp_variant == FBP_BACKPROJECTOR_AUTO && g.ny > 1) {
    TuneShape shape;
    int rc = autotune_backprojector(ctx, s, g, mixed, &shape);
    if (rc == FBP_OK) {
      const TuneShape saved{ctx->bp_variant, ctx->quad_tile_ny, ctx->bp_stages};
      apply_shape(ctx, shape);
      rc = fbp::launch_backproject(ctx, g, s, ctx->vol, ylim, mixed);
      apply_shape(ctx, saved);
    }
    s.pack_ready = false;
    // the outer slices can have wider windows than the tuning slab: the
    // untuned selection still applies there
    if (rc != FBP_ERR_UNSUPPORTED) return rc;
  }
  return fbp::launch_backproject(ctx, g, s, ctx->vol, ylim, mixed);
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

}  // namespace

namespace fbp {

int set_error(fbp_context* ctx, int code, const std::string& msg) {
  if (ctx)
    ctx->last_error = msg;
  else
    g_thread_error = msg;
  return code;
}

int cuda_check(fbp_context* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FBP_OK;
  cudaGetLastError();
  int code = e == cudaErrorMemoryAllocation ? FBP_ERR_OUT_OF_MEMORY : FBP_ERR_CUDA;
  return set_error(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

void* scratch(fbp_context* ctx, size_t bytes) {
  if (bytes <= ctx->scratch_bytes) return ctx->d_scratch;
  cudaFree(ctx->d_scratch);
  ctx->d_scratch = nullptr;
  ctx->scratch_bytes = 0;
  size_t b = std::max<size_t>(bytes, 1 << 20);
  if (cudaMalloc(&ctx->d_scratch, b) != cudaSuccess) {
    cudaGetLastError();
    set_error(ctx, FBP_ERR_OUT_OF_MEMORY, "cudaMalloc of scratch memory failed");
    ctx->d_scratch = nullptr;
    return nullptr;
  }
  ctx->scratch_bytes = b;
  return ctx->d_scratch;
}

static int encode_tiled(fbp_context* ctx, CUtensorMap* map, CUtensorMapDataType dtype, int rank, void* base,
                        const uint64_t* dims, const uint64_t* strides_bytes, const uint32_t* box,
                        CUtensorMapSwizzle swizzle, CUtensorMapL2promotion l2) {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!g_encode) return set_error(ctx, FBP_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t gdim[5], gstr[4];
  cuuint32_t bdim[5], estr[5];
  for (int i = 0; i < rank; ++i) {
    gdim[i] = dims[i];
    bdim[i] = box[i];
    estr[i] = 1;
    if (i + 1 < rank) gstr[i] = strides_bytes[i];
  }
  CUresult r = g_encode(map, dtype, rank, base, gdim, gstr, bdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, l2,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(ctx, FBP_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return FBP_OK;
}

int make_tensor_map_3d(fbp_context* ctx, CUtensorMap* map, CUtensorMapDataType dtype, void* base,
                       const uint64_t dims[3], const uint64_t strides_bytes[2], const uint32_t box[3]) {
  return encode_tiled(ctx, map, dtype, 3, base, dims, strides_bytes, box, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B);
}

int make_tensor_map_4d(fbp_context* ctx, CUtensorMap* map, CUtensorMapDataType dtype, void* base,
                       const uint64_t dims[4], const uint64_t strides_bytes[3], const uint32_t box[4]) {
  return encode_tiled(ctx, map, dtype, 4, base, dims, strides_bytes, box, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B);
}

int make_tensor_map_2d_bf16_sw128(fbp_context* ctx, CUtensorMap* map, void* base, uint64_t inner, uint64_t outer,
                                  uint64_t pitch_bytes, uint32_t box_inner, uint32_t box_outer) {
  const uint64_t dims[2] = {inner, outer};
  const uint64_t strides[1] = {pitch_bytes};
  const uint32_t box[2] = {box_inner, box_outer};
  return encode_tiled(ctx, map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box,
                      CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B);
}

int prepare_packed(fbp_context* ctx, Stack& s, int layout) {
  const bool quad = fbp::is_quad_layout(layout);
  const int fpitch = quad ? s.u + 1 : round_up(s.u, 4);
  const size_t need = quad ? (size_t)(s.n / 4) * (s.v + 1) * (size_t)(s.u + 1) * Stack::elem_bytes(layout)
                           : (size_t)fpitch * s.filt_rows() * Stack::elem_bytes(layout);
  if (!s.filt || s.filt_bytes < need) {
    cudaFree(s.filt);
    s.filt = nullptr;
    s.filt_bytes = 0;
    if (cuda_check(ctx, cudaMalloc(&s.filt, need), "cudaMalloc(packed views)")) return FBP_ERR_OUT_OF_MEMORY;
    s.filt_bytes = need;
  }
  if (!s.inv_scale || s.scale_cap < s.n) {
    cudaFree(s.inv_scale);
    s.inv_scale = nullptr;
    s.scale_cap = 0;
    if (cuda_check(ctx, cudaMalloc(&s.inv_scale, sizeof(float) * 2 * s.n), "cudaMalloc(view scales)"))
      return FBP_ERR_OUT_OF_MEMORY;
    s.scale_cap = s.n;
  }
  float* scale = s.inv_scale + s.n;
  // the four-term difference of the gradient layout is at most 4 max|value|;
  // the 24-bit layout keeps the FP32 exponent and needs no scale
  if (layout != kLayoutQuadG24)
    if (int rc = launch_view_scales(ctx, rowset_of(s), quad ? 8192.f : 16384.f, scale, s.inv_scale)) return rc;
  if (int rc = launch_pack(ctx, s, layout, s.filt, fpitch, scale)) return rc;
  s.filt_layout = layout;
  s.filt_pitch = fpitch;
  return FBP_OK;
}

}  // namespace fbp

extern "C" {

// ------------------------------------------------------------------ context
int fbp_create(fbp_context** out, int device) {
  if (!out) {
    g_thread_error = "null output pointer";
    return FBP_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    g_thread_error = "no CUDA device";
    return FBP_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) {
    g_thread_error = "device index out of range";
    return FBP_ERR_INVALID_ARGUMENT;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  if (prop.major != 10) {
    g_thread_error = std::string("libfbp_b200 is built for sm_100a (B200); device is ") + prop.name;
    return FBP_ERR_UNSUPPORTED;
  }
  DeviceGuard guard(device);
  fbp_context* ctx = new fbp_context();
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  ctx->device_cc = prop.major * 10 + prop.minor;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&ctx->d_err, sizeof(int)) != cudaSuccess ||
      cudaMemset(ctx->d_err, 0, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&ctx->d_minmax, 2 * sizeof(int)) != cudaSuccess) {
    g_thread_error = std::string("context setup failed: ") + cudaGetErrorString(cudaGetLastError());
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    cudaFree(ctx->d_err);
    cudaFree(ctx->d_minmax);
    delete ctx;
    return FBP_ERR_CUDA;
  }
  ctx->own_stream = true;
  ctx->proj.sinogram = false;
  ctx->sino.sinogram = true;
  *out = ctx;
  return FBP_OK;
}

int fbp_destroy(fbp_context* ctx) {
  if (!ctx) return FBP_OK;
  {
    DeviceGuard guard(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_stack(ctx->proj);
    free_stack(ctx->sino);
    cudaFree(ctx->vol);
    cudaFree(ctx->d_err);
    cudaFree(ctx->d_minmax);
    cudaFree(ctx->d_trig);
    cudaFree(ctx->d_span);
    cudaFree(ctx->d_stage2d);
    cudaFree(ctx->ftab.twiddle);
    cudaFree(ctx->ftab.hbr);
    cudaFree(ctx->ftab.kernel);
    cudaFree(ctx->ttab.th);
    cudaFree(ctx->d_scratch);
    cudaFreeHost(ctx->h_pinned);
    cudaFree(ctx->d_batch);
    cudaFreeHost(ctx->h_batch);
    if (ctx->ev_batch_copy) cudaEventDestroy(ctx->ev_batch_copy);
    if (ctx->ev_sync) cudaEventDestroy(ctx->ev_sync);
    if (ctx->copy_stream) {
      cudaStreamSynchronize(ctx->copy_stream);
      cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return FBP_OK;
}

const char* fbp_last_error(const fbp_context* ctx) {
  return ctx ? ctx->last_error.c_str() : g_thread_error.c_str();
}

int fbp_set_stream(fbp_context* ctx, void* stream) {
  FBP_CTX(ctx);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  if (stream) {
    ctx->stream = static_cast<cudaStream_t>(stream);
    ctx->own_stream = false;
  } else {
    ctx->own_stream = true;
    return fbp::cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream create");
  }
  return FBP_OK;
}

int fbp_synchronize(fbp_context* ctx) {
  FBP_CTX(ctx);
  FBP_TRY(fbp::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"));
  return check_device_error(ctx);
}

int fbp_set_precision(fbp_context* ctx, int precision) {
  FBP_CTX(ctx);
  if (precision != FBP_PRECISION_FP32 && precision != FBP_PRECISION_MIXED && precision != FBP_PRECISION_MIXED24)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "unknown precision");
  ctx->precision = precision;
  return FBP_OK;
}

int fbp_set_filter_impl(fbp_context* ctx, int impl) {
  FBP_CTX(ctx);
  if (impl < FBP_FILTER_IMPL_AUTO || impl > FBP_FILTER_IMPL_TOEPLITZ)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "unknown filter implementation");
  ctx->filter_impl = impl;
  return FBP_OK;
}

int fbp_set_filter_padding(fbp_context* ctx, int padded_length) {
  FBP_CTX(ctx);
  if (padded_length < 0 || (padded_length & (padded_length - 1)))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "padding must be 0 or a power of two");
  ctx->pad_len = padded_length;
  return FBP_OK;
}

int fbp_set_clip_after_backprojection(fbp_context* ctx, int enable) {
  FBP_CTX(ctx);
  ctx->clip_after_bp = enable ? 1 : 0;
  return FBP_OK;
}

int fbp_set_backprojector(fbp_context* ctx, int variant) {
  FBP_CTX(ctx);
  if (variant < FBP_BACKPROJECTOR_AUTO || variant > FBP_BACKPROJECTOR_GENERIC_Y8)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "unknown backprojector variant");
  ctx->bp_variant = variant;
  for (auto& p : ctx->plans) p.valid = false;
  return FBP_OK;
}

int fbp_last_backprojection(const fbp_context* ctx, int* variant, int* layout, int* box_u, int* box_v,
                            int* tile_ny) {
  if (!ctx) return FBP_ERR_INVALID_ARGUMENT;
  if (ctx->last_bp[0] < 0) return FBP_ERR_STATE;
  if (variant) *variant = ctx->last_bp[0];
  if (layout) *layout = ctx->last_bp[1];
  if (box_u) *box_u = ctx->last_bp[2];
  if (box_v) *box_v = ctx->last_bp[3];
  if (tile_ny) *tile_ny = ctx->last_bp[4];
  return FBP_OK;
}

int fbp_set_autotune(fbp_context* ctx, int enable) {
  FBP_CTX(ctx);
  ctx->autotune = enable ? 1 : 0;
  return FBP_OK;
}

int fbp_set_autotune_cache(fbp_context* ctx, const char* path) {
  FBP_CTX(ctx);
  ctx->tune_cache = path ? path : "";
  ctx->tune_cache_loaded = false;
  return FBP_OK;
}

int fbp_autotune_stats(const fbp_context* ctx, int* timed, int* from_cache) {
  if (!ctx) return FBP_ERR_INVALID_ARGUMENT;
  if (timed) *timed = ctx->tune_timed;
  if (from_cache) *from_cache = ctx->tune_cached;
  return FBP_OK;
}

int fbp_set_view_ring(fbp_context* ctx, int stages) {
  FBP_CTX(ctx);
  if (stages != 0 && (stages < 2 || stages > 8))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "view ring stages must be 0 or 2..8");
  ctx->bp_stages = stages;
  return FBP_OK;
}

int fbp_set_symmetric_tile(fbp_context* ctx, int voxels_per_thread_y) {
  FBP_CTX(ctx);
  if (voxels_per_thread_y != 0 && voxels_per_thread_y != 8 && voxels_per_thread_y != 16)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "symmetric tile height must be 0, 8 or 16");
  ctx->quad_tile_ny = voxels_per_thread_y;
  return FBP_OK;
}

int fbp_memory_in_use(const fbp_context* ctx, size_t* bytes) {
  if (!ctx || !bytes) return FBP_ERR_INVALID_ARGUMENT;
  size_t b = 0;
  if (ctx->vol) b += ctx->vol_cap;
  for (const Stack* s : {&ctx->proj, &ctx->sino}) {
    if (s->f32) b += s->f32_cap;
    if (s->filt) b += s->filt_bytes;
    if (s->inv_scale) b += sizeof(float) * 2 * s->scale_cap;
  }
  b += ctx->scratch_bytes;
  *bytes = b;
  return FBP_OK;
}

// ------------------------------------------------------------------ buffers
int fbp_generate_blank_volume(fbp_context* ctx, int x, int y, int z) {
  FBP_CTX(ctx);
  return ensure_volume(ctx, x, y, z, true);
}

int fbp_generate_blank_projections(fbp_context* ctx, int x, int y, int n) {
  FBP_CTX(ctx);
  return alloc_stack(ctx, ctx->proj, x, y, n);
}

int fbp_generate_blank_sinograms(fbp_context* ctx, int x, int y, int n) {
  FBP_CTX(ctx);
  return alloc_stack(ctx, ctx->sino, x, y, n);
}

int fbp_free_volume(fbp_context* ctx) {
  FBP_CTX(ctx);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->vol);
  ctx->vol = nullptr;
  ctx->vol_cap = 0;
  ctx->vx = ctx->vy = ctx->vz = 0;
  ctx->minmax_valid = false;
  return FBP_OK;
}

int fbp_free_projections(fbp_context* ctx) {
  FBP_CTX(ctx);
  cudaStreamSynchronize(ctx->stream);
  free_stack(ctx->proj);
  return FBP_OK;
}

int fbp_free_sinograms(fbp_context* ctx) {
  FBP_CTX(ctx);
  cudaStreamSynchronize(ctx->stream);
  free_stack(ctx->sino);
  return FBP_OK;
}

int fbp_get_volume_size(const fbp_context* ctx, int* x, int* y, int* z) {
  if (!ctx || !x || !y || !z) return FBP_ERR_INVALID_ARGUMENT;
  *x = ctx->vx;
  *y = ctx->vy;
  *z = ctx->vz;
  return FBP_OK;
}

int fbp_get_projections_size(const fbp_context* ctx, int* u, int* v, int* n) {
  if (!ctx || !u || !v || !n) return FBP_ERR_INVALID_ARGUMENT;
  *u = ctx->proj.u;
  *v = ctx->proj.v;
  *n = ctx->proj.n;
  return FBP_OK;
}

int fbp_get_sinograms_size(const fbp_context* ctx, int* u, int* v, int* n) {
  if (!ctx || !u || !v || !n) return FBP_ERR_INVALID_ARGUMENT;
  *u = ctx->sino.u;
  *v = ctx->sino.v;
  *n = ctx->sino.n;
  return FBP_OK;
}

// ---------------------------------------------------------------- transfers
int fbp_upload_projections(fbp_context* ctx, const float* src, int u, int v, int n, int on_dev) {
  FBP_CTX(ctx);
  return upload_stack(ctx, ctx->proj, src, u, v, n, on_dev);
}

int fbp_upload_sinograms(fbp_context* ctx, const float* src, int u, int v, int n, int on_dev) {
  FBP_CTX(ctx);
  return upload_stack(ctx, ctx->sino, src, u, v, n, on_dev);
}

int fbp_download_projections(fbp_context* ctx, float* dst, int on_dev) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->proj, "download_projections"));
  return download_rows(ctx, ctx->proj, 0, ctx->proj.rows(), dst, on_dev);
}

int fbp_download_sinograms(fbp_context* ctx, float* dst, int on_dev) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->sino, "download_sinograms"));
  return download_rows(ctx, ctx->sino, 0, ctx->sino.rows(), dst, on_dev);
}

int fbp_store_projection(fbp_context* ctx, const float* src, int index, int on_dev) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->proj, "store_projection"));
  if (index < 0 || index >= ctx->proj.n) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "projection index out of range");
  return upload_rows(ctx, ctx->proj, (size_t)index * ctx->proj.v, ctx->proj.v, src, on_dev);
}

int fbp_load_projection(fbp_context* ctx, int index, float* dst, int on_dev) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->proj, "load_projection"));
  if (index < 0 || index >= ctx->proj.n) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "projection index out of range");
  return download_rows(ctx, ctx->proj, (size_t)index * ctx->proj.v, ctx->proj.v, dst, on_dev);
}

int fbp_store_sinogram(fbp_context* ctx, const float* src, int y, int on_dev) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->sino, "store_sinogram"));
  if (y < 0 || y >= ctx->sino.v) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "sinogram index out of range");
  return upload_rows(ctx, ctx->sino, (size_t)y * ctx->sino.n, ctx->sino.n, src, on_dev);
}

int fbp_load_sinogram(fbp_context* ctx, int y, float* dst, int on_dev) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->sino, "load_sinogram"));
  if (y < 0 || y >= ctx->sino.v) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "sinogram index out of range");
  return download_rows(ctx, ctx->sino, (size_t)y * ctx->sino.n, ctx->sino.n, dst, on_dev);
}

// One projection [v][u] (view `index`) out of / into the sinogram stack
// [v][view][u]: rows index, index + views, ... (FBP3D.cpp:755-778).
int fbp_load_projection_from_sinograms(fbp_context* ctx, int index, float* dst, int on_dev) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->sino, "load_projection_from_sinograms"));
  if (index < 0 || index >= ctx->sino.n) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "projection index out of range");
  return download_rows(ctx, ctx->sino, (size_t)index, ctx->sino.v, dst, on_dev, (size_t)ctx->sino.n);
}

int fbp_store_projection_to_sinograms(fbp_context* ctx, const float* src, int index, int on_dev) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->sino, "store_projection_to_sinograms"));
  if (index < 0 || index >= ctx->sino.n) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "projection index out of range");
  return upload_rows(ctx, ctx->sino, (size_t)index, ctx->sino.v, src, on_dev, (size_t)ctx->sino.n);
}

static int volume_slice(fbp_context* ctx, int axis, int index, float* host_or_dev, int on_dev, bool load) {
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "volume is not allocated");
  if (!load) ctx->minmax_valid = false;
  if (!host_or_dev) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null pointer");
  const int nx = ctx->vx, ny = ctx->vy, nz = ctx->vz;
  const int lim = axis == 0 ? nx : axis == 1 ? ny : nz;
  if (index < 0 || index >= lim) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "slice index out of range");
  float* v = ctx->vol;
  cudaError_t e;
  const cudaMemcpyKind k = load ? kind_of(true, on_dev) : kind_of(on_dev, true);
  if (axis == 2) {  // z-slice [y][x]: contiguous
    float* p = v + (size_t)index * nx * ny;
    e = load ? cudaMemcpyAsync(host_or_dev, p, sizeof(float) * nx * ny, k, ctx->stream)
             : cudaMemcpyAsync(p, host_or_dev, sizeof(float) * nx * ny, k, ctx->stream);
  } else if (axis == 1) {  // y-slice [z][x]
    float* p = v + (size_t)index * nx;
    e = load ? cudaMemcpy2DAsync(host_or_dev, sizeof(float) * nx, p, sizeof(float) * nx * ny, sizeof(float) * nx, nz, k,
                                 ctx->stream)
             : cudaMemcpy2DAsync(p, sizeof(float) * nx * ny, host_or_dev, sizeof(float) * nx, sizeof(float) * nx, nz, k,
                                 ctx->stream);
  } else {  // x-slice [z][y]
    float* p = v + index;
    e = load ? cudaMemcpy2DAsync(host_or_dev, sizeof(float), p, sizeof(float) * nx, sizeof(float), (size_t)ny * nz, k,
                                 ctx->stream)
             : cudaMemcpy2DAsync(p, sizeof(float) * nx, host_or_dev, sizeof(float), sizeof(float), (size_t)ny * nz, k,
                                 ctx->stream);
  }
  FBP_TRY(fbp::cuda_check(ctx, e, "volume slice copy"));
  return sync_host(ctx, !on_dev);
}

int fbp_load_volume_slice_x(fbp_context* ctx, int i, float* d, int o) { FBP_CTX(ctx); return volume_slice(ctx, 0, i, d, o, true); }
int fbp_load_volume_slice_y(fbp_context* ctx, int i, float* d, int o) { FBP_CTX(ctx); return volume_slice(ctx, 1, i, d, o, true); }
int fbp_load_volume_slice_z(fbp_context* ctx, int i, float* d, int o) { FBP_CTX(ctx); return volume_slice(ctx, 2, i, d, o, true); }
int fbp_store_volume_slice_x(fbp_context* ctx, const float* s, int i, int o) { FBP_CTX(ctx); return volume_slice(ctx, 0, i, const_cast<float*>(s), o, false); }
int fbp_store_volume_slice_y(fbp_context* ctx, const float* s, int i, int o) { FBP_CTX(ctx); return volume_slice(ctx, 1, i, const_cast<float*>(s), o, false); }
int fbp_store_volume_slice_z(fbp_context* ctx, const float* s, int i, int o) { FBP_CTX(ctx); return volume_slice(ctx, 2, i, const_cast<float*>(s), o, false); }

int fbp_read_volume(fbp_context* ctx, float* dst, int on_dev) {
  FBP_CTX(ctx);
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "read_volume but the volume is not allocated");
  if (!dst) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null destination pointer");
  size_t bytes = sizeof(float) * (size_t)ctx->vx * ctx->vy * ctx->vz;
  FBP_TRY(fbp::cuda_check(ctx, cudaMemcpyAsync(dst, ctx->vol, bytes, kind_of(true, on_dev), ctx->stream), "volume download"));
  return sync_host(ctx, true);
}

int fbp_write_volume_data(fbp_context* ctx, const float* src, int on_dev) {
  FBP_CTX(ctx);
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "write_volume_data but the volume is not allocated");
  ctx->minmax_valid = false;
  if (!src) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null source pointer");
  size_t bytes = sizeof(float) * (size_t)ctx->vx * ctx->vy * ctx->vz;
  FBP_TRY(fbp::cuda_check(ctx, cudaMemcpyAsync(ctx->vol, src, bytes, kind_of(on_dev, true), ctx->stream), "volume upload"));
  return sync_host(ctx, !on_dev);
}

int fbp_volume_device_ptr(fbp_context* ctx, float** ptr) {
  FBP_CTX(ctx);
  if (!ptr) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null pointer");
  *ptr = ctx->vol;
  ctx->minmax_valid = false;  // the caller may write through the pointer
  return ctx->vol ? FBP_OK : fbp::set_error(ctx, FBP_ERR_STATE, "volume is not allocated");
}

int fbp_projections_device_ptr(fbp_context* ctx, float** ptr, int* pitch) {
  FBP_CTX(ctx);
  if (!ptr || !pitch) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null pointer");
  FBP_TRY(require_stack(ctx, ctx->proj, "projections_device_ptr"));
  FBP_TRY(materialize_f32(ctx, ctx->proj));
  *ptr = ctx->proj.f32;
  *pitch = ctx->proj.pitch;
  return FBP_OK;
}

// ----------------------------------------------------------- pipeline stages
int fbp_log_normalize_projections(fbp_context* ctx, float base) {
  FBP_CTX(ctx);
  return record_log(ctx, ctx->proj, base, "log_normalize_projections");
}

int fbp_log_normalize_sinograms(fbp_context* ctx, float base) {
  FBP_CTX(ctx);
  return record_log(ctx, ctx->sino, base, "log_normalize_sinograms");
}

int fbp_apply_fdk_weights_to_projections(fbp_context* ctx, float sod, float odd, float det_w) {
  FBP_CTX(ctx);
  return record_weights(ctx, ctx->proj, sod, odd, det_w, "apply_fdk_weights_to_projections");
}

int fbp_apply_fdk_weights_to_sinograms(fbp_context* ctx, float sod, float odd, float det_w) {
  FBP_CTX(ctx);
  return record_weights(ctx, ctx->sino, sod, odd, det_w, "apply_fdk_weights_to_sinograms");
}

int fbp_apply_filter_to_projections(fbp_context* ctx, int filter_type) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->proj, "apply_filter_to_projections"));
  return filter_stack(ctx, ctx->proj, filter_type);
}

int fbp_apply_filter_to_sinograms(fbp_context* ctx, int filter_type) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->sino, "apply_filter_to_sinograms"));
  return filter_stack(ctx, ctx->sino, filter_type);
}

int fbp_clip_negatives_of_volume(fbp_context* ctx) {
  FBP_CTX(ctx);
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "clip_negatives_of_volume but the volume is not allocated");
  ctx->minmax_valid = false;
  return fbp::launch_clip(ctx, ctx->vol, ctx->vx, ctx->vy, ctx->vz, ctx->vz);
}

// ------------------------------------------------ forward projection (f3)
// The reference sizes the detector like the volume: volume x columns, volume
// y rows (FBP3D.cpp:219, 274); parallel beam measures in voxels (detector
// width = volume width = x size, FBP3D.cpp:230-231).
static int forward(fbp_context* ctx, Stack& s, bool cone, float sod, float odd, float det_w, float vol_w, float rot,
                   int count, float offset) {
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "project_forward but the volume is not allocated");
  if (count <= 0) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "projection count must be positive");
  if (cone && (!(sod > 0.f) || !(odd >= 0.f) || !(det_w > 0.f) || !(vol_w > 0.f)))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "distances and widths must be positive");
  const int nu = ctx->vx, nv = ctx->vy;
  FBP_TRY(alloc_stack(ctx, s, nu, nv, count, false));  // generate_blank_*: every sample is written
  const double vox = cone ? (double)vol_w / ctx->vx : 1.0;
  const double du = cone ? (double)det_w / nu : 1.0;
  return fbp::launch_forward(ctx, ctx->vol, ctx->vx, ctx->vy, ctx->vz, vox, cone, sod, (double)sod + odd, du, du,
                             2.0 * kPi * (double)rot, offset, nu, nv, count, s.f32, s.pitch, s.sinogram);
}

int fbp_project_forward_cone_to_projections(fbp_context* ctx, float sod, float odd, float det_w, float vol_w,
                                            float rot, int count, float offset) {
  FBP_CTX(ctx);
  return forward(ctx, ctx->proj, true, sod, odd, det_w, vol_w, rot, count, offset);
}

int fbp_project_forward_cone_to_sinograms(fbp_context* ctx, float sod, float odd, float det_w, float vol_w,
                                          float rot, int count, float offset) {
  FBP_CTX(ctx);
  return forward(ctx, ctx->sino, true, sod, odd, det_w, vol_w, rot, count, offset);
}

int fbp_project_forward_parallel_to_projections(fbp_context* ctx, float rot, int count, float offset) {
  FBP_CTX(ctx);
  return forward(ctx, ctx->proj, false, 0.f, 0.f, 0.f, 0.f, rot, count, offset);
}

int fbp_project_forward_parallel_to_sinograms(fbp_context* ctx, float rot, int count, float offset) {
  FBP_CTX(ctx);
  return forward(ctx, ctx->sino, false, 0.f, 0.f, 0.f, 0.f, rot, count, offset);
}

int fbp2d_project_forward(fbp_context* ctx, const float* image, int nx, int nz, float* sinogram, int bins, int views,
                          const fbp_geometry* g) {
  FBP_CTX(ctx);
  if (!image || !sinogram || !g || nx <= 0 || nz <= 0 || bins <= 0 || views <= 0)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "bad 2D forward projection arguments");
  if (!(g->detector_width > 0.f) || !(g->volume_width > 0.f))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "detector and volume widths must be positive");
  const bool cone = g->kind == FBP_GEOMETRY_CONE;
  if (cone && !(g->source_distance > 0.f))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "source distance must be positive");
  const double vox = (double)g->volume_width / nx, du = (double)g->detector_width / bins;
  return fbp::launch_forward(ctx, image, nx, 1, nz, vox, cone, g->source_distance,
                             (double)g->source_distance + g->detector_distance, du, du,
                             2.0 * kPi * (double)g->full_rotation_count, g->rotation_offset_radian, bins, 1, views,
                             sinogram, bins, false);
}

// ---------------------------------------------------------- sharding (e)
int fbp_set_detector_rows(fbp_context* ctx, int row_offset, int total_rows) {
  FBP_CTX(ctx);
  if (total_rows < 0 || row_offset < 0 || (total_rows == 0 && row_offset != 0) ||
      (total_rows > 0 && row_offset >= total_rows))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "bad detector row band");
  ctx->det_row_off = row_offset;
  ctx->det_rows_total = total_rows;
  return FBP_OK;
}

int fbp_set_volume_slab(fbp_context* ctx, int y_offset, int y_count) {
  FBP_CTX(ctx);
  if (y_offset < 0 || y_count < 0 || (y_count == 0 && y_offset != 0))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "bad volume slab");
  ctx->slab_y0 = y_offset;
  ctx->slab_ny = y_count;
  return FBP_OK;
}

int fbp_plan_slabs(const fbp_geometry* g, int detector_cols, int detector_rows, int volume_h, int volume_v,
                   int slabs, int* out) {
  if (!g || !out || detector_cols <= 0 || detector_rows <= 0 || volume_h <= 0 || volume_v <= 0 || slabs <= 0 ||
      slabs > volume_v)
    return FBP_ERR_INVALID_ARGUMENT;
  const bool cone = g->kind == FBP_GEOMETRY_CONE;
  const double du = (double)g->detector_width / detector_cols, dv = du;  // square detector pixels
  const double vox = (double)g->volume_width / volume_h;
  const double sod = g->source_distance, sdd = (double)g->source_distance + g->detector_distance;
  if (!(du > 0.0) || !(vox > 0.0) || (cone && !(sod > 0.0))) return FBP_ERR_INVALID_ARGUMENT;
  const double cv = 0.5 * detector_rows - 0.5;
  // farthest voxel centre from the rotation axis bounds the source distance over every view
  const double rad = std::sqrt(2.0) * (0.5 * volume_h - 0.5) * vox;
  const double dmin = cone ? (sod - rad) / sod : 1.0, dmax = cone ? (sod + rad) / sod : 1.0;
  const double G = cone ? sdd / (sod * dv) : 1.0 / dv;
  for (int k = 0; k < slabs; ++k) {
    const int y0 = (int)((long long)volume_v * k / slabs), y1 = (int)((long long)volume_v * (k + 1) / slabs);
    int r0 = 0, r1 = detector_rows;  // whole detector when a voxel may lie at or behind the source
    if (dmin > 0.0) {
      double vmin = 1e300, vmax = -1e300;
      for (int y : {y0, y1 - 1})
        for (double d : {dmin, dmax}) {
          const double v = G * (y + 0.5 - 0.5 * volume_v) * vox / d + cv;
          vmin = std::min(vmin, v);
          vmax = std::max(vmax, v);
        }
      // bilinear taps use rows floor(v) and floor(v) + 1; one row of margin each side
      r0 = (int)std::max(0.0, std::floor(vmin) - 1.0);
      r1 = (int)std::min((double)detector_rows, std::floor(vmax) + 3.0);
      if (r1 <= r0) {  // slab projects off the detector: keep one (all-zero-weight) row
        r0 = std::min(std::max(r0, 0), detector_rows - 1);
        r1 = r0 + 1;
      }
    }
    out[4 * k] = y0;
    out[4 * k + 1] = y1;
    out[4 * k + 2] = r0;
    out[4 * k + 3] = r1;
  }
  return FBP_OK;
}

// ---------------------------------------------------------- file I/O (f2)
int fbp_projection_file_index(const char* path) { return path ? fbp::projection_file_index(path) : -1; }

static int read_files(fbp_context* ctx, Stack& s, const char* directory, int fw, int fh, int ch, int bpc, int tw,
                      int th, int count) {
  FBP_TRY(alloc_stack(ctx, s, tw, th, count));  // generate_blank_projections / _sinograms
  s.filtered = false;
  s.log_pending = s.weights_pending = false;
  FBP_TRY(fbp::read_projection_files(ctx, directory, fw, fh, ch, bpc, tw, th, count, s.f32, s.pitch, s.sinogram));
  return sync_host(ctx, true);
}

int fbp_read_projections(fbp_context* ctx, const char* directory, int file_width, int file_height,
                         int file_channel_count, int byte_per_channel, int target_width, int target_height,
                         int projection_count) {
  FBP_CTX(ctx);
  return read_files(ctx, ctx->proj, directory, file_width, file_height, file_channel_count, byte_per_channel,
                    target_width, target_height, projection_count);
}

int fbp_read_projections_as_sinograms(fbp_context* ctx, const char* directory, int file_width, int file_height,
                                      int file_channel_count, int byte_per_channel, int target_width,
                                      int target_height, int projection_count) {
  FBP_CTX(ctx);
  return read_files(ctx, ctx->sino, directory, file_width, file_height, file_channel_count, byte_per_channel,
                    target_width, target_height, projection_count);
}

int fbp_write_volume(fbp_context* ctx, const char* directory) {
  FBP_CTX(ctx);
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "write_volume but the volume is not allocated");
  FBP_TRY(fbp::write_volume_files(ctx, directory));
  return sync_host(ctx, true);
}

// -------------------------------------------------- histogram normalisation
static int volume_extremes_on_device(fbp_context* ctx) {
  if (ctx->minmax_valid) return FBP_OK;  // folded in by the last backprojection
  FBP_TRY(fbp::launch_volume_minmax(ctx, ctx->vol, (long long)ctx->vx * ctx->vy * ctx->vz, ctx->d_minmax));
  ctx->minmax_valid = true;
  return FBP_OK;
}

int fbp_volume_min_max(fbp_context* ctx, float* min_value, float* max_value) {
  FBP_CTX(ctx);
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "volume_min_max but the volume is not allocated");
  if (!min_value || !max_value) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null pointer");
  FBP_TRY(volume_extremes_on_device(ctx));
  int keys[2];
  FBP_TRY(fbp::cuda_check(ctx, cudaMemcpyAsync(keys, ctx->d_minmax, sizeof(keys), cudaMemcpyDeviceToHost, ctx->stream),
                          "min/max readback"));
  FBP_TRY(sync_host(ctx, true));
  auto value = [](int k) {
    const int b = k >= 0 ? k : k ^ 0x7fffffff;
    float f;
    std::memcpy(&f, &b, sizeof(f));
    return f;
  };
  if (keys[0] > keys[1]) {  // no finite value
    *min_value = *max_value = 0.f;
    return FBP_OK;
  }
  *min_value = value(keys[0]);
  *max_value = value(keys[1]);
  return FBP_OK;
}

int fbp_normalize_histogram(fbp_context* ctx) {
  FBP_CTX(ctx);
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "normalize_histogram but the volume is not allocated");
  FBP_TRY(volume_extremes_on_device(ctx));
  FBP_TRY(fbp::launch_normalize(ctx, ctx->vol, (long long)ctx->vx * ctx->vy * ctx->vz, ctx->d_minmax, 0.f, 0.f));
  ctx->minmax_valid = false;
  return FBP_OK;
}

int fbp_normalize_histogram_range(fbp_context* ctx, float min_value, float max_value) {
  FBP_CTX(ctx);
  if (!ctx->vol) return fbp::set_error(ctx, FBP_ERR_STATE, "normalize_histogram but the volume is not allocated");
  FBP_TRY(fbp::launch_normalize(ctx, ctx->vol, (long long)ctx->vx * ctx->vy * ctx->vz, nullptr, min_value, max_value));
  ctx->minmax_valid = false;
  return FBP_OK;
}

int fbp_project_backward_cone_fdk_from_projections(fbp_context* ctx, float sod, float odd, float det_w, float vol_w,
                                                   float rot, int h, int v, float offset) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->proj, "project_backward_cone_fdk_from_projections"));
  return backproject(ctx, ctx->proj, cone_geom(ctx->proj, sod, odd, det_w, vol_w, rot, h, v, offset));
}

}  // extern "C"

namespace fbp {
int plan_cone_projections(fbp_context* c, const fbp_geometry& ge, int h, int v, BPLaunchPlan* plan) {
  DeviceGuard guard(c->device);
  FBP_TRY(require_stack(c, c->proj, "cone backprojection"));
  fbp::BPGeom g = cone_geom(c->proj, ge.source_distance, ge.detector_distance, ge.detector_width, ge.volume_width,
                            ge.full_rotation_count, h, v, ge.rotation_offset_radian);
  int ylim = 0;
  bool mixed = false;
  FBP_TRY(setup_backproject(c, c->proj, g, &ylim, &mixed));
  return fbp::plan_backproject(c, g, c->proj, c->vol, ylim, mixed, plan);
}
}  // namespace fbp

extern "C" {

int fbp_project_backward_cone_fdk_batch(fbp_context* const* contexts, const fbp_geometry* geometries,
                                        const int* volume_h, const int* volume_v, int count, fbp_context* launcher) {
  FBP_CTX(launcher);
  if (!contexts || !geometries || !volume_h || !volume_v || count <= 0)
    return fbp::set_error(launcher, FBP_ERR_INVALID_ARGUMENT, "bad batch arguments");
  for (int i = 0; i < count; ++i) {
    if (!contexts[i] || contexts[i]->device != launcher->device)
      return fbp::set_error(launcher, FBP_ERR_INVALID_ARGUMENT, "batch contexts must be on the launcher's device");
    if (geometries[i].kind != FBP_GEOMETRY_CONE)
      return fbp::set_error(launcher, FBP_ERR_INVALID_ARGUMENT, "batched backprojection takes cone-beam geometries");
  }
  struct Plans {
    std::vector<fbp::BPLaunchPlan*> p;
    ~Plans() {
      for (auto* x : p) fbp::free_bp_plan(x);
    }
  } plans;
  // plan every job on its own stream (weights, filter, packing, footprint pass)
  for (int i = 0; i < count; ++i) {
    fbp_context* c = contexts[i];
    plans.p.push_back(fbp::new_bp_plan());
    if (int rc = fbp::plan_cone_projections(c, geometries[i], volume_h[i], volume_v[i], plans.p.back()))
      return fbp::set_error(launcher, rc, std::string("batch job ") + std::to_string(i) + ": " + c->last_error);
  }
  auto event = [&](fbp_context* c) -> cudaEvent_t {
    if (!c->ev_sync) cudaEventCreateWithFlags(&c->ev_sync, cudaEventDisableTiming);
    return c->ev_sync;
  };
  // jobs that share a batch key run in one persistent launch on the
  // launcher's stream (after their own streams' work); the rest alone
  std::vector<bool> done(count, false);
  for (int i = 0; i < count; ++i) {
    if (done[i]) continue;
    const long long key = fbp::bp_plan_batch_key(*plans.p[i]);
    if (key == 0) {
      done[i] = true;
      FBP_TRY(fbp::launch_bp_plan(contexts[i], *plans.p[i]));
      continue;
    }
    std::vector<fbp::BPLaunchPlan*> group;
    std::vector<fbp_context*> members;
    for (int k = i; k < count; ++k)
      if (!done[k] && fbp::bp_plan_batch_key(*plans.p[k]) == key) {
        done[k] = true;
        group.push_back(plans.p[k]);
        members.push_back(contexts[k]);
      }
    for (fbp_context* c : members)
      if (c != launcher) {
        cudaEvent_t ev = event(c);
        if (fbp::cuda_check(launcher, ev ? cudaEventRecord(ev, c->stream) : cudaErrorInvalidResourceHandle,
                            "batch ready event") ||
            fbp::cuda_check(launcher, cudaStreamWaitEvent(launcher->stream, ev, 0), "batch ready wait"))
          return FBP_ERR_CUDA;
      }
    FBP_TRY(fbp::launch_bp_batch(launcher, group.data(), (int)group.size()));
    cudaEvent_t lev = event(launcher);
    if (fbp::cuda_check(launcher, lev ? cudaEventRecord(lev, launcher->stream) : cudaErrorInvalidResourceHandle,
                        "batch done event"))
      return FBP_ERR_CUDA;
    for (fbp_context* c : members) {
      if (c != launcher && fbp::cuda_check(launcher, cudaStreamWaitEvent(c->stream, lev, 0), "batch done wait"))
        return FBP_ERR_CUDA;
      c->last_bp[0] = FBP_BACKPROJECTOR_SYMMETRIC;
      c->minmax_valid = false;
    }
  }
  return FBP_OK;
}

int fbp_project_backward_cone_fdk_from_sinograms(fbp_context* ctx, float sod, float odd, float det_w, float vol_w,
                                                 float rot, int h, int v, float offset) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->sino, "project_backward_cone_fdk_from_sinograms"));
  return backproject(ctx, ctx->sino, cone_geom(ctx->sino, sod, odd, det_w, vol_w, rot, h, v, offset));
}

static fbp::BPGeom parallel_geom(const Stack& s, float rot, int h, int v, float offset) {
  // The reference passes projection_plane_width = volume_width = x size
  // (FBP3D.cpp:481-482): the detector spans the volume width, in voxel units.
  fbp::BPGeom g{};
  g.kind = FBP_GEOMETRY_PARALLEL;
  g.vox = 1.0;
  g.du = (double)h / s.u;
  g.dv = (double)v / s.v;
  g.span = 2.0 * kPi * (double)rot;
  g.offset = offset;
  g.nu = s.u;
  g.nv = s.v;
  g.nviews = s.n;
  g.nx = h;
  g.ny = v;
  g.nz = h;
  return g;
}

int fbp_project_backward_parallel_from_projections(fbp_context* ctx, float rot, int h, int v, float offset) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->proj, "project_backward_parallel_from_projections"));
  if (h <= 0 || v <= 0) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "volume resolution must be positive");
  return backproject(ctx, ctx->proj, parallel_geom(ctx->proj, rot, h, v, offset));
}

int fbp_project_backward_parallel_from_sinograms(fbp_context* ctx, float rot, int h, int v, float offset) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->sino, "project_backward_parallel_from_sinograms"));
  if (h <= 0 || v <= 0) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "volume resolution must be positive");
  return backproject(ctx, ctx->sino, parallel_geom(ctx->sino, rot, h, v, offset));
}

int fbp_reconstruct_fdk_to_host(fbp_context* ctx, const float* projections, int cols, int rows, int count,
                                const fbp_geometry* g, int filter_type, int h, int v, float* volume, int slabs) {
  FBP_CTX(ctx);
  if (!projections || !volume || !g) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null pointer");
  if (slabs < 1 || slabs > 64 || v <= 0 || h <= 0 || slabs > v)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "slabs must be in [1, min(64, v)]");
  if (ctx->det_rows_total > 0 || ctx->slab_ny > 0)
    return fbp::set_error(ctx, FBP_ERR_STATE, "reconstruct_fdk_to_host with a detector band or volume slab set");
  Stack& s = ctx->proj;
  // upload (the host buffer should be pinned), weights, filter
  if (!(s.f32 && s.u == cols && s.v == rows && s.n == count)) FBP_TRY(alloc_stack(ctx, s, cols, rows, count, false));
  s.filtered = false;
  s.log_pending = s.weights_pending = false;
  FBP_TRY(fbp::cuda_check(ctx,
                          copy_rows(s.f32, (size_t)s.pitch * 4, projections, (size_t)cols * 4, (size_t)cols * 4,
                                            s.rows(), cudaMemcpyHostToDevice, ctx->stream),
                          "projection upload"));
  const bool cone = g->kind == FBP_GEOMETRY_CONE;
  if (cone)
    FBP_TRY(record_weights(ctx, s, g->source_distance, g->detector_distance, g->detector_width, "reconstruct_fdk_to_host"));
  FBP_TRY(filter_stack(ctx, s, filter_type));
  fbp::BPGeom gg;
  if (cone) {
    gg = cone_geom(s, g->source_distance, g->detector_distance, g->detector_width, g->volume_width,
                   g->full_rotation_count, h, v, g->rotation_offset_radian);
  } else {
    gg = parallel_geom(s, g->full_rotation_count, h, v, g->rotation_offset_radian);
    gg.vox = (double)g->volume_width / h;
    gg.du = (double)g->detector_width / s.u;
    gg.dv = gg.du;
  }
  if (cone && !(gg.sod > 0.0 && gg.sdd >= gg.sod))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "source distance must be positive");
  if (!(gg.du > 0.0) || !(gg.vox > 0.0))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "detector and volume widths must be positive");
  FBP_TRY(ensure_volume(ctx, h, v, h, false));
  if (!ctx->copy_stream) {
    DeviceGuard guard(ctx->device);
    FBP_TRY(fbp::cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "copy stream"));
  }
  const bool mixed = ctx->precision != FBP_PRECISION_FP32;
  std::vector<cudaEvent_t> done(slabs, nullptr);
  int rc = FBP_OK;
  const TuneShape saved{ctx->bp_variant, ctx->quad_tile_ny, ctx->bp_stages};
  if (ctx->autotune && ctx->bp_variant == FBP_BACKPROJECTOR_AUTO && v > 1) {
    TuneShape shape;
    rc = autotune_backprojector(ctx, s, gg, mixed, &shape);
    if (rc == FBP_OK) apply_shape(ctx, shape);
  }
  // y-slab k is backprojected straight into the whole volume, then copied to
  // the host on the copy stream while slab k + 1 computes
  for (int k = 0; k < slabs && rc == FBP_OK; ++k) {
    const int y0 = (int)((long long)v * k / slabs), y1 = (int)((long long)v * (k + 1) / slabs);
    fbp::BPGeom gs = gg;
    gs.ny_total = v;
    gs.y_off = y0;
    gs.ny = y1 - y0;
    gs.vol_ystride = v;
    const int ylim = ctx->clip_after_bp ? std::max(0, std::min(gs.ny, gs.nz - y0)) : 0;
    rc = fbp::launch_backproject(ctx, gs, s, ctx->vol + (size_t)y0 * h, ylim, mixed);
    if (rc == FBP_ERR_UNSUPPORTED && ctx->bp_variant != saved.variant) {
      // a tuned choice that an outer slab's windows do not allow
      apply_shape(ctx, saved);
      rc = fbp::launch_backproject(ctx, gs, s, ctx->vol + (size_t)y0 * h, ylim, mixed);
    }
    s.pack_ready = mixed && !s.filtered;  // the first slab packed the views: the others reuse them
    if (rc) break;
    if ((rc = fbp::cuda_check(ctx, cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming), "event")) ||
        (rc = fbp::cuda_check(ctx, cudaEventRecord(done[k], ctx->stream), "event")) ||
        (rc = fbp::cuda_check(ctx, cudaStreamWaitEvent(ctx->copy_stream, done[k], 0), "event wait")))
      break;
    rc = fbp::cuda_check(ctx,
                         copy_rows(volume + (size_t)y0 * h, (size_t)v * h * 4, ctx->vol + (size_t)y0 * h,
                                           (size_t)v * h * 4, (size_t)(y1 - y0) * h * 4, h, cudaMemcpyDeviceToHost,
                                           ctx->copy_stream),
                         "slab readback");
  }
  s.pack_ready = false;
  apply_shape(ctx, saved);
  ctx->minmax_valid = false;
  cudaStreamSynchronize(ctx->copy_stream);
  for (cudaEvent_t e : done)
    if (e) cudaEventDestroy(e);
  if (rc) return rc;
  return sync_host(ctx, true);
}

int fbp_reconstruct_fdk(fbp_context* ctx, const fbp_geometry* g, int filter_type, int h, int v) {
  FBP_CTX(ctx);
  if (!g) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null geometry");
  FBP_TRY(require_stack(ctx, ctx->proj, "reconstruct_fdk"));
  if (g->kind == FBP_GEOMETRY_CONE) {
    FBP_TRY(record_weights(ctx, ctx->proj, g->source_distance, g->detector_distance, g->detector_width, "reconstruct_fdk"));
    FBP_TRY(filter_stack(ctx, ctx->proj, filter_type));
    return backproject(ctx, ctx->proj,
                       cone_geom(ctx->proj, g->source_distance, g->detector_distance, g->detector_width, g->volume_width,
                                 g->full_rotation_count, h, v, g->rotation_offset_radian));
  }
  FBP_TRY(filter_stack(ctx, ctx->proj, filter_type));
  fbp::BPGeom pg = parallel_geom(ctx->proj, g->full_rotation_count, h, v, g->rotation_offset_radian);
  pg.vox = (double)g->volume_width / h;
  pg.du = (double)g->detector_width / ctx->proj.u;
  pg.dv = pg.du;
  return backproject(ctx, ctx->proj, pg);
}

// ----------------------------------------------------------------------- 2D
static int stage_2d(fbp_context* ctx, const float* sino, int bins, int views, Stack& st, size_t offset_bytes) {
  st = Stack();
  st.u = bins;
  st.v = 1;
  st.n = views;
  st.pitch = round_up(bins, 4);
  st.filtered = false;
  const size_t need = offset_bytes + st.bytes32();
  if (ctx->stage2d_bytes < need) {
    cudaFree(ctx->d_stage2d);
    ctx->d_stage2d = nullptr;
    ctx->stage2d_bytes = 0;
    if (fbp::cuda_check(ctx, cudaMalloc(&ctx->d_stage2d, need), "cudaMalloc(2D staging)")) return FBP_ERR_OUT_OF_MEMORY;
    ctx->stage2d_bytes = need;
  }
  char* base = reinterpret_cast<char*>(ctx->d_stage2d);
  st.f32 = reinterpret_cast<float*>(base + offset_bytes);
  return fbp::cuda_check(ctx,
                         copy_rows(st.f32, (size_t)st.pitch * 4, sino, (size_t)bins * 4, (size_t)bins * 4,
                                           views, cudaMemcpyDeviceToDevice, ctx->stream),
                         "2D sinogram staging");
}

int fbp2d_filter_sinogram(fbp_context* ctx, float* sino, int bins, int views, int filter_type, float fan_sdd,
                          float det_w) {
  FBP_CTX(ctx);
  if (!sino || bins <= 0 || views <= 0) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "bad sinogram");
  if (filter_type < 0 || filter_type > FBP_FILTER_RAMP_SAMPLED)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "unknown filter type");
  const int n = ctx->pad_len > 0 ? ctx->pad_len : next_pow2_reference(bins);
  if (n < bins) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "padded length smaller than the row");
  FBP_TRY(fbp::ensure_filter_tables(ctx, n, filter_type));
  fbp::RowSet rs{};
  rs.data = sino;
  rs.pitch = bins;
  rs.rows = views;
  rs.m = bins;
  rs.n_views = views;
  rs.n_v = 1;
  rs.sinogram = false;
  if (fan_sdd > 0.f) {
    if (!(det_w > 0.f)) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "detector width must be positive");
    rs.weight = true;
    rs.w_sdd = fan_sdd;
    rs.w_du = det_w / bins;
    rs.w_dv = 0.f;
  }
  // the context's precision / implementation switch, as for the 3D stacks:
  // MIXED and MIXED24 filter on the tensor cores (split-BF16 Toeplitz product)
  int impl = ctx->filter_impl;
  if (impl == FBP_FILTER_IMPL_AUTO)
    impl = (ctx->precision != FBP_PRECISION_FP32 && fbp::toeplitz_supported(bins)) ? FBP_FILTER_IMPL_TOEPLITZ
                                                                                     : FBP_FILTER_IMPL_FFT;
  if (impl != FBP_FILTER_IMPL_TOEPLITZ) return fbp::launch_filter_fft(ctx, rs, n);
  if (!fbp::toeplitz_supported(bins))
    return fbp::set_error(ctx, FBP_ERR_UNSUPPORTED, "Toeplitz filter needs 64 <= bins <= 8192");
  // the GEMM's row split reads 16-byte vectors: stage the rows at a pitch of
  // a multiple of 4 floats, filter them in place there and copy them back
  Stack st;
  FBP_TRY(stage_2d(ctx, sino, bins, views, st, 0));
  rs.data = st.f32;
  rs.pitch = st.pitch;
  FBP_TRY(fbp::launch_filter_toeplitz(ctx, rs, n, filter_type));
  return fbp::cuda_check(ctx,
                         copy_rows(sino, (size_t)bins * 4, st.f32, (size_t)st.pitch * 4, (size_t)bins * 4,
                                           views, cudaMemcpyDeviceToDevice, ctx->stream),
                         "2D filtered rows copy-back");
}

int fbp2d_project_backward(fbp_context* ctx, const float* sino, int bins, int views, const fbp_geometry* geom,
                           float* image, int nx, int nz) {
  FBP_CTX(ctx);
  if (!sino || !image || !geom || bins <= 0 || views <= 0 || nx <= 0 || nz <= 0)
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "bad 2D backprojection arguments");
  if (!(geom->detector_width > 0.f) || !(geom->volume_width > 0.f))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "detector and volume widths must be positive");
  fbp::BPGeom g{};
  g.kind = geom->kind == FBP_GEOMETRY_CONE ? FBP_GEOMETRY_CONE : FBP_GEOMETRY_PARALLEL;
  g.sod = geom->source_distance;
  g.sdd = (double)geom->source_distance + geom->detector_distance;
  if (g.kind == FBP_GEOMETRY_CONE && !(g.sod > 0.0))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "source distance must be positive");
  g.du = (double)geom->detector_width / bins;
  g.dv = 1.0;
  g.vox = (double)geom->volume_width / nx;
  g.span = 2.0 * kPi * (double)geom->full_rotation_count;
  g.offset = geom->rotation_offset_radian;
  g.nu = bins;
  g.nv = 1;
  g.nviews = views;
  g.nx = nx;
  g.ny = 1;
  g.nz = nz;
  // the 2D kernel reads the rows where they are; a geometry whose tile windows
  // could be very wide (source near the image) takes the general path
  const int rc = fbp::launch_bp2d(ctx, g, sino, bins, image);
  if (rc != FBP_ERR_UNSUPPORTED) return rc;
  Stack st;
  FBP_TRY(stage_2d(ctx, sino, bins, views, st, 0));
  return fbp::launch_backproject(ctx, g, st, image, 0, false);
}

int fbp2d_parallelize_fan_beam_sinogram(fbp_context* ctx, const float* fan, int bins, int views,
                                        const fbp_geometry* geom, float* par, int out_bins, float out_w) {
  FBP_CTX(ctx);
  if (!fan || !par || !geom || bins <= 0 || views <= 0 || out_bins <= 0 || !(out_w > 0.f))
    return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "bad rebinning arguments");
  fbp::BPGeom g{};
  g.sod = geom->source_distance;
  g.sdd = (double)geom->source_distance + geom->detector_distance;
  g.du = (double)geom->detector_width / bins;
  g.span = 2.0 * kPi * (double)geom->full_rotation_count;
  g.offset = geom->rotation_offset_radian;
  return fbp::launch_rebin_fan(ctx, fan, bins, views, g, par, out_bins, (double)out_w / out_bins);
}

// ------------------------------------------------------------------ FFT rows
int fbp_fft_rows(fbp_context* ctx, float* rows, int n, int count, int inverse) {
  FBP_CTX(ctx);
  if (!rows) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null rows");
  return fbp::launch_fft_rows(ctx, reinterpret_cast<float2*>(rows), n, count, inverse);
}

int fbp_fft_shift_rows(fbp_context* ctx, float* rows, int n, int count, int shift) {
  FBP_CTX(ctx);
  if (!rows) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null rows");
  return fbp::launch_fft_shift_rows(ctx, reinterpret_cast<float2*>(rows), n, count, shift);
}

// ------------------------------------------------------------------ phantoms
int fbp_project_ellipsoids_to_projections(fbp_context* ctx, const double* ell, int count, const fbp_geometry* geom) {
  FBP_CTX(ctx);
  FBP_TRY(require_stack(ctx, ctx->proj, "project_ellipsoids_to_projections"));
  if (!geom || (count > 0 && !ell)) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "null argument");
  if (count < 0 || count > 64) return fbp::set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "ellipsoid count must be in [0, 64]");
  Stack& s = ctx->proj;
  fbp::BPGeom g{};
  g.kind = geom->kind;
  g.sod = geom->source_distance;
  g.sdd = (double)geom->source_distance + geom->detector_distance;
  g.du = (double)geom->detector_width / s.u;
  g.dv = g.du;
  g.span = 2.0 * kPi * (double)geom->full_rotation_count;
  g.offset = geom->rotation_offset_radian;
  g.nu = s.u;
  g.nv = s.v;
  g.nviews = s.n;
  double* d = static_cast<double*>(fbp::scratch(ctx, sizeof(double) * 16 * std::max(count, 1)));
  if (!d) return FBP_ERR_OUT_OF_MEMORY;
  if (count > 0)
    FBP_TRY(fbp::cuda_check(ctx, cudaMemcpyAsync(d, ell, sizeof(double) * 16 * count, cudaMemcpyHostToDevice, ctx->stream),
                            "ellipsoid upload"));
  s.filtered = false;
  s.log_pending = s.weights_pending = false;
  FBP_TRY(fbp::launch_project_ellipsoids(ctx, d, count, g, s.f32, s.pitch));
  // the host array is only borrowed for the call
  return fbp::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
}

}  // extern "C"
