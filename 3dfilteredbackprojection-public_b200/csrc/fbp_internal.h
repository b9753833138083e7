// Internal declarations shared by the CUDA translation units of libfbp_b200.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fbp_b200.h"

namespace fbp {

// Device-side error codes written to the context's error word.
enum DeviceError : int {
  kDevOk = 0,
  kDevTimeout = 1,    // an mbarrier / flag wait ran out of iterations
  kDevFootprint = 2,  // a staged detector window was smaller than a tile's footprint
  kDevGeometry = 3,   // a voxel lies at or behind the source plane
};

// Layout of filtered views kept for the backprojector. A pair layout has
// nv + 1 element rows per view; element e at column u holds the samples of
// detector rows e - 1 and e (zero outside the detector), so one
// shared-memory load yields both rows of a bilinear tap for v in [e-1, e).
enum FiltLayout : int {
  kLayoutRaw32 = 0,   // plain FP32 rows (unfiltered data, 2D staging)
  kLayoutPair32 = 1,  // float2 (8 bytes / sample), FP32 form
  kLayoutPair16 = 2,  // half2 (4 bytes / sample) with a per-view scale, MIXED form
  // Four views interleaved per detector element, for the four-fold symmetric
  // backprojector (MIXED form). Views k = g + s K/4 (s = 0..3) form group g;
  // element (g, e, c + 1) holds, for each slot s, the 2 x 2 neighbourhood of
  // rows e - 1, e and columns c, c + 1 as four FP16 values with the view's
  // scale: a, b - a, c' - a, d - c' - b + a (a = (e-1, c), b = (e, c),
  // c' = (e-1, c+1), d = (e, c+1); zero outside the detector). 32 bytes per
  // element, stored as two planes per element row (slots 0, 1 | slots 2, 3,
  // 16 bytes per column), so neighbouring columns are 16 bytes apart; a
  // bilinear tap is a + fu (c' - a) + fv ((b - a) + fu (...)).
  kLayoutQuadG16 = 3,
  // The same four-view gradient quantities (MIXED24 form) as 24-bit values:
  // an FP32 whose low byte is dropped on store and rebuilt on load as a copy
  // of its lowest stored byte; the pack picks the stored value whose rebuilt
  // float is nearest, so the error is that of rounding to 16 significant
  // bits. No scale (the FP32 exponent is kept). 4 slots x 4 values x 3 bytes
  // = 48 bytes per element, three 16-byte planes per element row.
  kLayoutQuadG24 = 4,
};

constexpr bool is_quad_layout(int layout) { return layout == kLayoutQuadG16 || layout == kLayoutQuadG24; }

// A stack of detector rows. Projections are [view][v][u] (rows ordered view
// major), sinograms [v][view][u] (rows ordered v major). Rows of u samples
// are padded to `pitch` elements so that every row starts 16-byte aligned.
// After filtering, the stack's content is the filtered buffer `filt` (in a
// pair layout) and f32 still holds the unfiltered input.
struct Stack {
  float* f32 = nullptr;
  int u = 0, v = 0, n = 0;
  int pitch = 0;  // f32 row pitch in elements (multiple of 4)
  bool sinogram = false;
  bool filtered = false;          // content lives in filt
  void* filt = nullptr;
  size_t filt_bytes = 0;
  int filt_layout = kLayoutPair32;
  int filt_pitch = 0;             // elements per row of filt (multiple of 4)
  float* inv_scale = nullptr;     // per view (x2: [inv | scale]) for the FP16 layouts
  int scale_cap = 0;              // views inv_scale has room for
  size_t f32_cap = 0;             // bytes allocated at f32 (buffers only grow: no cudaFree between jobs)
  bool pack_ready = false;        // filt already holds the packed FP16 views of f32 (slabs of one reconstruction)
  // Log normalisation and FDK weights recorded by their calls and applied
  // inside the filter kernel's load (log first, then weight), or by a
  // standalone pass when something else reads the rows first.
  bool log_pending = false;
  double log_base = 1.0;
  bool weights_pending = false;
  double w_sdd = 0, w_du = 0, w_dv = 0;
  double w_voff = 0;  // rows held are a band of a taller detector: centre offset in rows
  size_t rows() const { return (size_t)v * n; }
  size_t bytes32() const { return (size_t)pitch * rows() * sizeof(float); }
  static int elem_bytes(int layout) {
    return layout == kLayoutQuadG24 ? 48 : layout == kLayoutQuadG16 ? 32 : layout == kLayoutPair32 ? 8 : 4;
  }
  // element rows of the filtered buffer (pair layouts carry one extra row per view)
  size_t filt_rows() const { return (size_t)(v + 1) * n; }
};

struct FilterTables {
  int n = 0, filter = -1;
  int cap = 0;                // entries allocated (grow only: no cudaFree between jobs)
  float2* twiddle = nullptr;  // n/2 entries exp(-2 pi i k / n)
  float* hbr = nullptr;       // n entries H[bitrev(k)] / n
  float* kernel = nullptr;    // n entries: spatial kernel g = IDFT(H) (circular)
};

// Toeplitz operands of the tensor-core filter: Bt[i][k] = g[(i - k) mod n]
// for i < m, k < kp (zero for k >= m), as BF16 hi rows then BF16 lo rows.
struct ToeplitzTables {
  int m = 0, n = 0, filter = -1;
  void* th = nullptr;  // 2 * m * kp BF16 values, then 9 x m FP32 columns T P_j (row baseline basis)
  size_t cap = 0;      // bytes allocated at th (grow only)
};

}  // namespace fbp

// Backprojector window boxes: widths and heights per plan (a grid of
// kBoxGrid x kBoxGrid tensor maps), chosen from a histogram of the window
// sizes whose bins cover widths and heights below kBoxHist.
constexpr int kBoxGrid = 8;
constexpr int kBoxHist = 128;

struct fbp_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;
  int precision = FBP_PRECISION_FP32;
  int filter_impl = FBP_FILTER_IMPL_AUTO;
  int pad_len = 0;
  int clip_after_bp = 1;
  int bp_variant = FBP_BACKPROJECTOR_AUTO;
  int quad_tile_ny = 0;  // symmetric backprojector: voxels per thread along y (8 or 16; 0 = 16)
  int det_row_off = 0, det_rows_total = 0;  // fbp_set_detector_rows (0 rows: the whole detector)
  int slab_y0 = 0, slab_ny = 0;             // fbp_set_volume_slab (0 slices: the whole volume)
  int last_bp[5] = {-1, -1, 0, 0, 0};  // variant, layout, box_u, box_v, tile height of the last backprojection
  int bp_stages = 0;                    // generic backprojector: view ring stages (0: as many as fit, up to 8)
  int autotune = 0;                    // time the backprojector shapes per geometry on first use
  int device_cc = 0;                   // compute capability (major * 10 + minor), part of the tuning key
  static constexpr int kTuneKey = 23;  // geometry, form, layout, slab, GPU
  struct TuneShape {
    int variant = FBP_BACKPROJECTOR_AUTO;
    int quad_ny = 0;  // symmetric: voxels per thread along y
    int stages = 0;   // generic: view ring stages
  };
  struct TuneEntry {
    double key[kTuneKey];
    TuneShape shape;
    float ms = 0.f;
  };
  std::vector<TuneEntry> tuned;        // autotuner choices per geometry
  std::string tune_cache;              // file of tuning choices shared between processes ("" = none)
  bool tune_cache_loaded = false;
  int tune_timed = 0, tune_cached = 0; // geometries timed / taken from the choices known
  int num_sms = 148;
  unsigned long long launches = 0;  // kernels launched by this context

  float* vol = nullptr;
  int vx = 0, vy = 0, vz = 0;
  size_t vol_cap = 0;  // bytes allocated at vol

  fbp::Stack proj;
  fbp::Stack sino;

  int* d_err = nullptr;          // device error word
  int* d_minmax = nullptr;       // volume min / max as order-preserving int keys
  bool minmax_valid = false;     // d_minmax describes the current volume
  double2* d_trig = nullptr;     // per-view (cos, sin) in FP64
  int trig_cap = 0;
  double trig_key[3] = {-1, 0, 0};  // (views, span, offset) of the table in d_trig
  int* d_span = nullptr;         // footprint pre-pass results (spans + per-tile needs)
  size_t span_cap = 0;           // ints in d_span
  float* d_stage2d = nullptr;    // 2D sinograms restaged with 16-byte row pitch
  size_t stage2d_bytes = 0;
  fbp::FilterTables ftab;
  fbp::ToeplitzTables ttab;
  void* d_scratch = nullptr;     // generic scratch (row shifts, Toeplitz operands)
  size_t scratch_bytes = 0;
  void* h_pinned = nullptr;      // small pinned staging for per-call tables
  size_t h_pinned_bytes = 0;

  // cached backprojection plans: the largest detector window of any
  // (tile, view) for a geometry (samples, rows including row v + 1); several,
  // so that the slabs of a streamed reconstruction keep theirs
  struct BPPlan {
    bool valid = false;
    double key[20] = {0};
    int box_u = 0, box_v = 0;
    // window (width, height) counts over the (tile, view) pairs, kBoxHist^2,
    // and the box grid chosen from them for one layout and box limits
    std::vector<unsigned> hist;
    int sel_layout = -1, sel_u = 0, sel_v = 0;
    int sel_w[kBoxGrid] = {0}, sel_h[kBoxGrid] = {0};
  } plans[64];  // geometries seen by this context (a serving worker meets dozens)
  int plan_next = 0;
  cudaStream_t copy_stream = nullptr;  // slab readback beside the backprojection (created on first use)
  // batched backprojection launched from this context (grow only)
  void* d_batch = nullptr;             // job table, tensor maps and work counter
  size_t batch_cap = 0;
  void* h_batch = nullptr;             // pinned staging of the table
  size_t h_batch_cap = 0;
  cudaEvent_t ev_batch_copy = nullptr; // the staged table has gone up
  cudaEvent_t ev_sync = nullptr;       // cross-stream ordering of batched jobs
};

namespace fbp {

// ---- error helpers (fbp_api.cu) ----
int set_error(fbp_context* ctx, int code, const std::string& msg);
int cuda_check(fbp_context* ctx, cudaError_t e, const char* what);
// Error check after a kernel launch; counts the launch.
inline int launched(fbp_context* ctx, const char* what) {
  ctx->launches++;
  return cuda_check(ctx, cudaGetLastError(), what);
}
void* scratch(fbp_context* ctx, size_t bytes);

// ---- filter (fbp_filter.cu) ----
struct RowSet {
  float* data;          // f32 rows (input; also output when out16 == nullptr)
  long long pitch;      // elements
  long long rows;
  int m;                // samples per row
  // row -> (view, iv) for weights and per-view scales
  int n_views, n_v;
  bool sinogram;        // rows ordered v-major
  // optional fused pre-ops
  bool log_norm = false;
  float log_base = 1.f;
  bool weight = false;
  float w_sdd = 0, w_du = 0, w_dv = 0;
  float w_voff = 0;  // detector-centre offset of the rows (row band of a taller detector)
  // output: in place into `data` (out == nullptr) or into a pair layout
  void* out = nullptr;
  int out_layout = kLayoutRaw32;
  long long out_pitch = 0;            // elements
  const float* view_scale = nullptr;  // kLayoutPair16: values are multiplied by it before rounding
};
int ensure_filter_tables(fbp_context* ctx, int n, int filter);
int launch_filter_fft(fbp_context* ctx, const RowSet& rs, int n);
int launch_filter_toeplitz(fbp_context* ctx, const RowSet& rs, int n, int filter);
int launch_elementwise_pre(fbp_context* ctx, const RowSet& rs);  // weight / log-norm only
// Per-view scales for FP16 storage: scale = largest power of two with
// scale * max|row value of the view| <= limit; inv = 1 / scale.
int launch_view_scales(fbp_context* ctx, const RowSet& rs, float limit, float* view_scale, float* inv_scale);
// Pack the stack's f32 rows into a compact backprojector layout: kLayoutPair16
// with row pitch `pitch` elements or kLayoutQuadG16 (FP16 with the per-view
// scales view_scale), or kLayoutQuadG24 (24-bit, no scale).
int launch_pack(fbp_context* ctx, const Stack& s, int layout, void* out, long long pitch, const float* view_scale);
int launch_fft_rows(fbp_context* ctx, float2* data, int n, int rows, int inverse);
int launch_fft_shift_rows(fbp_context* ctx, float2* data, int n, int rows, int shift);
// Copy filtered rows [row0, row0 + nrows) of a pair layout back to FP32 rows.
// rows row0, row0 + row_step, ... (nrows of them) of the filtered buffer, as FP32 rows of dst
int launch_unpack_rows(fbp_context* ctx, const Stack& s, size_t row0, size_t nrows, float* dst, long long dst_pitch,
                       long long row_step = 1);
bool toeplitz_supported(int m);

// ---- backprojection (fbp_backproject.cu) ----
struct BPGeom {
  int kind;           // FBP_GEOMETRY_CONE / FBP_GEOMETRY_PARALLEL
  double sod, sdd;    // cone only
  double du, dv, vox;
  double span, offset;
  int nu, nv, nviews;
  int nx, ny, nz;
  // sharding: the stack holds detector rows [row_off, row_off + nv) of nv_total
  // rows, and the volume y-slices [y_off, y_off + ny) of ny_total (0: whole)
  int row_off = 0, nv_total = 0;
  int y_off = 0, ny_total = 0;
  int vol_ystride = 0;  // y-slices between z planes of the output (0: ny); a slab of a whole volume
};
// Backproject the stack's content (filt when filtered, else f32 rows). In
// the MIXED form (`mixed`) f32 content is first packed into the FP16 layout
// the selected kernel reads (prepare_packed); sums are FP32 in every form.
int launch_backproject(fbp_context* ctx, const BPGeom& g, Stack& st, float* vol, int clip_ylimit, bool mixed);
// The same in two steps: plan (footprint pass, packing, tensor maps; work on
// ctx's stream) and launch. Plans with the same non-zero batch key can also run
// together in one persistent launch on another context's stream.
struct BPLaunchPlan;
BPLaunchPlan* new_bp_plan();
void free_bp_plan(BPLaunchPlan* p);
int plan_backproject(fbp_context* ctx, const BPGeom& g, Stack& st, float* vol, int clip_ylimit, bool mixed,
                     BPLaunchPlan* plan);
int launch_bp_plan(fbp_context* ctx, const BPLaunchPlan& p);
long long bp_plan_batch_key(const BPLaunchPlan& p);
long long bp_plan_tiles(const BPLaunchPlan& p);  // work items (tile orbits x y-slabs) of a batchable plan
// Plan ctx's cone-beam FDK backprojection of its projections (pending
// weights / filter, the volume buffer, footprint pass, packing) in the
// reference API's geometry terms, without launching it (fbp_api.cu).
int plan_cone_projections(fbp_context* ctx, const fbp_geometry& g, int h, int v, BPLaunchPlan* plan);
// tile_begin / tile_end: the range of each job's tiles this launch computes
// (nullptr: all of them)
int launch_bp_batch(fbp_context* launcher, BPLaunchPlan* const* plans, int n, const long long* tile_begin = nullptr,
                    const long long* tile_end = nullptr);
// (fbp_api.cu) size the stack's packed buffer for `layout`, compute the
// per-view scales and pack the f32 rows into it.
int prepare_packed(fbp_context* ctx, Stack& s, int layout);
int launch_clip(fbp_context* ctx, float* vol, int nx, int ny, int nz, int y_limit);
// 2D backprojection (g.ny == 1) of filtered rows [views][pitch] into image
// [nz][nx]; FBP_ERR_UNSUPPORTED (nothing launched) when a tile's detector
// window could exceed 512 samples (the caller takes the general path).
int launch_bp2d(fbp_context* ctx, const BPGeom& g, const float* sino, long long pitch, float* image);
// Per-view FP64 (cos, sin) table of g's view set in ctx->d_trig.
int ensure_trig(fbp_context* ctx, const BPGeom& g);
int launch_rebin_fan(fbp_context* ctx, const float* fan, int bins, int views, const BPGeom& g,
                     float* par, int out_bins, double du_out);

// ---- volume post-processing (fbp_volume.cu) ----
// Order-preserving key of a float (int comparison == float comparison).
__device__ __forceinline__ int minmax_key(float f) {
  const int b = __float_as_int(f);
  return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ __forceinline__ float minmax_value(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }
// Warp-reduce (lo, hi) and fold it into the device pair mm (all 32 lanes call;
// a lane without values passes +inf / -inf; NaN is ignored).
__device__ __forceinline__ void fold_minmax(int* mm, float lo, float hi) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0 && lo <= hi) {
    atomicMin(mm, minmax_key(lo));
    atomicMax(mm + 1, minmax_key(hi));
  }
}
int launch_minmax_init(fbp_context* ctx, int* mm);
int launch_volume_minmax(fbp_context* ctx, const float* vol, long long n, int* mm);
// Rescale in place with the range from the device pair mm, or (mm == nullptr) from mn, mx.
int launch_normalize(fbp_context* ctx, float* vol, long long n, const int* mm, float mn, float mx);

// ---- forward projection (fbp_forward.cu) ----
int launch_forward(fbp_context* ctx, const float* vol, int nx, int ny, int nz, double vox, bool cone, double sod,
                   double sdd, double du, double dv, double span, double offset, int nu, int nv, int nviews,
                   float* out, long long pitch, bool sinogram);

// ---- file ingest / slice output (fbp_io.cu) ----
int projection_file_index(const std::string& path);  // -1 when the name carries no index
int read_projection_files(fbp_context* ctx, const char* directory, int fw, int fh, int channels, int bpc, int tw,
                          int th, int count, float* dst, long long pitch, bool sinogram);
int write_volume_files(fbp_context* ctx, const char* directory);

// ---- phantoms (fbp_phantom.cu) ----
int launch_project_ellipsoids(fbp_context* ctx, const double* d_ell, int count, const BPGeom& g,
                              float* out, int pitch);

// ---- TMA helpers ----
int make_tensor_map_3d(fbp_context* ctx, CUtensorMap* map, CUtensorMapDataType dtype, void* base,
                       const uint64_t dims[3], const uint64_t strides_bytes[2], const uint32_t box[3]);
int make_tensor_map_4d(fbp_context* ctx, CUtensorMap* map, CUtensorMapDataType dtype, void* base,
                       const uint64_t dims[4], const uint64_t strides_bytes[3], const uint32_t box[4]);
// 2D BF16 rows (inner x outer, row pitch in bytes) with 128-byte swizzle.
int make_tensor_map_2d_bf16_sw128(fbp_context* ctx, CUtensorMap* map, void* base, uint64_t inner, uint64_t outer,
                                  uint64_t pitch_bytes, uint32_t box_inner, uint32_t box_outer);

}  // namespace fbp
