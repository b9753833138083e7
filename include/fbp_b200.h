/*
 * fbp_b200.h - C ABI of the B200 CT reconstruction core (FDK cone-beam,
 * 3D parallel-beam, 2D parallel-beam and 2D flat-detector fan-beam FBP).
 *
 * Every entry point returns an int status (FBP_OK == 0) and never aborts;
 * fbp_last_error() gives the message of the last failure. Pointers passed in
 * are borrowed for the duration of the call only. A context owns its device
 * buffers (volume, projections, sinograms) the way class FBP3D owns its
 * textures (reference Source/FilteredBackProjection/FBP3D.h:87-89), is bound
 * to one CUDA device and one stream, and must be used from one host thread
 * at a time.
 *
 * Reference citations are paths inside furkanunsal42/3DFilteredBackProjection-Public.
 *
 * Conventions: volume buffers are x-fastest [z][y][x] with y the rotation
 * axis (reference Texture3D(h, v, h), FBP3D.cpp:531); projection stacks are
 * [view][v][u] (Texture2DArray(u, v, N), FBP3D.cpp:40); sinogram stacks are
 * [v][view][u] (Texture3D(u, N, v), FBP3D.cpp:54); 2D sinograms are
 * [view][bin] and 2D images [row][column].
 */
#ifndef FBP_B200_H
#define FBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define FBP_OK 0
#define FBP_ERR_INVALID_ARGUMENT (-1)
#define FBP_ERR_STATE (-2)        /* required buffer missing; the reference prints and ASSERTs (FBP3D.cpp:214-217) */
#define FBP_ERR_CUDA (-3)
#define FBP_ERR_OUT_OF_MEMORY (-4)
#define FBP_ERR_DEVICE_TIMEOUT (-5) /* a bounded device-side wait expired */
#define FBP_ERR_UNSUPPORTED (-6)
#define FBP_ERR_DEVICE_CHECK (-7)   /* a device-side bounds / footprint check failed */

/* ---- filter types: 0..2 keep the values of FBP2D::FilterType (FBP2D.h:10-14) */
#define FBP_FILTER_RAM_LAK 0
#define FBP_FILTER_SHEPP_LOGAN 1
#define FBP_FILTER_COSINE 2
#define FBP_FILTER_HANN 3
#define FBP_FILTER_RAMP_SAMPLED 4 /* |k|/n sampled in frequency (FastFourierTransformImage.cpp:35,45) */

/* ---- precision forms ------------------------------------------------------ */
/* FP32: FP32 FFT filter, FP32 filtered views, FP32 accumulation.           */
/* MIXED: split-BF16 tensor-core Toeplitz filter (FP32 accumulate), FP16    */
/*        filtered views with a per-view power-of-two scale, FP32            */
/*        accumulation.                                                      */
/* MIXED24: split-BF16 Toeplitz filter, 24-bit filtered views (FP32 with   */
/*        the low byte dropped: 16 significant bits, FP32 exponent) for the  */
/*        four-fold symmetric backprojector (FP32 views otherwise), FP32     */
/*        accumulation. 12 bytes of shared-memory gathers per update (FP32   */
/*        16, MIXED 8), for inputs whose noise leaves FP16 storage short of  */
/*        1e-4 relative error.                                              */
#define FBP_PRECISION_FP32 0
#define FBP_PRECISION_MIXED 1
#define FBP_PRECISION_MIXED24 2

/* ---- filter implementations ---------------------------------------------- */
#define FBP_FILTER_IMPL_AUTO 0     /* FFT for FP32, Toeplitz GEMM for MIXED */
#define FBP_FILTER_IMPL_FFT 1      /* batched shared-memory FFT             */
#define FBP_FILTER_IMPL_TOEPLITZ 2 /* tcgen05 split-BF16 Toeplitz GEMM       */

/* ---- backprojector variants ----------------------------------------------- */
#define FBP_BACKPROJECTOR_AUTO 0      /* symmetric when the geometry allows it      */
#define FBP_BACKPROJECTOR_GENERIC 1   /* one 16x16x16 tile per CTA, any geometry    */
#define FBP_BACKPROJECTOR_SYMMETRIC 2 /* four-fold orbit of tiles per CTA: square  */
                                      /* volume, views % 4 == 0 over one full turn */
#define FBP_BACKPROJECTOR_GENERIC_Y8 3 /* generic with 16x16x8 tiles (8 voxels per  */
                                       /* thread along y), any geometry            */

/* ---- geometry kinds ------------------------------------------------------- */
#define FBP_GEOMETRY_CONE 0     /* flat-panel cone beam, circular orbit         */
#define FBP_GEOMETRY_PARALLEL 1 /* parallel beam (3D: stacked 2D)               */

typedef struct fbp_context fbp_context;

/* Geometry of one backprojection, in the reference's terms
 * (FBP3D.h:58, FBP3D.cpp:536-552). Lengths in any unit (mm in the tests).
 *   source_distance    source to rotation axis (xray_source_distance, SOD)
 *   detector_distance  rotation axis to detector (detector_panel_distance);
 *                      SDD = source_distance + detector_distance
 *   detector_width     width of the nu detector columns; pixels are square
 *   volume_width       width of the nx voxels; voxels are isotropic
 *   views cover angles offset + 2*pi*full_rotation_count*k/K, k < K.
 * For FBP_GEOMETRY_PARALLEL the two distances are ignored. */
typedef struct fbp_geometry {
  int kind;
  float source_distance;
  float detector_distance;
  float detector_width;
  float volume_width;
  float full_rotation_count;
  float rotation_offset_radian;
} fbp_geometry;

/* ---- context ---------------------------------------------------------------
 * Replaces the FBP3D object (FBP3D.h:16-20): fbp_create ~ FBP3D(), which in
 * the reference compiles ~40 compute shaders in member initialisers. */
int fbp_create(fbp_context** ctx, int device);
int fbp_destroy(fbp_context* ctx);
/* Last error message of ctx (or of the calling thread when ctx is NULL). */
const char* fbp_last_error(const fbp_context* ctx);
/* Run all work of ctx on this cudaStream_t (NULL: the context's own stream). */
int fbp_set_stream(fbp_context* ctx, void* cuda_stream);
int fbp_synchronize(fbp_context* ctx);
int fbp_set_precision(fbp_context* ctx, int precision);
int fbp_set_filter_impl(fbp_context* ctx, int impl);
/* Padding of detector rows before filtering: 0 = the reference's next power
 * of two >= width (FastFourierTransformGPU.cpp:258-262, circular wrap-around
 * included), otherwise an explicit power of two >= width. */
int fbp_set_filter_padding(fbp_context* ctx, int padded_length);
/* 1 (default): project_backward_* end with clip_negatives_of_volume as the
 * reference does (FBP3D.cpp:489,521,558,592); 0: leave negatives. */
int fbp_set_clip_after_backprojection(fbp_context* ctx, int enable);
/* Backprojector variant (FBP_BACKPROJECTOR_*); AUTO by default. */
int fbp_set_backprojector(fbp_context* ctx, int variant);
/* 1: with the variant AUTO, the first backprojection of each geometry (form,
 * staged layout, detector band and volume slab included) times the
 * applicable kernels - symmetric, generic with 16 and with 8 voxels per
 * thread along y - on a central slab of up to 48 y-slices and keeps the
 * fastest for later calls of that geometry; 0 (default): AUTO picks the
 * symmetric kernel when the geometry allows it. No counterpart in the
 * reference, whose backprojection is one fixed shader. */
int fbp_set_autotune(fbp_context* ctx, int enable);
/* With autotuning on: the shapes the tuner times are the symmetric kernel
 * with 16 or 8 voxels per thread along y and the generic kernel with 16 or 8
 * voxels per thread, each with its full view ring or a 4-stage one. A cache
 * file (path; NULL or "" = none) keeps the choices across processes: they are
 * read from it on the first tuning and each new choice is appended as one
 * line (key of geometry, form, layout, slab and GPU; shape; time), so another
 * process with the same geometry takes the cached shape without timing. */
int fbp_set_autotune_cache(fbp_context* ctx, const char* path);
/* Geometries the tuner timed, and geometries whose shape came from the
 * choices already known (this context's or the cache file's). */
int fbp_autotune_stats(const fbp_context* ctx, int* timed, int* from_cache);
/* View ring stages of the generic backprojector (2..8; 0 = as many as fit). */
int fbp_set_view_ring(fbp_context* ctx, int stages);
/* Voxels per thread along y of the four-fold symmetric backprojector: 16
 * (one CTA per SM, 64 accumulators a thread) or 8 (two CTAs per SM); 0 (the
 * default) = 16. No counterpart in the reference. */
int fbp_set_symmetric_tile(fbp_context* ctx, int voxels_per_thread_y);
/* Device bytes held by ctx's buffers. */
int fbp_memory_in_use(const fbp_context* ctx, size_t* bytes);
/* What the last backprojection ran (no counterpart in the reference, whose
 * backprojection is one fixed shader): *variant = FBP_BACKPROJECTOR_GENERIC,
 * _GENERIC_Y8 or _SYMMETRIC; *layout = staged view layout (0 FP32 rows,
 * 1 FP32 row pairs, 2 FP16 row pairs, 3 FP16 four-view gradient quads,
 * 4 24-bit four-view gradient quads);
 * *box_u x *box_v = largest staged detector window in elements; *tile_ny =
 * voxels per thread along y. Any output pointer may be NULL. FBP_ERR_STATE
 * before the first backprojection. */
int fbp_last_backprojection(const fbp_context* ctx, int* variant, int* layout, int* box_u, int* box_v,
                            int* tile_ny);

/* ---- buffers (FBP3D.cpp:16-56, 197-210) ----------------------------------- */
int fbp_generate_blank_volume(fbp_context* ctx, int x_size, int y_size, int z_size);
int fbp_generate_blank_projections(fbp_context* ctx, int x_size, int y_size, int projection_amount);
int fbp_generate_blank_sinograms(fbp_context* ctx, int x_size, int y_size, int projection_amount);
int fbp_free_volume(fbp_context* ctx);
int fbp_free_projections(fbp_context* ctx);
int fbp_free_sinograms(fbp_context* ctx);
int fbp_get_volume_size(const fbp_context* ctx, int* x, int* y, int* z);
int fbp_get_projections_size(const fbp_context* ctx, int* u, int* v, int* count);
int fbp_get_sinograms_size(const fbp_context* ctx, int* u, int* v, int* count); /* u x v detector, count views */

/* ---- transfers --------------------------------------------------------------
 * `*_on_device` = 1: the pointer is device memory of ctx's device, else host
 * memory (pinned memory gives asynchronous copies). Host-memory transfers
 * are complete when the call returns. */
/* Whole stack [view][v][u]; (re)allocates the projections. Replaces the
 * per-batch upload + store_projection loop of read_projections
 * (FBP3D.cpp:105-118). */
int fbp_upload_projections(fbp_context* ctx, const float* src, int u, int v, int count, int src_on_device);
/* Whole stack [v][view][u]; (re)allocates the sinograms (FBP3D.cpp:126-176). */
int fbp_upload_sinograms(fbp_context* ctx, const float* src, int u, int v, int count, int src_on_device);
int fbp_download_projections(fbp_context* ctx, float* dst, int dst_on_device);
int fbp_download_sinograms(fbp_context* ctx, float* dst, int dst_on_device);
int fbp_store_projection(fbp_context* ctx, const float* src, int projection_index, int src_on_device); /* FBP3D.cpp:718-728 */
int fbp_load_projection(fbp_context* ctx, int projection_index, float* dst, int dst_on_device);      /* FBP3D.cpp:706-716 */
int fbp_store_sinogram(fbp_context* ctx, const float* src, int y_index, int src_on_device);           /* FBP3D.cpp:742-753 */
int fbp_load_sinogram(fbp_context* ctx, int y_index, float* dst, int dst_on_device);                  /* FBP3D.cpp:730-740 */
/* One projection [v][u] (view projection_index) gathered from / scattered into the
 * sinogram stack [v][view][u]; read_projections_as_sinograms stores each file this way
 * (FBP3D.cpp:167). */
int fbp_load_projection_from_sinograms(fbp_context* ctx, int projection_index, float* dst,
                                       int dst_on_device);                                             /* FBP3D.cpp:755-765 */
int fbp_store_projection_to_sinograms(fbp_context* ctx, const float* src, int projection_index,
                                      int src_on_device);                                              /* FBP3D.cpp:767-778 */
/* Slices of the volume: x-slice is [z][y], y-slice [z][x], z-slice [y][x]
 * (FBP3D.cpp:639-704). */
int fbp_load_volume_slice_x(fbp_context* ctx, int x_index, float* dst, int dst_on_device);
int fbp_load_volume_slice_y(fbp_context* ctx, int y_index, float* dst, int dst_on_device);
int fbp_load_volume_slice_z(fbp_context* ctx, int z_index, float* dst, int dst_on_device);
int fbp_store_volume_slice_x(fbp_context* ctx, const float* src, int x_index, int src_on_device);
int fbp_store_volume_slice_y(fbp_context* ctx, const float* src, int y_index, int src_on_device);
int fbp_store_volume_slice_z(fbp_context* ctx, const float* src, int z_index, int src_on_device);
/* Whole volume [z][y][x] (replaces the per-y-slice readback of write_volume,
 * FBP3D.cpp:178-195, without the file output). */
int fbp_read_volume(fbp_context* ctx, float* dst, int dst_on_device);
int fbp_write_volume_data(fbp_context* ctx, const float* src, int src_on_device);
/* Device pointers of ctx's buffers (valid until the buffer is reallocated or
 * freed). Projections may be row-padded: *row_pitch is in floats. */
int fbp_volume_device_ptr(fbp_context* ctx, float** ptr);
int fbp_projections_device_ptr(fbp_context* ctx, float** ptr, int* row_pitch);

/* ---- pipeline stages (FBP3D.cpp) ------------------------------------------- */
int fbp_log_normalize_projections(fbp_context* ctx, float base_value);                                 /* :333-349 */
int fbp_log_normalize_sinograms(fbp_context* ctx, float base_value);                                   /* :351-367 */
int fbp_apply_fdk_weights_to_projections(fbp_context* ctx, float xray_source_distance,
                                         float detector_panel_distance, float detector_width);         /* :369-387 */
int fbp_apply_fdk_weights_to_sinograms(fbp_context* ctx, float xray_source_distance,
                                       float detector_panel_distance, float detector_width);           /* FBP3D.h:53 */
int fbp_apply_filter_to_projections(fbp_context* ctx, int filter_type);                               /* :389-414 */
int fbp_apply_filter_to_sinograms(fbp_context* ctx, int filter_type);                                 /* :417-442 */
int fbp_clip_negatives_of_volume(fbp_context* ctx);                                                    /* :444-458 */
/* ---- forward projection (FBP3D.cpp:212-330, FBP2D.cpp:54-94) -----------------------------
 * Ray-driven: each detector pixel's ray (backprojector conventions) is clipped to the volume
 * box and cut into n = ceil(length / (voxel / 2)) equal steps; the trilinearly interpolated
 * volume (zero outside) is summed at the step midpoints times the step. As in the reference
 * the detector is sized like the volume (x columns, y rows) and the stack is (re)allocated;
 * parallel beam measures in voxels (detector width = volume width). */
int fbp_project_forward_cone_to_projections(fbp_context* ctx, float xray_source_distance,
                                            float detector_panel_distance, float detector_width, float volume_width,
                                            float full_rotation_count, int projection_count,
                                            float rotation_offset_radian);                  /* FBP3D.cpp:266-297 */
int fbp_project_forward_cone_to_sinograms(fbp_context* ctx, float xray_source_distance,
                                          float detector_panel_distance, float detector_width, float volume_width,
                                          float full_rotation_count, int projection_count,
                                          float rotation_offset_radian);                    /* FBP3D.cpp:299-330 */
int fbp_project_forward_parallel_to_projections(fbp_context* ctx, float full_rotation_count, int projection_count,
                                                float rotation_offset_radian);              /* FBP3D.cpp:212-238 */
int fbp_project_forward_parallel_to_sinograms(fbp_context* ctx, float full_rotation_count, int projection_count,
                                              float rotation_offset_radian);                /* FBP3D.cpp:240-264 */
/* FBP2D::project_forward (FBP2D.cpp:54-94) on caller device buffers: image [nz][nx] pixels
 * of volume_width/nx, sinogram [views][bins]; parallel beam, or flat-detector fan beam for
 * FBP_GEOMETRY_CONE. */
int fbp2d_project_forward(fbp_context* ctx, const float* image, int nx, int nz, float* sinogram, int bins, int views,
                          const fbp_geometry* geometry);

/* ---- sharding (no counterpart in the reference, which runs on one GL context) ----------
 * One volume over several GPUs without a collective on the data path: y-slab k of the
 * volume needs only the detector rows its voxels project to. fbp_plan_slabs splits
 * volume_v y-slices into `slabs` balanced slabs and writes, per slab, out[4k..4k+3] =
 * {y0, y1, row0, row1}: slices [y0, y1) and detector rows [row0, row1) (cone magnification
 * bound over every view, bilinear neighbour and one row of margin included). Host only.
 * On the rank of slab k: fbp_set_detector_rows(ctx, row0, detector_rows) declares that the
 * stacks hold that row band (the FDK weight and the backprojector use the global row), and
 * fbp_set_volume_slab(ctx, y0, y1 - y0) makes project_backward_* (called with the whole
 * volume's resolution) compute only those y-slices; the context's volume is the slab.
 * Offsets 0 and counts 0 restore the whole detector / volume. */
int fbp_plan_slabs(const fbp_geometry* geometry, int detector_cols, int detector_rows, int volume_h, int volume_v,
                   int slabs, int* out);
int fbp_set_detector_rows(fbp_context* ctx, int row_offset, int total_rows);
int fbp_set_volume_slab(fbp_context* ctx, int y_offset, int y_count);

/* ---- reconstruction server (no counterpart in the reference) --------------------------
 * Continuous batching of independent jobs on one GPU: `slots` worker threads, each with its
 * own context and CUDA stream; queued jobs start in arrival order as a slot and HBM budget
 * (hbm_budget_bytes, 0 = 80 % of the free memory) free up, looking up to 8 jobs past a head
 * that does not fit; a job larger than the budget runs alone. Jobs admitted together overlap
 * on the device, and each result equals the same job run alone. Slots keep their buffers
 * (grow only). Host buffers should be pinned so that copies overlap other jobs' kernels. */
#define FBP_JOB_CONE 0        /* FDK: input [views][det_rows][det_cols], output [vol_h][vol_v][vol_h] */
#define FBP_JOB_FAN2D 1       /* flat-detector fan FBP: input [views][det_cols], output [vol_h][vol_h] */
#define FBP_JOB_PARALLEL2D 2  /* parallel-beam FBP, same shapes as FAN2D */
#define FBP_JOB_HOST_WAIT 3   /* holds a slot and reserve_bytes for `views` microseconds (scheduler tests) */
typedef struct fbp_request {
  int kind;                /* FBP_JOB_* */
  int precision;           /* FBP_PRECISION_* */
  int filter_type;         /* FBP_FILTER_* */
  int clip;                /* cone: clip negatives after backprojection (the reference's default: 1) */
  fbp_geometry geometry;   /* cone: reference-API distances; 2D: detector_width, volume_width, turns */
  int det_cols, det_rows, views;
  int vol_h, vol_v;
  long long reserve_bytes; /* HBM working set to reserve; 0 = estimate from the sizes */
  const float* input;      /* host */
  float* output;           /* host */
} fbp_request;
typedef struct fbp_job_result {
  int status;                                      /* FBP_OK or the job's error code */
  double queued_ms, started_ms, finished_ms;       /* since the server was created */
  char error[128];
} fbp_job_result;
typedef struct fbp_server fbp_server;
int fbp_server_create(fbp_server** server, int device, size_t hbm_budget_bytes, int slots);
/* device < 0: no GPU, only FBP_JOB_HOST_WAIT jobs (tests of the scheduler). */
/* enable 1 (default): cone jobs' backprojections go through the server's
 * engine into the persistent multi-job backprojector (as in
 * fbp_project_backward_cone_fdk_batch), their tiles launched in chunks of
 * about chunk_updates voxel-view updates (<= 0: 6e10, about 20 ms) mixed
 * with the other waiting jobs' tiles; a cone job of more than 1e10
 * updates runs its own slab pipeline instead (volume readback under the
 * backprojection); 0: each job launches its own kernels. */
int fbp_server_set_batching(fbp_server* server, int enable, double chunk_updates);
/* With batching on, the cone jobs of at most max_updates voxel-view updates
 * go through the engine (<= 0: 1e10); larger ones run their own slab
 * pipelines. Independent jobs on their own streams already share the SMs
 * when their grids are small; the engine pays for jobs too small to fill
 * the GPU alone. No counterpart in the reference (one reconstruction per
 * GL context). */
int fbp_server_set_batch_limit(fbp_server* server, double max_updates);
/* Since the server was created: device time of the batched backprojection
 * launches (each launch timed on its stream, summed), host time the cone
 * jobs of the batching path spent in their uploads and volume readbacks
 * (summed over workers), batched launches, and jobs that took that path.
 * Any output pointer may be NULL. */
int fbp_server_stats(fbp_server* server, double* batch_gpu_ms, double* upload_ms, double* readback_ms,
                     long long* batch_launches, long long* batched_jobs);
int fbp_server_submit(fbp_server* server, const fbp_request* request, long long* ticket);
/* Blocks until the job ends; the ticket is consumed. A second caller waiting
 * on a ticket that another caller already waits on gets FBP_ERR_STATE; an
 * unknown (or consumed) ticket gives FBP_ERR_INVALID_ARGUMENT. */
int fbp_server_wait(fbp_server* server, long long ticket, fbp_job_result* result);
int fbp_server_destroy(fbp_server* server); /* runs the queued jobs, then stops */

/* ---- file I/O (FBP3D.cpp:74-195) -------------------------------------------------------
 * FBP3D::read_projections / read_projections_as_sinograms (FBP3D.cpp:74-176): allocate the
 * stack (target_width x target_height x projection_count) and fill it from the files of
 * `directory`. A file's projection index is the 4 characters before a 4-character extension
 * (FBP3D.cpp:97-104); other files are ignored; a missing index is an error. Each file is raw
 * file_width x file_height pixels of file_channel_count channels of byte_per_channel (1 or 2,
 * little endian) bytes; channel 0 is used, normalised by 255 / 65535, and resampled
 * bilinearly (pixel centres aligned, edges clamped) when the sizes differ. Host threads read
 * into pinned buffers overlapped with the device conversion. */
int fbp_read_projections(fbp_context* ctx, const char* directory, int file_width, int file_height,
                         int file_channel_count, int byte_per_channel, int target_width, int target_height,
                         int projection_count);
int fbp_read_projections_as_sinograms(fbp_context* ctx, const char* directory, int file_width, int file_height,
                                      int file_channel_count, int byte_per_channel, int target_width,
                                      int target_height, int projection_count);
/* FBP3D::write_volume (FBP3D.cpp:178-195): one raw uint16 file per y-slice (x fastest, then z),
 * round(clamp(v, 0, 1) * 65535), named directory + "/CTAnalyzer_Slice#" + 6-digit index + ".raw"
 * (the reference always appends the separator). */
int fbp_write_volume(fbp_context* ctx, const char* directory);
/* The projection index a file name carries under the read_projections rule, or -1 (host only). */
int fbp_projection_file_index(const char* path);

/* Volume extremes, FBP3D::compute_min_value_of_volume / compute_max_value_of_volume
 * (FBP3D.cpp:780-800): NaN ignored; 0, 0 for a volume without finite values. */
int fbp_volume_min_max(fbp_context* ctx, float* min_value, float* max_value);
/* FBP3D::normalize_histogram() (FBP3D.cpp:802-815): v' = (v - min) / (max - min) over the
 * volume's extremes, in FP32 (0 everywhere when max <= min). The range stays on the device;
 * right after a backprojection it comes from the backprojector's store epilogue. */
int fbp_normalize_histogram(fbp_context* ctx);
/* FBP3D::normalize_histogram(min texture, max texture) (FBP3D.cpp:817-826): given range. */
int fbp_normalize_histogram_range(fbp_context* ctx, float min_value, float max_value);
int fbp_project_backward_cone_fdk_from_projections(fbp_context* ctx, float xray_source_distance,
    float detector_panel_distance, float detector_width, float volume_width, float full_rotation_count,
    int volume_resolution_horizontal, int volume_resolution_vertical, float rotation_offset_radian);  /* :524-559 */
int fbp_project_backward_cone_fdk_from_sinograms(fbp_context* ctx, float xray_source_distance,
    float detector_panel_distance, float detector_width, float volume_width, float full_rotation_count,
    int volume_resolution_horizontal, int volume_resolution_vertical, float rotation_offset_radian);  /* :561-593 */
int fbp_project_backward_parallel_from_projections(fbp_context* ctx, float full_rotation_count,
    int volume_resolution_horizontal, int volume_resolution_vertical, float rotation_offset_radian);  /* :460-490 */
int fbp_project_backward_parallel_from_sinograms(fbp_context* ctx, float full_rotation_count,
    int volume_resolution_horizontal, int volume_resolution_vertical, float rotation_offset_radian);  /* :492-522 */
/* Several cone-beam FDK backprojections at once (no counterpart in the
 * reference, one reconstruction per GL context): for each i, what
 * fbp_project_backward_cone_fdk_from_projections(contexts[i], geometries[i]...,
 * volume_h[i], volume_v[i]) computes - pending weights / log and the filter,
 * each job's clip setting and precision form - but the jobs that run the
 * four-fold symmetric backprojector with the same staged layout share ONE
 * persistent launch on `launcher`'s stream: OCC CTAs per SM take (job, tile
 * orbit, y-slab) work items from a device-side queue, so jobs of uneven size
 * (volume, detector, views) fill the GPU together and small jobs use the SMs
 * that a large job's last tiles leave idle. Each job's volume is bit-identical
 * to the same job batched with any others or alone. Other jobs launch on their
 * own streams. Asynchronous: each context's later work is ordered after the
 * batch. A device-side wait that expires in the batched launch is reported by
 * the launcher; geometry checks by the job's context. All contexts on one
 * device; the launcher may be one of them. */
int fbp_project_backward_cone_fdk_batch(fbp_context* const* contexts, const fbp_geometry* geometries,
                                        const int* volume_h, const int* volume_v, int count, fbp_context* launcher);
/* One call for the whole cone-beam FDK (weight + filter + backprojection +
 * optional clip) on the resident projections, geometry as above. */
int fbp_reconstruct_fdk(fbp_context* ctx, const fbp_geometry* geometry, int filter_type,
                        int volume_resolution_horizontal, int volume_resolution_vertical);
/* Host buffers in, host volume out, overlapped (no counterpart in the reference): upload the
 * [count][rows][cols] projections (pinned host memory recommended), FDK weights (cone),
 * filter, then backproject the volume in `slabs` y-ranges (1..64) written straight into the
 * context's h x v x h volume, each slab copied to `volume` ([z][y][x], host) on a second
 * stream while the next slab computes. Returns when `volume` is complete. */
int fbp_reconstruct_fdk_to_host(fbp_context* ctx, const float* projections, int cols, int rows, int count,
                                const fbp_geometry* geometry, int filter_type, int h, int v, float* volume,
                                int slabs);

/* ---- 2D (FBP2D.h:17-41) on caller-owned device buffers ---------------------
 * sinogram [views][bins], image [rows][cols]; filtered in place. */
/* Weight (fan: SDD/sqrt(SDD^2+u^2)) and filter every row; fan_sdd <= 0 means
 * parallel beam (no weight). Combines FBP2D::apply_filter on the shifted
 * spectrum with the surrounding FFFT calls (Mains/fbp_parallel2d_main.cpp:31-41).
 * The context's filter implementation / precision choose the arithmetic as for
 * the 3D stacks: the FP32 FFT, or (MIXED, MIXED24, or FBP_FILTER_IMPL_TOEPLITZ)
 * the tcgen05 split-BF16 Toeplitz product, which needs 64 <= bins <= 8192. */
int fbp2d_filter_sinogram(fbp_context* ctx, float* sinogram, int bins, int views, int filter_type,
                          float fan_sdd, float detector_width);
/* The same filtering without a context and without allocating device memory,
 * for callers that must not allocate while they run (hosts that own all GPU
 * memory through their own pool, real-time read-out loops where an
 * allocation would synchronise the device, plugin hosts that forbid it).
 * No counterpart in the reference. Runs on the current device and the given
 * cudaStream_t (NULL: the legacy default stream); its tables live in an
 * 80 KiB file-scope device array, so padded_length (0: next power of two >=
 * bins) may be at most 4096 - longer rows are rejected with
 * FBP_ERR_UNSUPPORTED. Every call looks up that array's device address in
 * the current context; the first call on a device also loads the library's
 * device code there, so make it before any stream capture. All calls share
 * the array: calls whose work overlaps on the GPU race and must be
 * serialised. A CUDA error pending from the caller's earlier work is
 * reported (and cleared) before any launch. Errors are reported through
 * fbp_last_error(NULL). */
int fbp2d_filter_sinogram_noalloc(float* sinogram, int bins, int views, int filter_type, float fan_sdd,
                                  float detector_width, int padded_length, void* cuda_stream);
/* 2D backprojection (FBP2D.cpp:96-122 for parallel beam; flat-detector fan
 * beam for FBP_GEOMETRY_CONE). image has cols x rows = nx x nz pixels of
 * size volume_width/nx. */
int fbp2d_project_backward(fbp_context* ctx, const float* sinogram, int bins, int views,
                           const fbp_geometry* geometry, float* image, int nx, int nz);
/* Fan (flat detector) -> parallel sinogram rebinning (FBP2D.cpp:31-52).
 * Output has out_bins bins of pitch out_detector_width/out_bins and the same
 * number of views. */
int fbp2d_parallelize_fan_beam_sinogram(fbp_context* ctx, const float* fan, int bins, int views,
                                        const fbp_geometry* geometry, float* parallel, int out_bins,
                                        float out_detector_width);

/* ---- GPU FFT over rows (FastFourierTransformGPU.h:13-48) -------------------
 * Interleaved complex64 rows [rows][n], n a power of two <= 4096. */
int fbp_fft_rows(fbp_context* ctx, float* complex_rows, int n, int rows, int inverse);
int fbp_fft_shift_rows(fbp_context* ctx, float* complex_rows, int n, int rows, int shift_amount);

/* ---- analytic phantom projections (test/bench input generator) -------------
 * Line integrals of ellipsoids (rows of 16 doubles: density, semi-axes a b c,
 * centre x y z, 3x3 rotation row-major whose columns are the axes) through
 * the cone geometry, FP64 arithmetic, written as FP32 into the resident
 * projections (which must already be allocated with u, v, count). Replaces
 * render_ellipsoid + project_forward_cone_to_projections (FBP3D.cpp:609-628,
 * 269-299) for generating inputs. */
int fbp_project_ellipsoids_to_projections(fbp_context* ctx, const double* ellipsoids, int count,
                                          const fbp_geometry* geometry);

/* ---- diagnostics --------------------------------------------------------- */
/* Number of kernels ctx has launched since it was created. */
int fbp_kernel_launch_count(const fbp_context* ctx, uint64_t* count);
/* Measured shared-memory load bandwidth of the device (bytes/s, all SMs,
 * conflict-free 32-bit loads): the roofline denominator of the
 * backprojector, whose bilinear taps are shared-memory gathers. */
int fbp_measure_smem_bandwidth(fbp_context* ctx, double* bytes_per_second);

#ifdef __cplusplus
}
#endif

#endif /* FBP_B200_H */
