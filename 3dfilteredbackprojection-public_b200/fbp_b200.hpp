// fbp_b200.hpp - header-only C++ drop-in for the reference's FBP3D / FBP2D /
// FFFT classes (furkanunsal42/3DFilteredBackProjection-Public:
// Source/FilteredBackProjection/FBP3D.h:16-170, FBP2D.h:8-72,
// Source/FastFourierTransformGPU/FastFourierTransformGPU.h:10-67) over the C
// ABI in include/fbp_b200.h.
//
// Method names and argument order are the reference's. GL textures become
// plain float pointers (host memory, or device memory with on_device = true)
// with the sizes of the buffers the object owns; the object owns its device
// buffers like the reference owns its textures, and is non-copyable
// (FBP3D.h:19). Non-zero status codes throw fbp::Error (the reference printed
// and ASSERTed).
#pragma once

#include <memory>
#include <stdexcept>
#include <string>

#include "fbp_b200.h"

namespace fbp {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& msg) : std::runtime_error(msg), status(status) {}
  int status;
};

inline void check(fbp_context* ctx, int status) {
  if (status != FBP_OK) throw Error(status, fbp_last_error(ctx));
}

class Context {
 public:
  explicit Context(int device = 0) {
    fbp_context* c = nullptr;
    int rc = fbp_create(&c, device);
    if (rc != FBP_OK) throw Error(rc, fbp_last_error(nullptr));
    ctx_.reset(c);
  }
  fbp_context* get() const { return ctx_.get(); }

 private:
  struct Del {
    void operator()(fbp_context* c) const { fbp_destroy(c); }
  };
  std::unique_ptr<fbp_context, Del> ctx_;
};

class FBP2D {
 public:
  enum FilterType {  // FBP2D.h:10-14 (+ HANN, RAMP_SAMPLED)
    RAM_LAK = FBP_FILTER_RAM_LAK,
    SHEPP_LOGAN = FBP_FILTER_SHEPP_LOGAN,
    COSINE = FBP_FILTER_COSINE,
    HANN = FBP_FILTER_HANN,
    RAMP_SAMPLED = FBP_FILTER_RAMP_SAMPLED,
  };

  explicit FBP2D(int device = 0) : owned_(std::make_shared<Context>(device)), ctx_(owned_->get()) {}
  explicit FBP2D(fbp_context* shared) : ctx_(shared) {}

  // Precision form of apply_filter: FBP_PRECISION_FP32 (FFT) or MIXED /
  // MIXED24 (tcgen05 split-BF16 Toeplitz product); no counterpart in the reference.
  void set_precision(int precision) { check(ctx_, fbp_set_precision(ctx_, precision)); }
  void set_filter_impl(int impl) { check(ctx_, fbp_set_filter_impl(ctx_, impl)); }
  // Weight (fan beam when fan_sdd > 0) and filter every row of a device
  // sinogram [views][bins] in place (FBP2D::apply_filter with the FFT calls
  // around it, FBP2D.cpp:124-144).
  void apply_filter(float* device_sinogram, int bins, int views, FilterType filter_type = RAM_LAK,
                    float fan_sdd = 0.f, float detector_width = 0.f) {
    check(ctx_, fbp2d_filter_sinogram(ctx_, device_sinogram, bins, views, filter_type, fan_sdd, detector_width));
  }
  // 2D backprojection into a device image [rows][cols] (FBP2D.cpp:96-122).
  void project_backward(const float* device_sinogram, int bins, int views, const fbp_geometry& geometry,
                        float* device_image, int cols, int rows) {
    check(ctx_, fbp2d_project_backward(ctx_, device_sinogram, bins, views, &geometry, device_image, cols, rows));
  }
  // FBP2D::project_backward(sinogram, out) with the reference's fixed
  // arguments (FBP2D.cpp:107-111): full_rotation_count 1.0, offset 0.006 rad,
  // detector width = image width * sqrt(2), volume width = image width.
  void project_backward(const float* device_sinogram, int bins, int views, float* device_image, int size) {
    fbp_geometry g{FBP_GEOMETRY_PARALLEL, 0.f, 0.f, size * 1.41421356f, (float)size, 1.0f, 0.006f};
    project_backward(device_sinogram, bins, views, g, device_image, size, size);
  }
  void parallelize_fan_beam_sinogram(const float* device_fan, int bins, int views, float* device_parallel,
                                     float xray_source_distance, float detector_panel_distance,
                                     float detector_width, float volume_width, float total_rotation_count) {
    fbp_geometry g{FBP_GEOMETRY_CONE, xray_source_distance, detector_panel_distance, detector_width, volume_width,
                   total_rotation_count, 0.f};
    // parallel detector width = volume width * sqrt(2) (FBP2D.cpp:49)
    check(ctx_, fbp2d_parallelize_fan_beam_sinogram(ctx_, device_fan, bins, views, &g, device_parallel, bins,
                                                    volume_width * 1.41421356f));
  }
  void synchronize() { check(ctx_, fbp_synchronize(ctx_)); }

 private:
  std::shared_ptr<Context> owned_;
  fbp_context* ctx_;
};

class FFFT {
 public:
  explicit FFFT(int device = 0) : owned_(std::make_shared<Context>(device)), ctx_(owned_->get()) {}
  explicit FFFT(fbp_context* shared) : ctx_(shared) {}
  // interleaved complex64 device rows [rows][n]
  void fft_radix2(float* rows, int n, int count) { check(ctx_, fbp_fft_rows(ctx_, rows, n, count, 0)); }
  void inverse_fft_radix2(float* rows, int n, int count) { check(ctx_, fbp_fft_rows(ctx_, rows, n, count, 1)); }
  void fft_shift(float* rows, int n, int count) { check(ctx_, fbp_fft_shift_rows(ctx_, rows, n, count, n / 2)); }
  void fft_shift(float* rows, int n, int count, int shift_amount) {
    check(ctx_, fbp_fft_shift_rows(ctx_, rows, n, count, shift_amount));
  }
  void inverse_fft_shift(float* rows, int n, int count) {
    check(ctx_, fbp_fft_shift_rows(ctx_, rows, n, count, -(n / 2)));
  }
  void inverse_fft_shift(float* rows, int n, int count, int shift_amount) {
    check(ctx_, fbp_fft_shift_rows(ctx_, rows, n, count, -shift_amount));
  }

 private:
  std::shared_ptr<Context> owned_;
  fbp_context* ctx_;
};

class FBP3D {
 public:
  FBP3D(const FBP3D& other) = delete;
  FBP3D& operator=(const FBP3D&) = delete;
  explicit FBP3D(int device = 0)
      : ctx_(std::make_shared<Context>(device)), fbp_solver(ctx_->get()), fft_solver(ctx_->get()) {}

  fbp_context* context() const { return ctx_->get(); }

  void generate_blank_volume(int x_size, int y_size, int z_size) {
    check(c(), fbp_generate_blank_volume(c(), x_size, y_size, z_size));
  }
  void generate_blank_projections(int x_size, int y_size, int projection_amount) {
    check(c(), fbp_generate_blank_projections(c(), x_size, y_size, projection_amount));
  }
  void generate_blank_sinograms(int x_size, int y_size, int projection_amount) {
    check(c(), fbp_generate_blank_sinograms(c(), x_size, y_size, projection_amount));
  }
  void free_volume() { check(c(), fbp_free_volume(c())); }
  // FBP3D.h: read_projections / read_projections_as_sinograms / write_volume (FBP3D.cpp:74-195)
  void read_projections(const std::string& upper_directory, int file_width, int file_height, int file_channel_count,
                        int byte_per_channel, int target_projection_width, int target_projection_height,
                        int projection_count) {
    check(c(), fbp_read_projections(c(), upper_directory.c_str(), file_width, file_height, file_channel_count,
                                    byte_per_channel, target_projection_width, target_projection_height,
                                    projection_count));
  }
  void read_projections_as_sinograms(const std::string& upper_directory, int file_width, int file_height,
                                     int file_channel_count, int byte_per_channel, int target_projection_width,
                                     int target_projection_height, int projection_count) {
    check(c(), fbp_read_projections_as_sinograms(c(), upper_directory.c_str(), file_width, file_height,
                                                 file_channel_count, byte_per_channel, target_projection_width,
                                                 target_projection_height, projection_count));
  }
  void write_volume(const std::string& upper_directory) { check(c(), fbp_write_volume(c(), upper_directory.c_str())); }
  void free_projections() { check(c(), fbp_free_projections(c())); }
  void free_sinograms() { check(c(), fbp_free_sinograms(c())); }

  // Replaces read_projections' decode + upload loop (FBP3D.cpp:74-124): the
  // caller decodes, this uploads [count][v][u].
  void upload_projections(const float* data, int u, int v, int count, bool on_device = false) {
    check(c(), fbp_upload_projections(c(), data, u, v, count, on_device));
  }
  void upload_sinograms(const float* data, int u, int v, int count, bool on_device = false) {
    check(c(), fbp_upload_sinograms(c(), data, u, v, count, on_device));
  }

  void log_normalize_projections(float base_value) { check(c(), fbp_log_normalize_projections(c(), base_value)); }
  void log_normalize_sinograms(float base_value) { check(c(), fbp_log_normalize_sinograms(c(), base_value)); }
  void apply_fdk_weights_to_projections(float xray_source_distance, float detector_panel_distance,
                                        float detector_width) {
    check(c(), fbp_apply_fdk_weights_to_projections(c(), xray_source_distance, detector_panel_distance,
                                                    detector_width));
  }
  void apply_fdk_weights_to_sinograms(float xray_source_distance, float detector_panel_distance,
                                      float detector_width) {
    check(c(), fbp_apply_fdk_weights_to_sinograms(c(), xray_source_distance, detector_panel_distance,
                                                  detector_width));
  }
  void apply_filter_to_projections(FBP2D::FilterType filter_type) {
    check(c(), fbp_apply_filter_to_projections(c(), filter_type));
  }
  void apply_filter_to_sinograms(FBP2D::FilterType filter_type) {
    check(c(), fbp_apply_filter_to_sinograms(c(), filter_type));
  }
  void clip_negatives_of_volume() { check(c(), fbp_clip_negatives_of_volume(c())); }
  void normalize_histogram() { check(c(), fbp_normalize_histogram(c())); }                       // FBP3D.h:81
  void normalize_histogram(float min_value, float max_value) {                                  // FBP3D.h:82
    check(c(), fbp_normalize_histogram_range(c(), min_value, max_value));
  }

  void project_backward_parallel_from_projections(float full_rotation_count, int volume_resolution_horizontal,
                                                  int volume_resolution_vertical, float rotation_offset_radian = 0.0f) {
    check(c(), fbp_project_backward_parallel_from_projections(c(), full_rotation_count, volume_resolution_horizontal,
                                                              volume_resolution_vertical, rotation_offset_radian));
  }
  void project_backward_cone_fdk_from_projections(float xray_source_distance, float detector_panel_distance,
                                                  float detector_width, float volume_width, float full_rotation_count,
                                                  int volume_resolution_horizontal, int volume_resolution_vertical,
                                                  float rotation_offset_radian = 0.0f) {
    check(c(), fbp_project_backward_cone_fdk_from_projections(
                   c(), xray_source_distance, detector_panel_distance, detector_width, volume_width,
                   full_rotation_count, volume_resolution_horizontal, volume_resolution_vertical,
                   rotation_offset_radian));
  }
  void project_backward_parallel_from_sinograms(float full_rotation_count, int volume_resolution_horizontal,
                                                int volume_resolution_vertical, float rotation_offset_radian = 0.0f) {
    check(c(), fbp_project_backward_parallel_from_sinograms(c(), full_rotation_count, volume_resolution_horizontal,
                                                            volume_resolution_vertical, rotation_offset_radian));
  }
  void project_backward_cone_fdk_from_sinograms(float xray_source_distance, float detector_panel_distance,
                                                float detector_width, float volume_width, float full_rotation_count,
                                                int volume_resolution_horizontal, int volume_resolution_vertical,
                                                float rotation_offset_radian = 0.0f) {
    check(c(), fbp_project_backward_cone_fdk_from_sinograms(
                   c(), xray_source_distance, detector_panel_distance, detector_width, volume_width,
                   full_rotation_count, volume_resolution_horizontal, volume_resolution_vertical,
                   rotation_offset_radian));
  }

  // slices: x -> [z][y], y -> [z][x], z -> [y][x]
  void load_volume_slice_x(int x_index, float* out, bool on_device = false) {
    check(c(), fbp_load_volume_slice_x(c(), x_index, out, on_device));
  }
  void load_volume_slice_y(int y_index, float* out, bool on_device = false) {
    check(c(), fbp_load_volume_slice_y(c(), y_index, out, on_device));
  }
  void load_volume_slice_z(int z_index, float* out, bool on_device = false) {
    check(c(), fbp_load_volume_slice_z(c(), z_index, out, on_device));
  }
  void store_volume_slice_x(const float* src, int x_index, bool on_device = false) {
    check(c(), fbp_store_volume_slice_x(c(), src, x_index, on_device));
  }
  void store_volume_slice_y(const float* src, int y_index, bool on_device = false) {
    check(c(), fbp_store_volume_slice_y(c(), src, y_index, on_device));
  }
  void store_volume_slice_z(const float* src, int z_index, bool on_device = false) {
    check(c(), fbp_store_volume_slice_z(c(), src, z_index, on_device));
  }
  void load_projection(int projection_index, float* out, bool on_device = false) {
    check(c(), fbp_load_projection(c(), projection_index, out, on_device));
  }
  void store_projection(const float* src, int projection_index, bool on_device = false) {
    check(c(), fbp_store_projection(c(), src, projection_index, on_device));
  }
  void load_sinogram(int y_index, float* out, bool on_device = false) {
    check(c(), fbp_load_sinogram(c(), y_index, out, on_device));
  }
  void store_sinogram(const float* src, int y_index, bool on_device = false) {
    check(c(), fbp_store_sinogram(c(), src, y_index, on_device));
  }
  // FBP3D.cpp:755-778: one [v][u] projection out of / into the sinogram stack
  void load_projection_from_sinograms(int projection_index, float* out, bool on_device = false) {
    check(c(), fbp_load_projection_from_sinograms(c(), projection_index, out, on_device));
  }
  void store_projection_to_sinograms(const float* src, int projection_index, bool on_device = false) {
    check(c(), fbp_store_projection_to_sinograms(c(), src, projection_index, on_device));
  }
  void read_volume(float* out, bool on_device = false) { check(c(), fbp_read_volume(c(), out, on_device)); }

  void set_precision(int precision) { check(c(), fbp_set_precision(c(), precision)); }
  void synchronize() { check(c(), fbp_synchronize(c())); }

 private:
  fbp_context* c() const { return ctx_->get(); }
  std::shared_ptr<Context> ctx_;

 public:
  // members named as in the reference (FBP3D.h:84-85), sharing the context
  FBP2D fbp_solver;
  FFFT fft_solver;
};

}  // namespace fbp
