// Volume post-processing: min / max of the volume and histogram
// normalisation, FBP3D::compute_min_value_of_volume /
// compute_max_value_of_volume / normalize_histogram
// (Source/FilteredBackProjection/FBP3D.cpp:780-826). The reference keeps the
// extremes in R32UI textures and rescales in a shader that it does not ship;
// here v' = (v - min) / (max - min) in FP32 (0 everywhere when max <= min).
//
// The extremes are kept on the device as a pair of order-preserving integer
// keys (int compare == float compare, NaN ignored). The backprojector folds
// the values it stores into the same pair, so normalising a fresh
// reconstruction needs no reduction pass; the normalise kernel reads the pair
// itself (no host round trip).

#include "fbp_internal.h"

#include <algorithm>
#include <climits>

namespace fbp {
namespace {

__global__ void minmax_init_kernel(int* mm) {
  mm[0] = INT_MAX;
  mm[1] = INT_MIN;
}

__global__ void __launch_bounds__(256) minmax_reduce_kernel(const float* __restrict__ v, long long n, int* mm) {
  float lo = __int_as_float(0x7f800000), hi = -lo;  // +inf, -inf
  const long long n4 = n >> 2;
  const float4* v4 = reinterpret_cast<const float4*>(v);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
    const float4 q = __ldg(v4 + i);
    lo = fminf(fminf(lo, q.x), fminf(q.y, fminf(q.z, q.w)));
    hi = fmaxf(fmaxf(hi, q.x), fmaxf(q.y, fmaxf(q.z, q.w)));
  }
  for (long long i = (n4 << 2) + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    lo = fminf(lo, v[i]);
    hi = fmaxf(hi, v[i]);
  }
  fold_minmax(mm, lo, hi);
}

// v' = (v - min) / (max - min); the range comes from the device pair (mm) or
// from the arguments.
__global__ void __launch_bounds__(256) normalize_kernel(float* __restrict__ v, long long n, const int* mm, float mn,
                                                        float mx) {
  if (mm) {
    mn = minmax_value(mm[0]);
    mx = minmax_value(mm[1]);
  }
  const float range = mx - mn;
  const bool flat = !(range > 0.f);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long n4 = n >> 2;
  float4* v4 = reinterpret_cast<float4*>(v);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
    float4 q = v4[i];
    q.x = flat ? 0.f : __fdiv_rn(q.x - mn, range);
    q.y = flat ? 0.f : __fdiv_rn(q.y - mn, range);
    q.z = flat ? 0.f : __fdiv_rn(q.z - mn, range);
    q.w = flat ? 0.f : __fdiv_rn(q.w - mn, range);
    v4[i] = q;
  }
  for (long long i = (n4 << 2) + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
    v[i] = flat ? 0.f : __fdiv_rn(v[i] - mn, range);
}

int grid_for_n(fbp_context* ctx, long long n) {
  const long long b = ((n >> 2) + 255) / 256;
  return (int)std::max(1LL, std::min(b, (long long)ctx->num_sms * 8));
}

}  // namespace

int launch_minmax_init(fbp_context* ctx, int* mm) {
  minmax_init_kernel<<<1, 1, 0, ctx->stream>>>(mm);
  return launched(ctx, "minmax_init_kernel");
}

int launch_volume_minmax(fbp_context* ctx, const float* vol, long long n, int* mm) {
  if (int rc = launch_minmax_init(ctx, mm)) return rc;
  minmax_reduce_kernel<<<grid_for_n(ctx, n), 256, 0, ctx->stream>>>(vol, n, mm);
  return launched(ctx, "minmax_reduce_kernel");
}

int launch_normalize(fbp_context* ctx, float* vol, long long n, const int* mm, float mn, float mx) {
  normalize_kernel<<<grid_for_n(ctx, n), 256, 0, ctx->stream>>>(vol, n, mm, mn, mx);
  return launched(ctx, "normalize_kernel");
}

}  // namespace fbp
