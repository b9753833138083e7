// Device helpers shared by the row-filter kernels: fused pre-operations on
// load and stores into the backprojector's pair layouts.
#pragma once

#include "fbp_internal.h"

namespace fbp {

// The pending pre-operations (log normalisation, then FDK weight) on the raw
// sample x of row r, column i.
__device__ __forceinline__ float pre_op(const RowSet& rs, long long r, int i, float x) {
  if (rs.log_norm) {
    float y = fmaxf(x, 1e-30f * rs.log_base);
    x = -logf(y / rs.log_base);
  }
  if (rs.weight) {
    int iv = rs.sinogram ? (int)(r / rs.n_views) : (int)(r % rs.n_v);
    float u = (i + 0.5f - 0.5f * rs.m) * rs.w_du;
    float v = (iv + 0.5f - 0.5f * rs.n_v + rs.w_voff) * rs.w_dv;
    x *= rs.w_sdd * rsqrtf(rs.w_sdd * rs.w_sdd + u * u + v * v);
  }
  return x;
}

__device__ __forceinline__ float load_pre(const RowSet& rs, long long r, int i) {
  return pre_op(rs, r, i, rs.data[r * rs.pitch + i]);
}

__device__ __forceinline__ int row_view(const RowSet& rs, long long r) {
  return rs.sinogram ? (int)(r % rs.n_views) : (int)(r / rs.n_v);
}

// Write filtered sample i of row r: in place (FP32 rows) or into a pair
// layout of nv + 1 element rows per view, element e = (row e - 1, row e).
// Sample (view, iv) is the .x half of element iv + 1 and the .y half of
// element iv; row 0 also zeroes the .x half of element 0 and the last row
// the .y half of element nv.
__device__ __forceinline__ long long pair_row(const RowSet& rs, int view, int e) {
  return rs.sinogram ? (long long)e * rs.n_views + view : (long long)view * (rs.n_v + 1) + e;
}

__device__ __forceinline__ void store_row_sample(const RowSet& rs, long long r, int i, float y) {
  if (rs.out_layout == kLayoutRaw32) {
    rs.data[r * rs.pitch + i] = y;
    return;
  }
  const int iv = rs.sinogram ? (int)(r / rs.n_views) : (int)(r % rs.n_v);
  const int view = row_view(rs, r);
  const long long below = pair_row(rs, view, iv + 1) * rs.out_pitch + i;  // element iv + 1: .x
  const long long here = pair_row(rs, view, iv) * rs.out_pitch + i;       // element iv: .y
  if (rs.out_layout == kLayoutPair32) {
    float2* o = static_cast<float2*>(rs.out);
    o[below].x = y;
    o[here].y = y;
    if (iv == 0) o[here].x = 0.f;
    if (iv == rs.n_v - 1) o[below].y = 0.f;
  } else {
    __half2* o = static_cast<__half2*>(rs.out);
    const __half h = __float2half_rn(y * rs.view_scale[view]);
    const __half z = __float2half_rn(0.f);
    o[below].x = h;
    o[here].y = h;
    if (iv == 0) o[here].x = z;
    if (iv == rs.n_v - 1) o[below].y = z;
  }
}

}  // namespace fbp
