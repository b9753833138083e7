// Diagnostics: kernel-launch counter and a shared-memory bandwidth probe.
//
// The probe measures the device's shared-memory load bandwidth with
// conflict-free 32-bit loads (every lane of a warp reads a different bank,
// immediate offsets, four independent accumulators), on every SM at full
// occupancy. It is the roofline denominator of the backprojector, whose four
// bilinear taps per voxel-view update are shared-memory gathers.

#include "fbp_internal.h"

namespace fbp {
namespace {

constexpr int kProbeWords = 8192;  // 32 KB of shared memory per CTA

__device__ __forceinline__ float lds(uint32_t addr) {
  float v;
  asm volatile("ld.volatile.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}

__global__ void __launch_bounds__(256) smem_probe_kernel(int iters, float* sink) {
  __shared__ float buf[kProbeWords];
  for (int i = threadIdx.x; i < kProbeWords; i += blockDim.x) buf[i] = (float)(i & 7);
  __syncthreads();
  // lane l reads bank l; the 8 warps read different 128-byte lines; 16
  // volatile loads per iteration with immediate offsets
  const uint32_t base = (uint32_t)__cvta_generic_to_shared(buf) + 4u * ((threadIdx.x & 31) + ((threadIdx.x >> 5) << 5));
  float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int j = 0; j < 16; j += 4) {
      a0 += lds(base + (j + 0) * 2048);
      a1 += lds(base + (j + 1) * 2048);
      a2 += lds(base + (j + 2) * 2048);
      a3 += lds(base + (j + 3) * 2048);
    }
  }
  const float r = a0 + a1 + a2 + a3;
  if (r == -1.f) sink[threadIdx.x] = r;  // never true; keeps the sums live
}

}  // namespace
}  // namespace fbp

extern "C" {

int fbp_kernel_launch_count(const fbp_context* ctx, uint64_t* count) {
  if (!ctx || !count) return FBP_ERR_INVALID_ARGUMENT;
  *count = ctx->launches;
  return FBP_OK;
}

int fbp_measure_smem_bandwidth(fbp_context* ctx, double* bytes_per_second) {
  if (!ctx || !bytes_per_second) return FBP_ERR_INVALID_ARGUMENT;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  float* sink = static_cast<float*>(fbp::scratch(ctx, 4096));
  if (!sink) return FBP_ERR_OUT_OF_MEMORY;
  const int blocks = ctx->num_sms * 4, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fbp::smem_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(iters, sink);  // warm-up
  cudaEventRecord(e0, ctx->stream);
  const int reps = 5;
  for (int r = 0; r < reps; ++r) fbp::smem_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(iters, sink);
  cudaEventRecord(e1, ctx->stream);
  ctx->launches += 1 + reps;
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (prev >= 0) cudaSetDevice(prev);
  if (int rc = fbp::cuda_check(ctx, e != cudaSuccess ? e : cudaGetLastError(), "smem_probe_kernel")) return rc;
  const double bytes = (double)blocks * threads * iters * 16.0 * 4.0 * reps;
  *bytes_per_second = bytes / (ms * 1e-3);
  return FBP_OK;
}

}  // extern "C"
