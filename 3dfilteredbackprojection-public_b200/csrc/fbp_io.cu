// File ingest and slice output: FBP3D::read_projections,
// read_projections_as_sinograms and write_volume
// (Source/FilteredBackProjection/FBP3D.cpp:74-195).
//
// Reading. Every file of the directory whose name has at least 8 characters
// names its projection index by the 4 characters before a 4-character
// extension ("...0123.raw"), as the reference parses it (FBP3D.cpp:97-104);
// files whose index does not parse or is out of range are ignored, and a
// missing index is an error (the reference would load an empty path). A file
// holds file_width x file_height pixels of file_channel_count channels of
// byte_per_channel bytes (1 or 2, little endian), rows in file order; the
// first channel is used and normalised like the reference's UNSIGNED_SHORT /
// UNSIGNED_BYTE texture upload (v / 65535, v / 255). When the file size
// differs from the target size the image is resampled bilinearly (pixel
// centres aligned, edges clamped); the reference's Image::resize comes from
// its absent GraphicsCortex library, so this resampling is this library's
// definition.
//
// Pipeline: host threads read batches of files into one of two pinned
// buffers; each batch is copied to the device asynchronously and one kernel
// converts and resamples it straight into the projection (or sinogram)
// stack, while the threads read the next batch into the other buffer.
//
// Writing. One file per y-slice (x fastest, then z), the reference's
// "CTAnalyzer_Slice#" + 6-digit index + ".raw" names (FBP3D.cpp:185-193), as
// GL's float -> normalised unsigned short conversion: round(clamp(v, 0, 1) x
// 65535). The reference always appends '/' to the directory (its check at
// FBP3D.cpp:183 is always true); so does this. Slices are converted on the GPU
// in batches and written by host threads while the next batch converts.

#include "fbp_internal.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <filesystem>
#include <string>
#include <thread>
#include <vector>

namespace fbp {
namespace {

struct IngestArgs {
  const unsigned char* raw;  // batch of files, file_bytes apart
  long long file_bytes;
  int fw, fh, channels, bpc;
  int tw, th;
  int first, count;          // projection indices of this batch
  float* dst;                // stack rows
  long long pitch;           // floats per row
  bool sinogram;             // rows ordered [v][view]
  int nviews;
  float rx, ry;              // file pixels per target pixel
};

__device__ __forceinline__ float texel(const IngestArgs& a, const unsigned char* f, int x, int y) {
  const long long o = ((long long)y * a.fw + x) * a.channels * a.bpc;
  if (a.bpc == 2) return __fdiv_rn((float)(f[o] | (f[o + 1] << 8)), 65535.f);
  return __fdiv_rn((float)f[o], 255.f);
}

__global__ void ingest_kernel(IngestArgs a) {
  const long long per = (long long)a.tw * a.th;
  const long long total = per * a.count;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t / per);
    const int r = (int)(t - (long long)k * per);
    const int v = r / a.tw, u = r - v * a.tw;
    const unsigned char* f = a.raw + (long long)k * a.file_bytes;
    float val;
    if (a.fw == a.tw && a.fh == a.th) {
      val = texel(a, f, u, v);
    } else {
      const float sx = fminf(fmaxf(__fsub_rn(__fmul_rn((float)u + 0.5f, a.rx), 0.5f), 0.f), (float)(a.fw - 1));
      const float sy = fminf(fmaxf(__fsub_rn(__fmul_rn((float)v + 0.5f, a.ry), 0.5f), 0.f), (float)(a.fh - 1));
      const int x0 = (int)sx, y0 = (int)sy;
      const int x1 = min(x0 + 1, a.fw - 1), y1 = min(y0 + 1, a.fh - 1);
      const float ax = sx - (float)x0, ay = sy - (float)y0;
      const float top = __fadd_rn(__fmul_rn(1.f - ax, texel(a, f, x0, y0)), __fmul_rn(ax, texel(a, f, x1, y0)));
      const float bot = __fadd_rn(__fmul_rn(1.f - ax, texel(a, f, x0, y1)), __fmul_rn(ax, texel(a, f, x1, y1)));
      val = __fadd_rn(__fmul_rn(1.f - ay, top), __fmul_rn(ay, bot));
    }
    const int view = a.first + k;
    const long long row = a.sinogram ? (long long)v * a.nviews + view : (long long)view * a.th + v;
    a.dst[row * a.pitch + u] = val;
  }
}

// y-slices [y0, y0 + ns) of a [z][y][x] volume -> uint16 slices [s][z][x]
__global__ void slices_u16_kernel(const float* vol, int nx, int ny, int nz, int y0, int ns, unsigned short* out) {
  const long long per = (long long)nx * nz;
  const long long total = per * ns;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t / per);
    const long long r = t - (long long)s * per;
    const int z = (int)(r / nx), x = (int)(r - (long long)z * nx);
    const float v = fminf(fmaxf(vol[((long long)z * ny + (y0 + s)) * nx + x], 0.f), 1.f);
    out[t] = (unsigned short)__float2uint_rn(__fmul_rn(v, 65535.f));
  }
}

// Run fn(i) for i in [0, n) on up to `threads` host threads.
template <class F>
void parallel_for(int n, int threads, F fn) {
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  const int nt = std::max(1, std::min(threads, n));
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&] {
      for (int i = next++; i < n; i = next++) fn(i);
    });
  for (auto& th : pool) th.join();
}

int host_threads() { return (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency())); }

}  // namespace

int projection_file_index(const std::string& path) {
  if (path.size() < 8) return -1;
  const std::string digits = path.substr(path.size() - 8, 4);
  int v = 0, used = 0;
  for (char ch : digits) {
    if (ch < '0' || ch > '9') break;
    v = v * 10 + (ch - '0');
    ++used;
  }
  return used ? v : -1;
}

int read_projection_files(fbp_context* ctx, const char* directory, int fw, int fh, int channels, int bpc, int tw,
                          int th, int count, float* dst, long long pitch, bool sinogram) {
  namespace fs = std::filesystem;
  std::error_code ec;
  if (!directory || !fs::is_directory(fs::path(directory), ec))
    return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, std::string("projection directory \"") +
                                                      (directory ? directory : "(null)") + "\" doesn't exist");
  if (fw <= 0 || fh <= 0 || channels <= 0 || (bpc != 1 && bpc != 2) || tw <= 0 || th <= 0 || count <= 0)
    return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "bad file or target dimensions (byte_per_channel must be 1 or 2)");
  std::vector<std::string> files(count);
  for (const auto& entry : fs::directory_iterator(fs::path(directory), ec)) {
    const std::string p = entry.path().string();
    const int idx = projection_file_index(p);
    if (idx >= 0 && idx < count) files[idx] = p;
  }
  for (int i = 0; i < count; ++i)
    if (files[i].empty())
      return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "no projection file for index " + std::to_string(i));

  const long long fbytes = (long long)fw * fh * channels * bpc;
  const int batch = (int)std::max(1LL, std::min<long long>(count, (256LL << 20) / fbytes));
  unsigned char* pinned[2] = {nullptr, nullptr};
  unsigned char* staging = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr};
  int rc = FBP_OK;
  auto cleanup = [&] {
    cudaStreamSynchronize(ctx->stream);
    for (int b = 0; b < 2; ++b) {
      cudaFreeHost(pinned[b]);
      if (copied[b]) cudaEventDestroy(copied[b]);
    }
    cudaFree(staging);
  };
  const size_t bbytes = (size_t)batch * fbytes;
  if (cuda_check(ctx, cudaMallocHost(&pinned[0], bbytes), "cudaMallocHost(ingest)") ||
      cuda_check(ctx, cudaMallocHost(&pinned[1], bbytes), "cudaMallocHost(ingest)") ||
      cuda_check(ctx, cudaMalloc(&staging, 2 * bbytes), "cudaMalloc(ingest staging)") ||
      cuda_check(ctx, cudaEventCreateWithFlags(&copied[0], cudaEventDisableTiming), "event") ||
      cuda_check(ctx, cudaEventCreateWithFlags(&copied[1], cudaEventDisableTiming), "event")) {
    cleanup();
    return FBP_ERR_OUT_OF_MEMORY;
  }
  for (int b0 = 0, slot = 0; b0 < count && rc == FBP_OK; b0 += batch, slot ^= 1) {
    const int n = std::min(batch, count - b0);
    // the pinned buffer is free once its previous copy has completed
    if ((rc = cuda_check(ctx, cudaEventSynchronize(copied[slot]), "ingest buffer wait"))) break;
    std::atomic<bool> failed{false};
    parallel_for(n, host_threads(), [&](int i) {
      FILE* f = std::fopen(files[b0 + i].c_str(), "rb");
      const size_t got = f ? std::fread(pinned[slot] + (size_t)i * fbytes, 1, (size_t)fbytes, f) : 0;
      if (f) std::fclose(f);
      if (got != (size_t)fbytes) failed = true;
    });
    if (failed) {
      rc = set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "a projection file is shorter than " + std::to_string(fbytes) +
                                                        " bytes or unreadable (batch from index " + std::to_string(b0) + ")");
      break;
    }
    unsigned char* dev = staging + (size_t)slot * bbytes;
    if ((rc = cuda_check(ctx, cudaMemcpyAsync(dev, pinned[slot], (size_t)n * fbytes, cudaMemcpyHostToDevice, ctx->stream),
                         "ingest copy")))
      break;
    if ((rc = cuda_check(ctx, cudaEventRecord(copied[slot], ctx->stream), "event"))) break;
    IngestArgs a;
    a.raw = dev;
    a.file_bytes = fbytes;
    a.fw = fw;
    a.fh = fh;
    a.channels = channels;
    a.bpc = bpc;
    a.tw = tw;
    a.th = th;
    a.first = b0;
    a.count = n;
    a.dst = dst;
    a.pitch = pitch;
    a.sinogram = sinogram;
    a.nviews = count;
    a.rx = (float)fw / (float)tw;
    a.ry = (float)fh / (float)th;
    const long long work = (long long)tw * th * n;
    const int blocks = (int)std::max(1LL, std::min<long long>((work + 255) / 256, (long long)ctx->num_sms * 16));
    ingest_kernel<<<blocks, 256, 0, ctx->stream>>>(a);
    if ((rc = launched(ctx, "ingest_kernel"))) break;
  }
  cleanup();
  return rc;
}

int write_volume_files(fbp_context* ctx, const char* directory) {
  if (!directory || !*directory) return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "empty directory");
  const int nx = ctx->vx, ny = ctx->vy, nz = ctx->vz;
  std::string dir(directory);
  dir.push_back('/');  // the reference always appends a separator (FBP3D.cpp:183)
  const long long sbytes = (long long)nx * nz * 2;
  const int batch = (int)std::max(1LL, std::min<long long>(ny, (128LL << 20) / sbytes));
  unsigned short* pinned[2] = {nullptr, nullptr};
  unsigned short* dev = nullptr;
  auto cleanup = [&] {
    cudaStreamSynchronize(ctx->stream);
    cudaFreeHost(pinned[0]);
    cudaFreeHost(pinned[1]);
    cudaFree(dev);
  };
  const size_t bbytes = (size_t)batch * sbytes;
  if (cuda_check(ctx, cudaMallocHost(&pinned[0], bbytes), "cudaMallocHost(slices)") ||
      cuda_check(ctx, cudaMallocHost(&pinned[1], bbytes), "cudaMallocHost(slices)") ||
      cuda_check(ctx, cudaMalloc(&dev, 2 * bbytes), "cudaMalloc(slices)")) {
    cleanup();
    return FBP_ERR_OUT_OF_MEMORY;
  }
  int rc = FBP_OK;
  std::thread writer;
  std::atomic<bool> write_failed{false};
  for (int y0 = 0, slot = 0; y0 < ny && rc == FBP_OK; y0 += batch, slot ^= 1) {
    const int n = std::min(batch, ny - y0);
    unsigned short* d = dev + (size_t)slot * batch * nx * nz;
    const long long work = (long long)nx * nz * n;
    const int blocks = (int)std::max(1LL, std::min<long long>((work + 255) / 256, (long long)ctx->num_sms * 16));
    slices_u16_kernel<<<blocks, 256, 0, ctx->stream>>>(ctx->vol, nx, ny, nz, y0, n, d);
    if ((rc = launched(ctx, "slices_u16_kernel"))) break;
    // the writer of the batch two back used this pinned buffer
    if (writer.joinable()) writer.join();
    if ((rc = cuda_check(ctx, cudaMemcpyAsync(pinned[slot], d, (size_t)n * sbytes, cudaMemcpyDeviceToHost, ctx->stream),
                         "slice download")))
      break;
    if ((rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "slice download"))) break;
    if (write_failed) break;
    writer = std::thread([&, slot, y0, n] {
      parallel_for(n, host_threads(), [&](int i) {
        char name[64];
        std::snprintf(name, sizeof(name), "CTAnalyzer_Slice#%06d.raw", y0 + i);
        const std::string path = dir + name;
        FILE* f = std::fopen(path.c_str(), "wb");
        const size_t put = f ? std::fwrite(pinned[slot] + (size_t)i * nx * nz, 1, (size_t)sbytes, f) : 0;
        if (!f || std::fclose(f) != 0 || put != (size_t)sbytes) write_failed = true;
      });
    });
  }
  if (writer.joinable()) writer.join();
  cleanup();
  if (rc == FBP_OK && write_failed)
    rc = set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "could not write slice files under \"" + dir + "\"");
  return rc;
}

}  // namespace fbp
