// Detector-row filtering: FDK cosine weight + ramp-type filter.
//
// Replaces the reference's per-view chain (FBP3D::apply_filter_to_projections,
// Source/FilteredBackProjection/FBP3D.cpp:389-414): load, real->complex blit,
// pad, FFFT::fft (radix-2 over texture rows, FastFourierTransformGPU.cpp:3-52),
// fft_shift, FBP2D::apply_filter (FBP2D.cpp:124-144), inverse shift, inverse
// FFT (conj-FFT-conj-divide, FastFourierTransformGPU.cpp:30-36), blit, store:
// ~45 full-texture passes per view. Here one kernel reads each row once and
// writes it once.
//
// Algorithm: two real rows are packed as the real and imaginary parts of one
// complex row (the filter response H is real and even, so the filtered rows
// come back as the real and imaginary parts). Forward transform is a
// decimation-in-frequency radix-2 FFT (natural order in, bit-reversed out),
// the spectrum is multiplied by H[bitrev(k)]/n, and the inverse is a
// decimation-in-time radix-2 FFT (bit-reversed in, natural order out), so no
// bit-reversal permutation is ever executed. Row padding to n samples is the
// reference's (next power of two >= width, FastFourierTransformGPU.cpp:258-262).
//
// The filter response and the spatial kernel are generated on the GPU in
// FP64 from the band-limited ramp kernel (h(0) = 1/4, h(odd k) = -1/(pi k)^2,
// Kak & Slaney eq. 3.61) wrapped onto the n-point circle, times the window.

#include "fbp_internal.h"
#include "fbp_rows.cuh"

#include <cmath>
#include <cstdio>

namespace fbp {
namespace {

__device__ __forceinline__ double ramp_tap(long long k) {
  if (k == 0) return 0.25;
  if ((k & 1) == 0) return 0.0;
  const double pi = 3.14159265358979323846;
  double kk = (double)k;
  return -1.0 / (pi * pi * kk * kk);
}

__device__ __forceinline__ double filter_window(int filter, double f) {
  const double pi = 3.14159265358979323846;
  switch (filter) {
    case FBP_FILTER_SHEPP_LOGAN:
      return f == 0.0 ? 1.0 : sin(pi * f) / (pi * f);
    case FBP_FILTER_COSINE:
      return cospi(f);
    case FBP_FILTER_HANN:
      return 0.5 * (1.0 + cospi(2.0 * f));
    default:
      return 1.0;
  }
}

// H[k] for k < n (one thread per k), FP64.
__global__ void response_kernel(int n, int filter, double* H) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  long long kk = k <= n / 2 ? k : (long long)k - n;
  double f = fabs((double)kk) / n;
  if (filter == FBP_FILTER_RAMP_SAMPLED) {
    H[k] = f;
    return;
  }
  double s = 0.25;  // j = 0 term (cos 0 = 1)
  for (int j = 1; j < n; j += 2) {
    long long jj = j <= n / 2 ? j : (long long)j - n;
    long long p = ((long long)j * k) % n;
    s += ramp_tap(jj) * cospi(2.0 * (double)p / n);
  }
  H[k] = s * filter_window(filter, f);
}

// From H: hbr (bit-reversed, divided by n), twiddles, spatial kernel g.
__global__ void tables_kernel(int n, int log2n, const double* H, float* hbr, float2* tw, float* g) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const unsigned r = log2n > 0 ? __brev((unsigned)k) >> (32 - log2n) : 0u;  // n = 1: the one sample
  hbr[k] = (float)(H[r] / n);
  if (k < n / 2) {
    double s, c;
    sincospi(-2.0 * (double)k / n, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
  double acc = 0.0;
  for (int j = 0; j < n; j++) {
    long long p = ((long long)j * k) % n;
    acc += H[j] * cospi(2.0 * (double)p / n);
  }
  g[k] = (float)(acc / n);
}

__global__ void twiddle_kernel(int n, float2* tw) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n / 2) return;
  double s, c;
  sincospi(-2.0 * (double)k / n, &s, &c);
  tw[k] = make_float2((float)c, (float)s);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Shared memory of filter_fft_kernel: per-stage twiddle tables (n - 1
// float2: 2^lh entries for stage lh at offset 2^lh - 1), then the rows'
// buffer (P x n float2) from a 16-byte boundary.
__host__ __device__ constexpr size_t fft_buf_offset(int n) { return (sizeof(float2) * n + 15) / 16 * 16; }
__host__ __device__ constexpr size_t fft_smem_bytes(int n, int pairs) {
  return fft_buf_offset(n) + sizeof(float2) * n * pairs;
}

struct FilterKArgs {
  RowSet rs;
  int n, log2n, pairs_per_cta;
  long long npairs;
  const float2* tw;
  const float* hbr;
};

// Butterfly passes over the P rows of `buf` (n = 2^L complex samples each).
// Two radix-2 stages are done per pass on four elements in registers (the
// same operations in the same order as two separate radix-2 stages, with half
// the shared-memory round trips and barriers).
//
// Bank conflicts: sample a of the buffer lives at fsw(a), its low four bits
// XORed with 5 x bits 4-5 of a. A half-warp of 8-byte accesses is
// conflict-free when its 16 addresses differ in the low four bits; the
// butterflies touch blk R s + j + r s (j < s, 16 / s consecutive blocks per
// half-warp for s < 16): for s >= 16 the 16 addresses are one aligned run
// (the XOR permutes it), for s = 4 (R = 4) bits 2-3 become r ^ (blk & 3), for
// s = 1 (R = 4, the middle pass) bits 0-1 become r ^ (blk >> 2 & 3); radix-2
// passes only run at s >= n / 2. Each stage reads its own contiguous twiddle
// table (stage lh: T[i] = exp(-2 pi i i / 2^(lh + 1)), i < 2^lh), so lanes
// with consecutive j read consecutive twiddles.
__device__ __forceinline__ int fsw(int a) { return a ^ (((a >> 4) & 3) * 5); }
struct FftRows {
  float2* buf;
  const float2* tws;  // per-stage tables, stage lh at offset 2^lh - 1
  int n, L, P;
  __device__ __forceinline__ const float2* T(int lh) const { return tws + ((1 << lh) - 1); }
  __device__ __forceinline__ float2& at(int a) const { return buf[fsw(a)]; }
};

// forward DIF radix-2 stage lh (half-size h = 2^lh)
__device__ __forceinline__ void fwd_r2(const FftRows& f, int lh) {
  const int h = 1 << lh, half = f.n >> 1;
  const float2* T = f.T(lh);
  for (int b = threadIdx.x; b < f.P * half; b += blockDim.x) {
    const int p = b >> (f.L - 1), q = b & (half - 1);
    const int j = q & (h - 1), blk = q >> lh;
    const int d = p * f.n + (blk << (lh + 1)) + j;
    const float2 x0 = f.at(d), x1 = f.at(d + h);
    f.at(d) = make_float2(x0.x + x1.x, x0.y + x1.y);
    f.at(d + h) = cmul(make_float2(x0.x - x1.x, x0.y - x1.y), T[j]);
  }
}

// forward DIF stages lh and lh - 1 (lh >= 1) on blocks of 2^(lh + 1)
__device__ __forceinline__ void fwd_r4(const FftRows& f, int lh) {
  const int h = 1 << lh, h2 = h >> 1, quarter = f.n >> 2;
  const float2 *T = f.T(lh), *T1 = f.T(lh - 1);
  for (int b = threadIdx.x; b < f.P * quarter; b += blockDim.x) {
    const int p = b / quarter, q = b - p * quarter;
    const int j = q & (h2 - 1), blk = q >> (lh - 1);
    const int d = p * f.n + (blk << (lh + 1)) + j;
    const float2 e0 = f.at(d), e1 = f.at(d + h2), e2 = f.at(d + h), e3 = f.at(d + h + h2);
    const float2 t0 = make_float2(e0.x + e2.x, e0.y + e2.y);
    const float2 t2 = cmul(make_float2(e0.x - e2.x, e0.y - e2.y), T[j]);
    const float2 t1 = make_float2(e1.x + e3.x, e1.y + e3.y);
    const float2 t3 = cmul(make_float2(e1.x - e3.x, e1.y - e3.y), T[j + h2]);
    const float2 w = T1[j];
    f.at(d) = make_float2(t0.x + t1.x, t0.y + t1.y);
    f.at(d + h2) = cmul(make_float2(t0.x - t1.x, t0.y - t1.y), w);
    f.at(d + h) = make_float2(t2.x + t3.x, t2.y + t3.y);
    f.at(d + h + h2) = cmul(make_float2(t2.x - t3.x, t2.y - t3.y), w);
  }
}

// inverse DIT radix-2 stage lh
__device__ __forceinline__ void inv_r2(const FftRows& f, int lh) {
  const int h = 1 << lh, half = f.n >> 1;
  const float2* T = f.T(lh);
  for (int b = threadIdx.x; b < f.P * half; b += blockDim.x) {
    const int p = b >> (f.L - 1), q = b & (half - 1);
    const int j = q & (h - 1), blk = q >> lh;
    const int d = p * f.n + (blk << (lh + 1)) + j;
    const float2 x0 = f.at(d);
    const float2 x1 = cmulc(f.at(d + h), T[j]);
    f.at(d) = make_float2(x0.x + x1.x, x0.y + x1.y);
    f.at(d + h) = make_float2(x0.x - x1.x, x0.y - x1.y);
  }
}

// inverse DIT stages lh and lh + 1 on blocks of 2^(lh + 2)
__device__ __forceinline__ void inv_r4(const FftRows& f, int lh) {
  const int h = 1 << lh, quarter = f.n >> 2;
  const float2 *T = f.T(lh), *T1 = f.T(lh + 1);
  for (int b = threadIdx.x; b < f.P * quarter; b += blockDim.x) {
    const int p = b / quarter, q = b - p * quarter;
    const int j = q & (h - 1), blk = q >> lh;
    const int d = p * f.n + (blk << (lh + 2)) + j;
    const float2 e0 = f.at(d), e1 = f.at(d + h), e2 = f.at(d + 2 * h), e3 = f.at(d + 3 * h);
    const float2 w = T[j];
    const float2 x1 = cmulc(e1, w), x3 = cmulc(e3, w);
    const float2 a0 = make_float2(e0.x + x1.x, e0.y + x1.y), a1 = make_float2(e0.x - x1.x, e0.y - x1.y);
    const float2 a2 = make_float2(e2.x + x3.x, e2.y + x3.y), a3 = make_float2(e2.x - x3.x, e2.y - x3.y);
    const float2 y = cmulc(a2, T1[j]), z = cmulc(a3, T1[j + h]);
    f.at(d) = make_float2(a0.x + y.x, a0.y + y.y);
    f.at(d + 2 * h) = make_float2(a0.x - y.x, a0.y - y.y);
    f.at(d + h) = make_float2(a1.x + z.x, a1.y + z.y);
    f.at(d + 3 * h) = make_float2(a1.x - z.x, a1.y - z.y);
  }
}

// The last two forward stages (1, 0), the response H (bit-reversed, / n) and
// the first two inverse stages (0, 1) of each block of four, in registers.
__device__ __forceinline__ void middle_r4(const FftRows& f, const float* hb) {
  const int quarter = f.n >> 2;
  const float2 w1 = f.T(1)[1], w0 = f.T(0)[0];
  for (int b = threadIdx.x; b < f.P * quarter; b += blockDim.x) {
    const int p = b / quarter, q = b - p * quarter;
    const int d = p * f.n + 4 * q;
    const float4 h4 = __ldg(reinterpret_cast<const float4*>(hb) + q);  // the response from global memory (L1)
    const float hq[4] = {h4.x, h4.y, h4.z, h4.w};
    const float2 e0 = f.at(d), e1 = f.at(d + 1), e2 = f.at(d + 2), e3 = f.at(d + 3);
    // forward stage 1 (pairs 0-2 with w0, 1-3 with w1), stage 0 (pairs 0-1, 2-3 with w0)
    const float2 t0 = make_float2(e0.x + e2.x, e0.y + e2.y);
    const float2 t2 = cmul(make_float2(e0.x - e2.x, e0.y - e2.y), w0);
    const float2 t1 = make_float2(e1.x + e3.x, e1.y + e3.y);
    const float2 t3 = cmul(make_float2(e1.x - e3.x, e1.y - e3.y), w1);
    float2 s0 = make_float2(t0.x + t1.x, t0.y + t1.y);
    float2 s1 = cmul(make_float2(t0.x - t1.x, t0.y - t1.y), w0);
    float2 s2 = make_float2(t2.x + t3.x, t2.y + t3.y);
    float2 s3 = cmul(make_float2(t2.x - t3.x, t2.y - t3.y), w0);
    s0 = make_float2(s0.x * hq[0], s0.y * hq[0]);
    s1 = make_float2(s1.x * hq[1], s1.y * hq[1]);
    s2 = make_float2(s2.x * hq[2], s2.y * hq[2]);
    s3 = make_float2(s3.x * hq[3], s3.y * hq[3]);
    // inverse stage 0 (pairs 0-1, 2-3 with w0), stage 1 (pairs 0-2 with w0, 1-3 with w1)
    const float2 x1 = cmulc(s1, w0), x3 = cmulc(s3, w0);
    const float2 a0 = make_float2(s0.x + x1.x, s0.y + x1.y), a1 = make_float2(s0.x - x1.x, s0.y - x1.y);
    const float2 a2 = make_float2(s2.x + x3.x, s2.y + x3.y), a3 = make_float2(s2.x - x3.x, s2.y - x3.y);
    const float2 y = cmulc(a2, w0), z = cmulc(a3, w1);
    f.at(d) = make_float2(a0.x + y.x, a0.y + y.y);
    f.at(d + 2) = make_float2(a0.x - y.x, a0.y - y.y);
    f.at(d + 1) = make_float2(a1.x + z.x, a1.y + z.y);
    f.at(d + 3) = make_float2(a1.x - z.x, a1.y - z.y);
  }
}

// One CTA filters `pairs_per_cta` row pairs per iteration, grid-stride.
__global__ void __launch_bounds__(256) filter_fft_kernel(FilterKArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = a.n;
  float2* tws = reinterpret_cast<float2*>(smem_raw);
  float2* buf = reinterpret_cast<float2*>(smem_raw + fft_buf_offset(n));
  // stage lh's table from the n / 2 twiddles exp(-2 pi i k / n)
  for (int i = threadIdx.x; i < n - 1; i += blockDim.x) {
    const int lh = 31 - __clz(i + 1), k = i + 1 - (1 << lh);
    tws[i] = a.tw[k << (a.log2n - 1 - lh)];
  }
  const float* hb = a.hbr;
  const RowSet& rs = a.rs;
  const int P = a.pairs_per_cta;
  const FftRows f{buf, tws, n, a.log2n, P};
  const long long ngroups = (a.npairs + P - 1) / P;
  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    __syncthreads();
    // load P pairs: real part row 2p, imaginary part row 2p + 1, zero padded
    for (int idx = threadIdx.x; idx < P * n; idx += blockDim.x) {
      int p = idx / n, i = idx - p * n;
      long long pr = grp * P + p;
      float re = 0.f, im = 0.f;
      if (pr < a.npairs && i < rs.m) {
        long long r0 = 2 * pr;
        re = load_pre(rs, r0, i);
        if (r0 + 1 < rs.rows) im = load_pre(rs, r0 + 1, i);
      }
      f.at(idx) = make_float2(re, im);
    }
    __syncthreads();
    // forward DIF (natural order in, bit-reversed out): an odd stage first,
    // then pairs of stages down to stage 2
    int lh = f.L - 1;
    if (f.L & 1) {
      fwd_r2(f, lh--);
      __syncthreads();
    }
    for (; lh >= 3; lh -= 2) {
      fwd_r4(f, lh);
      __syncthreads();
    }
    int next;  // first inverse stage still to do
    if (lh == 1) {
      middle_r4(f, hb);
      next = 2;
    } else {  // n <= 2: the response on its own
      for (int idx = threadIdx.x; idx < P * n; idx += blockDim.x) {
        const float hv = hb[idx & (n - 1)];
        const float2 x = f.at(idx);
        f.at(idx) = make_float2(x.x * hv, x.y * hv);
      }
      next = 0;
    }
    __syncthreads();
    // inverse DIT (bit-reversed in, natural order out): pairs of stages, then an odd last one
    for (; next + 1 < f.L; next += 2) {
      inv_r4(f, next);
      __syncthreads();
    }
    if (next < f.L) {
      inv_r2(f, next);
      __syncthreads();
    }
    // store
    for (int idx = threadIdx.x; idx < P * n; idx += blockDim.x) {
      int p = idx / n, i = idx - p * n;
      long long pr = grp * P + p;
      if (pr >= a.npairs || i >= rs.m) continue;
      float2 y = f.at(idx);
      long long r0 = 2 * pr;
      store_row_sample(rs, r0, i, y.x);
      if (r0 + 1 < rs.rows) store_row_sample(rs, r0 + 1, i, y.y);
    }
  }
}

__global__ void elementwise_pre_kernel(RowSet rs) {
  long long total = rs.rows * (long long)rs.m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e / rs.m;
    int i = (int)(e - r * rs.m);
    rs.data[r * rs.pitch + i] = load_pre(rs, r, i);
  }
}

// Per-view max |pre-processed sample| (as float bits: non-negative floats
// order like integers). One warp reduces one row, lane 0 folds it into a
// shared per-view table, and each block flushes its table once.
__global__ void view_absmax_kernel(RowSet rs, unsigned* vmax) {
  extern __shared__ unsigned smax[];
  for (int i = threadIdx.x; i < rs.n_views; i += blockDim.x) smax[i] = 0u;
  __syncthreads();
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (long long r = blockIdx.x * (long long)warps + (threadIdx.x >> 5); r < rs.rows;
       r += (long long)gridDim.x * warps) {
    float m = 0.f;
    for (int i = lane; i < rs.m; i += 32) m = fmaxf(m, fabsf(load_pre(rs, r, i)));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0 && m > 0.f) atomicMax(smax + row_view(rs, r), __float_as_uint(m));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < rs.n_views; i += blockDim.x)
    if (smax[i]) atomicMax(vmax + i, smax[i]);
}

// scale = largest power of two with scale * max|value| <= limit (so FP16,
// max 65504, holds every stored value and its neighbour differences).
__global__ void view_scale_kernel(const unsigned* vmax, int nviews, float limit, float* scale, float* inv) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nviews) return;
  const float bound = __uint_as_float(vmax[k]);
  float s = 1.f;
  if (bound > 0.f && isfinite(bound)) {
    int e = (int)floorf(log2f(limit / bound));
    e = max(-100, min(100, e));
    s = ldexpf(1.f, e);
  }
  scale[k] = s;
  inv[k] = 1.f / s;
}

constexpr int kPackRows = 8;  // element rows per block of the quad packers

// f32 rows -> pair16: element (view, e, c) = (row e - 1, row e - row e - 1) * scale.
__global__ void pack_pair16_kernel(const float* src, long long spitch, int m, int n_views, int n_v, bool sinogram,
                                   const float* scale, __half2* out, long long opitch) {
  // grid: x over columns, y over element rows e, z over views
  const int e = blockIdx.y, view = blockIdx.z;
  const long long er = sinogram ? (long long)e * n_views + view : (long long)view * (n_v + 1) + e;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m; c += gridDim.x * blockDim.x) {
    auto row = [&](int iv) -> long long { return sinogram ? (long long)iv * n_views + view : (long long)view * n_v + iv; };
    const float lo = e >= 1 ? src[row(e - 1) * spitch + c] : 0.f;
    const float hi = e < n_v ? src[row(e) * spitch + c] : 0.f;
    const float sc = scale[view];
    // (row e - 1, row e minus row e - 1 as read back): the second value's
    // rounding does not add to the first's (error feedback, as the quads)
    const __half hl = __float2half_rn(lo * sc);
    const __half hd = __float2half_rn(fmaf(hi, sc, -__half2float(hl)));
    out[er * opitch + c] = __halves2half2(hl, hd);
  }
}

// f32 rows -> quad-interleaved gradient layout: one thread per (group g,
// element row e, element column s), writing the 32 bytes of the four slots
// as two 16-byte plane entries.
//
// Each slot holds a 2x2 neighbourhood (a, b: rows e - 1, e of column c; c',
// d: the same rows of column c + 1) as four FP16 values that the
// backprojector reads back as a_r, a_r + c1, a_r + g0 and a_r + c1 + g0 + g1.
// The differences are taken against the values as they will be read back
// (error feedback): a_r = fp16(a), c1 = fp16(c' - a_r), g0 = fp16(b - a_r),
// g1 = fp16(d - (a_r + c1 + g0)). Only a carries a's own rounding error, and
// a bilinear tap weights it by (1 - fu)(1 - fv); the other three corners err
// by the rounding of a difference. On ramp-filtered noisy C4-class views
// this halves the per-tap error of independently rounded differences
// (2.4e-4 -> 1.2e-4 relative).
__global__ void pack_quadg16_kernel(const float* src, long long spitch, int m, int n_views, int n_v, bool sinogram,
                                    const float* scale, uint4* out) {
  // grid: x over element columns, y over runs of kPackRows element rows (each
  // row's samples are loaded once and carried to the next row), z over view
  // groups g
  const int Q = n_views >> 2, P = m + 1;
  const int g = blockIdx.z, e0 = blockIdx.y * kPackRows, e1 = min(e0 + kPackRows, n_v + 1);
  float k[4];
#pragma unroll
  for (int slot = 0; slot < 4; ++slot) k[slot] = scale[g + slot * Q];
  for (int sc = blockIdx.x * blockDim.x + threadIdx.x; sc < P; sc += gridDim.x * blockDim.x) {
    const int c = sc - 1;  // element column sc covers columns c, c + 1
    // samples of row iv at columns c, c + 1 for the four slots (zero outside)
    auto load = [&](int iv, float (&lo)[4], float (&hi)[4]) {
#pragma unroll
      for (int slot = 0; slot < 4; ++slot) {
        const int view = g + slot * Q;
        const bool ok = iv >= 0 && iv < n_v;
        const long long r = sinogram ? (long long)iv * n_views + view : (long long)view * n_v + iv;
        lo[slot] = ok && c >= 0 ? src[r * spitch + c] : 0.f;
        hi[slot] = ok && c + 1 < m ? src[r * spitch + c + 1] : 0.f;
      }
    };
    float pa[4], pc[4], pb[4], pd[4];
    load(e0 - 1, pa, pc);
    for (int e = e0; e < e1; ++e) {
      load(e, pb, pd);
      uint32_t w[8];
#pragma unroll
      for (int slot = 0; slot < 4; ++slot) {
        const float kk = k[slot];
        const __half ha = __float2half_rn(pa[slot] * kk);
        const float ar = __half2float(ha);
        const __half hc1 = __float2half_rn(fmaf(pc[slot], kk, -ar));
        const __half hg0 = __float2half_rn(fmaf(pb[slot], kk, -ar));
        const float c1 = __half2float(hc1), g0 = __half2float(hg0);
        const __half hg1 = __float2half_rn(fmaf(pd[slot], kk, -((ar + c1) + g0)));
        const __half2 x1 = __halves2half2(ha, hg0);   // (a_r, g0): the row e - 1 value and the row step
        const __half2 x2 = __halves2half2(hc1, hg1);  // (c1, g1): their steps along u
        w[2 * slot] = *reinterpret_cast<const uint32_t*>(&x1);
        w[2 * slot + 1] = *reinterpret_cast<const uint32_t*>(&x2);
        pa[slot] = pb[slot];
        pc[slot] = pd[slot];
      }
      // two planes per element row: slots 0, 1 then slots 2, 3, 16 bytes per column each
      const long long ge = (long long)g * (n_v + 1) + e;
      out[(2 * ge) * P + sc] = make_uint4(w[0], w[1], w[2], w[3]);
      out[(2 * ge + 1) * P + sc] = make_uint4(w[4], w[5], w[6], w[7]);
    }
  }
}

// 24-bit store of an FP32 value for kLayoutQuadG24: the top three bytes S of
// a stored value are read back as the float with bits (S << 8) | (S & 0xff).
// That map is monotonic in S, so the nearest of the three candidates around
// the truncation x >> 8 is the nearest representable value (ties to the
// lower magnitude); the sign byte is carried along unchanged.
__device__ __forceinline__ uint32_t store24(float x) {
  const uint32_t b = __float_as_uint(x), sign = b & 0x80000000u, mag = b & 0x7fffffffu;
  const uint32_t t = mag >> 8;
  uint32_t best = t, err = 0xffffffffu;
#pragma unroll
  for (int d = -1; d <= 1; ++d) {
    const uint32_t s = t + d;
    if ((d < 0 && t == 0) || s > 0x7fffffu) continue;
    const uint32_t back = (s << 8) | (s & 0xffu);
    const uint32_t e = back > mag ? back - mag : mag - back;
    if (e < err) {
      err = e;
      best = s;
    }
  }
  return (sign >> 8) | best;  // 24 bits: sign, exponent, 15 significand bits
}

// f32 rows -> kLayoutQuadG24: one thread per (group g, element row e, element
// column s); the 16 values (slot-major: a, b - a, c' - a, d - c' - b + a) are
// stored as 3-byte little-endian fields of 12 words, written as three
// 16-byte plane entries.
__global__ void pack_quadg24_kernel(const float* src, long long spitch, int m, int n_views, int n_v, bool sinogram,
                                    uint4* out) {
  // grid: x over element columns, y over runs of kPackRows element rows, z
  // over view groups g (as pack_quadg16_kernel)
  const int Q = n_views >> 2, P = m + 1;
  const int g = blockIdx.z, e0 = blockIdx.y * kPackRows, e1 = min(e0 + kPackRows, n_v + 1);
  for (int sc = blockIdx.x * blockDim.x + threadIdx.x; sc < P; sc += gridDim.x * blockDim.x) {
    const int c = sc - 1;
    auto load = [&](int iv, float (&lo)[4], float (&hi)[4]) {
#pragma unroll
      for (int slot = 0; slot < 4; ++slot) {
        const int view = g + slot * Q;
        const bool ok = iv >= 0 && iv < n_v;
        const long long r = sinogram ? (long long)iv * n_views + view : (long long)view * n_v + iv;
        lo[slot] = ok && c >= 0 ? src[r * spitch + c] : 0.f;
        hi[slot] = ok && c + 1 < m ? src[r * spitch + c + 1] : 0.f;
      }
    };
    float pa[4], pc[4], pb[4], pd[4];
    load(e0 - 1, pa, pc);
    for (int e = e0; e < e1; ++e) {
      load(e, pb, pd);
      uint32_t w[12];
#pragma unroll
      for (int i = 0; i < 12; ++i) w[i] = 0u;
#pragma unroll
      for (int slot = 0; slot < 4; ++slot) {
        const float val[4] = {pa[slot], pb[slot] - pa[slot], pc[slot] - pa[slot],
                              (pd[slot] - pc[slot]) - (pb[slot] - pa[slot])};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t s24 = store24(val[q]);
          const int byte = 3 * (4 * slot + q), wi = byte >> 2, sh = 8 * (byte & 3);
          w[wi] |= s24 << sh;
          if (sh > 8) w[wi + 1] |= s24 >> (32 - sh);
        }
        pa[slot] = pb[slot];
        pc[slot] = pd[slot];
      }
      const long long ge = (long long)g * (n_v + 1) + e;
      out[(3 * ge) * P + sc] = make_uint4(w[0], w[1], w[2], w[3]);
      out[(3 * ge + 1) * P + sc] = make_uint4(w[4], w[5], w[6], w[7]);
      out[(3 * ge + 2) * P + sc] = make_uint4(w[8], w[9], w[10], w[11]);
    }
  }
}

// Natural-order complex FFT of rows (FFFT::fft_radix2 / inverse_fft_radix2,
// FastFourierTransformGPU.cpp:3-36): inverse = conj, FFT, conj, divide by n.
__global__ void __launch_bounds__(256) fft_rows_kernel(float2* data, int n, int log2n, int rows,
                                                       int inverse, const float2* twg) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int half = n >> 1;
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* buf = tw + half;
  for (int i = threadIdx.x; i < half; i += blockDim.x) tw[i] = twg[i];
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    __syncthreads();
    float2* row = data + (long long)r * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      float2 x = row[i];
      if (inverse) x.y = -x.y;
      buf[i] = x;
    }
    __syncthreads();
    for (int lh = log2n - 1; lh >= 0; --lh) {
      const int h = 1 << lh, tsh = log2n - 1 - lh;
      for (int q = threadIdx.x; q < half; q += blockDim.x) {
        int j = q & (h - 1), blk = q >> lh;
        float2* d = buf + (blk << (lh + 1)) + j;
        float2 x0 = d[0], x1 = d[h];
        d[0] = make_float2(x0.x + x1.x, x0.y + x1.y);
        d[h] = cmul(make_float2(x0.x - x1.x, x0.y - x1.y), tw[j << tsh]);
      }
      __syncthreads();
    }
    const float sc = inverse ? 1.f / n : 1.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      unsigned br = __brev((unsigned)i) >> (32 - log2n);
      float2 x = buf[br];
      if (inverse) x = make_float2(x.x * sc, -x.y * sc);
      row[i] = x;
    }
  }
}

// out[(i + s) mod n] = in[i] per row (FFFT::fft_shift, FastFourierTransformGPU.cpp:93-142).
__global__ void fft_shift_kernel(float2* data, int n, int rows, int shift) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* buf = reinterpret_cast<float2*>(smem_raw);
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    __syncthreads();
    float2* row = data + (long long)r * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) buf[i] = row[i];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int j = (int)((((long long)i + shift) % n + n) % n);
      row[j] = buf[i];
    }
  }
}

__global__ void unpack_rows_kernel(const void* src, int layout, long long spitch, const float* inv_scale,
                                   int n_views, int n_v, bool sinogram, long long row0, long long row_step,
                                   long long nrows, int m, float* dst, long long dpitch) {
  long long total = nrows * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e / m;
    int i = (int)(e - r * m);
    long long gr = row0 + r * row_step;
    const int view = sinogram ? (int)(gr % n_views) : (int)(gr / n_v);
    const int iv = sinogram ? (int)(gr / n_views) : (int)(gr % n_v);
    // row iv is the .x half of element iv + 1
    const long long er = sinogram ? (long long)(iv + 1) * n_views + view : (long long)view * (n_v + 1) + iv + 1;
    float x;
    if (layout == kLayoutPair32)
      x = static_cast<const float2*>(src)[er * spitch + i].x;
    else
      x = __half2float(static_cast<const __half2*>(src)[er * spitch + i].x) * inv_scale[view];
    dst[r * dpitch + i] = x;
  }
}

int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return l;
}

int grid_for(fbp_context* ctx, long long work, int per_block) {
  long long b = (work + per_block - 1) / per_block;
  long long cap = (long long)ctx->num_sms * 16;
  return (int)std::max(1LL, std::min(b, cap));
}

}  // namespace

int ensure_filter_tables(fbp_context* ctx, int n, int filter) {
  FilterTables& t = ctx->ftab;
  if (t.n == n && t.filter == filter) return FBP_OK;
  if (n < 1 || (n & (n - 1)) || n > 8192)
    return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "filter length must be a power of two in [1, 8192]");
  if (filter < 0 || filter > FBP_FILTER_RAMP_SAMPLED)
    return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "unknown filter type");
  if (n > t.cap) {  // grow only: a context serving many row lengths stops allocating
    cudaFree(t.twiddle);
    cudaFree(t.hbr);
    cudaFree(t.kernel);
    t.twiddle = nullptr;
    t.hbr = nullptr;
    t.kernel = nullptr;
    t.n = 0;
    t.cap = 0;
    if (cuda_check(ctx, cudaMalloc(&t.twiddle, sizeof(float2) * (n / 2 + 1)), "cudaMalloc(twiddle)") ||
        cuda_check(ctx, cudaMalloc(&t.hbr, sizeof(float) * n), "cudaMalloc(hbr)") ||
        cuda_check(ctx, cudaMalloc(&t.kernel, sizeof(float) * n), "cudaMalloc(kernel)"))
      return FBP_ERR_OUT_OF_MEMORY;
    t.cap = n;
  }
  double* H = static_cast<double*>(scratch(ctx, sizeof(double) * n));
  if (!H) return FBP_ERR_OUT_OF_MEMORY;
  int blocks = (n + 127) / 128;
  response_kernel<<<blocks, 128, 0, ctx->stream>>>(n, filter, H);
  tables_kernel<<<blocks, 128, 0, ctx->stream>>>(n, ilog2(n), H, t.hbr, t.twiddle, t.kernel);
  ctx->launches += 1;  // two launches above
  if (int rc = launched(ctx, "filter tables")) return rc;
  t.n = n;
  t.filter = filter;
  return FBP_OK;
}

int launch_filter_fft(fbp_context* ctx, const RowSet& rs, int n) {
  if (n < rs.m) return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "padded length smaller than the row");
  if (n > 4096) return set_error(ctx, FBP_ERR_UNSUPPORTED, "FFT filter supports padded lengths up to 4096");
  if (rs.rows == 0) return FBP_OK;
  FilterKArgs a;
  a.rs = rs;
  a.n = n;
  a.log2n = ilog2(n);
  a.pairs_per_cta = std::max(1, std::min(8, 4096 / n));
  a.npairs = (rs.rows + 1) / 2;
  a.tw = ctx->ftab.twiddle;
  a.hbr = ctx->ftab.hbr;
  size_t smem = fft_smem_bytes(n, a.pairs_per_cta);
  // per device and process-wide: set on every launch (same value from every context)
  cudaFuncSetAttribute(filter_fft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
  long long groups = (a.npairs + a.pairs_per_cta - 1) / a.pairs_per_cta;
  int grid = (int)std::min<long long>(groups, (long long)ctx->num_sms * 4);
  filter_fft_kernel<<<grid, 256, smem, ctx->stream>>>(a);
  return launched(ctx, "filter_fft_kernel");
}

int launch_elementwise_pre(fbp_context* ctx, const RowSet& rs) {
  if (rs.rows == 0) return FBP_OK;
  elementwise_pre_kernel<<<grid_for(ctx, rs.rows * rs.m, 256), 256, 0, ctx->stream>>>(rs);
  return launched(ctx, "elementwise_pre_kernel");
}

int launch_view_scales(fbp_context* ctx, const RowSet& rs, float limit, float* view_scale, float* inv_scale) {
  if (rs.n_views > 16384) return set_error(ctx, FBP_ERR_UNSUPPORTED, "at most 16384 views in MIXED precision");
  unsigned* vmax = static_cast<unsigned*>(scratch(ctx, sizeof(unsigned) * rs.n_views + 64));
  if (!vmax) return FBP_ERR_OUT_OF_MEMORY;
  if (int rc = cuda_check(ctx, cudaMemsetAsync(vmax, 0, sizeof(unsigned) * rs.n_views, ctx->stream), "memset"))
    return rc;
  const int blocks = (int)std::max(1LL, std::min<long long>((rs.rows + 7) / 8, (long long)ctx->num_sms * 4));
  const size_t sm = sizeof(unsigned) * rs.n_views;
  cudaFuncSetAttribute(view_absmax_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
  view_absmax_kernel<<<blocks, 256, sm, ctx->stream>>>(rs, vmax);
  view_scale_kernel<<<(rs.n_views + 127) / 128, 128, 0, ctx->stream>>>(vmax, rs.n_views, limit, view_scale, inv_scale);
  ctx->launches += 1;  // two launches above
  return launched(ctx, "view scale kernels");
}

int launch_pack(fbp_context* ctx, const Stack& s, int layout, void* out, long long pitch, const float* view_scale) {
  if (layout == kLayoutPair16) {
    if (s.v + 1 > 65535 || s.n > 65535)
      return set_error(ctx, FBP_ERR_UNSUPPORTED, "the pair layout takes up to 65534 rows and 65535 views");
    const dim3 grid((s.u + 255) / 256, s.v + 1, s.n);
    pack_pair16_kernel<<<grid, 256, 0, ctx->stream>>>(s.f32, s.pitch, s.u, s.n, s.v, s.sinogram, view_scale,
                                                      static_cast<__half2*>(out), pitch);
    return launched(ctx, "pack_pair16_kernel");
  }
  if (layout == kLayoutQuadG16) {
    if (s.n % 4) return set_error(ctx, FBP_ERR_UNSUPPORTED, "the interleaved layout needs a multiple of 4 views");
    if (s.v + 1 > 65535 || s.n / 4 > 65535)
      return set_error(ctx, FBP_ERR_UNSUPPORTED, "the interleaved layout takes up to 65534 rows and 262140 views");
    const dim3 grid((s.u + 1 + 255) / 256, (s.v + 1 + kPackRows - 1) / kPackRows, s.n / 4);
    pack_quadg16_kernel<<<grid, 256, 0, ctx->stream>>>(s.f32, s.pitch, s.u, s.n, s.v, s.sinogram, view_scale,
                                                       static_cast<uint4*>(out));
    return launched(ctx, "pack_quadg16_kernel");
  }
  if (layout == kLayoutQuadG24) {
    if (s.n % 4) return set_error(ctx, FBP_ERR_UNSUPPORTED, "the interleaved layout needs a multiple of 4 views");
    if (s.v + 1 > 65535 || s.n / 4 > 65535)
      return set_error(ctx, FBP_ERR_UNSUPPORTED, "the interleaved layout takes up to 65534 rows and 262140 views");
    const dim3 grid((s.u + 1 + 255) / 256, (s.v + 1 + kPackRows - 1) / kPackRows, s.n / 4);
    pack_quadg24_kernel<<<grid, 256, 0, ctx->stream>>>(s.f32, s.pitch, s.u, s.n, s.v, s.sinogram,
                                                       static_cast<uint4*>(out));
    return launched(ctx, "pack_quadg24_kernel");
  }
  return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "unknown packed layout");
}

int launch_fft_rows(fbp_context* ctx, float2* data, int n, int rows, int inverse) {
  if (n < 2 || (n & (n - 1)) || n > 8192)
    return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "FFT length must be a power of two in [2, 8192]");
  if (rows <= 0) return FBP_OK;
  // twiddles for n (independent of the filter tables' n)
  float2* tw = static_cast<float2*>(scratch(ctx, sizeof(float2) * (n / 2)));
  if (!tw) return FBP_ERR_OUT_OF_MEMORY;
  twiddle_kernel<<<(n / 2 + 127) / 128, 128, 0, ctx->stream>>>(n, tw);
  size_t smem = sizeof(float2) * (n / 2 + n);
  cudaFuncSetAttribute(fft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
  fft_rows_kernel<<<std::min(rows, ctx->num_sms * 4), 256, smem, ctx->stream>>>(data, n, ilog2(n), rows, inverse,
                                                                                 tw);
  ctx->launches += 1;  // twiddle_kernel
  return launched(ctx, "fft_rows_kernel");
}

int launch_fft_shift_rows(fbp_context* ctx, float2* data, int n, int rows, int shift) {
  if (n <= 0 || n > 8192) return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "row length must be in [1, 8192]");
  if (rows <= 0) return FBP_OK;
  cudaFuncSetAttribute(fft_shift_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
  fft_shift_kernel<<<std::min(rows, ctx->num_sms * 4), 256, sizeof(float2) * n, ctx->stream>>>(data, n, rows,
                                                                                                shift);
  return launched(ctx, "fft_shift_kernel");
}

int launch_unpack_rows(fbp_context* ctx, const Stack& s, size_t row0, size_t nrows, float* dst,
                       long long dst_pitch, long long row_step) {
  if (nrows == 0) return FBP_OK;
  unpack_rows_kernel<<<grid_for(ctx, (long long)nrows * s.u, 256), 256, 0, ctx->stream>>>(
      s.filt, s.filt_layout, s.filt_pitch, s.inv_scale, s.n, s.v, s.sinogram, (long long)row0, row_step,
      (long long)nrows, s.u, dst, dst_pitch);
  return launched(ctx, "unpack_rows_kernel");
}

}  // namespace fbp

// ---------------------------------------------------------------------------
// Allocation-free variant of fbp2d_filter_sinogram.
//
// Some callers cannot allocate device memory while they run: hosts that hand
// out all GPU memory from their own pool at start-up, real-time acquisition
// loops where a cudaMalloc / cudaFree would synchronise the device and stall
// the detector read-out, and plugins whose host forbids allocations after
// initialisation. This entry point needs no context and allocates nothing:
// the filter tables it generates (FP64 response, twiddles, bit-reversed
// response) live in the file-scope array below, which every GPU that loads
// the library holds until the process exits.
//
// Capacity: padded row lengths up to kNoAllocMaxN = 4096 samples (rows up to
// 4096 bins with the default padding). The array is shared by all calls on a
// device and keeps the last call's tables; each call rewrites every table
// entry it reads before reading it, so nothing needs clearing. Calls whose
// work overlaps on the GPU (other streams, other host threads) race on the
// array and must be serialised by the caller.

namespace {
constexpr int kNoAllocMaxN = 4096;
constexpr size_t kNoAllocH = 0;                                         // double[4096]
constexpr size_t kNoAllocTw = kNoAllocH + sizeof(double) * kNoAllocMaxN;  // float2[2048]
constexpr size_t kNoAllocHbr = kNoAllocTw + sizeof(float2) * (kNoAllocMaxN / 2);  // float[4096]
constexpr size_t kNoAllocG = kNoAllocHbr + sizeof(float) * kNoAllocMaxN;           // float[4096]
constexpr size_t kNoAllocBytes = kNoAllocG + sizeof(float) * kNoAllocMaxN;         // 80 KiB
}  // namespace

static __device__ __align__(256) unsigned char fbp_noalloc_filter_scratch[kNoAllocBytes];

extern "C" int fbp2d_filter_sinogram_noalloc(float* sinogram, int bins, int views, int filter_type, float fan_sdd,
                                              float detector_width, int padded_length, void* cuda_stream) {
  using namespace fbp;
  if (!sinogram || bins <= 0 || views <= 0)
    return set_error(nullptr, FBP_ERR_INVALID_ARGUMENT, "bad sinogram");
  if (filter_type < 0 || filter_type > FBP_FILTER_RAMP_SAMPLED)
    return set_error(nullptr, FBP_ERR_INVALID_ARGUMENT, "unknown filter type");
  if (fan_sdd > 0.f && !(detector_width > 0.f))
    return set_error(nullptr, FBP_ERR_INVALID_ARGUMENT, "detector width must be positive");
  int n = padded_length;
  if (n <= 0) {  // the reference's rule: next power of two >= bins (1 for one bin)
    int l = 0;
    for (long t = 2L * bins - 1; t > 1; t >>= 1) l++;
    n = l < 31 ? 1 << l : 0;
  }
  if (n < bins || n < 1 || (n & (n - 1)))
    return set_error(nullptr, FBP_ERR_INVALID_ARGUMENT, "padded length must be a power of two >= the row width");
  if (n > kNoAllocMaxN)
    return set_error(nullptr, FBP_ERR_UNSUPPORTED,
                     "padded row length " + std::to_string(n) +
                         " exceeds the 4096-sample maximum of fbp2d_filter_sinogram_noalloc");
  // an error left by the caller's own earlier work would otherwise be read
  // back below and reported as this call's
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(nullptr, FBP_ERR_CUDA,
                     std::string("a CUDA error was pending before fbp2d_filter_sinogram_noalloc: ") +
                         cudaGetErrorString(e));
  // Device address of the scratch array in the current device's context (the
  // array's host-side name is not a device address). Looked up on every
  // call: a context torn down and made again (cudaDeviceReset) may load the
  // module elsewhere. The first call on a device loads the module's device
  // code, which is why that call should come before any stream capture.
  void* base = nullptr;
  e = cudaGetSymbolAddress(&base, fbp_noalloc_filter_scratch);
  if (e != cudaSuccess) return cuda_check(nullptr, e, "cudaGetSymbolAddress(filter scratch)");
  unsigned char* b = static_cast<unsigned char*>(base);
  double* H = reinterpret_cast<double*>(b + kNoAllocH);
  float2* tw = reinterpret_cast<float2*>(b + kNoAllocTw);
  float* hbr = reinterpret_cast<float*>(b + kNoAllocHbr);
  float* g = reinterpret_cast<float*>(b + kNoAllocG);
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  int dev = 0, sms = 148;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_check(nullptr, e, "cudaGetDevice");
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return cuda_check(nullptr, e, "cudaDeviceGetAttribute(multiprocessor count)");

  const int blocks = (n + 127) / 128;
  response_kernel<<<blocks, 128, 0, stream>>>(n, filter_type, H);
  tables_kernel<<<blocks, 128, 0, stream>>>(n, ilog2(n), H, hbr, tw, g);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return cuda_check(nullptr, e, "fbp2d_filter_sinogram_noalloc: filter tables");

  RowSet rs{};
  rs.data = sinogram;
  rs.pitch = bins;
  rs.rows = views;
  rs.m = bins;
  rs.n_views = views;
  rs.n_v = 1;
  rs.sinogram = false;
  if (fan_sdd > 0.f) {
    rs.weight = true;
    rs.w_sdd = fan_sdd;
    rs.w_du = detector_width / bins;
    rs.w_dv = 0.f;
  }
  FilterKArgs a;
  a.rs = rs;
  a.n = n;
  a.log2n = ilog2(n);
  a.pairs_per_cta = std::max(1, std::min(8, 4096 / n));
  a.npairs = (rs.rows + 1) / 2;
  a.tw = tw;
  a.hbr = hbr;
  const size_t smem = fft_smem_bytes(n, a.pairs_per_cta);
  if ((e = cudaFuncSetAttribute(filter_fft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024)) !=
      cudaSuccess)
    return cuda_check(nullptr, e, "fbp2d_filter_sinogram_noalloc: shared memory attribute");
  const long long groups = (a.npairs + a.pairs_per_cta - 1) / a.pairs_per_cta;
  const int grid = (int)std::min<long long>(groups, (long long)sms * 4);
  filter_fft_kernel<<<grid, 256, smem, stream>>>(a);
  return cuda_check(nullptr, cudaGetLastError(), "fbp2d_filter_sinogram_noalloc: filter_fft_kernel");
}
