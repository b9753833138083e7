// Voxel-driven, distance-weighted backprojection with bilinear detector
// interpolation, for flat-panel cone beam (FDK) and parallel beam, in 3D and
// 2D (a 2D image is a volume with one y-slice and a one-row detector).
//
// Replaces the reference's per-view dispatch loop
// FBP3D::project_backward_cone_fdk_from_projections (Source/FilteredBackProjection/
// FBP3D.cpp:524-559, one full read-modify-write of the volume per view) and the
// 3D / 2D parallel variants (FBP3D.cpp:460-522, FBP2D.cpp:96-122). The GLSL
// bodies are not in the reference; the arithmetic is the textbook FDK one.
//
// Design (one launch for all views):
//   * A CTA owns a TX x TZ tile of voxel columns and NY voxels along the
//     rotation axis (y); each consumer thread owns one column segment of NY
//     voxels and keeps its NY sums in registers across every view, so the
//     volume is written exactly once (clip epilogue fused into the store).
//   * Warp specialisation: one producer warp computes, in FP64, the tile's
//     detector footprint and tile-local projective coefficients for 32 views
//     at a time (one view per lane), re-based on the tile corner and on the
//     staged window so that the FP32 coordinates the consumers form stay small
//     and accurate, and copies each view's footprint window (box_u x box_v
//     elements) into a ring of shared-memory stages with TMA
//     (cp.async.bulk.tensor, no multicast). Samples outside the detector
//     arrive as zeros from the TMA out-of-bounds fill. Full / empty mbarriers
//     per stage replace block barriers; consumer warps never wait for one
//     another.
//   * Filtered views are stored in a pair layout (element (v, u) holds rows v
//     and v + 1), so a bilinear tap is two shared-memory loads (8-byte float2
//     or 4-byte half2). Per view a consumer thread forms 1/D, its detector
//     column u (constant along the column), the distance weight and the v
//     step once; per voxel it steps v with one FMA and takes floor / fraction
//     with the 1.5 * 2^23 rounding constant (no conversion instructions).
//   * Every mbarrier wait is bounded; on expiry the CTA records an error and
//     leaves, and every CTA checks the error word before starting.

#include "fbp_internal.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>
#include <vector>

namespace fbp {
namespace {

constexpr int kMaxStages = 8;                // shared-memory ring stages (one view each)
constexpr int kMaxDynamicSmem = 227 * 1024;  // sm_100: largest dynamic shared memory of one CTA
constexpr uint32_t kWaitLimit = 1u << 22;  // mbarrier polls before giving up

struct ViewCoef {
  float Dx, Dz, D0;  // D = L / SOD (cone) or 1 (parallel), affine in (x', z')
  float Nx, Nz, N0;  // u_local * D
  float Vx, Vz, V0;  // v_local * D at the tile's first y
  float wscale;      // extra per-view weight (FP16 views: 1 / scale)
  int skip;          // tile footprint misses the detector
  int box;           // staged window: width (elements) | rows << 16
};

// Per-view window boxes: a grid of tensor maps over the same filtered stack,
// 8 widths x 8 heights chosen per geometry from the histogram of window sizes
// that the footprint pass collects (the largest of each = the largest
// window); the producer stages each (tile, view) window with the smallest box
// that holds it, so a copy moves little more than what the view needs.
constexpr int kNW = kBoxGrid, kNH = kBoxGrid;
struct BoxMaps {
  CUtensorMap map[kNW * kNH];  // [width index][height index]
  int w[kNW];                  // box widths in elements of the layout
  int h[kNH];                  // box heights in element rows
};

struct BPArgs {
  float* vol;
  int nx, ny, nz;
  int nu, nv, nviews;
  int kind;
  double sod, sdd, du, dv, vox;
  double cu, cv;          // (nu - 1) / 2, (nv - 1) / 2
  float dvn;              // v step per voxel times D
  float scale;            // pi / K * filter spacing factor
  const double2* trig;    // (cos, sin) per view
  const float* inv_scale; // FP16 per-view 1/scale or nullptr
  int box_u, box_v, align;  // largest window (elements, element rows)
  int box_bytes;            // smem bytes reserved per staged window (multiple of 128)
  int chunk;              // ring stages
  int ntx, ntz;           // tiles along x and z
  int sino_layout;        // tensor coordinates (u, view, v) instead of (u, v, view)
  int pair_rows;          // 1: an element carries rows v and v + 1 (pair layouts)
  int clip_ylimit;        // clip negatives where iy < clip_ylimit
  int* err;
  // interleaved layout in global memory, for windows too large to stage:
  // 16-byte entries, [group][element row][plane][element column]
  const uint4* qg;
  int qg_pitch, qg_rows;  // element columns per plane row, element rows per group
  int resident;           // CTAs resident on the GPU at once (view-group skew of the interleaved walk)
  int band;               // tile orbits along z in one band of the symmetric kernel's tile order
  int* minmax;            // fold the stored values' min / max into this pair (or nullptr)
  int y_off, ny_total;    // the volume is y-slices [y_off, y_off + ny) of ny_total
  int vol_ystride;        // y-slices between z planes of the output buffer
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false (and records kDevTimeout) after kWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  for (uint32_t i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  atomicCAS(err, 0, kDevTimeout);
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ int floor_div(int a, int b) {  // b > 0
  int q = a / b;
  return (a % b != 0 && a < 0) ? q - 1 : q;
}

// Tile geometry for view k in FP64: the affine coefficients of D (= L/SOD
// for cone beam, 1 for parallel beam), of u*D and of v*D in tile-local voxel
// offsets (x', z', y'), and the detector extremes over the tile's corner
// voxels. A projective map attains its extremes over a box at the corners.
struct TileGeo {
  double Dx, Dz, D0, Ux, Uz, U0, G, Yc;
  double umin, umax, vmin, vmax, dmin;
};

__device__ void tile_geo(const BPArgs& a, int k, int ix0, int iy0, int iz0, int ex, int ey, int ez, TileGeo& t) {
  const double c = a.trig[k].x, s = a.trig[k].y;
  const double Xc = (ix0 + 0.5 - 0.5 * a.nx) * a.vox;
  const double Zc = (iz0 + 0.5 - 0.5 * a.nz) * a.vox;
  t.Yc = (a.y_off + iy0 + 0.5 - 0.5 * a.ny_total) * a.vox;
  if (a.kind == FBP_GEOMETRY_CONE) {
    const double K = a.sdd / (a.sod * a.du);
    t.Dx = a.vox * c / a.sod;
    t.Dz = a.vox * s / a.sod;
    t.D0 = (a.sod + Xc * c + Zc * s) / a.sod;
    t.Ux = -a.vox * s * K;
    t.Uz = a.vox * c * K;
    t.U0 = (-Xc * s + Zc * c) * K;
    t.G = a.sdd / (a.sod * a.dv);
  } else {
    t.Dx = 0.0;
    t.Dz = 0.0;
    t.D0 = 1.0;
    t.Ux = -a.vox * s / a.du;
    t.Uz = a.vox * c / a.du;
    t.U0 = (-Xc * s + Zc * c) / a.du;
    t.G = 1.0 / a.dv;
  }
  t.umin = 1e300;
  t.umax = -1e300;
  t.vmin = 1e300;
  t.vmax = -1e300;
  t.dmin = 1e300;
#pragma unroll
  for (int cx = 0; cx < 2; ++cx)
#pragma unroll
    for (int cz = 0; cz < 2; ++cz) {
      const double x = cx ? ex : 0, z = cz ? ez : 0;
      const double D = t.Dx * x + t.Dz * z + t.D0;
      t.dmin = fmin(t.dmin, D);
      // one FP64 reciprocal per corner column instead of three divisions (the
      // producer computes this for every quad, skipped ones included)
      const double rD = 1.0 / D;
      const double u = (t.Ux * x + t.Uz * z + t.U0) * rD + a.cu;
      t.umin = fmin(t.umin, u);
      t.umax = fmax(t.umax, u);
#pragma unroll
      for (int cy = 0; cy < 2; ++cy) {
        const double y = cy ? ey : 0;
        const double v = t.G * (t.Yc + a.vox * y) * rD + a.cv;
        t.vmin = fmin(t.vmin, v);
        t.vmax = fmax(t.vmax, v);
      }
    }
}

constexpr double kSlack = 1.0 / 64;  // detector samples of margin around the footprint

__device__ __forceinline__ bool tile_skip(const BPArgs& a, const TileGeo& t) {
  return t.dmin <= 1e-6 || t.umax <= -1.0 || t.umin >= (double)a.nu || t.vmax <= -1.0 || t.vmin >= (double)a.nv;
}

// Window origin (u0 aligned down for TMA) and the samples the tile needs.
__device__ __forceinline__ void tile_window(const BPArgs& a, const TileGeo& t, int& u0, int& v0, int& need_u,
                                            int& need_v) {
  u0 = floor_div((int)floor(t.umin - kSlack), a.align) * a.align;
  v0 = (int)floor(t.vmin - kSlack);
  need_u = (int)floor(t.umax + kSlack) + 2 - u0;
  need_v = (int)floor(t.vmax + kSlack) + 2 - v0;
}

// Coefficients for view k of this tile; returns skip.
__device__ bool tile_view_coef(const BPArgs& a, int k, int ix0, int iy0, int iz0, int ex, int ey, int ez,
                               ViewCoef& vc, int& u0, int& v0, int& need_u, int& need_v, bool& overflow,
                               bool& behind) {
  TileGeo t;
  tile_geo(a, k, ix0, iy0, iz0, ex, ey, ez, t);
  behind = t.dmin <= 1e-6;
  const bool skip = tile_skip(a, t);
  tile_window(a, t, u0, v0, need_u, need_v);
  overflow = !skip && (need_u > a.box_u || need_v - a.pair_rows > a.box_v);
  const double du0 = a.cu - u0, dv0 = a.cv - v0;
  vc.Dx = (float)t.Dx;
  vc.Dz = (float)t.Dz;
  vc.D0 = (float)t.D0;
  vc.Nx = (float)(t.Ux + du0 * t.Dx);
  vc.Nz = (float)(t.Uz + du0 * t.Dz);
  vc.N0 = (float)(t.U0 + du0 * t.D0);
  vc.Vx = (float)(dv0 * t.Dx);
  vc.Vz = (float)(dv0 * t.Dz);
  vc.V0 = (float)(t.G * t.Yc + dv0 * t.D0);
  vc.wscale = a.inv_scale ? a.inv_scale[k] : 1.0f;
  vc.skip = skip;
  return skip;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ float lds_f32(uint32_t addr) {
  float v;
  asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}
__device__ __forceinline__ float2 lds_f32x2(uint32_t addr) {
  float2 v;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}
__device__ __forceinline__ __half2 lds_h2(uint32_t addr) {
  uint32_t v;
  asm("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(addr));
  return *reinterpret_cast<__half2*>(&v);
}

// Two FP32 FMAs in one instruction (sm_100 packed f32x2), d = a * b + c per lane.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  unsigned long long ra, rb, rc, rd;
  asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(rc) : "f"(c.x), "f"(c.y));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(rd) : "l"(ra), "l"(rb), "l"(rc));
  float2 d;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(rd));
  return d;
}

__device__ __forceinline__ unsigned long long pack2(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long r) {
  float2 d;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(r));
  return d;
}
// a + b per lane rounded toward zero or to nearest, and a - b rounded to nearest (packed f32x2)
__device__ __forceinline__ float2 fadd2_rz(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
  return unpack2(d);
}
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
  return unpack2(d);
}
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
  return unpack2(d);
}

// Value I (0..15) of a kLayoutQuadG24 element held in 12 words: its three
// bytes sit at byte 3 I, and the float is rebuilt as (bytes << 8) | low byte.
template <int I>
__device__ __forceinline__ float dec24(const uint32_t (&w)[12]) {
  constexpr int B = 3 * I, W = B >> 2, O = B & 3;
  constexpr int W1 = W + 1 < 12 ? W + 1 : W;  // the last value needs no second word
  constexpr unsigned sel = O | (O << 4) | ((O + 1) << 8) | ((O + 2) << 12);
  return __uint_as_float(__byte_perm(w[W], w[W1], sel));
}

__device__ __forceinline__ uint4 lds_u4(uint32_t addr) {
  uint4 v;
  asm("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr));
  return v;
}

// Hardware approximate reciprocal (max 1 ulp error; D is a distance ratio near 1).
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// FP16 x FP16 + FP32 with one rounding to FP32.
__device__ __forceinline__ float fma_f16_f32(__half a, __half b, float c) {
  float d;
  asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d) : "h"(__half_as_ushort(a)), "h"(__half_as_ushort(b)), "f"(c));
  return d;
}

constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr uint32_t kMagicBits = 0x4B400000u;

// One bilinear update of a voxel whose window-local row coordinate is v >= 0:
// accum += W * sample(u, v). v + kMagic rounded toward zero is
// kMagic + floor(v), so its bit pattern minus kMagicBits is the row index and
// c0 + bits * RB the address of the element at (floor(v), iu) (c0 folds the
// window base, the column and -kMagicBits * RB); no conversion instructions.
// wa, wb already carry W for the FP32 layouts.
template <int LAYOUT>
__device__ __forceinline__ void tap(float v, uint32_t c0, uint32_t RB, float wa, float wb, float fu, float W,
                                    float& accum) {
  const float t = __fadd_rz(v, kMagic);
  const float fv = v - (t - kMagic);  // in [0, 1)
  const uint32_t addr = __float_as_uint(t) * RB + c0;
  if constexpr (LAYOUT == kLayoutRaw32) {
    const float p00 = lds_f32(addr), p01 = lds_f32(addr + 4);
    const float p10 = lds_f32(addr + RB), p11 = lds_f32(addr + RB + 4);
    const float r0 = fmaf(wb, p01, wa * p00);
    const float r1 = fmaf(wb, p11, wa * p10);
    accum += fmaf(fv, r1 - r0, r0);
  } else if constexpr (LAYOUT == kLayoutPair32) {
    const float2 X = lds_f32x2(addr), Y = lds_f32x2(addr + 8);  // (p00, p10), (p01, p11)
    const float r0 = fmaf(wb, Y.x, wa * X.x);
    const float r1 = fmaf(wb, Y.y, wa * X.y);
    accum += fmaf(fv, r1 - r0, r0);
  } else {
    // element = (row v, row v + 1 minus row v); the u-lerp of both in FP32
    const float2 x = __half22float2(lds_h2(addr)), y = __half22float2(lds_h2(addr + 4));
    const float2 ag = ffma2(make_float2(fu, fu), fsub2(y, x), x);
    accum = fmaf(W, fmaf(fv, ag.y, ag.x), accum);
  }
}

template <int LAYOUT, int TX, int TZ, int NY>
__global__ void __launch_bounds__(TX* TZ + 32, 2) bp_kernel(const __grid_constant__ BoxMaps maps, const BPArgs a) {
  static_assert(TX % 8 == 0 && TZ % 4 == 0, "warp tile is 8 x 4 columns");
  constexpr int NCW = TX * TZ / 32;  // consumer warps
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int S = a.chunk;  // ring stages (one view each)
  const int bx = blockIdx.x % a.ntx, bz = blockIdx.x / a.ntx;
  const int ix0 = bx * TX, iz0 = bz * TZ, iy0 = blockIdx.y * NY;

  ViewCoef* coef = reinterpret_cast<ViewCoef*>(smem + (size_t)S * a.box_bytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(coef + S);
  uint64_t* empty = full + S;
  volatile int* s_abort = reinterpret_cast<volatile int*>(empty + S);

  if (tid == 0) {
    *s_abort = *(volatile int*)a.err != 0;
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (*s_abort) return;

  if (warp == NCW) {
    // ---------------------------------------------------------------- producer
    // Lane l computes view kb + l of each batch of 32; then the views are
    // staged in order, each with the smallest box of the grid that holds it.
    int issued = 0;
    for (int kb = 0; kb < a.nviews && !*s_abort; kb += 32) {
      const int k = kb + lane;
      ViewCoef vc;
      int u0 = 0, v0 = 0, wi = 0, hi = 0;
      bool skip = true;
      vc.skip = 1;
      if (k < a.nviews) {
        bool overflow = false, behind = false;
        int need_u = 0, need_v = 0;
        // full tile extents: every consumer thread's samples lie in the window
        skip = tile_view_coef(a, k, ix0, iy0, iz0, TX - 1, NY - 1, TZ - 1, vc, u0, v0, need_u, need_v, overflow,
                              behind);
        if (overflow) atomicCAS(a.err, 0, kDevFootprint);
        if (behind) atomicCAS(a.err, 0, kDevGeometry);
        if (overflow || behind) skip = true, vc.skip = 1;
        const int rows = need_v - a.pair_rows;  // element rows to stage
        while (wi < kNW - 1 && maps.w[wi] < need_u) ++wi;
        while (hi < kNH - 1 && maps.h[hi] < rows) ++hi;
        vc.box = maps.w[wi] | (maps.h[hi] << 16);
      }
      const int nb = min(32, a.nviews - kb);
      for (int i = 0; i < nb; ++i) {
        const int kk = kb + i;
        const int s = kk % S;
        if (kk >= S && !mbar_wait(&empty[s], ((kk / S) & 1) ^ 1, a.err)) {
          *s_abort = 1;
          break;
        }
        if (lane == i) coef[s] = vc;
        const int sk = __shfl_sync(0xffffffffu, (int)skip, i);
        const int cu0 = __shfl_sync(0xffffffffu, u0, i), cv0 = __shfl_sync(0xffffffffu, v0, i);
        const int mi = __shfl_sync(0xffffffffu, wi * kNH + hi, i);
        __syncwarp();
        if (lane == 0) {
          if (sk) {
            mbar_arrive(&full[s]);
          } else {
            const CUtensorMap* m = &maps.map[mi];
            const uint32_t bytes = (uint32_t)(maps.w[mi / kNH] * maps.h[mi % kNH] * (LAYOUT == kLayoutPair32 ? 8 : 4));
            mbar_arrive_expect_tx(&full[s], bytes);
            const int x = LAYOUT == kLayoutPair32 ? 2 * cu0 : cu0;  // float2 elements are two floats
            const int e0 = cv0 + a.pair_rows;                      // pair layouts: row v is element row v + 1
            void* dst = smem + (size_t)s * a.box_bytes;
            if (a.sino_layout)
              tma_load_3d(dst, m, x, kk, e0, &full[s]);
            else
              tma_load_3d(dst, m, x, e0, kk, &full[s]);
          }
        }
        __syncwarp();
        issued = kk + 1;
      }
    }
    // leave only when every copy issued into this CTA's memory has landed
    for (int kk = max(0, issued - S); kk < issued; ++kk) mbar_wait(&full[kk % S], (kk / S) & 1, a.err);
    return;
  }

  // ------------------------------------------------------------------ consumers
  constexpr int WX = TX / 8;
  const int tx = (warp % WX) * 8 + (lane & 7);
  const int tz = (warp / WX) * 4 + (lane >> 3);
  const float fx = (float)tx, fz = (float)tz;
  constexpr int ESZ = LAYOUT == kLayoutPair32 ? 8 : 4;
  // rows of a window usable as floor(v): all for pair layouts, all but the
  // last for the raw layout (it also reads row v + 1)
  constexpr int kRowTail = LAYOUT == kLayoutRaw32 ? 1 : 0;

  float acc[NY];
#pragma unroll
  for (int j = 0; j < NY; ++j) acc[j] = 0.f;

  int s = 0;
  uint32_t ph = 0;
  bool bad = false;
  for (int k = 0; k < a.nviews; ++k) {
    if (!mbar_wait(&full[s], ph, a.err)) {
      *s_abort = 1;
      break;
    }
    const ViewCoef g = coef[s];
    if (!g.skip) {
      const float D = fmaf(g.Dx, fx, fmaf(g.Dz, fz, g.D0));
      const float rD = __frcp_rn(D);
      const float ul = fmaf(g.Nx, fx, fmaf(g.Nz, fz, g.N0)) * rD;
      const float vl = fmaf(g.Vx, fx, fmaf(g.Vz, fz, g.V0)) * rD;
      const float dvv = a.dvn * rD;
      const float W = rD * rD * g.wscale;
      const float fuf = floorf(ul);
      const int iu = (int)fuf;
      const float fu = ul - fuf;
      const float vlast = fmaf((float)(NY - 1), dvv, vl);
      const int BU = g.box & 0xffff, BV = g.box >> 16;
      const uint32_t RB = (uint32_t)(BU * ESZ);
      // exclusive bound on v, kSlack / 2 inside the window: the footprint pass
      // leaves kSlack, so the guard never trips for a voxel of the tile, and
      // the rounded row index can never pass the last staged row
      const float vmax_ok = (float)(BV - kRowTail) - (float)(kSlack / 2);
      if (iu >= 0 && iu <= BU - 2 && vl >= 0.f && vlast < vmax_ok) {
        const float wa = W - W * fu, wb = W * fu;
        const uint32_t c0 = smem_u32(smem + (size_t)s * a.box_bytes) + (uint32_t)(iu * ESZ) - kMagicBits * RB;
#pragma unroll
        for (int j = 0; j < NY; ++j) tap<LAYOUT>(fmaf((float)j, dvv, vl), c0, RB, wa, wb, fu, W, acc[j]);
      } else {
        bad = true;  // cannot happen when the footprint pass is right; recorded below
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (++s == S) {
      s = 0;
      ph ^= 1;
    }
  }
  if (bad) atomicCAS(a.err, 0, kDevFootprint);
  if (*s_abort) return;

  const int ix = ix0 + tx, iz = iz0 + tz;
  float lo = __int_as_float(0x7f800000), hi = -lo;
  if (ix < a.nx && iz < a.nz) {
    float* out = a.vol + ((size_t)iz * a.vol_ystride) * a.nx + ix;
#pragma unroll
    for (int j = 0; j < NY; ++j) {
      const int iy = iy0 + j;
      if (iy < a.ny) {
        float r = acc[j] * a.scale;
        if (iy < a.clip_ylimit) r = fmaxf(r, 0.f);
        out[(size_t)iy * a.nx] = r;
        lo = fminf(lo, r);
        hi = fmaxf(hi, r);
      }
    }
  }
  if (a.minmax) fold_minmax(a.minmax, lo, hi);
}

// ---------------------------------------------------------------------------
// Four-fold symmetric backprojector.
//
// On a circular orbit with K views over one turn (K % 4 == 0) and a square
// volume (nx == nz), voxel P = (X, Z) at view k and the voxel rotated by 90
// degrees, (-Z, X), at view k + K/4 project to the same detector coordinate
// (t = X cos + Z sin and s = -X sin + Z cos are unchanged). A CTA therefore
// owns an orbit of four 16 x 16 x NY tiles (a tile of the lower-left quadrant
// and its three rotations) and walks all K views m of the representative
// tile: the producer computes the tile footprint and coefficients once per m
// and stages the windows of views m + r K/4 (mod K), r = 0..3 (same origin
// and box), which feed the r-th rotated tile; each consumer thread forms its
// detector column, weights and v steps once per m and applies every
// floor / fraction / address to four accumulator sets. Windows live in a byte ring
// (entries of variable size, freed in order), so typical small windows keep
// several quads in flight while the largest still fits.

constexpr int kQuadEntries = 8;  // outstanding view-quads per CTA

// Quad record flags.
constexpr int kQSkip = 1;    // the tile footprint misses the detector (or failed a check): no taps
constexpr int kQDirect = 2;  // interleaved layout: window not staged, consumers gather it from global memory
constexpr int kQFirst = 4;   // first quad of a work item (a tile orbit and y-slab of one job)
constexpr int kQLast = 8;    // last quad of a work item: the consumers store its voxels next
constexpr int kQExit = 16;   // multi-job launch: the queue is empty, the CTA leaves

// 16-byte aligned so that consumers read a record with vector loads (96 bytes)
struct alignas(16) QuadCoef {
  float Dx, Dz, D0, Nx, Nz, N0, Vx, Vz, V0;
  float ws[4];  // per-view extra weight of the four views (FP16 views: 1 / scale)
  int flags;    // kQ* bits
  int sub;      // bytes between the entry's four windows
  int u0, e0;   // direct: element column / element row of the window origin
  // consumer constants of the window, formed once by the producer
  uint32_t cbase;  // ring address of element column 0 minus kMagicBits element rows
  uint32_t rb;     // bytes per staged element row
  uint32_t plane;  // interleaved layout: bytes between the 16-byte planes of an element row
  int bu2;         // last element column a tap may start at (box width - 2)
  float vmax;      // exclusive bound on the window-local v of a tap
  float dvn;       // the job's v step per voxel times D
  int item;        // work item of this quad
};
static_assert(sizeof(QuadCoef) == 96, "six 16-byte loads per record");

// Multi-job launch (several reconstructions in one persistent launch): one
// entry per job in global memory; work item item0 + i of job j is the job's
// tile t0 + i (tiles ordered y-slab, then z, then x), so a launch can carry
// a whole job or a range of its tiles.
struct QuadJob {
  BPArgs a;
  long long item0;  // first work item of the job in this launch
  long long t0;     // its tile
  int nbh;          // representative tiles per axis
  int nty;          // y-slabs
};
struct QuadQueue {
  const QuadJob* jobs;    // sorted by item0
  const BoxMaps* maps;    // one grid of tensor maps per job
  int njobs;
  long long nitems;
  unsigned long long* next;  // work-item counter (zero before the launch)
  int* err;                  // device error word of the launch
  int ring;                  // ring bytes of every CTA
};

__device__ __forceinline__ int find_job(const QuadQueue& qq, long long item) {
  int lo = 0, hi = qq.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (qq.jobs[mid].item0 <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <bool MULTI>
__device__ __forceinline__ const BPArgs& job_args(const BPArgs& a, const QuadQueue& qq, int jb) {
  if constexpr (MULTI) return qq.jobs[jb].a;
  else return a;
}
template <bool MULTI>
__device__ __forceinline__ const BoxMaps& job_maps(const BoxMaps& m, const QuadQueue& qq, int jb) {
  if constexpr (MULTI) return qq.maps[jb];
  else return m;
}

// Tile of a work item and the first view (group) of its walk. The walk starts
// at an offset advanced by about K views per `resident` CTAs in tile order
// (interleaved layout: by view groups): tiles that run at the same time then
// read the same views (their windows share L2) instead of all starting at view
// 0. The offset depends only on the tile, so results are the same whichever
// CTA, launch or batch computes it.
//
// Tile order within a y-slab: bands of `band` orbit rows along z, walked
// column by column along x, so the ~`resident` tiles that run at once form a
// near-square patch of the slab (band ~ sqrt(resident)); their windows of one
// view group then span about half the detector columns a slab-wide row of
// tiles would, and DRAM reads of the filtered views fall in proportion.
struct ItemTile {
  int ix0, iy0, iz0;
  int g0, k0;
};
template <bool QG, int NY>
__device__ __forceinline__ ItemTile item_tile(const BPArgs& ja, long long t, int nbh) {
  ItemTile it;
  const long long per = (long long)nbh * nbh;
  const int by = (int)(t / per);
  const int rem = (int)(t - (long long)by * per);
  const int H = min(max(1, ja.band), nbh);
  const int b = rem / (H * nbh);
  const int hb = min(H, nbh - b * H);  // orbit rows in this band (the last may be short)
  const int r2 = rem - b * H * nbh;
  const int bx = r2 / hb, bz = b * H + (r2 - bx * hb);
  it.ix0 = bx * 16;
  it.iz0 = bz * 16;
  it.iy0 = by * NY;
  const int K = ja.nviews;
  it.g0 = QG ? (int)((t * (K >> 2) / max(1, ja.resident)) % (K >> 2)) : 0;
  it.k0 = QG ? 0 : (int)((t * K / max(1, ja.resident)) % K);
  return it;
}

// 288 threads. OCC = 2 CTAs per SM: 9 warps each put 5 warps on some SM
// sub-partitions (16K registers each), so at most 96 registers per thread,
// and each CTA gets half of the shared memory. OCC = 1: up to 168 registers
// and all of the shared memory, for 16 voxels per thread along y (64
// accumulators a thread, the window staged once for twice the voxels).
//
// MULTI = false: one job, one work item (tile orbit and y-slab) per CTA, from
// the block index. MULTI = true: a persistent launch of OCC CTAs per SM over
// the work items of several jobs (uneven sizes, each with its own geometry,
// views and tensor maps, all of one staged layout); the producer takes the
// next item from the queue's counter and streams its quads into the ring
// without a pause between items, the consumers reset their sums at an item's
// first quad and store its voxels after its last. An item's arithmetic and
// view order do not depend on the launch, so a job's volume is the same bits
// alone or batched with others.
template <int LAYOUT, int NY, int OCC, bool MULTI>
__global__ void __launch_bounds__(256 + 32, OCC)
    bp_quad_kernel(const __grid_constant__ BoxMaps maps, const __grid_constant__ BPArgs a,
                   const __grid_constant__ QuadQueue qq) {
  constexpr int TX = 16, TZ = 16, NCW = 8, E = kQuadEntries;
  // QG: the four views of a quad come interleaved in one window (one copy,
  // two 16-byte loads per voxel step feed all four taps). The quads are
  // walked group-major, q = g + m K/4 for m = 0..3, so the slot of rotation
  // r, (m + r) mod 4, is a compile-time index in each of the four unrolled steps.
  // QG24: the same with three 16-byte planes of 24-bit values and no scale.
  constexpr bool QG24 = LAYOUT == kLayoutQuadG24;
  constexpr bool QG = LAYOUT == kLayoutQuadG16 || QG24;
  constexpr int ESZ = QG24 ? 48 : QG ? 32 : LAYOUT == kLayoutPair32 ? 8 : 4;
  constexpr int NPL = QG24 ? 3 : 2;  // 16-byte planes per element row
  constexpr int kRowTail = LAYOUT == kLayoutRaw32 ? 1 : 0;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int R = MULTI ? qq.ring : a.box_bytes;  // ring bytes
  int* const err = MULTI ? qq.err : a.err;

  QuadCoef* coef = reinterpret_cast<QuadCoef*>(smem + R);
  uint64_t* full = reinterpret_cast<uint64_t*>(coef + E);
  uint64_t* empty = full + E;
  // end_pos: ring byte position (64-bit: a persistent CTA allocates far more
  // than 2^31 bytes over its items) where each entry's windows end
  long long* end_pos = reinterpret_cast<long long*>(empty + E);
  volatile int* s_abort = reinterpret_cast<volatile int*>(end_pos + E);

  if (tid == 0) {
    *s_abort = *(volatile int*)err != 0;
    for (int e = 0; e < E; ++e) {
      mbar_init(&full[e], 1);
      mbar_init(&empty[e], NCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (*s_abort) return;

  if (warp == NCW) {
    // ---------------------------------------------------------------- producer
    // head / tail: ring bytes allocated / freed; hpos = head mod R; oldest:
    // first quad not yet known to be released; seq: quads issued since the
    // launch (all items)
    long long head = 0, tail = 0;
    int hpos = 0, oldest = 0, seq = 0;
    bool more = true, first = true;
    while (more && !*s_abort) {
      // the next work item: this CTA's tile, or the queue's next item
      long long item;
      if constexpr (MULTI) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(qq.next, 1ull);
        item = (long long)__shfl_sync(0xffffffffu, t, 0);
        if (item >= qq.nitems) break;
      } else {
        if (!first) break;
        item = (long long)blockIdx.y * gridDim.x + blockIdx.x;
      }
      first = false;
      const int jb = MULTI ? find_job(qq, item) : 0;
      const BPArgs& ja = job_args<MULTI>(a, qq, jb);
      const BoxMaps& jm = job_maps<MULTI>(maps, qq, jb);
      const long long t_local = MULTI ? item - qq.jobs[jb].item0 + qq.jobs[jb].t0 : item;
      const ItemTile til = item_tile<QG, NY>(ja, t_local, MULTI ? qq.jobs[jb].nbh : ja.ntx >> 1);
      const int K = ja.nviews, Q = K >> 2;
      for (int kb = 0; kb < K && !*s_abort; kb += 32) {
        const int it = kb + lane;  // quad of the item (ring entry order)
        // view of the representative tile; rotation r uses view (k + r Q) mod K
        const int gq = QG ? ((it >> 2) + til.g0) % Q : 0;  // view group of quad it
        const int k = QG ? gq + (it & 3) * Q : (it + til.k0) % K;
        QuadCoef qc;
        int u0 = 0, v0 = 0, mi = 0, need = 0, sub = 0, tx_bytes = 0;
        bool skip = true, direct = false;
        qc.flags = kQSkip;
        qc.rb = 0;
        if (it < K) {
          ViewCoef vc;
          bool overflow = false, behind = false;
          int need_u = 0, need_v = 0;
          skip = tile_view_coef(ja, k, til.ix0, til.iy0, til.iz0, TX - 1, NY - 1, TZ - 1, vc, u0, v0, need_u,
                                need_v, overflow, behind);
          // checks of the job's geometry go to the job's error word
          if (overflow) atomicCAS(ja.err, 0, kDevFootprint);
          if (behind) atomicCAS(ja.err, 0, kDevGeometry);
          if (overflow || behind) skip = true;
          int wi = 0, hi = 0;
          const int rows = need_v - ja.pair_rows;
          while (wi < kNW - 1 && jm.w[wi] < need_u) ++wi;
          while (hi < kNH - 1 && jm.h[hi] < rows) ++hi;
          mi = wi * kNH + hi;
          tx_bytes = jm.w[wi] * jm.h[hi] * ESZ;
          sub = (tx_bytes + 127) & ~127;
          // interleaved layout: a window wider than the widest box or larger than
          // the ring (rare near-source tiles) is read from global memory instead
          direct = QG && !skip && (need_u > jm.w[kNW - 1] || rows > jm.h[kNH - 1] || sub > R);
          need = (skip || direct) ? 0 : (QG ? sub : 4 * sub);
          qc.Dx = vc.Dx; qc.Dz = vc.Dz; qc.D0 = vc.D0;
          qc.Nx = vc.Nx; qc.Nz = vc.Nz; qc.N0 = vc.N0;
          qc.Vx = vc.Vx; qc.Vz = vc.Vz; qc.V0 = vc.V0;
#pragma unroll
          for (int r = 0; r < 4; ++r) qc.ws[r] = ja.inv_scale ? ja.inv_scale[(k + r * Q) % K] : 1.0f;
          qc.flags = (skip ? kQSkip : 0) | (direct ? kQDirect : 0) | (it == 0 ? kQFirst : 0) |
                     (it == K - 1 ? kQLast : 0);
          // window: width (elements) and rows
          const int BU = direct ? need_u : jm.w[wi], BV = direct ? rows : jm.h[hi];
          qc.sub = sub;
          qc.u0 = u0 + 1;
          qc.e0 = v0 + ja.pair_rows;
          qc.rb = (uint32_t)(BU * ESZ);
          qc.plane = (uint32_t)(BU * 16);
          qc.bu2 = BU - 2;
          qc.vmax = (float)(BV - kRowTail) - (float)(kSlack / 2);
          qc.dvn = ja.dvn;
          qc.item = (int)item;
        }
        const int nb = min(32, K - kb);
        for (int i = 0; i < nb; ++i) {
          const int q = seq + i;  // ring sequence number
          const int e = q % E;
          const int qneed = __shfl_sync(0xffffffffu, need, i);
          // allocate qneed contiguous ring bytes: wrap to 0 when the tail end is too short
          const bool wrap = hpos + qneed > R;
          const long long start = wrap ? head + (R - hpos) : head;
          bool ok = true;
          while (oldest < q && (oldest <= q - E || start + qneed - tail > R)) {
            if (!mbar_wait(&empty[oldest % E], (oldest / E) & 1, err)) {
              ok = false;
              break;
            }
            tail = end_pos[oldest % E];
            ++oldest;
          }
          if (!ok) {
            *s_abort = 1;
            more = false;
            break;
          }
          if (oldest == q) tail = start;  // nothing outstanding: the whole ring is free
          const int off = wrap ? 0 : hpos;  // start mod R
          if (lane == i) {
            qc.cbase = smem_u32(smem) + (uint32_t)off - kMagicBits * qc.rb;
            coef[e] = qc;
          }
          if (lane == 0) end_pos[e] = start + qneed;
          head = start + qneed;
          hpos = off + qneed == R ? 0 : off + qneed;
          const int sk = __shfl_sync(0xffffffffu, (int)(skip || direct), i);
          const int cu0 = __shfl_sync(0xffffffffu, u0, i), cv0 = __shfl_sync(0xffffffffu, v0, i);
          const int cmi = __shfl_sync(0xffffffffu, mi, i), csub = __shfl_sync(0xffffffffu, sub, i);
          const int ctx = __shfl_sync(0xffffffffu, tx_bytes, i);
          // view of the representative tile at quad kb + i (the interleaved layout addresses its group)
          const int ck = QG ? 0 : __shfl_sync(0xffffffffu, k, i);
          __syncwarp();
          if (lane == 0) {
            if (sk) {
              mbar_arrive(&full[e]);
            } else if (QG) {
              // group gq, slots = views gq + s Q; element column u0 + 1 holds columns u0, u0 + 1
              mbar_arrive_expect_tx(&full[e], (uint32_t)ctx);
              tma_load_4d(smem + off, &jm.map[cmi], 2 * (cu0 + 1), 0, cv0 + ja.pair_rows,
                          (((kb + i) >> 2) + til.g0) % Q, &full[e]);
            } else {
              mbar_arrive_expect_tx(&full[e], (uint32_t)(4 * ctx));
              const CUtensorMap* m = &jm.map[cmi];
              const int x = LAYOUT == kLayoutPair32 ? 2 * cu0 : cu0;
              const int e0 = cv0 + ja.pair_rows;
#pragma unroll
              for (int r = 0; r < 4; ++r) {
                void* dst = smem + off + r * csub;
                const int kv = (ck + r * Q) % K;
                if (ja.sino_layout)
                  tma_load_3d(dst, m, x, kv, e0, &full[e]);
                else
                  tma_load_3d(dst, m, x, e0, kv, &full[e]);
              }
            }
          }
          __syncwarp();
        }
        if (!more) break;
        seq += nb;
      }
    }
    if (MULTI && !*s_abort) {
      // queue empty: one record that tells the consumers to leave
      const int q = seq, e = q % E;
      bool ok = true;
      while (oldest < q && oldest <= q - E) {
        if (!mbar_wait(&empty[oldest % E], (oldest / E) & 1, err)) {
          ok = false;
          break;
        }
        ++oldest;
      }
      if (ok) {
        if (lane == 0) {
          coef[e].flags = kQExit | kQSkip;
          mbar_arrive(&full[e]);
        }
        __syncwarp();
        ++seq;
      } else {
        *s_abort = 1;
      }
    }
    // leave only when every copy issued into this CTA's memory has landed
    for (int q = max(0, seq - E); q < seq; ++q) mbar_wait(&full[q % E], (q / E) & 1, err);
    return;
  }

  // ------------------------------------------------------------------ consumers
  // a warp owns 8 x 4 columns; for the interleaved layout each quarter-warp
  // (one shared-memory phase of 16-byte loads) is a compact 4 x 2 patch, whose
  // detector columns stay within 8 elements (no bank conflicts)
  const int tx = QG ? (warp & 1) * 8 + ((lane >> 3) & 1) * 4 + (lane & 3) : (warp & 1) * 8 + (lane & 7);
  const int tz = QG ? (warp >> 1) * 4 + (lane >> 4) * 2 + ((lane >> 2) & 1) : (warp >> 1) * 4 + (lane >> 3);
  const float fx = (float)tx, fz = (float)tz;
  // plain FP32 sums: four rotations x NY voxels in registers (a
  // compensated sum was measured to change no digit of the MIXED form's
  // error, which the FP16 views set, and cost 5% at C4)
  float acc[4][NY];
  // a new work item: zero every sum of this thread
  auto reset = [&]() {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int j = 0; j < NY; ++j) acc[r][j] = 0.f;
  };
  reset();
  int e = 0;
  uint32_t ph = 0;
  bool bad = false, stop = false, last = false, leave = false;
  int grp = 0;        // interleaved layout: view group of the current four quads
  long long item = -1;  // work item being accumulated
  int jb = 0;         // its job
  // one quad: wait for its window, apply it to the 4 x NY voxels, release it
  auto step = [&](auto mc) {
    constexpr int M = decltype(mc)::value;
    if (!mbar_wait(&full[e], ph, err)) {
      *s_abort = 1;
      stop = true;
      return;
    }
    const QuadCoef g = coef[e];
    if constexpr (MULTI) {  // one job's single item: set up before the loop, the loop counts its quads
      if (g.flags & (kQExit | kQFirst)) {
        if (g.flags & kQExit) {  // no more items (always at a group start)
          leave = true;
        } else {
          item = g.item;
          jb = find_job(qq, item);
          const BPArgs& ja = qq.jobs[jb].a;
          const ItemTile til = item_tile<QG, NY>(ja, item - qq.jobs[jb].item0 + qq.jobs[jb].t0, qq.jobs[jb].nbh);
          grp = til.g0;
        }
      }
      last = (g.flags & kQLast) != 0;
    }
    if (!(g.flags & kQSkip)) {
      // explicit roundings (no contraction): the same bits in every instantiation
      const float D = fmaf(g.Dx, fx, fmaf(g.Dz, fz, g.D0));
      const float rD = rcp_approx(D);
      const float ul = __fmul_rn(fmaf(g.Nx, fx, fmaf(g.Nz, fz, g.N0)), rD);
      const float vl = __fmul_rn(fmaf(g.Vx, fx, fmaf(g.Vz, fz, g.V0)), rD);
      const float dvv = __fmul_rn(g.dvn, rD);
      const float W = __fmul_rn(rD, rD);
      const float fuf = floorf(ul);
      const int iu = (int)fuf;
      const float fu = ul - fuf;
      const float vlast = fmaf((float)(NY - 1), dvv, vl);
      const uint32_t RB = g.rb;
      if (iu >= 0 && iu <= g.bu2 && vl >= 0.f && vlast < g.vmax) {
        const uint32_t c0 = g.cbase + (uint32_t)(iu * (QG ? 16 : ESZ));
        const __half2 fu2 = __float2half2_rn(fu);
        if constexpr (QG) {
          float Wr[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) Wr[r] = __fmul_rn(W, g.ws[r]);
          // (A, G) of the four rotations at one voxel from the 2 x 16 bytes of
          // its element (slot of rotation r: (M + r) mod 4): A = u-lerp of row
          // e - 1, G = u-lerp of the row difference
          auto decode = [&](const uint4& L0, const uint4& L1, const uint4& L2, float (&A)[4], float (&G)[4]) {
            if constexpr (QG24) {
              const uint32_t wv[12] = {L0.x, L0.y, L0.z, L0.w, L1.x, L1.y, L1.z, L1.w, L2.x, L2.y, L2.z, L2.w};
              // (A, G) = (a, b - a) + fu (c' - a, d - c' - b + a) for the slot of rotation r
              auto slot = [&](auto slc, float& Ar, float& Gr) {
                constexpr int SL = decltype(slc)::value;
                const float2 ag = ffma2(make_float2(fu, fu), make_float2(dec24<4 * SL + 2>(wv), dec24<4 * SL + 3>(wv)),
                                        make_float2(dec24<4 * SL>(wv), dec24<4 * SL + 1>(wv)));
                Ar = ag.x;
                Gr = ag.y;
              };
              slot(std::integral_constant<int, (M + 0) & 3>{}, A[0], G[0]);
              slot(std::integral_constant<int, (M + 1) & 3>{}, A[1], G[1]);
              slot(std::integral_constant<int, (M + 2) & 3>{}, A[2], G[2]);
              slot(std::integral_constant<int, (M + 3) & 3>{}, A[3], G[3]);
            } else {
              const uint32_t wv[8] = {L0.x, L0.y, L0.z, L0.w, L1.x, L1.y, L1.z, L1.w};
#pragma unroll
              for (int r = 0; r < 4; ++r) {
                const int sl = (M + r) & 3;
                const __half2 X1 = *reinterpret_cast<const __half2*>(&wv[2 * sl]);      // (a, b - a)
                const __half2 X2 = *reinterpret_cast<const __half2*>(&wv[2 * sl + 1]);  // (c' - a, d - c' - b + a)
                const float2 P = __half22float2(X1);
                A[r] = fma_f16_f32(__low2half(fu2), __low2half(X2), P.x);
                G[r] = fma_f16_f32(__low2half(fu2), __high2half(X2), P.y);
              }
            }
          };
          // rotation pairs (0, 1), (2, 3) of one voxel: v-lerp and weighted sum as packed pairs
          auto rot_pairs = [&](const float (&A)[4], const float (&G)[4], float fv, int j) {
#pragma unroll
            for (int pr = 0; pr < 2; ++pr) {
              float& d0 = acc[2 * pr][j];
              float& d1 = acc[2 * pr + 1][j];
              const float2 t = ffma2(make_float2(fv, fv), make_float2(G[2 * pr], G[2 * pr + 1]),
                                     make_float2(A[2 * pr], A[2 * pr + 1]));
              const float2 d = ffma2(make_float2(Wr[2 * pr], Wr[2 * pr + 1]), t, make_float2(d0, d1));
              d0 = d.x;
              d1 = d.y;
            }
          };
          if (!(g.flags & kQDirect)) {
            const uint32_t plane = g.plane;
            static_assert(NY % 2 == 0, "voxels stepped in pairs");
            const float2 magic2 = make_float2(kMagic, kMagic);
            // v of voxels j and j + 1, stepped by 2 dvv from (vl, vl + dvv): no
            // per-pair constants (a few ulps of v from the repeated additions)
            const float dv2 = 2.f * dvv;
            const float2 step2 = make_float2(dv2, dv2);
            float2 v2 = make_float2(vl, vl + dvv);
#pragma unroll
            for (int j = 0; j < NY; j += 2) {
              // floor and fraction of voxels j and j + 1 with packed FP32 ops
              if (j) v2 = fadd2(v2, step2);
              const float2 t2 = fadd2_rz(v2, magic2);
              const float2 fv2 = fsub2(v2, fsub2(t2, magic2));
              const uint32_t a0 = __float_as_uint(t2.x) * RB + c0, a1 = __float_as_uint(t2.y) * RB + c0;
              // slots 0, 1 | slots 2, 3 (QG24: the 48 bytes of the element)
              const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
              float A0[4], G0[4];
              decode(lds_u4(a0), lds_u4(a0 + plane), QG24 ? lds_u4(a0 + 2 * plane) : z4, A0, G0);
              rot_pairs(A0, G0, fv2.x, j);
              decode(lds_u4(a1), lds_u4(a1 + plane), QG24 ? lds_u4(a1 + 2 * plane) : z4, A0, G0);
              rot_pairs(A0, G0, fv2.y, j + 1);
            }
          } else {
            // window not staged: read the elements from global memory (zero
            // outside the stored extent, as the TMA fill would give)
            const BPArgs& ja = job_args<MULTI>(a, qq, jb);
            const int col = g.u0 + iu;
            const bool col_ok = col >= 0 && col < ja.qg_pitch;
            const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
            for (int j = 0; j < NY; ++j) {
              const float v = fmaf((float)j, dvv, vl);
              const float t = __fadd_rz(v, kMagic);
              const float fv = v - (t - kMagic);
              const int row = g.e0 + (int)(__float_as_uint(t) - kMagicBits);
              uint4 L0 = zero, L1 = zero, L2 = zero;
              if (col_ok && row >= 0 && row < ja.qg_rows) {
                const uint4* p = ja.qg + ((size_t)grp * ja.qg_rows + row) * NPL * ja.qg_pitch + col;
                L0 = __ldg(p);
                L1 = __ldg(p + ja.qg_pitch);
                if (QG24) L2 = __ldg(p + 2 * ja.qg_pitch);
              }
              float A[4], G[4];
              decode(L0, L1, L2, A, G);
              rot_pairs(A, G, fv, j);
            }
          }
        } else {
          const uint32_t sub = (uint32_t)g.sub;
          float wa[4], wb[4], Wr[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            Wr[r] = __fmul_rn(W, g.ws[r]);
            wb[r] = __fmul_rn(Wr[r], fu);
            wa[r] = __fsub_rn(Wr[r], wb[r]);
          }
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            const float v = fmaf((float)j, dvv, vl);
#pragma unroll
            for (int r = 0; r < 4; ++r)
              tap<LAYOUT>(v, c0 + r * sub, RB, wa[r], wb[r], fu, Wr[r],
                          acc[r][j]);
          }
        }
      } else {
        bad = true;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[e]);
    if (++e == E) {
      e = 0;
      ph ^= 1;
    }
  };
  // the item's sums into its voxels: four rotated columns,
  // (x, z) -> (n-1-z, x) -> (n-1-x, n-1-z) -> (z, n-1-x)
  auto store = [&]() {
    const BPArgs& ja = job_args<MULTI>(a, qq, jb);
    const ItemTile til = item_tile<QG, NY>(ja, MULTI ? item - qq.jobs[jb].item0 + qq.jobs[jb].t0 : item,
                                           MULTI ? qq.jobs[jb].nbh : a.ntx >> 1);
    const int n = ja.nx;
    const int ix = til.ix0 + tx, iz = til.iz0 + tz;
    const int cx[4] = {ix, n - 1 - iz, n - 1 - ix, iz};
    const int cz[4] = {iz, ix, n - 1 - iz, n - 1 - ix};
    float* const vol = ja.vol;
    const int ystride = ja.vol_ystride, ny = ja.ny, ylim = ja.clip_ylimit;
    const float scale = ja.scale;
    float lo = __int_as_float(0x7f800000), hi = -lo;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      float* out = vol + ((size_t)cz[r] * ystride) * n + cx[r];
#pragma unroll
      for (int j = 0; j < NY; ++j) {
        const int iy = til.iy0 + j;
        if (iy < ny) {
          float val = acc[r][j] * scale;
          if (iy < ylim) val = fmaxf(val, 0.f);
          out[(size_t)iy * n] = val;
          lo = fminf(lo, val);
          hi = fmaxf(hi, val);
        }
      }
    }
    if (ja.minmax) fold_minmax(ja.minmax, lo, hi);
  };
  if constexpr (!MULTI) {
    // one work item, K quads (as many as views): a loop of known length
    item = (long long)blockIdx.y * gridDim.x + blockIdx.x;
    const int K = a.nviews;
    if constexpr (QG) {
      grp = item_tile<QG, NY>(a, item, a.ntx >> 1).g0;
      const int Q = K >> 2;
      for (int q = 0; q < K; q += 4) {
        step(std::integral_constant<int, 0>{});
        if (stop) break;
        step(std::integral_constant<int, 1>{});
        if (stop) break;
        step(std::integral_constant<int, 2>{});
        if (stop) break;
        step(std::integral_constant<int, 3>{});
        if (stop) break;
        if (++grp == Q) grp = 0;
      }
    } else {
      for (int q = 0; q < K; ++q) {
        step(std::integral_constant<int, 0>{});
        if (stop) break;
      }
    }
    if (bad) atomicCAS(a.err, 0, kDevFootprint);
    if (stop || *s_abort) return;
    store();
    return;
  }
  for (;;) {
    if constexpr (QG) {
      // a group of four quads (an item's quads come in whole groups)
      step(std::integral_constant<int, 0>{});
      if (stop || leave) break;
      step(std::integral_constant<int, 1>{});
      if (stop) break;
      step(std::integral_constant<int, 2>{});
      if (stop) break;
      step(std::integral_constant<int, 3>{});
      if (stop) break;
      const int Qj = job_args<MULTI>(a, qq, jb).nviews >> 2;
      if (++grp == Qj) grp = 0;
    } else {
      step(std::integral_constant<int, 0>{});
      if (stop || leave) break;
    }
    if (last) {
      if (bad) atomicCAS(job_args<MULTI>(a, qq, jb).err, 0, kDevFootprint);
      bad = false;
      if (*s_abort) break;
      store();
      if (!MULTI) break;
      reset();
      last = false;
    }
  }
  if (bad) atomicCAS(err, 0, kDevFootprint);
}

// Footprint pre-pass: one warp per tile (lanes over views) finds the
// largest window any (tile, view) needs; same FP64 code as the
// backprojector's producer, so the largest box always fits. With `hist`, it
// also counts the windows by (width, height), clamped to kBoxHist - 1, in a
// shared-memory histogram (kBoxHist^2 counters) added to `hist` at the end.
template <int TX, int TZ, int NY>
__global__ void footprint_kernel(BPArgs a, int nty, int* spans, unsigned* hist) {
  extern __shared__ unsigned sh_hist[];
  if (hist)
    for (int i = threadIdx.x; i < kBoxHist * kBoxHist; i += blockDim.x) sh_hist[i] = 0u;
  __syncthreads();
  const long long ntiles = (long long)a.ntx * a.ntz * nty;
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  int gu = 0, gv = 0;
  for (long long T = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); T < ntiles; T += warps) {
    const int by = (int)(T / ((long long)a.ntx * a.ntz));
    const int rr = (int)(T - (long long)by * a.ntx * a.ntz);
    const int bz = rr / a.ntx, bx = rr - bz * a.ntx;
    const int ix0 = bx * TX, iz0 = bz * TZ, iy0 = by * NY;
    for (int k = lane; k < a.nviews; k += 32) {
      TileGeo g;
      // full tile extents, as the backprojector's producer uses them
      tile_geo(a, k, ix0, iy0, iz0, TX - 1, NY - 1, TZ - 1, g);
      if (g.dmin <= 1e-6) atomicCAS(a.err, 0, kDevGeometry);
      if (tile_skip(a, g)) continue;
      int u0, v0, nu_, nv_;
      tile_window(a, g, u0, v0, nu_, nv_);
      gu = max(gu, nu_);
      gv = max(gv, nv_);
      if (hist)
        atomicAdd(&sh_hist[min(max(nu_, 0), kBoxHist - 1) * kBoxHist + min(max(nv_, 0), kBoxHist - 1)], 1u);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    gu = max(gu, __shfl_xor_sync(0xffffffffu, gu, o));
    gv = max(gv, __shfl_xor_sync(0xffffffffu, gv, o));
  }
  if (lane == 0) {
    atomicMax(spans, gu);
    atomicMax(spans + 1, gv);
  }
  __syncthreads();
  if (hist)
    for (int i = threadIdx.x; i < kBoxHist * kBoxHist; i += blockDim.x)
      if (sh_hist[i]) atomicAdd(&hist[i], sh_hist[i]);
}

__global__ void clip_kernel(float* vol, int nx, int ny, int nz, int ylim) {
  const long long total = (long long)nx * ny * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long iy = (e / nx) % ny;
    if (iy < ylim) vol[e] = fmaxf(vol[e], 0.f);
  }
}

// Fan (flat detector) -> parallel rebinning; see the C ABI comment.
__global__ void rebin_fan_kernel(const float* fan, int bins, int views, double sod, double sdd, double du,
                                 double span, double offset, float* par, int out_bins, double du_out) {
  const long long total = (long long)views * out_bins;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int k = (int)(e / out_bins), j = (int)(e % out_bins);
    double th = offset + span * k / views;
    double s = (j + 0.5 - out_bins / 2.0) * du_out;
    float val = 0.f;
    if (fabs(s) < sod) {
      double gam = asin(s / sod);
      double beta = th - gam;
      double ui = sdd * tan(gam) / du + bins / 2.0 - 0.5;
      double bi = (beta - offset) / (span / views);
      double bf = floor(bi), ab = bi - bf;
      long long b0 = (long long)bf;
      double fu = floor(ui), au = ui - fu;
      long long iu = (long long)fu;
      double acc = 0.0;
      for (int t = 0; t < 2; ++t) {
        long long bb = (((b0 + t) % views) + views) % views;
        const float* row = fan + bb * bins;
        double p0 = (iu >= 0 && iu < bins) ? row[iu] : 0.0;
        double p1 = (iu + 1 >= 0 && iu + 1 < bins) ? row[iu + 1] : 0.0;
        double r = p0 * (1 - au) + p1 * au;
        acc += t ? r * ab : r * (1 - ab);
      }
      val = (float)acc;
    }
    par[e] = val;
  }
}

template <int LAYOUT, int TX, int TZ, int NY>
cudaError_t launch_cfg(const BoxMaps& maps, const BPArgs& a, size_t smem, cudaStream_t stream) {
  auto kern = bp_kernel<LAYOUT, TX, TZ, NY>;
  // The attribute is process-wide: contexts on other threads launch this kernel
  // with other sizes, so it is always raised to the device maximum (a launch
  // still uses only its own dynamic size).
  (void)smem;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  dim3 grid(a.ntx * a.ntz, (a.ny + NY - 1) / NY);
  kern<<<grid, TX * TZ + 32, smem, stream>>>(maps, a);
  return cudaGetLastError();
}

template <int LAYOUT, int NY, int OCC>
cudaError_t launch_quad_cfg(const BoxMaps& maps, const BPArgs& a, size_t smem, cudaStream_t stream) {
  auto kern = bp_quad_kernel<LAYOUT, NY, OCC, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
  if (e != cudaSuccess) return e;
  // all of L1 as shared memory, so that two CTAs of up to 113 KB share an SM
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  dim3 grid((a.ntx / 2) * (a.ntz / 2), (a.ny + NY - 1) / NY);
  kern<<<grid, 256 + 32, smem, stream>>>(maps, a, QuadQueue{});
  return cudaGetLastError();
}

template <int NY, int OCC>
cudaError_t launch_quad_ny(int layout, const BoxMaps& maps, const BPArgs& a, size_t smem, cudaStream_t stream) {
  switch (layout) {
    case kLayoutPair32:
      return launch_quad_cfg<kLayoutPair32, NY, OCC>(maps, a, smem, stream);
    case kLayoutPair16:
      return launch_quad_cfg<kLayoutPair16, NY, OCC>(maps, a, smem, stream);
    case kLayoutQuadG16:
      return launch_quad_cfg<kLayoutQuadG16, NY, OCC>(maps, a, smem, stream);
    case kLayoutQuadG24:
      return launch_quad_cfg<kLayoutQuadG24, NY, OCC>(maps, a, smem, stream);
    default:
      return launch_quad_cfg<kLayoutRaw32, NY, OCC>(maps, a, smem, stream);
  }
}

cudaError_t launch_quad(int layout, int ny_tile, const BoxMaps& maps, const BPArgs& a, size_t smem,
                        cudaStream_t stream) {
  return ny_tile == 16 ? launch_quad_ny<16, 1>(layout, maps, a, smem, stream)
                       : launch_quad_ny<8, 2>(layout, maps, a, smem, stream);
}

template <int TX, int TZ, int NY>
cudaError_t launch_layout(int layout, const BoxMaps& maps, const BPArgs& a, size_t smem, cudaStream_t stream) {
  switch (layout) {
    case kLayoutPair32:
      return launch_cfg<kLayoutPair32, TX, TZ, NY>(maps, a, smem, stream);
    case kLayoutPair16:
      return launch_cfg<kLayoutPair16, TX, TZ, NY>(maps, a, smem, stream);
    default:
      return launch_cfg<kLayoutRaw32, TX, TZ, NY>(maps, a, smem, stream);
  }
}

}  // namespace

// A box width whose shared-memory row stride (planes x width sixteen-byte
// units) is 3, 4 or 5 mod 8.
static bool bank_friendly(int planes, int w) {
  const int r = (planes * w) % 8;
  return r >= 3 && r <= 5;
}

// Per-view (cos, sin) of theta_k = offset + span k / K in FP64, computed on
// the device (no host staging, so a new view set needs no stream sync) and
// kept while the view set stays the same.
__global__ void trig_kernel(double2* trig, int n, double offset, double span) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double sn, cs;
  sincos(offset + span * k / n, &sn, &cs);
  trig[k] = make_double2(cs, sn);
}

int ensure_trig(fbp_context* ctx, const BPGeom& g) {
  if (ctx->trig_cap < g.nviews) {
    cudaFree(ctx->d_trig);
    ctx->d_trig = nullptr;
    ctx->trig_cap = 0;
    ctx->trig_key[0] = -1;
    if (cuda_check(ctx, cudaMalloc(&ctx->d_trig, sizeof(double2) * g.nviews), "cudaMalloc(trig)"))
      return FBP_ERR_OUT_OF_MEMORY;
    ctx->trig_cap = g.nviews;
  }
  if (ctx->trig_key[0] == g.nviews && ctx->trig_key[1] == g.span && ctx->trig_key[2] == g.offset) return FBP_OK;
  trig_kernel<<<(g.nviews + 127) / 128, 128, 0, ctx->stream>>>(ctx->d_trig, g.nviews,
                                                                g.offset, g.span);
  if (int rc = launched(ctx, "trig_kernel")) return rc;
  ctx->trig_key[0] = g.nviews;
  ctx->trig_key[1] = g.span;
  ctx->trig_key[2] = g.offset;
  return FBP_OK;
}

// Thresholds t_0 < ... < t_{n-1} = the last candidate, taken from `cand`
// (ascending), minimising sum_v weight[v] * (smallest t_i >= v) over the
// values v = 0 .. weight.size() - 1 (weights of values above the last
// candidate are ignored): dynamic program over the candidates. Fewer
// candidates than n repeat the last threshold.
static void best_thresholds(const std::vector<double>& weight, const std::vector<int>& cand, int n, int* out) {
  const int C = (int)cand.size();
  // W[j] = total weight of the values <= cand[j]
  std::vector<double> W(C, 0.0);
  for (int j = 0; j < C; ++j) {
    double acc = 0.0;
    for (int v = 0; v < (int)weight.size() && v <= cand[j]; ++v) acc += weight[v];
    W[j] = acc;
  }
  const double inf = 1e300;
  std::vector<double> dp((size_t)(n + 1) * C, inf);
  std::vector<int> from((size_t)(n + 1) * C, -1);
  for (int j = 0; j < C; ++j) dp[(size_t)1 * C + j] = cand[j] * W[j];
  for (int m = 2; m <= n; ++m)
    for (int j = 0; j < C; ++j)
      for (int i = 0; i < j; ++i) {
        const double c = dp[(size_t)(m - 1) * C + i] + cand[j] * (W[j] - W[i]);
        if (c < dp[(size_t)m * C + j]) {
          dp[(size_t)m * C + j] = c;
          from[(size_t)m * C + j] = i;
        }
      }
  // the most thresholds that the candidates allow, ending at the last one
  int m = std::min(n, C);
  int j = C - 1;
  std::vector<int> t;
  for (; m >= 1 && j >= 0; --m) {
    t.push_back(cand[j]);
    j = from[(size_t)m * C + j];
  }
  std::sort(t.begin(), t.end());
  for (int i = 0; i < n; ++i) out[i] = t[std::min(i, (int)t.size() - 1)];
}

// The backprojector's box grid for one plan: kBoxGrid widths (multiples of
// align, the largest = mbu) and kBoxGrid heights (the largest = mbv) that
// minimise the staged window area summed over the footprint histogram, by
// alternating the width and the height programs (each exact for the other
// fixed). Windows larger than the largest box are left out (they take the
// direct path or fail the footprint check). Without a histogram: a linear
// grid, each of the quarters 1/4 .. 4/4 of the largest window in each
// dimension taken twice.
static void choose_boxes(const std::vector<unsigned>& hist, int mbu, int mbv, int align, int pair_rows, int planes,
                         int* w, int* h) {
  const int n = kBoxGrid, B = kBoxHist;
  for (int i = 0; i < n; ++i) {
    const int quarter = i / 2 + 1;
    const int wi = (mbu * quarter + 3) / 4;
    w[i] = std::max(align, (wi + align - 1) / align * align);
    h[i] = std::max(1, (mbv * quarter + 3) / 4);
  }
  w[n - 1] = mbu;
  h[n - 1] = mbv;
  if ((int)hist.size() != B * B) return;
  // counts over (width rounded up to align, rows staged)
  const int U = std::max(mbu, 1) + 1, V = std::max(mbv, 1) + 1;
  std::vector<double> cnt((size_t)U * V, 0.0);
  double total = 0.0;
  for (int nu = 0; nu < B; ++nu)
    for (int nv = 0; nv < B; ++nv) {
      const unsigned c = hist[(size_t)nu * B + nv];
      if (!c) continue;
      const int u = std::max(align, (nu + align - 1) / align * align);
      const int r = std::max(1, nv - pair_rows);
      if (u > mbu || r > mbv) continue;
      cnt[(size_t)u * V + r] += c;
      total += c;
    }
  if (total <= 0.0) return;
  // widths: multiples of align; with planes > 0 (interleaved layouts, 16-byte
  // planes) only those whose row stride is 3 to 5 mod 8 sixteen-byte units,
  // so that the quarter-warp's two voxel rows (same detector column, next
  // element row) fall in different bank groups (a simulation of the C4
  // access pattern: 1.22 wavefronts per 16-byte load phase at 4 mod 8, 1.23
  // at 3 or 5, against 1.31 at 2 or 6 and 1.44 at 0)
  std::vector<int> cu, cv;
  for (int u = align; u <= mbu; u += align)
    if (planes <= 0 || bank_friendly(planes, u)) cu.push_back(u);
  if (cu.empty() || cu.back() != mbu) cu.push_back(mbu);
  for (int r = 1; r <= mbv; ++r) cv.push_back(r);
  auto pick = [](const int* t, int n, int x) {
    for (int i = 0; i < n; ++i)
      if (t[i] >= x) return t[i];
    return t[n - 1];
  };
  for (int it = 0; it < 3; ++it) {
    std::vector<double> wu(U, 0.0), wv(V, 0.0);
    for (int u = 0; u < U; ++u)
      for (int r = 0; r < V; ++r) {
        const double c = cnt[(size_t)u * V + r];
        if (c) wu[u] += c * pick(h, n, r);
      }
    best_thresholds(wu, cu, n, w);
    for (int u = 0; u < U; ++u)
      for (int r = 0; r < V; ++r) {
        const double c = cnt[(size_t)u * V + r];
        if (c) wv[r] += c * pick(w, n, u);
      }
    best_thresholds(wv, cv, n, h);
  }
}

// A planned backprojection: everything a launch needs (arguments, tensor
// maps, shared memory) after the footprint pass and the packing.
struct BPLaunchPlan {
  BPArgs a;
  BoxMaps maps;
  size_t smem = 0;
  int layout = 0, ny_tile = 0, occ = 2;
  bool use_quad = false, is2d = false;
};

BPLaunchPlan* new_bp_plan() { return new BPLaunchPlan(); }
void free_bp_plan(BPLaunchPlan* p) { delete p; }

int plan_backproject(fbp_context* ctx, const BPGeom& g, Stack& st, float* vol, int clip_ylimit, bool mixed,
                     BPLaunchPlan* plan_out) {
  const double pi = 3.14159265358979323846;
  // MIXED24: 24-bit views for the symmetric kernel (FP32 rows otherwise)
  const bool c24 = mixed && ctx->precision == FBP_PRECISION_MIXED24;
  // Four-fold symmetric path: square volume, views over one turn (or
  // 4m + 1 turns) with K % 4 == 0, an even number of 16-wide tiles per axis.
  const bool is2d = g.ny == 1;
  const double turns = g.span / (2.0 * pi);
  const long long iturns = llround(turns);
  const bool symmetric = !is2d && g.nx == g.nz && g.nx % 32 == 0 && g.nviews % 4 == 0 &&
                         fabs(turns - (double)iturns) < 1e-9 && iturns % 4 == 1;
  const bool quad = symmetric && (ctx->bp_variant == FBP_BACKPROJECTOR_AUTO ||
                                  ctx->bp_variant == FBP_BACKPROJECTOR_SYMMETRIC);
  if (ctx->bp_variant == FBP_BACKPROJECTOR_SYMMETRIC && !symmetric)
    return set_error(ctx, FBP_ERR_UNSUPPORTED,
                     "the four-fold symmetric backprojector needs nx == nz (a multiple of 32), views % 4 == 0 and "
                     "views over one full turn");
  // MIXED forms over f32 rows: packed for the selected kernel below
  const bool packed = mixed && !st.filtered && (quad || !c24);
  const int layout = st.filtered ? st.filt_layout
                     : packed    ? (quad ? (c24 ? kLayoutQuadG24 : kLayoutQuadG16) : kLayoutPair16)
                                 : kLayoutRaw32;
  const int esize = Stack::elem_bytes(layout);
  BPArgs a{};
  a.vol = vol;
  a.nx = g.nx;
  a.ny = g.ny;
  a.nz = g.nz;
  a.nu = g.nu;
  a.nv = g.nv;
  a.nviews = g.nviews;
  a.kind = g.kind;
  a.sod = g.sod;
  a.sdd = g.sdd;
  a.du = g.du;
  a.dv = g.dv;
  a.vox = g.vox;
  a.cu = 0.5 * g.nu - 0.5;
  // row band of a taller detector / y-slab of a taller volume (sharding)
  a.cv = 0.5 * (g.nv_total > 0 ? g.nv_total : g.nv) - 0.5 - g.row_off;
  a.y_off = g.y_off;
  a.vol_ystride = g.vol_ystride > 0 ? g.vol_ystride : g.ny;
  a.ny_total = g.ny_total > 0 ? g.ny_total : g.ny;
  if (g.kind == FBP_GEOMETRY_CONE) {
    a.dvn = (float)(g.sdd / (g.sod * g.dv) * g.vox);
    a.scale = (float)(pi / g.nviews * g.sdd / (g.sod * g.du));
  } else {
    a.dvn = (float)(g.vox / g.dv);
    a.scale = (float)(pi / g.nviews / g.du);
  }
  a.inv_scale = (layout == kLayoutPair16 || layout == kLayoutQuadG16) ? st.inv_scale : nullptr;
  // TMA: x * element size must be a multiple of 16 bytes (the interleaved
  // layouts' x counts 8-byte words, two per 16-byte plane element: always even)
  a.align = is_quad_layout(layout) ? 1 : layout == kLayoutPair32 ? 2 : 4;
  a.sino_layout = st.sinogram ? 1 : 0;
  a.pair_rows = layout == kLayoutRaw32 ? 0 : 1;
  a.clip_ylimit = clip_ylimit;
  a.err = ctx->d_err;

  // per-view trig in FP64 (cached per view set)
  if (int rc = ensure_trig(ctx, g)) return rc;
  a.trig = ctx->d_trig;

  // tile configuration: 16 x 16 columns, NY voxels along y (1 for 2D)
  // symmetric kernel: 16 voxels per thread along y with one CTA per SM, or 8
  // with two (a per-context choice; 0 = 16)
  const int quad_ny = ctx->quad_tile_ny == 8 ? 8 : 16;
  const int TX = 16, TZ = 16,
            NY = is2d ? 1 : quad ? quad_ny : (ctx->bp_variant == FBP_BACKPROJECTOR_GENERIC_Y8 ? 8 : 16);
  a.ntx = (g.nx + TX - 1) / TX;
  a.ntz = (g.nz + TZ - 1) / TZ;
  const int nty = (g.ny + NY - 1) / NY;

  // footprint pre-pass (cached per geometry and layout)
  double key[20] = {(double)g.kind, g.sod, g.sdd, g.du, g.dv, g.vox, g.span, g.offset, (double)g.nu,
                    (double)g.nv, (double)g.nviews, (double)g.nx, (double)g.ny, (double)g.nz,
                    (double)a.align, (double)NY, (double)g.row_off, (double)g.nv_total, (double)g.y_off,
                    (double)g.ny_total};
  fbp_context::BPPlan* found = nullptr;
  for (auto& p : ctx->plans) {
    bool same = p.valid;
    for (int i = 0; i < 20 && same; ++i) same = p.key[i] == key[i];
    if (same) {
      found = &p;
      break;
    }
  }
  // a plan made without the histogram (not a symmetric candidate then) is
  // redone in place when the symmetric kernel may now run
  const bool redo = found && quad && found->hist.empty();
  const bool hit = found != nullptr && !redo;
  fbp_context::BPPlan& plan = found ? *found : ctx->plans[ctx->plan_next];
  if (!hit) {
    if (!found) ctx->plan_next = (ctx->plan_next + 1) % (int)(sizeof(ctx->plans) / sizeof(ctx->plans[0]));
    plan.valid = false;
    // 4 span words, then the (width, height) histogram
    constexpr int kSpanWords = 4 + kBoxHist * kBoxHist;
    if (ctx->span_cap < kSpanWords) {
      cudaFree(ctx->d_span);
      ctx->d_span = nullptr;
      ctx->span_cap = 0;
      if (cuda_check(ctx, cudaMalloc(&ctx->d_span, sizeof(int) * kSpanWords), "cudaMalloc(footprint spans)"))
        return FBP_ERR_OUT_OF_MEMORY;
      ctx->span_cap = kSpanWords;
    }
    // the window histogram only for the symmetric kernel (its interleaved
    // layouts fit their boxes to it); the other plans take quarter steps
    unsigned* d_hist = quad ? reinterpret_cast<unsigned*>(ctx->d_span + 4) : nullptr;
    cudaMemsetAsync(ctx->d_span, 0, (d_hist ? kSpanWords : 4) * sizeof(int), ctx->stream);
    const long long ntiles = (long long)a.ntx * a.ntz * nty;
    // few blocks: each adds its whole shared histogram to the global one
    const int blocks = (int)std::max(1LL, std::min<long long>((ntiles + 7) / 8, (long long)ctx->num_sms * 2));
    const size_t hist_smem = sizeof(unsigned) * kBoxHist * kBoxHist;
    auto fk = is2d ? footprint_kernel<16, 16, 1> : NY == 8 ? footprint_kernel<16, 16, 8> : footprint_kernel<16, 16, 16>;
    if (cuda_check(ctx, cudaFuncSetAttribute(fk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist_smem),
                   "footprint_kernel shared memory"))
      return FBP_ERR_CUDA;
    fk<<<blocks, 256, hist_smem, ctx->stream>>>(a, nty, ctx->d_span, d_hist);
    if (int rc = launched(ctx, "footprint_kernel")) return rc;
    const int words = d_hist ? kSpanWords : 4;
    std::vector<int> hs(words);
    if (cuda_check(ctx, cudaMemcpyAsync(hs.data(), ctx->d_span, sizeof(int) * words, cudaMemcpyDeviceToHost,
                                        ctx->stream),
                   "spans") ||
        cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "footprint sync"))
      return FBP_ERR_CUDA;
    plan.box_u = std::max(hs[0], 2);
    plan.box_v = std::max(hs[1], 2);
    if (d_hist)
      plan.hist.assign(reinterpret_cast<const unsigned*>(hs.data() + 4),
                       reinterpret_cast<const unsigned*>(hs.data() + kSpanWords));
    else
      plan.hist.clear();
    plan.sel_layout = -1;
    plan.valid = true;
    for (int i = 0; i < 20; ++i) plan.key[i] = key[i];
  }
  const int bu = (plan.box_u + a.align - 1) / a.align * a.align;
  // a pair element carries row v + 1 with it: one row less to stage
  const int bv = layout == kLayoutRaw32 ? plan.box_v : std::max(1, plan.box_v - 1);
  if (!is_quad_layout(layout) && ((layout == kLayoutPair32 ? 2 * bu : bu) > 256 || bv > 256))
    return set_error(ctx, FBP_ERR_UNSUPPORTED,
                     "detector footprint of a voxel tile exceeds the 256-element TMA box; geometry magnification "
                     "too large for the staged backprojector");
  a.box_u = bu;
  a.box_v = bv;
  // two CTAs per SM: each gets half of the 228 KB shared memory; the
  // symmetric kernel with 16 voxels per thread runs one CTA per SM
  const int occ = (quad && NY == 16) ? 1 : 2;
  const size_t smem_cap = occ == 1 ? (size_t)kMaxDynamicSmem : 113 * 1024;
  const size_t max_box = (size_t)(bu * bv * esize + 127) / 128 * 128;
  size_t smem = 0;
  bool use_quad = quad;
  if (use_quad) {
    // byte ring for the windows + entry records
    const size_t fixed = kQuadEntries * (sizeof(QuadCoef) + 2 * sizeof(uint64_t) + sizeof(long long)) + 64;
    const size_t ring = (smem_cap - fixed) / 128 * 128;
    // the interleaved layout gathers windows that do not fit from global memory
    const size_t entry = is_quad_layout(layout) ? 0 : 4 * max_box;
    if (entry > ring) {
      use_quad = false;  // the largest quad does not fit: generic path
      if (ctx->bp_variant == FBP_BACKPROJECTOR_SYMMETRIC)
        return set_error(ctx, FBP_ERR_UNSUPPORTED, "detector windows too large for the symmetric backprojector");
    } else {
      a.box_bytes = (int)ring;
      smem = ring + fixed;
    }
  }
  if (!use_quad) {
    if (quad) {
      // re-plan with the generic tile height
      const int saved = ctx->bp_variant;
      ctx->bp_variant = FBP_BACKPROJECTOR_GENERIC;
      const int rc = plan_backproject(ctx, g, st, vol, clip_ylimit, mixed, plan_out);
      ctx->bp_variant = saved;
      return rc;
    }
    a.box_bytes = (int)max_box;
    const size_t per_stage = a.box_bytes + sizeof(ViewCoef) + 2 * sizeof(uint64_t);
    int stages = (int)std::min<size_t>(kMaxStages, (smem_cap - 64) / per_stage);
    if (ctx->bp_stages > 0) stages = std::min(stages, ctx->bp_stages);
    if (stages < 2)
      return set_error(ctx, FBP_ERR_UNSUPPORTED, "staged detector window does not fit in shared memory");
    a.chunk = stages;
    smem = (size_t)stages * per_stage + 64;
  }

  if (packed && !(st.pack_ready && st.filt_layout == layout))
    if (int rc = prepare_packed(ctx, st, layout)) return rc;
  a.inv_scale = (layout == kLayoutPair16 || layout == kLayoutQuadG16) ? st.inv_scale : nullptr;  // set by the pack
  a.resident = occ * ctx->num_sms;  // CTAs resident at once (view-group skew of the symmetric kernel)
  a.band = std::max(1, (int)std::lround(std::sqrt((double)a.resident)));
  if (is_quad_layout(layout)) {
    a.qg = static_cast<const uint4*>(st.filt);
    a.qg_pitch = st.filt_pitch;
    a.qg_rows = st.v + 1;
  }
  // the grid of boxes over the filtered stack (4-byte elements; float2 as two floats)
  const bool from_filt = st.filtered || packed;
  const void* base = from_filt ? st.filt : (const void*)st.f32;
  const int pitch_el = from_filt ? st.filt_pitch : st.pitch;
  const uint64_t pitch_bytes = (uint64_t)pitch_el * esize;
  const uint64_t ux = layout == kLayoutPair32 ? 2ull * st.u : (uint64_t)st.u;
  const uint64_t rows_v = layout == kLayoutRaw32 ? (uint64_t)st.v : (uint64_t)st.v + 1;  // element rows per view
  BoxMaps maps;
  // interleaved layout: boxes of at most 128 x 256 elements (TMA: 256 words per
  // box row) and at most the ring; larger windows are gathered directly
  // (the widest box of the interleaved layouts is widened, within 128, to a
  // bank-friendly row stride, as choose_boxes picks the narrower ones)
  const int planes = is_quad_layout(layout) ? (int)(esize / 16) : 0;
  int mbu = is_quad_layout(layout) ? std::min(bu, 128) : bu;
  if (planes > 0)
    for (int wider = mbu; wider <= 128 && wider < mbu + 8; ++wider)
      if (bank_friendly(planes, wider)) {
        mbu = wider;
        break;
      }
  const int mbv = is_quad_layout(layout) ? std::min(bv, std::max(1, (int)(a.box_bytes / (esize * mbu)))) : bv;
  if (!(plan.sel_layout == layout && plan.sel_u == mbu && plan.sel_v == mbv)) {
    // the interleaved layouts take the boxes fitted to the histogram (C4: the
    // MIXED backprojection 1405 -> 1289 ms); the others keep the quarter steps
    // of the largest window, measured faster for the FP32 pairs (1835 vs 1884
    // ms at C4: their shared-memory row stride, 8 bytes x the box width, meets
    // bank conflicts at some fitted widths)
    static const std::vector<unsigned> no_hist;
    choose_boxes(is_quad_layout(layout) ? plan.hist : no_hist, mbu, mbv, a.align, a.pair_rows, planes, plan.sel_w,
                 plan.sel_h);
    plan.sel_layout = layout;
    plan.sel_u = mbu;
    plan.sel_v = mbv;
  }
  for (int i = 0; i < kNW; ++i) maps.w[i] = plan.sel_w[i];
  for (int j = 0; j < kNH; ++j) maps.h[j] = plan.sel_h[j];
  for (int i = 0; i < kNW; ++i)
    for (int j = 0; j < kNH; ++j) {
      if (is_quad_layout(layout)) {  // [group][element row][plane][element column][2 x 8 bytes]
        const uint32_t planes = (uint32_t)esize / 16;
        const uint64_t d4[4] = {2ull * pitch_el, planes, rows_v, (uint64_t)st.n / 4};
        const uint64_t s4[3] = {16ull * pitch_el, (uint64_t)esize * pitch_el, (uint64_t)esize * pitch_el * rows_v};
        const uint32_t b4[4] = {2u * maps.w[i], planes, (uint32_t)maps.h[j], 1};
        if (int rc = make_tensor_map_4d(ctx, &maps.map[i * kNH + j], CU_TENSOR_MAP_DATA_TYPE_UINT64,
                                        const_cast<void*>(base), d4, s4, b4))
          return rc;
        continue;
      }
      const uint32_t box_x = layout == kLayoutPair32 ? 2 * maps.w[i] : maps.w[i];  // in 4-byte elements
      uint64_t dims[3], strides[2];
      uint32_t box[3];
      if (st.sinogram) {  // [v][view][u]
        dims[0] = ux;
        dims[1] = st.n;
        dims[2] = rows_v;
        strides[0] = pitch_bytes;
        strides[1] = pitch_bytes * st.n;
        box[0] = box_x;
        box[1] = 1;
        box[2] = maps.h[j];
      } else {  // [view][v][u]
        dims[0] = ux;
        dims[1] = rows_v;
        dims[2] = st.n;
        strides[0] = pitch_bytes;
        strides[1] = pitch_bytes * rows_v;
        box[0] = box_x;
        box[1] = maps.h[j];
        box[2] = 1;
      }
      if (int rc = make_tensor_map_3d(ctx, &maps.map[i * kNH + j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                      const_cast<void*>(base), dims, strides, box))
        return rc;
    }
  // the stored values' extremes feed histogram normalisation of the context's volume
  if (vol == ctx->vol && ctx->d_minmax) {
    if (int rc = launch_minmax_init(ctx, ctx->d_minmax)) return rc;
    a.minmax = ctx->d_minmax;
  }
  BPLaunchPlan& p = *plan_out;
  p.a = a;
  p.maps = maps;
  p.smem = smem;
  p.layout = layout;
  p.ny_tile = NY;
  p.occ = occ;
  p.use_quad = use_quad;
  p.is2d = is2d;
  return FBP_OK;
}

int launch_bp_plan(fbp_context* ctx, const BPLaunchPlan& p) {
  const int NY = p.ny_tile;
  ctx->last_bp[0] = p.use_quad  ? FBP_BACKPROJECTOR_SYMMETRIC
                    : NY == 8   ? FBP_BACKPROJECTOR_GENERIC_Y8
                                : FBP_BACKPROJECTOR_GENERIC;
  ctx->last_bp[1] = p.layout;
  ctx->last_bp[2] = p.a.box_u;
  ctx->last_bp[3] = p.a.box_v;
  ctx->last_bp[4] = NY;
  cudaError_t e = p.use_quad ? launch_quad(p.layout, NY, p.maps, p.a, p.smem, ctx->stream)
                  : p.is2d   ? launch_layout<16, 16, 1>(p.layout, p.maps, p.a, p.smem, ctx->stream)
                  : NY == 8  ? launch_layout<16, 16, 8>(p.layout, p.maps, p.a, p.smem, ctx->stream)
                             : launch_layout<16, 16, 16>(p.layout, p.maps, p.a, p.smem, ctx->stream);
  if (e == cudaSuccess) ctx->launches++;
  ctx->minmax_valid = e == cudaSuccess && p.a.minmax != nullptr;
  return cuda_check(ctx, e, "bp_kernel");
}

int launch_backproject(fbp_context* ctx, const BPGeom& g, Stack& st, float* vol, int clip_ylimit, bool mixed) {
  BPLaunchPlan p;
  if (int rc = plan_backproject(ctx, g, st, vol, clip_ylimit, mixed, &p)) return rc;
  return launch_bp_plan(ctx, p);
}

long long bp_plan_batch_key(const BPLaunchPlan& p) {
  if (!p.use_quad) return 0;  // the persistent launch runs the four-fold symmetric kernel
  return 1 + p.layout + 16LL * p.ny_tile + 4096LL * p.occ + 65536LL * p.a.box_bytes;
}

namespace {

template <int LAYOUT, int NY, int OCC>
cudaError_t launch_quad_multi_cfg(const QuadQueue& qq, size_t smem, int grid, cudaStream_t stream) {
  auto kern = bp_quad_kernel<LAYOUT, NY, OCC, true>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  static const BoxMaps no_maps{};
  static const BPArgs no_args{};
  kern<<<grid, 256 + 32, smem, stream>>>(no_maps, no_args, qq);
  return cudaGetLastError();
}

template <int NY, int OCC>
cudaError_t launch_quad_multi_ny(int layout, const QuadQueue& qq, size_t smem, int grid, cudaStream_t stream) {
  switch (layout) {
    case kLayoutPair32:
      return launch_quad_multi_cfg<kLayoutPair32, NY, OCC>(qq, smem, grid, stream);
    case kLayoutQuadG16:
      return launch_quad_multi_cfg<kLayoutQuadG16, NY, OCC>(qq, smem, grid, stream);
    case kLayoutQuadG24:
      return launch_quad_multi_cfg<kLayoutQuadG24, NY, OCC>(qq, smem, grid, stream);
    default:
      return cudaErrorInvalidValue;  // other layouts run one launch per job
  }
}

}  // namespace

// Several jobs' symmetric backprojections (plans with one batch key) in one
// persistent launch on the launcher's stream: OCC CTAs per SM walk a queue
// of (job, tile orbit, y-slab) work items, largest jobs first in the order
// given. The job table goes up through the launcher's pinned staging.
long long bp_plan_tiles(const BPLaunchPlan& p) {
  return (long long)(p.a.ntx >> 1) * (p.a.ntx >> 1) * ((p.a.ny + p.ny_tile - 1) / p.ny_tile);
}

int launch_bp_batch(fbp_context* L, BPLaunchPlan* const* plans, int n, const long long* tile_begin,
                    const long long* tile_end) {
  if (n <= 0) return FBP_OK;
  const BPLaunchPlan& p0 = *plans[0];
  const long long key = bp_plan_batch_key(p0);
  if (key == 0) return set_error(L, FBP_ERR_INVALID_ARGUMENT, "backprojection plan cannot run in a batch");
  if (p0.layout != kLayoutPair32 && p0.layout != kLayoutQuadG16 && p0.layout != kLayoutQuadG24)
    return set_error(L, FBP_ERR_UNSUPPORTED, "batched backprojection supports FP32 pairs and interleaved quads");
  const size_t jobs_bytes = (sizeof(QuadJob) * n + 63) / 64 * 64;
  const size_t maps_bytes = sizeof(BoxMaps) * n;
  const size_t bytes = jobs_bytes + maps_bytes + 64;
  if (L->batch_cap < bytes) {
    cudaFree(L->d_batch);
    L->d_batch = nullptr;
    L->batch_cap = 0;
    if (cuda_check(L, cudaMalloc(&L->d_batch, bytes), "cudaMalloc(batch table)")) return FBP_ERR_OUT_OF_MEMORY;
    L->batch_cap = bytes;
  }
  if (L->h_batch_cap < bytes) {
    // the previous table may still be on its way up
    if (L->h_batch && cuda_check(L, cudaStreamSynchronize(L->stream), "batch staging sync")) return FBP_ERR_CUDA;
    cudaFreeHost(L->h_batch);
    L->h_batch = nullptr;
    L->h_batch_cap = 0;
    if (cuda_check(L, cudaMallocHost(&L->h_batch, bytes), "cudaMallocHost(batch table)")) return FBP_ERR_OUT_OF_MEMORY;
    L->h_batch_cap = bytes;
  } else if (L->ev_batch_copy) {
    if (cuda_check(L, cudaEventSynchronize(L->ev_batch_copy), "batch staging reuse")) return FBP_ERR_CUDA;
  }
  unsigned char* h = static_cast<unsigned char*>(L->h_batch);
  QuadJob* hj = reinterpret_cast<QuadJob*>(h);
  BoxMaps* hm = reinterpret_cast<BoxMaps*>(h + jobs_bytes);
  long long items = 0;
  for (int i = 0; i < n; ++i) {
    const BPLaunchPlan& p = *plans[i];
    if (bp_plan_batch_key(p) != key)
      return set_error(L, FBP_ERR_INVALID_ARGUMENT, "a batch needs one staged layout, tile height and ring size");
    hj[i] = QuadJob{};
    hj[i].a = p.a;
    hj[i].a.minmax = nullptr;  // no histogram range for batched jobs
    hj[i].item0 = items;
    hj[i].nbh = p.a.ntx >> 1;
    hj[i].nty = (p.a.ny + p.ny_tile - 1) / p.ny_tile;
    const long long all = bp_plan_tiles(p);
    const long long t0 = tile_begin ? std::max(0LL, tile_begin[i]) : 0;
    const long long t1 = tile_end ? std::min(all, tile_end[i]) : all;
    if (t1 <= t0) return set_error(L, FBP_ERR_INVALID_ARGUMENT, "empty tile range in a batch");
    hj[i].t0 = t0;
    hm[i] = p.maps;
    items += t1 - t0;
  }
  *reinterpret_cast<unsigned long long*>(h + jobs_bytes + maps_bytes) = 0ull;
  unsigned char* d = static_cast<unsigned char*>(L->d_batch);
  if (cuda_check(L, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, L->stream), "batch table upload"))
    return FBP_ERR_CUDA;
  if (!L->ev_batch_copy && cuda_check(L, cudaEventCreateWithFlags(&L->ev_batch_copy, cudaEventDisableTiming),
                                      "batch event"))
    return FBP_ERR_CUDA;
  if (cuda_check(L, cudaEventRecord(L->ev_batch_copy, L->stream), "batch event record")) return FBP_ERR_CUDA;
  QuadQueue qq;
  qq.jobs = reinterpret_cast<const QuadJob*>(d);
  qq.maps = reinterpret_cast<const BoxMaps*>(d + jobs_bytes);
  qq.njobs = n;
  qq.nitems = items;
  qq.next = reinterpret_cast<unsigned long long*>(d + jobs_bytes + maps_bytes);
  qq.err = L->d_err;
  qq.ring = p0.a.box_bytes;
  const int grid = (int)std::min<long long>(items, (long long)p0.occ * L->num_sms);
  cudaError_t e = p0.ny_tile == 16 ? launch_quad_multi_ny<16, 1>(p0.layout, qq, p0.smem, grid, L->stream)
                                   : launch_quad_multi_ny<8, 2>(p0.layout, qq, p0.smem, grid, L->stream);
  if (e == cudaSuccess) L->launches++;
  return cuda_check(L, e, "bp_quad_kernel (batch)");
}

// ---------------------------------------------------------------------------
// 2D backprojection (parallel beam and flat-detector fan beam, FBP2D.cpp:96-122
// and FBP2D.cpp:31-52 with FBP3D's FDK weight restricted to v = 0).
//
// The whole filtered sinogram of a 2D job (at most a few MB) sits in L2, so the
// 3D kernels' TMA window ring, footprint pass and per-view producer would cost
// more than the taps. A CTA owns a 32 x 32 pixel tile; per chunk of kChunk2D
// views one warp computes each view's tile-local projective coefficients in
// FP64 (one view per lane, re-based to the tile origin so FP32 stays
// accurate) and the detector window the tile needs; all threads then stage the
// chunk's windows (zero outside the detector) in shared memory and each thread
// accumulates four pixels of one column: per view one reciprocal of the
// distance ratio (fan beam), one bilinear tap from shared memory, one FMA.
constexpr int kTile2D = 32;    // pixels per tile side
constexpr int kChunk2D = 64;   // views per staged chunk
constexpr int kPix2D = 4;      // pixels per thread along z
constexpr int kWin2DMax = 512; // widest staged window (samples): 64 x 512 floats = 128 KB

struct BP2DArgs {
  const float* sino;  // [views][pitch] filtered rows
  long long pitch;
  float* image;       // [nz][nx]
  const double2* trig;
  double sod, sdd, du, vox, cu;
  int nu, nviews, nx, nz;
  int wmax;           // staged window width (floats) of one view
  float scale;
  int* err;
};

template <bool CONE>
__global__ void __launch_bounds__(256) bp2d_kernel(const BP2DArgs a) {
  extern __shared__ __align__(16) unsigned char smem2d[];
  float* win = reinterpret_cast<float*>(smem2d);                       // kChunk2D x wmax
  float4* cof = reinterpret_cast<float4*>(win + kChunk2D * a.wmax);    // (Nx, Nz, N0, bu2) per view
  float4* dco = cof + kChunk2D;                                        // (Dx, Dz, D0, u0 bits) per view
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ix0 = blockIdx.x * kTile2D, iz0 = blockIdx.y * kTile2D;
  const int tx = lane, tz = warp * kPix2D;
  float acc[kPix2D];
#pragma unroll
  for (int j = 0; j < kPix2D; ++j) acc[j] = 0.f;
  bool bad = false;
  const double Xc = (ix0 + 0.5 - 0.5 * a.nx) * a.vox, Zc = (iz0 + 0.5 - 0.5 * a.nz) * a.vox;
  for (int k0 = 0; k0 < a.nviews; k0 += kChunk2D) {
    const int nk = min(kChunk2D, a.nviews - k0);
    __syncthreads();  // the previous chunk's windows are no longer read
    if (warp == 0) {
      for (int v = lane; v < nk; v += 32) {
        const double c = a.trig[k0 + v].x, s = a.trig[k0 + v].y;
        double Dx = 0.0, Dz = 0.0, D0 = 1.0, Ux, Uz, U0;
        if (CONE) {
          const double K = a.sdd / (a.sod * a.du);
          Dx = a.vox * c / a.sod;
          Dz = a.vox * s / a.sod;
          D0 = (a.sod + Xc * c + Zc * s) / a.sod;
          Ux = -a.vox * s * K;
          Uz = a.vox * c * K;
          U0 = (-Xc * s + Zc * c) * K;
        } else {
          Ux = -a.vox * s / a.du;
          Uz = a.vox * c / a.du;
          U0 = (-Xc * s + Zc * c) / a.du;
        }
        // detector window over the tile's four corners (u is monotonic along
        // each edge, so the corners bound it)
        double umin = 1e300, umax = -1e300, dmin = 1e300;
        for (int cc = 0; cc < 4; ++cc) {
          const double x = (cc & 1) ? kTile2D - 1 : 0, z = (cc & 2) ? kTile2D - 1 : 0;
          const double D = Dx * x + Dz * z + D0;
          dmin = fmin(dmin, D);
          const double u = (Ux * x + Uz * z + U0) / D + a.cu;
          umin = fmin(umin, u);
          umax = fmax(umax, u);
        }
        // one sample of margin on each side for the FP32 rounding of u
        const int u0 = (int)floor(umin) - 1;
        const int need = (int)floor(umax) + 3 - u0;
        if (dmin <= 1e-6 || need > a.wmax) atomicCAS(a.err, 0, kDevFootprint);
        const double du0 = a.cu - u0;  // u - u0 = (N . (x, z, 1)) / D with N re-based
        cof[v] = make_float4((float)(Ux + du0 * Dx), (float)(Uz + du0 * Dz), (float)(U0 + du0 * D0),
                             __int_as_float(min(need, a.wmax) - 2));
        dco[v] = make_float4((float)Dx, (float)Dz, (float)D0, __int_as_float(u0));
      }
    }
    __syncthreads();
    // stage the chunk's windows: row k0 + v, the samples u0 .. u0 + need - 1
    // that its taps can read (zero outside the detector)
    for (int i = tid; i < nk * a.wmax; i += blockDim.x) {
      const int v = i / a.wmax, e = i - v * a.wmax;
      if (e > __float_as_int(cof[v].w) + 1) continue;
      const int u = __float_as_int(dco[v].w) + e;
      win[i] = (u >= 0 && u < a.nu) ? __ldg(a.sino + (long long)(k0 + v) * a.pitch + u) : 0.f;
    }
    __syncthreads();
    const float fx = (float)tx;
    for (int v = 0; v < nk; ++v) {
      const float4 N = cof[v], D = dco[v];
      const int bu2 = __float_as_int(N.w);
      const float* w = win + v * a.wmax;
#pragma unroll
      for (int j = 0; j < kPix2D; ++j) {
        const float fz = (float)(tz + j);
        const float num = fmaf(N.x, fx, fmaf(N.y, fz, N.z));
        float u, W;
        if (CONE) {
          const float rD = __frcp_rn(fmaf(D.x, fx, fmaf(D.y, fz, D.z)));
          u = num * rD;
          W = rD * rD;
        } else {
          u = num;
          W = 1.f;
        }
        const float fu = floorf(u);
        const int iu = (int)fu;
        if (iu >= 0 && iu <= bu2) {
          const float t = u - fu, a0 = w[iu], a1 = w[iu + 1];
          acc[j] = fmaf(W, fmaf(t, a1 - a0, a0), acc[j]);
        } else {
          bad = true;
        }
      }
    }
  }
  if (bad) atomicCAS(a.err, 0, kDevFootprint);
  const int ix = ix0 + tx;
  if (ix < a.nx)
#pragma unroll
    for (int j = 0; j < kPix2D; ++j) {
      const int iz = iz0 + tz + j;
      if (iz < a.nz) a.image[(size_t)iz * a.nx + ix] = acc[j] * a.scale;
    }
}

int launch_bp2d(fbp_context* ctx, const BPGeom& g, const float* sino, long long pitch, float* image) {
  const double pi = 3.14159265358979323846;
  const bool cone = g.kind == FBP_GEOMETRY_CONE;
  // widest window of a tile over all views: the tile diagonal magnified at the
  // image point nearest the source
  const double diag = (kTile2D - 1) * std::sqrt(2.0) * g.vox;
  double width = diag / g.du;
  if (cone) {
    const double r = 0.5 * std::sqrt((double)g.nx * g.nx + (double)g.nz * g.nz) * g.vox + diag;
    const double dmin = (g.sod - r) / g.sod;
    if (dmin < 0.05) return FBP_ERR_UNSUPPORTED;  // the source inside or near the image: general path
    width *= g.sdd / (g.sod * dmin);
  }
  const int wmax = ((int)std::ceil(width) + 4 + 3) / 4 * 4;
  if (wmax > kWin2DMax) return FBP_ERR_UNSUPPORTED;
  if (int rc = ensure_trig(ctx, g)) return rc;
  BP2DArgs a;
  a.sino = sino;
  a.pitch = pitch;
  a.image = image;
  a.trig = ctx->d_trig;
  a.sod = g.sod;
  a.sdd = g.sdd;
  a.du = g.du;
  a.vox = g.vox;
  a.cu = 0.5 * g.nu - 0.5;
  a.nu = g.nu;
  a.nviews = g.nviews;
  a.nx = g.nx;
  a.nz = g.nz;
  a.wmax = wmax;
  a.scale = cone ? (float)(pi / g.nviews * g.sdd / (g.sod * g.du)) : (float)(pi / g.nviews / g.du);
  a.err = ctx->d_err;
  const size_t smem = sizeof(float) * kChunk2D * wmax + 2 * sizeof(float4) * kChunk2D;
  auto kern = cone ? bp2d_kernel<true> : bp2d_kernel<false>;
  if (int rc = cuda_check(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)(sizeof(float) * kChunk2D * kWin2DMax + 2 * sizeof(float4) * kChunk2D)),
                          "bp2d_kernel shared memory"))
    return rc;
  const dim3 grid((g.nx + kTile2D - 1) / kTile2D, (g.nz + kTile2D - 1) / kTile2D);
  kern<<<grid, 256, smem, ctx->stream>>>(a);
  return launched(ctx, "bp2d_kernel");
}

int launch_clip(fbp_context* ctx, float* vol, int nx, int ny, int nz, int y_limit) {
  long long total = (long long)nx * ny * nz;
  int blocks = (int)std::min<long long>((total + 255) / 256, (long long)ctx->num_sms * 16);
  if (total == 0) return FBP_OK;
  clip_kernel<<<blocks, 256, 0, ctx->stream>>>(vol, nx, ny, nz, y_limit);
  return launched(ctx, "clip_kernel");
}

int launch_rebin_fan(fbp_context* ctx, const float* fan, int bins, int views, const BPGeom& g, float* par,
                     int out_bins, double du_out) {
  long long total = (long long)views * out_bins;
  if (total == 0) return FBP_OK;
  int blocks = (int)std::min<long long>((total + 255) / 256, (long long)ctx->num_sms * 16);
  rebin_fan_kernel<<<blocks, 256, 0, ctx->stream>>>(fan, bins, views, g.sod, g.sdd, g.du, g.span, g.offset, par,
                                                    out_bins, du_out);
  return launched(ctx, "rebin_fan_kernel");
}

}  // namespace fbp
