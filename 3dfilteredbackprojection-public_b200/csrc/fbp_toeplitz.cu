// Row filtering as a dense product on the tensor cores (tcgen05).
//
// Filtering every detector row with the circular kernel g of the padded
// length n is Y = X T with T[k][i] = g[(i - k) mod n] (k, i < m): a dense,
// symmetric Toeplitz matrix (g is even). It replaces the per-view FFT chain of
// FBP3D::apply_filter_to_projections (Source/FilteredBackProjection/
// FBP3D.cpp:389-414) for the MIXED form. Precision: X and T are split into
// BF16 hi + lo parts (hi = bf16(x), lo = bf16(x - hi)), and
// Y = Xh Th + Xh Tl + Xl Th is accumulated in FP32 in tensor memory (the
// dropped Xl Tl term and the split residuals are ~2^-17 of |x|). Each row's
// smooth baseline b = sum_j c_j P_j (a degree-8 Chebyshev fit of the row, 9
// coefficients) is taken out before the split and its filtered contribution
// T b = sum_j c_j (T P_j) added back by the same tensor-core product: the K
// extent is extended by one 64-wide block whose first 9 columns hold the
// coefficients c_j (X side, split hi / lo) and the columns T P_j (T side,
// summed in FP64, split hi / lo). Detector rows sit on large, slowly varying
// values (line integrals of ~10, plateaus of opaque rays) against a high-pass
// output ten to a hundred times smaller, and the split's error follows
// |x - b| instead of |x|. On the noisy 2D fan case (768 bins, Poisson I0 =
// 1e5) the image error against the FP64 oracle is 3.2e-4 with the row mean
// alone and 4.1e-5 with the degree-8 baseline (numpy emulation of the same
// split); any baseline is exact in principle, since the same coefficients are
// subtracted and added back (to the split's 16 bits).
//
// Kernel: one CTA per 128 x 256 output tile. Warp 0 streams 64-wide K blocks
// of Xh, Xl, Th, Tl into a two-stage shared-memory ring with TMA (128-byte
// swizzle), warp 1 allocates 256 TMEM columns and issues
// tcgen05.mma.cta_group::1.kind::f16 (M 128, N 256, K 16: 12 per K block), and
// frees stages with tcgen05.commit; warps 4..7 (one warpgroup, each reading its
// 32 TMEM lanes) load the FP32 accumulators with tcgen05.ld, stage them
// through shared memory and write the backprojector's pair layout (FP16 with
// the per-view scale) with row-contiguous stores. All waits are bounded and
// TMEM is always released.

#include "fbp_internal.h"
#include "fbp_rows.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <utility>

namespace fbp {
namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 2;
constexpr int A_BYTES = BM * BK * 2;                     // 16 KB
constexpr int B_BYTES = BN * BK * 2;                     // 32 KB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // 96 KB
constexpr int TMEM_COLS = 256;
constexpr uint32_t kWait = 1u << 22;
constexpr int kEpiStride = 33;  // floats per staged row (bank-conflict-free)
constexpr int kBasis = 9;       // Chebyshev polynomials P_0 .. P_8 of the row baseline

// Inverse Gram matrix of the baseline basis on the row's samples (FP64 on the
// host, rounded to FP32): coefficients c = Ginv * (moments <x, P_j>).
struct BasisGram {
  float ginv[kBasis * kBasis];
};

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, int* err) {
  for (uint32_t i = 0; i < kWait; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  atomicCAS(err, 0, kDevTimeout);
  return false;
}
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* m, int x, int y, uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(su32(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(su32(b))
      : "memory");
}

// Shared-memory matrix descriptor, K-major operand with 128-byte swizzle:
// start address >> 4 (bits 0-13), stride between 8-row groups 1024 B >> 4
// (bits 32-45), descriptor version 1 (bits 46-47), swizzle mode 2 = 128B
// (bits 61-63). The leading-dimension offset is unused for swizzled K-major.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 in bits 17-22, M >> 4 in
// bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint64_t* b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(b)) : "memory");
}

struct GemmArgs {
  RowSet rs;        // output mapping (pair layout) of the whole stack
  long long row0;   // first stack row of this chunk
  int nrows;        // rows in this chunk
  int m;            // samples per row (N and K extent)
  int ntile_n;      // tiles along N
  int kblocks;          // 64-wide K blocks: the padded row and the baseline block
  int* err;
};

__global__ void __launch_bounds__(256, 1) toeplitz_gemm_kernel(const __grid_constant__ CUtensorMap mah,
                                                              const __grid_constant__ CUtensorMap mal,
                                                              const __grid_constant__ CUtensorMap mbh,
                                                              const __grid_constant__ CUtensorMap mbl,
                                                              const GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 128-byte swizzled operand tiles need 1024-byte aligned stages
  unsigned char* smem = smem_raw + ((1024 - (su32(smem_raw) & 1023)) & 1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* s_abort = reinterpret_cast<volatile int*>(tmem_holder + 1);
  const int nt = blockIdx.x % g.ntile_n, mt = blockIdx.x / g.ntile_n;
  const int rowt = mt * BM, col0 = nt * BN;
  const int KB = g.kblocks;

  if (tid == 0) {
    *s_abort = 0;
    for (int s = 0; s < STAGES; ++s) {
      bar_init(&full[s], 1);
      bar_init(&empty[s], 1);
    }
    bar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_holder)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_holder;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      int issued = 0;
      for (int kb = 0; kb < KB; ++kb) {
        const int s = kb % STAGES;
        if (kb >= STAGES && !bar_wait(&empty[s], ((kb / STAGES) & 1) ^ 1, g.err)) {
          *s_abort = 1;
          break;
        }
        unsigned char* st = smem + s * STAGE_BYTES;
        bar_expect_tx(&full[s], STAGE_BYTES);
        tma_2d(st, &mah, kb * BK, rowt, &full[s]);
        tma_2d(st + A_BYTES, &mal, kb * BK, rowt, &full[s]);
        tma_2d(st + 2 * A_BYTES, &mbh, kb * BK, col0, &full[s]);
        tma_2d(st + 2 * A_BYTES + B_BYTES, &mbl, kb * BK, col0, &full[s]);
        ++issued;
      }
      if (*s_abort) {
        // drain: the last copy into each stage must land before the CTA exits
        for (int s = 0; s < STAGES && s < issued; ++s) {
          const int uses = (issued - s + STAGES - 1) / STAGES;
          bar_wait(&full[s], (uses - 1) & 1, g.err);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer: D += Ah Bh + Ah Bl + Al Bh per K block
      bool ok = true;
      for (int kb = 0; kb < KB && ok; ++kb) {
        const int s = kb % STAGES;
        if (!bar_wait(&full[s], (kb / STAGES) & 1, g.err)) {
          *s_abort = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = su32(smem + s * STAGE_BYTES);
        const uint32_t ah = st, al = st + A_BYTES, bh = st + 2 * A_BYTES, bl = bh + B_BYTES;
#pragma unroll
        for (int term = 0; term < 3; ++term) {
          const uint32_t a = term == 2 ? al : ah;
          const uint32_t b = term == 1 ? bl : bh;
#pragma unroll
          for (int ks = 0; ks < BK / 16; ++ks)  // 16 BF16 = 32 bytes along K inside the swizzled row
            mma(tmem, smem_desc(a + ks * 32), smem_desc(b + ks * 32), (kb | term | ks) ? 1u : 0u);
        }
        mma_commit(&empty[s]);  // stage free once these MMAs have read it
      }
      mma_commit(done);  // accumulator complete (or abandoned after an abort)
    }
  } else if (warp >= 4) {
    // epilogue warpgroup: warp 4 + w reads TMEM lanes 32w .. 32w + 31
    const int w = warp - 4;
    const bool ok = bar_wait(done, 0, g.err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float* stage = reinterpret_cast<float*>(smem);  // ring is idle once `done` completed
    const int lrow = 32 * w + lane;                 // tile row of this thread
    for (int c = 0; c < BN / 32; ++c) {
      uint32_t v[32];
      const uint32_t addr = tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(c * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%"
          "19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) stage[lrow * kEpiStride + j] = __uint_as_float(v[j]);
      asm volatile("bar.sync 1, 128;" ::: "memory");
      // warp w writes tile rows w, w + 4, ...; lane = column: row-contiguous stores
      const int col = col0 + c * 32 + lane;
      if (ok && !*s_abort && col < g.m) {
        for (int r = w; r < BM; r += 4) {
          const int lr = rowt + r;
          if (lr < g.nrows) store_row_sample(g.rs, g.row0 + lr, col, stage[r * kEpiStride + lane]);
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// Chebyshev polynomials P_0 .. P_8 at t in [-1, 1]: P_{j+1} = 2 t P_j - P_{j-1}.
__device__ __forceinline__ void cheb9(float t, float (&p)[kBasis]) {
  const float t2 = t + t;
  p[0] = 1.f;
  p[1] = t;
#pragma unroll
  for (int j = 1; j + 1 < kBasis; ++j) p[j + 1] = fmaf(t2, p[j], -p[j - 1]);
}

// X rows (fused log / weight) -> BF16 hi and lo rows of x - b (zero past m),
// b = the row's degree-8 Chebyshev fit, whose coefficients (split the same
// way) fill the first columns of the row's baseline block [kp, kx). One warp
// per row, four samples per lane step: 16-byte loads, 8-byte stores.
// STAGE: the row's pre-processed samples wait in shared memory (kp floats per
// warp) between the fit and the split instead of being read and
// pre-processed twice.
template <bool STAGE>
__global__ void __launch_bounds__(256) split_rows_kernel(RowSet rs, long long row0, int nrows, int kp, int kx,
                                                         __nv_bfloat16* xh, __nv_bfloat16* xl,
                                                         const BasisGram gram) {
  extern __shared__ __align__(16) float rowbuf[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float4* buf = reinterpret_cast<float4*>(rowbuf + (size_t)wib * kp);
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  const float half_span = rs.m > 1 ? 0.5f * (float)(rs.m - 1) : 1.f;
  const float inv_half = 1.f / half_span;
  const int nq4 = kp >> 2;  // float4 groups of the padded row
  for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + wib; r < nrows; r += warps) {
    const long long gr = row0 + r;
    const float4* src = reinterpret_cast<const float4*>(rs.data + gr * rs.pitch);
    uint2* oh = reinterpret_cast<uint2*>(xh + r * kx);
    uint2* ol = reinterpret_cast<uint2*>(xl + r * kx);
    // moments <x, P_j> of the pre-processed row (zero past m)
    float mom[kBasis];
#pragma unroll
    for (int j = 0; j < kBasis; ++j) mom[j] = 0.f;
    for (int q = lane; q < nq4; q += 32) {
      float x[4] = {0.f, 0.f, 0.f, 0.f};
      if (4 * q < rs.m) {  // the row pitch is a multiple of 4: the 16-byte load stays in the row
        const float4 v = src[q];
        const float raw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if (4 * q + t < rs.m) x[t] = pre_op(rs, gr, 4 * q + t, raw[t]);
      }
      if (STAGE) buf[q] = make_float4(x[0], x[1], x[2], x[3]);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        float p[kBasis];
        cheb9(((float)(4 * q + t) - half_span) * inv_half, p);
#pragma unroll
        for (int j = 0; j < kBasis; ++j) mom[j] = fmaf(x[t], p[j], mom[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < kBasis; ++j)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mom[j] += __shfl_xor_sync(0xffffffffu, mom[j], o);
    float c[kBasis];
#pragma unroll
    for (int a = 0; a < kBasis; ++a) {
      float sum = 0.f;
#pragma unroll
      for (int b = 0; b < kBasis; ++b) sum = fmaf(gram.ginv[a * kBasis + b], mom[b], sum);
      c[a] = sum;
    }
    // the baseline block of the row (columns kp .. kp + 63): c_0 .. c_8, then zeros
    if (lane < (kx - kp) / 4) {
      float v[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        v[t] = 0.f;
#pragma unroll
        for (int a = 0; a < kBasis; ++a)
          if (4 * lane + t == a) v[t] = c[a];
      }
      __nv_bfloat16 h[4], l[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        h[t] = __float2bfloat16_rn(v[t]);
        l[t] = __float2bfloat16_rn(v[t] - __bfloat162float(h[t]));
      }
      oh[(kp >> 2) + lane] = *reinterpret_cast<const uint2*>(h);
      ol[(kp >> 2) + lane] = *reinterpret_cast<const uint2*>(l);
    }
    // x - b, split into BF16 hi and lo (each lane reads back what it wrote)
    for (int q = lane; q < nq4; q += 32) {
      float x[4] = {0.f, 0.f, 0.f, 0.f};
      if (STAGE) {
        const float4 v = buf[q];
        x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w;
      } else if (4 * q < rs.m) {
        const float4 v = src[q];
        const float raw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if (4 * q + t < rs.m) x[t] = pre_op(rs, gr, 4 * q + t, raw[t]);
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        float p[kBasis];
        cheb9(((float)(4 * q + t) - half_span) * inv_half, p);
        float b = 0.f;
#pragma unroll
        for (int j = 0; j < kBasis; ++j) b = fmaf(c[j], p[j], b);
        x[t] = 4 * q + t < rs.m ? x[t] - b : 0.f;
      }
      __nv_bfloat16 h[4], l[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        h[t] = __float2bfloat16_rn(x[t]);
        l[t] = __float2bfloat16_rn(x[t] - __bfloat162float(h[t]));
      }
      oh[q] = *reinterpret_cast<const uint2*>(h);
      ol[q] = *reinterpret_cast<const uint2*>(l);
    }
  }
}

// tp[j][i] = sum over k < m of P_j(t_k) T[k][i] = P_j(t_k) g[(i - k) mod n], in FP64.
__global__ void toeplitz_basis_kernel(const float* g, int n, int m, float* tp) {
  const double half = m > 1 ? 0.5 * (m - 1) : 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    double acc[kBasis];
    for (int j = 0; j < kBasis; ++j) acc[j] = 0.0;
    for (int k = 0; k < m; ++k) {
      const double t = (k - half) / half, gk = (double)g[(((i - k) % n) + n) % n];
      double pm = 1.0, pj = t;
      acc[0] += gk;
      acc[1] += t * gk;
      for (int j = 1; j + 1 < kBasis; ++j) {
        const double pn = 2.0 * t * pj - pm;
        acc[j + 1] += pn * gk;
        pm = pj;
        pj = pn;
      }
    }
    for (int j = 0; j < kBasis; ++j) tp[(size_t)j * m + i] = (float)acc[j];
  }
}

// Bt[i][k] = T[k][i] = g[(i - k) mod n] for k < m, (T P_j)[i] for k = kp + j
// (the baseline block), zero otherwise; split into BF16 hi and lo (k < kx).
__global__ void build_toeplitz_kernel(const float* g, int n, int m, int kp, int kx, const float* tp,
                                      __nv_bfloat16* th, __nv_bfloat16* tl) {
  const long long total = (long long)m * kx;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / kx), k = (int)(e - (long long)i * kx);
    float t = 0.f;
    if (k < m)
      t = g[(((i - k) % n) + n) % n];
    else if (k >= kp && k < kp + kBasis)
      t = tp[(size_t)(k - kp) * m + i];
    const __nv_bfloat16 h = __float2bfloat16_rn(t);
    th[e] = h;
    tl[e] = __float2bfloat16_rn(t - __bfloat162float(h));
  }
}


}  // namespace

bool toeplitz_supported(int m) { return m >= 64 && m <= 8192; }

namespace {
// Inverse Gram matrix of the Chebyshev P_0 .. P_8 at t_k = (k - (m - 1) / 2) / ((m - 1) / 2),
// k < m, in FP64 (Gauss-Jordan with partial pivoting; the matrix is nearly
// diagonal), rounded to FP32.
BasisGram basis_gram(int m) {
  double G[kBasis][2 * kBasis] = {};
  const double half = m > 1 ? 0.5 * (m - 1) : 1.0;
  for (int k = 0; k < m; ++k) {
    const double t = (k - half) / half;
    double p[kBasis];
    p[0] = 1.0;
    p[1] = t;
    for (int j = 1; j + 1 < kBasis; ++j) p[j + 1] = 2.0 * t * p[j] - p[j - 1];
    for (int a = 0; a < kBasis; ++a)
      for (int b = 0; b < kBasis; ++b) G[a][b] += p[a] * p[b];
  }
  for (int a = 0; a < kBasis; ++a) G[a][kBasis + a] = 1.0;
  for (int col = 0; col < kBasis; ++col) {
    int piv = col;
    for (int r = col + 1; r < kBasis; ++r)
      if (std::fabs(G[r][col]) > std::fabs(G[piv][col])) piv = r;
    for (int c = 0; c < 2 * kBasis; ++c) std::swap(G[col][c], G[piv][c]);
    const double d = G[col][col];
    for (int c = 0; c < 2 * kBasis; ++c) G[col][c] /= d;
    for (int r = 0; r < kBasis; ++r) {
      if (r == col) continue;
      const double f = G[r][col];
      for (int c = 0; c < 2 * kBasis; ++c) G[r][c] -= f * G[col][c];
    }
  }
  BasisGram out;
  for (int a = 0; a < kBasis; ++a)
    for (int b = 0; b < kBasis; ++b) out.ginv[a * kBasis + b] = (float)G[a][kBasis + b];
  return out;
}
}  // namespace

int launch_filter_toeplitz(fbp_context* ctx, const RowSet& rs, int n, int filter) {
  const int m = rs.m;
  if (!toeplitz_supported(m)) return set_error(ctx, FBP_ERR_UNSUPPORTED, "Toeplitz filter needs 64 <= width <= 8192");
  if (rs.rows == 0) return FBP_OK;
  const int kp = (m + BK - 1) / BK * BK;  // K padded to whole 64-blocks (16-byte pitch too)
  const int kx = kp + BK;                  // and one block for the row baseline
  ToeplitzTables& t = ctx->ttab;
  if (!(t.m == m && t.n == n && t.filter == filter)) {
    t.m = 0;
    const size_t bytes = sizeof(__nv_bfloat16) * (size_t)m * kx;
    const size_t need = 2 * bytes + sizeof(float) * kBasis * m;
    if (need > t.cap) {  // grow only
      cudaFree(t.th);
      t.th = nullptr;
      t.cap = 0;
      if (cuda_check(ctx, cudaMalloc(&t.th, need), "cudaMalloc(Toeplitz operands)")) return FBP_ERR_OUT_OF_MEMORY;
      t.cap = need;
    }
    if (int rc = ensure_filter_tables(ctx, n, filter)) return rc;
    float* tp = reinterpret_cast<float*>(static_cast<unsigned char*>(t.th) + 2 * bytes);
    toeplitz_basis_kernel<<<(m + 127) / 128, 128, 0, ctx->stream>>>(ctx->ftab.kernel, n, m, tp);
    if (int rc = launched(ctx, "toeplitz_basis_kernel")) return rc;
    build_toeplitz_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(ctx->ftab.kernel, n, m, kp, kx, tp,
                                                                     (__nv_bfloat16*)t.th,
                                                                     (__nv_bfloat16*)t.th + (size_t)m * kx);
    if (int rc = launched(ctx, "build_toeplitz_kernel")) return rc;
    t.m = m;
    t.n = n;
    t.filter = filter;
  }
  // rows in chunks so that the split operands stay small
  const long long chunk = std::min<long long>(rs.rows, 1LL << 16);
  const size_t sbytes = sizeof(__nv_bfloat16) * (size_t)chunk * kx;
  unsigned char* sp = static_cast<unsigned char*>(scratch(ctx, 2 * sbytes + 1024));
  if (!sp) return FBP_ERR_OUT_OF_MEMORY;
  __nv_bfloat16* xh = reinterpret_cast<__nv_bfloat16*>(sp);
  __nv_bfloat16* xl = reinterpret_cast<__nv_bfloat16*>(sp + sbytes);
  const BasisGram gram = basis_gram(m);
  const size_t stage_smem = kp <= 2048 ? sizeof(float) * 8 * (size_t)kp : 0;  // 8 warps x one padded row
  if (stage_smem) {
    // the attribute is process-wide and other contexts launch with other row
    // lengths: always the largest staged size (8 rows of 2048 samples)
    const cudaError_t ea = cudaFuncSetAttribute(split_rows_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)(sizeof(float) * 8 * 2048));
    if (ea != cudaSuccess) return cuda_check(ctx, ea, "split smem attribute");
  }
  CUtensorMap mah, mal, mbh, mbl;
  if (int rc = make_tensor_map_2d_bf16_sw128(ctx, &mah, xh, kx, chunk, (uint64_t)kx * 2, BK, BM)) return rc;
  if (int rc = make_tensor_map_2d_bf16_sw128(ctx, &mal, xl, kx, chunk, (uint64_t)kx * 2, BK, BM)) return rc;
  __nv_bfloat16* th = (__nv_bfloat16*)t.th;
  if (int rc = make_tensor_map_2d_bf16_sw128(ctx, &mbh, th, kx, m, (uint64_t)kx * 2, BK, BN)) return rc;
  if (int rc = make_tensor_map_2d_bf16_sw128(ctx, &mbl, th + (size_t)m * kx, kx, m, (uint64_t)kx * 2, BK, BN)) return rc;
  const size_t smem = STAGES * STAGE_BYTES + 1024 + 256;
  cudaError_t e = cudaFuncSetAttribute(toeplitz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_check(ctx, e, "toeplitz smem attribute");
  const int ntn = (m + BN - 1) / BN;
  for (long long r0 = 0; r0 < rs.rows; r0 += chunk) {
    const int nr = (int)std::min<long long>(chunk, rs.rows - r0);
    if (stage_smem)  // rows of up to 2048 samples wait in shared memory between the two passes
      split_rows_kernel<true><<<ctx->num_sms * 4, 256, stage_smem, ctx->stream>>>(rs, r0, nr, kp, kx, xh, xl, gram);
    else
      split_rows_kernel<false><<<ctx->num_sms * 16, 256, 0, ctx->stream>>>(rs, r0, nr, kp, kx, xh, xl, gram);
    if (int rc = launched(ctx, "split_rows_kernel")) return rc;
    GemmArgs ga;
    ga.rs = rs;
    ga.row0 = r0;
    ga.nrows = nr;
    ga.m = m;
    ga.ntile_n = ntn;
    ga.kblocks = kx / BK;
    ga.err = ctx->d_err;
    const int grid = ((nr + BM - 1) / BM) * ntn;
    toeplitz_gemm_kernel<<<grid, 256, smem, ctx->stream>>>(mah, mal, mbh, mbl, ga);
    if (int rc = launched(ctx, "toeplitz_gemm_kernel")) return rc;
  }
  return FBP_OK;
}

}  // namespace fbp
