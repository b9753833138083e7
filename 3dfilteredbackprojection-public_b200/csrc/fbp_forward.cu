// Ray-driven forward projection of the volume:
// FBP3D::project_forward_cone_to_projections / _to_sinogram and
// project_forward_parallel_to_projections / _to_sinogram
// (Source/FilteredBackProjection/FBP3D.cpp:212-330), FBP2D::project_forward
// (FBP2D.cpp:54-94). The reference's radon shaders are absent; the transform
// is defined in the backprojector's conventions (same angles, source, detector
// axes and pixel centres): the ray of detector pixel (iu, iv) at view k is
// clipped to the volume box, its length L cut into n = ceil(L / (vox / 2))
// equal steps, and the trilinearly interpolated volume (zero outside) summed
// at the step midpoints times the step.
//
// One thread per ray; a warp covers 8 detector columns x 4 rows of one view,
// so neighbouring rays read neighbouring voxels through L1. The per-ray
// setup (angles, ray-box clipping, n) is FP64, so the sample count matches
// the FP64 restatement; the march is FP32 (position stepped by FMA, eight
// clamped trilinear taps with zero weights outside the volume).

#include "fbp_internal.h"

#include <algorithm>

namespace fbp {
namespace {

struct FPArgs {
  const float* vol;
  int nx, ny, nz;
  double vox;
  int cone;
  double sod, sdd, du, dv, span, offset;
  int nu, nv, nviews;
  float* out;
  long long pitch;  // floats per detector row
  bool sinogram;    // rows ordered [v][view]
};

__global__ void __launch_bounds__(128) forward_kernel(const FPArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int iu = blockIdx.x * 8 + (lane & 7);
  const int iv = (blockIdx.y * 4 + warp) * 4 + (lane >> 3);
  const int k = blockIdx.z;
  if (iu >= a.nu || iv >= a.nv) return;
  double s, c;
  sincos(a.offset + a.span * k / a.nviews, &s, &c);
  const double u = (iu + 0.5 - 0.5 * a.nu) * a.du, v = (iv + 0.5 - 0.5 * a.nv) * a.dv;
  const double hx = 0.5 * a.nx * a.vox, hy = 0.5 * a.ny * a.vox, hz = 0.5 * a.nz * a.vox;
  double S[3], D[3];
  if (a.cone) {
    S[0] = -a.sod * c;
    S[1] = 0.0;
    S[2] = -a.sod * s;
    D[0] = (a.sdd - a.sod) * c - u * s - S[0];
    D[1] = v;
    D[2] = (a.sdd - a.sod) * s + u * c - S[2];
  } else {
    const double R = 2.0 * (hx + hy + hz);
    S[0] = -R * c - u * s;
    S[1] = v;
    S[2] = -R * s + u * c;
    D[0] = c;
    D[1] = 0.0;
    D[2] = s;
  }
  const double len = sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
  const double h[3] = {hx, hy, hz};
  double t0 = -1e300, t1 = 1e300;
  bool miss = false;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    D[q] /= len;
    if (fabs(D[q]) < 1e-300) {
      if (S[q] <= -h[q] || S[q] >= h[q]) miss = true;
      continue;
    }
    double ta = (-h[q] - S[q]) / D[q], tb = (h[q] - S[q]) / D[q];
    if (ta > tb) {
      const double tt = ta;
      ta = tb;
      tb = tt;
    }
    t0 = fmax(t0, ta);
    t1 = fmin(t1, tb);
  }
  float acc = 0.f;
  if (!miss && t1 > t0) {
    const long long n = (long long)ceil((t1 - t0) / (0.5 * a.vox));
    const double step = (t1 - t0) / n;
    const double tm = t0 + 0.5 * step;
    // position in voxel-index space (voxel centres at integers), FP32 from here
    const float fx0 = (float)((S[0] + tm * D[0]) / a.vox + 0.5 * a.nx - 0.5);
    const float fy0 = (float)((S[1] + tm * D[1]) / a.vox + 0.5 * a.ny - 0.5);
    const float fz0 = (float)((S[2] + tm * D[2]) / a.vox + 0.5 * a.nz - 0.5);
    const float dx = (float)(step * D[0] / a.vox), dy = (float)(step * D[1] / a.vox), dz = (float)(step * D[2] / a.vox);
    const long long sx = 1, sy = a.nx, sz = (long long)a.nx * a.ny;
    for (long long q = 0; q < n; ++q) {
      const float fq = (float)q;
      const float fx = fmaf(fq, dx, fx0), fy = fmaf(fq, dy, fy0), fz = fmaf(fq, dz, fz0);
      const float flx = floorf(fx), fly = floorf(fy), flz = floorf(fz);
      const int i0 = (int)flx, j0 = (int)fly, l0 = (int)flz;
      const float wx = fx - flx, wy = fy - fly, wz = fz - flz;
      // corners clamped into the volume, with zero weight where they fall outside
      const float ax0 = (unsigned)i0 < (unsigned)a.nx ? 1.f - wx : 0.f;
      const float ax1 = (unsigned)(i0 + 1) < (unsigned)a.nx ? wx : 0.f;
      const float ay0 = (unsigned)j0 < (unsigned)a.ny ? 1.f - wy : 0.f;
      const float ay1 = (unsigned)(j0 + 1) < (unsigned)a.ny ? wy : 0.f;
      const float az0 = (unsigned)l0 < (unsigned)a.nz ? 1.f - wz : 0.f;
      const float az1 = (unsigned)(l0 + 1) < (unsigned)a.nz ? wz : 0.f;
      const long long x0 = min(max(i0, 0), a.nx - 1) * sx, x1 = min(max(i0 + 1, 0), a.nx - 1) * sx;
      const long long y0 = min(max(j0, 0), a.ny - 1) * sy, y1 = min(max(j0 + 1, 0), a.ny - 1) * sy;
      const long long z0 = min(max(l0, 0), a.nz - 1) * sz, z1 = min(max(l0 + 1, 0), a.nz - 1) * sz;
      const float* p = a.vol;
      const float c00 = fmaf(ax1, __ldg(p + z0 + y0 + x1), ax0 * __ldg(p + z0 + y0 + x0));
      const float c01 = fmaf(ax1, __ldg(p + z0 + y1 + x1), ax0 * __ldg(p + z0 + y1 + x0));
      const float c10 = fmaf(ax1, __ldg(p + z1 + y0 + x1), ax0 * __ldg(p + z1 + y0 + x0));
      const float c11 = fmaf(ax1, __ldg(p + z1 + y1 + x1), ax0 * __ldg(p + z1 + y1 + x0));
      acc += fmaf(az1, fmaf(ay1, c11, ay0 * c10), az0 * fmaf(ay1, c01, ay0 * c00));
    }
    acc *= (float)step;
  }
  const long long row = a.sinogram ? (long long)iv * a.nviews + k : (long long)k * a.nv + iv;
  a.out[row * a.pitch + iu] = acc;
}

}  // namespace

int launch_forward(fbp_context* ctx, const float* vol, int nx, int ny, int nz, double vox, bool cone, double sod,
                   double sdd, double du, double dv, double span, double offset, int nu, int nv, int nviews,
                   float* out, long long pitch, bool sinogram) {
  if (nu <= 0 || nv <= 0 || nviews <= 0 || nviews > 65535)
    return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "forward projection: bad detector size or view count");
  FPArgs a;
  a.vol = vol;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.vox = vox;
  a.cone = cone ? 1 : 0;
  a.sod = sod;
  a.sdd = sdd;
  a.du = du;
  a.dv = dv;
  a.span = span;
  a.offset = offset;
  a.nu = nu;
  a.nv = nv;
  a.nviews = nviews;
  a.out = out;
  a.pitch = pitch;
  a.sinogram = sinogram;
  const dim3 grid((nu + 7) / 8, (nv + 15) / 16, nviews);
  forward_kernel<<<grid, 128, 0, ctx->stream>>>(a);
  return launched(ctx, "forward_kernel");
}

}  // namespace fbp
