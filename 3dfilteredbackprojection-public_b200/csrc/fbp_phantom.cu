// Analytic cone-beam projections of an ellipsoid phantom, FP64 arithmetic.
//
// Generates the synthetic projection stacks of the benchmarks on the device
// (a 1440-view 1536x1536 stack is 1.4e11 ray-ellipsoid intersections). The
// reference builds phantoms by rasterising ellipsoids into a volume and
// forward projecting it (FBP3D::generate_shepplogan / render_ellipsoid,
// Source/FilteredBackProjection/FBP3D.cpp:58-72, 609-628, then
// project_forward_cone_to_projections, FBP3D.cpp:269-299); exact line
// integrals avoid the voxelisation error of that route.
//
// Ellipsoid rows: [density, a, b, c, cx, cy, cz, R00..R22] with the columns
// of the row-major rotation R the ellipsoid axes in (x, y, z). Ray geometry
// follows the backprojector: source at -SOD*d, detector point
// (SDD-SOD)*d + u*e_u + v*y, d = (cos t, sin t) in (x, z), e_u = (-sin t, cos t).

#include "fbp_internal.h"

namespace fbp {
namespace {

constexpr int kMaxEll = 64;

__global__ void project_ellipsoids_kernel(const double* __restrict__ E, int ne, BPGeom g, float* out, int pitch) {
  __shared__ double se[kMaxEll * 16];
  for (int i = threadIdx.x; i < ne * 16; i += blockDim.x) se[i] = E[i];
  __syncthreads();
  const long long total = (long long)g.nviews * g.nv * g.nu;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int iu = (int)(e % g.nu);
    const long long r = e / g.nu;  // row = view * nv + iv
    const int iv = (int)(r % g.nv), k = (int)(r / g.nv);
    double s, c;
    sincos(g.offset + g.span * k / g.nviews, &s, &c);
    const double u = (iu + 0.5 - 0.5 * g.nu) * g.du, v = (iv + 0.5 - 0.5 * g.nv) * g.dv;
    double o[3], w[3];
    if (g.kind == FBP_GEOMETRY_CONE) {
      o[0] = -g.sod * c;
      o[1] = 0.0;
      o[2] = -g.sod * s;
      const double q0 = (g.sdd - g.sod) * c - u * s, q1 = v, q2 = (g.sdd - g.sod) * s + u * c;
      w[0] = q0 - o[0];
      w[1] = q1 - o[1];
      w[2] = q2 - o[2];
      const double il = rsqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
      w[0] *= il;
      w[1] *= il;
      w[2] *= il;
    } else {
      o[0] = -u * s;
      o[1] = v;
      o[2] = u * c;
      w[0] = c;
      w[1] = 0.0;
      w[2] = s;
    }
    double acc = 0.0;
    for (int n = 0; n < ne; ++n) {
      const double* p = se + 16 * n;
      const double* R = p + 7;
      const double d0 = o[0] - p[4], d1 = o[1] - p[5], d2 = o[2] - p[6];
      double A = 0.0, B = 0.0, C = -1.0;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double qi = (d0 * R[i] + d1 * R[3 + i] + d2 * R[6 + i]) / p[1 + i];
        const double vi = (w[0] * R[i] + w[1] * R[3 + i] + w[2] * R[6 + i]) / p[1 + i];
        A += vi * vi;
        B += qi * vi;
        C += qi * qi;
      }
      const double disc = B * B - A * C;
      if (disc > 0.0) acc += p[0] * 2.0 * sqrt(disc) / A;
    }
    out[r * pitch + iu] = (float)acc;
  }
}

}  // namespace

int launch_project_ellipsoids(fbp_context* ctx, const double* d_ell, int count, const BPGeom& g, float* out,
                              int pitch) {
  if (count < 0 || count > kMaxEll)
    return set_error(ctx, FBP_ERR_INVALID_ARGUMENT, "ellipsoid count must be in [0, 64]");
  const long long total = (long long)g.nviews * g.nv * g.nu;
  if (total == 0) return FBP_OK;
  int blocks = (int)std::min<long long>((total + 255) / 256, (long long)ctx->num_sms * 32);
  project_ellipsoids_kernel<<<blocks, 256, 0, ctx->stream>>>(d_ell, count, g, out, pitch);
  return launched(ctx, "project_ellipsoids_kernel");
}

}  // namespace fbp
