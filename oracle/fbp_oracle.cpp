// FP64 CPU oracle for the FDK / FBP hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker: only tests/, the smoke
// entry point and the bench's CPU-baseline leg load it. The product library
// never links or calls it.
//
// What it restates (paths relative to the reference project
// furkanunsal42/3DFilteredBackProjection-Public):
//   * Row filtering through the reference's radix-2 FFT algorithm:
//       FFT::fft_radix2            Source/FastFourierTransformCPU/FastFourierTransform.cpp:49-88
//       FFT::inverse_fft_radix2    FastFourierTransform.cpp:90-106 (conjugate, FFT, conjugate, /n)
//       FFT::fft_shift / inverse   FastFourierTransform.cpp:108-130 (vec[(i+s)%n] = copy[i])
//       padding to the next power of two
//                                  Source/FastFourierTransformGPU/FastFourierTransformGPU.cpp:258-267,269-280
//       spectrum shifted, multiplied by H, unshifted
//                                  Source/FilteredBackProjection/FBP3D.cpp:399-413
//     The twiddle pi is selectable: PI_MODE_EXACT (default) or PI_MODE_REPO,
//     which uses the reference's constant (float)3.14154965
//     (FastFourierTransform.h:9). PI_MODE_REPO is pinned bit-for-bit against
//     the reference FFT compiled from its own sources (oracle/Makefile).
//   * FDK cosine pre-weight      FBP3D.cpp:369-387 (shader body absent)
//   * cone FDK backprojection    FBP3D.cpp:524-559 (shader body absent)
//   * 3D parallel backprojection FBP3D.cpp:460-490
//   * 2D parallel backprojection FBP2D.cpp:96-122
//   * fan -> parallel rebinning  FBP2D.cpp:31-52
//   * negative clipping          FBP3D.cpp:444-458
//   * log normalisation          FBP3D.cpp:333-349
//
// Parity status: the FFT is pinned against the compiled reference. The
// weights, filter shapes, backprojectors and scaling lived in GLSL shaders
// that the reference does not ship (its README says the kernel sources are
// withheld), so for those the oracle is PARITY UNPINNED: it implements the
// textbook mathematics (Feldkamp-Davis-Kress 1984; Kak & Slaney ch. 3) in the
// conventions fixed below, and the CUDA library must match it.
//
// Conventions (shared with the CUDA library):
//   volume  vol[iz][iy][ix], x fastest; y is the rotation axis (detector v)
//   voxel centre  X = (ix + 0.5 - nx/2) * vox   (same for Y, Z)
//   projections   proj[view][iv][iu], u fastest
//   detector pixel centre  u = (iu + 0.5 - nu/2) * du, v likewise
//   view angle    theta_k = offset + span * k / K
//   central-ray direction d = (cos theta, sin theta) in the (x, z) plane;
//   source at -SOD*d, detector centre at (SDD - SOD)*d, detector u-axis
//   e_u = (-sin theta, cos theta), v-axis = +y.
//   bilinear detector interpolation with zero outside the detector.
//   backprojection scale = pi / K, times 1/(du * SOD/SDD) for cone and fan,
//   times 1/du for parallel; cone/fan views also weighted by (SOD/L)^2.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

const double kPiExact = 3.14159265358979323846;
// The reference's constant is a float literal stored in a double.
const double kPiRepo = (double)3.14154965f;

enum { PI_MODE_EXACT = 0, PI_MODE_REPO = 1 };

enum {
  FILTER_RAM_LAK = 0,
  FILTER_SHEPP_LOGAN = 1,
  FILTER_COSINE = 2,
  FILTER_HANN = 3,
  FILTER_RAMP_SAMPLED = 4,
};

struct cplx {
  double r, i;
};

inline cplx cmul(cplx a, cplx b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }

int floor_log2(long n) {
  int l = 0;
  for (unsigned long t = (unsigned long)n; t > 1UL; t >>= 1) l++;
  return l;
}

size_t reverse_bits(size_t x, int nbits) {
  size_t r = 0;
  for (int i = 0; i < nbits; i++, x >>= 1) r = (r << 1) | (x & 1U);
  return r;
}

// Radix-2 decimation-in-time FFT, the same operation order as
// FastFourierTransform.cpp:49-88: twiddle table polar(1, -2*PI*i/n) for
// i < n/2, bit-reversal swap, then stages size = 2..n, each reading the
// previous stage's values.
void fft_inplace(std::vector<cplx>& v, int pi_mode) {
  const size_t n = v.size();
  const int levels = floor_log2((long)n);
  const double PI = pi_mode == PI_MODE_REPO ? kPiRepo : kPiExact;
  std::vector<cplx> tw(n / 2);
  for (size_t i = 0; i < n / 2; i++) {
    double ph = -2 * PI * i / n;
    tw[i] = {std::cos(ph) * 1.0, std::sin(ph) * 1.0};
  }
  for (size_t i = 0; i < n; i++) {
    size_t j = reverse_bits(i, levels);
    if (j > i) std::swap(v[i], v[j]);
  }
  for (size_t size = 2; size <= n; size *= 2) {
    size_t half = size / 2, step = n / size;
    for (size_t i = 0; i < n; i += size) {
      for (size_t j = i, k = 0; j < i + half; j++, k += step) {
        cplx a = v[j];
        cplx t = cmul(v[j + half], tw[k]);
        v[j + half] = {a.r + (-t.r), a.i + (-t.i)};
        v[j] = {a.r + t.r, a.i + t.i};
      }
    }
    if (size == n) break;
  }
}

void ifft_inplace(std::vector<cplx>& v, int pi_mode) {
  for (auto& c : v) c.i *= -1;
  fft_inplace(v, pi_mode);
  for (auto& c : v) c.i *= -1;
  const double n = (double)v.size();
  for (auto& c : v) c = {c.r / n, c.i / n};
}

// vec[(i + s) % n] = copy[i]  (FastFourierTransform.cpp:113-120)
void shift_inplace(std::vector<cplx>& v, long s) {
  std::vector<cplx> c = v;
  const long n = (long)v.size();
  for (long i = 0; i < n; i++) {
    long j = ((i + s) % n + n) % n;
    v[j] = c[i];
  }
}

// Band-limited ramp kernel sampled at unit spacing (Kak & Slaney eq. 3.61
// with tau = 1): h(0) = 1/4, h(odd k) = -1/(pi k)^2, h(even k) = 0.
double ramp_tap(long k) {
  if (k == 0) return 0.25;
  if (k % 2 == 0) return 0.0;
  double kk = (double)k;
  return -1.0 / (kPiExact * kPiExact * kk * kk);
}

double window(int filter, double f) {  // f = |normalised frequency| in [0, 0.5]
  switch (filter) {
    case FILTER_SHEPP_LOGAN: {
      if (f == 0.0) return 1.0;
      double x = kPiExact * f;
      return std::sin(x) / x;
    }
    case FILTER_COSINE: return std::cos(kPiExact * f);
    case FILTER_HANN: return 0.5 * (1.0 + std::cos(2.0 * kPiExact * f));
    default: return 1.0;
  }
}

}  // namespace

extern "C" {

int orc_padded_length(int m) {
  // 1 << ceil_log2(m) with ceil_log2(m) = floor_log2(2m - 1)
  // (FastFourierTransformGPU.cpp:260,269-280).
  if (m <= 0) return 0;
  return 1 << floor_log2(2L * m - 1);
}

double orc_pi(int pi_mode) { return pi_mode == PI_MODE_REPO ? kPiRepo : kPiExact; }

// In-place forward / inverse FFT of one complex vector of power-of-two length.
int orc_fft(double* re, double* im, int n, int inverse, int pi_mode) {
  if (n <= 0 || (n & (n - 1))) return -1;
  std::vector<cplx> v(n);
  for (int i = 0; i < n; i++) v[i] = {re[i], im[i]};
  if (inverse) ifft_inplace(v, pi_mode); else fft_inplace(v, pi_mode);
  for (int i = 0; i < n; i++) { re[i] = v[i].r; im[i] = v[i].i; }
  return 0;
}

int orc_fft_shift(double* re, double* im, int n, int shift) {
  std::vector<cplx> v(n);
  for (int i = 0; i < n; i++) v[i] = {re[i], im[i]};
  shift_inplace(v, shift);
  for (int i = 0; i < n; i++) { re[i] = v[i].r; im[i] = v[i].i; }
  return 0;
}

// Filter frequency response H[k] (natural FFT order, length n, unit detector
// spacing). For the kernel-based filters H is the DFT of the circularly
// wrapped band-limited ramp kernel, multiplied by the window; it is real and
// even. FILTER_RAMP_SAMPLED is |k|/n, the frequency-sampled ramp of the
// reference's CPU lambda (FastFourierTransformImage.cpp:35,45) in the same
// units.
int orc_filter_response(double* H, int n, int filter) {
  if (n <= 0 || (n & (n - 1))) return -1;
  if (filter < 0 || filter > FILTER_RAMP_SAMPLED) return -2;
  std::vector<double> h(n);
  for (int j = 0; j < n; j++) {
    long jj = j <= n / 2 ? j : (long)j - n;
    h[j] = ramp_tap(jj);
  }
  for (int k = 0; k < n; k++) {
    long kk = k <= n / 2 ? k : (long)k - n;
    double f = std::fabs((double)kk) / n;
    if (filter == FILTER_RAMP_SAMPLED) { H[k] = f; continue; }
    double s = 0.0;
    for (int j = 0; j < n; j++) {
      // exact argument reduction: (j*k) mod n keeps the cosine argument small
      long p = ((long)j * k) % n;
      s += h[j] * std::cos(2.0 * kPiExact * (double)p / n);
    }
    H[k] = s * window(filter, f);
  }
  return 0;
}

// Spatial (circular) kernel g = IDFT(H), length n; g is real and even.
int orc_filter_kernel(double* g, int n, int filter) {
  std::vector<double> H(n);
  int rc = orc_filter_response(H.data(), n, filter);
  if (rc) return rc;
  for (int j = 0; j < n; j++) {
    double s = 0.0;
    for (int k = 0; k < n; k++) {
      long p = ((long)j * k) % n;
      s += H[k] * std::cos(2.0 * kPiExact * (double)p / n);
    }
    g[j] = s / n;
  }
  return 0;
}

// Row filtering along the reference's FFT path (FBP3D.cpp:399-413): zero-pad
// to n, FFT, shift by n/2, multiply by the shifted response, shift back,
// inverse FFT, keep the real part of the first m samples.
int orc_filter_rows(const double* in, double* out, long rows, int m, int n, int filter, int pi_mode) {
  if (n < m || (n & (n - 1))) return -1;
  std::vector<double> H(n);
  int rc = orc_filter_response(H.data(), n, filter);
  if (rc) return rc;
  // response laid out on the shifted spectrum: shifted[i] = natural[(i + n/2) % n]
  std::vector<double> Hs(n);
  for (int i = 0; i < n; i++) Hs[i] = H[(i + n / 2) % n];
#pragma omp parallel
  {
    std::vector<cplx> v(n);
#pragma omp for schedule(static)
    for (long r = 0; r < rows; r++) {
      for (int i = 0; i < n; i++) v[i] = {i < m ? in[r * m + i] : 0.0, 0.0};
      fft_inplace(v, pi_mode);
      shift_inplace(v, n / 2);
      for (int i = 0; i < n; i++) v[i] = {v[i].r * Hs[i], v[i].i * Hs[i]};
      shift_inplace(v, -(long)(n / 2));
      ifft_inplace(v, pi_mode);
      for (int i = 0; i < m; i++) out[r * m + i] = v[i].r;
    }
  }
  return 0;
}

// Same operator as a direct circular convolution with g = IDFT(H) (exact pi);
// an independent cross-check of orc_filter_rows in PI_MODE_EXACT.
int orc_filter_rows_direct(const double* in, double* out, long rows, int m, int n, int filter) {
  if (n < m || (n & (n - 1))) return -1;
  std::vector<double> g(n);
  int rc = orc_filter_kernel(g.data(), n, filter);
  if (rc) return rc;
#pragma omp parallel for schedule(static)
  for (long r = 0; r < rows; r++) {
    for (int i = 0; i < m; i++) {
      double s = 0.0;
      for (int j = 0; j < m; j++) s += in[r * m + j] * g[(((i - j) % n) + n) % n];
      out[r * m + i] = s;
    }
  }
  return 0;
}

// FDK cosine pre-weight SDD / sqrt(SDD^2 + u^2 + v^2) applied in place
// (FBP3D.cpp:369-387). nv == 1 with dv == 0 gives the fan-beam weight.
int orc_fdk_weight(double* p, int nu, int nv, int nviews, double sdd, double du, double dv) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < (long)nviews * nv; k++) {
    int iv = (int)(k % nv);
    double v = (iv + 0.5 - nv / 2.0) * dv;
    for (int iu = 0; iu < nu; iu++) {
      double u = (iu + 0.5 - nu / 2.0) * du;
      p[k * nu + iu] *= sdd / std::sqrt(sdd * sdd + u * u + v * v);
    }
  }
  return 0;
}

// -log(p / base) applied in place (FBP3D.cpp:333-349; base 97/255 in
// Mains/fbp_cone_fdk_main.cpp:25). Non-positive samples are floored at
// 1e-30 * base before the logarithm.
int orc_log_normalize(double* p, long count, double base) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < count; i++) {
    double x = std::max(p[i], 1e-30 * base);
    p[i] = -std::log(x / base);
  }
  return 0;
}

// Bilinear sample of one detector image with zeros outside it.
static inline double sample2(const double* img, int nu, int nv, double u, double v) {
  double fu = std::floor(u), fv = std::floor(v);
  long iu = (long)fu, iv = (long)fv;
  double au = u - fu, av = v - fv;
  auto at = [&](long a, long b) -> double {
    if (a < 0 || a >= nu || b < 0 || b >= nv) return 0.0;
    return img[b * nu + a];
  };
  double r0 = at(iu, iv) * (1 - au) + at(iu + 1, iv) * au;
  double r1 = at(iu, iv + 1) * (1 - au) + at(iu + 1, iv + 1) * au;
  return r0 * (1 - av) + r1 * av;
}

struct ConeGeom {
  double sod, sdd, du, dv, span, offset, vox;
  int nu, nv, nviews, nx, ny, nz;
};

static double cone_voxel(const double* q, const ConeGeom& g, const std::vector<double>& cs,
                         const std::vector<double>& sn, int ix, int iy, int iz) {
  double X = (ix + 0.5 - g.nx / 2.0) * g.vox;
  double Y = (iy + 0.5 - g.ny / 2.0) * g.vox;
  double Z = (iz + 0.5 - g.nz / 2.0) * g.vox;
  double acc = 0.0;
  const long vsz = (long)g.nu * g.nv;
  for (int k = 0; k < g.nviews; k++) {
    double t = X * cs[k] + Z * sn[k];
    double s = -X * sn[k] + Z * cs[k];
    double L = g.sod + t;
    if (L <= 0) continue;
    double u = g.sdd * s / L, v = g.sdd * Y / L;
    double ui = u / g.du + g.nu / 2.0 - 0.5;
    double vi = v / g.dv + g.nv / 2.0 - 0.5;
    double w = (g.sod / L) * (g.sod / L);
    acc += w * sample2(q + k * vsz, g.nu, g.nv, ui, vi);
  }
  double scale = kPiExact / g.nviews * g.sdd / (g.sod * g.du);
  return acc * scale;
}

static void view_trig(int nviews, double span, double offset, std::vector<double>& cs, std::vector<double>& sn) {
  cs.resize(nviews);
  sn.resize(nviews);
  for (int k = 0; k < nviews; k++) {
    double th = offset + span * k / nviews;
    cs[k] = std::cos(th);
    sn[k] = std::sin(th);
  }
}

// Voxel-driven cone-beam FDK backprojection of filtered projections q
// (FBP3D.cpp:524-559). vol is nx*ny*nz, x fastest.
int orc_bp_cone(const double* q, int nu, int nv, int nviews, double sod, double sdd, double du,
                double dv, double span, double offset, int nx, int ny, int nz, double vox,
                double* vol) {
  ConeGeom g{sod, sdd, du, dv, span, offset, vox, nu, nv, nviews, nx, ny, nz};
  std::vector<double> cs, sn;
  view_trig(nviews, span, offset, cs, sn);
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < ny; iy++)
      for (int ix = 0; ix < nx; ix++)
        vol[((long)iz * ny + iy) * nx + ix] = cone_voxel(q, g, cs, sn, ix, iy, iz);
  return 0;
}

// The same backprojection evaluated only at listed voxels (ix, iy, iz
// triplets); used to check large volumes on a sample.
int orc_bp_cone_points(const double* q, int nu, int nv, int nviews, double sod, double sdd,
                       double du, double dv, double span, double offset, int nx, int ny, int nz,
                       double vox, const int* ijk, long npts, double* out) {
  ConeGeom g{sod, sdd, du, dv, span, offset, vox, nu, nv, nviews, nx, ny, nz};
  std::vector<double> cs, sn;
  view_trig(nviews, span, offset, cs, sn);
#pragma omp parallel for schedule(dynamic, 16)
  for (long p = 0; p < npts; p++)
    out[p] = cone_voxel(q, g, cs, sn, ijk[3 * p], ijk[3 * p + 1], ijk[3 * p + 2]);
  return 0;
}

// 3D parallel-beam backprojection (FBP3D.cpp:460-490): stacked 2D parallel
// backprojection, detector row iv at height v = (iv + 0.5 - nv/2) * dv.
int orc_bp_parallel3d(const double* q, int nu, int nv, int nviews, double du, double dv,
                      double span, double offset, int nx, int ny, int nz, double vox, double* vol) {
  std::vector<double> cs, sn;
  view_trig(nviews, span, offset, cs, sn);
  const long vsz = (long)nu * nv;
  double scale = kPiExact / nviews / du;
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < ny; iy++)
      for (int ix = 0; ix < nx; ix++) {
        double X = (ix + 0.5 - nx / 2.0) * vox, Y = (iy + 0.5 - ny / 2.0) * vox;
        double Z = (iz + 0.5 - nz / 2.0) * vox;
        double acc = 0.0;
        for (int k = 0; k < nviews; k++) {
          double s = -X * sn[k] + Z * cs[k];
          acc += sample2(q + k * vsz, nu, nv, s / du + nu / 2.0 - 0.5, Y / dv + nv / 2.0 - 0.5);
        }
        vol[((long)iz * ny + iy) * nx + ix] = acc * scale;
      }
  return 0;
}

// 2D parallel-beam backprojection (FBP2D.cpp:96-122). img is nx (columns)
// by nz (rows), x fastest; sinogram q[view][bin].
int orc_bp_parallel2d(const double* q, int nbins, int nviews, double du, double span,
                      double offset, int nx, int nz, double pix, double* img) {
  return orc_bp_parallel3d(q, nbins, 1, nviews, du, 1.0, span, offset, nx, 1, nz, pix, img);
}

// 2D equidistant (flat-detector) fan-beam backprojection: the cone formula
// restricted to the central plane.
int orc_bp_fan2d(const double* q, int nbins, int nviews, double sod, double sdd, double du,
                 double span, double offset, int nx, int nz, double pix, double* img) {
  return orc_bp_cone(q, nbins, 1, nviews, sod, sdd, du, 1.0, span, offset, nx, 1, nz, pix, img);
}

// Fan (flat detector) -> parallel sinogram rebinning (FBP2D.cpp:31-52):
// parallel ray (theta_p, s) is the fan ray with gamma = asin(s / SOD) at
// source angle beta = theta_p - gamma, detector u = SDD * tan(gamma). Linear
// interpolation in u and in beta (periodic over the full turn), zeros off
// the detector. Output bins: n_out at pitch du_out, views as the input.
int orc_rebin_fan_to_parallel(const double* fan, int nbins, int nviews, double sod, double sdd,
                              double du, double span, double offset, int n_out, double du_out,
                              double* par) {
  const double dbeta = span / nviews;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nviews; k++) {
    double th = offset + span * k / nviews;
    for (int j = 0; j < n_out; j++) {
      double s = (j + 0.5 - n_out / 2.0) * du_out;
      double val = 0.0;
      if (std::fabs(s) < sod) {
        double gam = std::asin(s / sod);
        double beta = th - gam;
        double u = sdd * std::tan(gam);
        double ui = u / du + nbins / 2.0 - 0.5;
        double bi = (beta - offset) / dbeta;
        double bf = std::floor(bi);
        double ab = bi - bf;
        long b0 = (long)bf;
        auto row = [&](long b) -> double {
          long bb = ((b % nviews) + nviews) % nviews;
          return sample2(fan + bb * (long)nbins, nbins, 1, ui, 0.0);
        };
        val = row(b0) * (1 - ab) + row(b0 + 1) * ab;
      }
      par[(long)k * n_out + j] = val;
    }
  }
  return 0;
}

// max(v, 0) on y-slices iy < y_limit (FBP3D.cpp:444-458 loops y-slices up to
// the volume's z size).
int orc_clip_negatives(double* vol, int nx, int ny, int nz, int y_limit) {
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < std::min(ny, y_limit); iy++)
      for (int ix = 0; ix < nx; ix++) {
        double& x = vol[((long)iz * ny + iy) * nx + ix];
        if (x < 0) x = 0;
      }
  return 0;
}

// Whole cone-beam FDK pipeline from float projections: weight, filter,
// backproject (and optionally clip). Output in FP64.
int orc_fdk(const float* proj, int nu, int nv, int nviews, double sod, double sdd, double du,
            double dv, double span, double offset, int nx, int ny, int nz, double vox, int filter,
            int n_pad, int pi_mode, int clip, double* vol) {
  const long total = (long)nu * nv * nviews;
  std::vector<double> p(total), q(total);
  for (long i = 0; i < total; i++) p[i] = proj[i];
  orc_fdk_weight(p.data(), nu, nv, nviews, sdd, du, dv);
  int rc = orc_filter_rows(p.data(), q.data(), (long)nv * nviews, nu, n_pad, filter, pi_mode);
  if (rc) return rc;
  orc_bp_cone(q.data(), nu, nv, nviews, sod, sdd, du, dv, span, offset, nx, ny, nz, vox, vol);
  if (clip) orc_clip_negatives(vol, nx, ny, nz, nz);
  return 0;
}

// ---------------------------------------------------------------------------
// Analytic phantoms (FP64). Ellipse rows: [rho, a, b, cx, cz, phi];
// ellipsoid rows: [rho, a, b, c, cx, cy, cz, R00..R22] where the columns of
// R (row-major) are the ellipsoid's axes in (x, y, z) world coordinates.

static inline double chord2(double ox, double oz, double wx, double wz, const double* e) {
  double rho = e[0], a = e[1], b = e[2], cx = e[3], cz = e[4], phi = e[5];
  double c = std::cos(phi), s = std::sin(phi);
  double px = ox - cx, pz = oz - cz;
  double qx = (px * c + pz * s) / a, qz = (-px * s + pz * c) / b;
  double vx = (wx * c + wz * s) / a, vz = (-wx * s + wz * c) / b;
  double A = vx * vx + vz * vz, B = qx * vx + qz * vz, C = qx * qx + qz * qz - 1.0;
  double disc = B * B - A * C;
  if (disc <= 0) return 0.0;
  return rho * 2.0 * std::sqrt(disc) / A;
}

static inline double chord3(const double o[3], const double w[3], const double* e) {
  double rho = e[0];
  const double* ax = e + 1;
  const double* c = e + 4;
  const double* R = e + 7;
  double p[3] = {o[0] - c[0], o[1] - c[1], o[2] - c[2]};
  double q[3], v[3];
  for (int i = 0; i < 3; i++) {
    // component along axis i = column i of R
    q[i] = (p[0] * R[0 * 3 + i] + p[1] * R[1 * 3 + i] + p[2] * R[2 * 3 + i]) / ax[i];
    v[i] = (w[0] * R[0 * 3 + i] + w[1] * R[1 * 3 + i] + w[2] * R[2 * 3 + i]) / ax[i];
  }
  double A = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  double B = q[0] * v[0] + q[1] * v[1] + q[2] * v[2];
  double C = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] - 1.0;
  double disc = B * B - A * C;
  if (disc <= 0) return 0.0;
  return rho * 2.0 * std::sqrt(disc) / A;
}

int orc_project_ellipses_parallel2d(const double* E, int ne, int nbins, int nviews, double du,
                                    double span, double offset, float* sino) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nviews; k++) {
    double th = offset + span * k / nviews, c = std::cos(th), s = std::sin(th);
    for (int j = 0; j < nbins; j++) {
      double u = (j + 0.5 - nbins / 2.0) * du;
      double ox = -u * s, oz = u * c;  // u * e_u
      double acc = 0.0;
      for (int e = 0; e < ne; e++) acc += chord2(ox, oz, c, s, E + 6 * e);
      sino[(long)k * nbins + j] = (float)acc;
    }
  }
  return 0;
}

int orc_project_ellipses_fan2d(const double* E, int ne, int nbins, int nviews, double sod,
                               double sdd, double du, double span, double offset, float* sino) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nviews; k++) {
    double th = offset + span * k / nviews, c = std::cos(th), s = std::sin(th);
    double sx = -sod * c, sz = -sod * s;
    for (int j = 0; j < nbins; j++) {
      double u = (j + 0.5 - nbins / 2.0) * du;
      double qx = (sdd - sod) * c - u * s, qz = (sdd - sod) * s + u * c;
      double wx = qx - sx, wz = qz - sz, L = std::sqrt(wx * wx + wz * wz);
      wx /= L; wz /= L;
      double acc = 0.0;
      for (int e = 0; e < ne; e++) acc += chord2(sx, sz, wx, wz, E + 6 * e);
      sino[(long)k * nbins + j] = (float)acc;
    }
  }
  return 0;
}

// Cone-beam line integrals for every pixel of the listed views (views ==
// nullptr: all views). Output proj[view_slot][iv][iu].
int orc_project_ellipsoids_cone(const double* E, int ne, int nu, int nv, int nviews, double sod,
                                double sdd, double du, double dv, double span, double offset,
                                const int* views, int nsel, float* proj) {
  int count = views ? nsel : nviews;
#pragma omp parallel for collapse(2) schedule(static)
  for (int kk = 0; kk < count; kk++)
    for (int iv = 0; iv < nv; iv++) {
      int k = views ? views[kk] : kk;
      double th = offset + span * k / nviews, c = std::cos(th), s = std::sin(th);
      double src[3] = {-sod * c, 0.0, -sod * s};
      double v = (iv + 0.5 - nv / 2.0) * dv;
      for (int iu = 0; iu < nu; iu++) {
        double u = (iu + 0.5 - nu / 2.0) * du;
        double q[3] = {(sdd - sod) * c - u * s, v, (sdd - sod) * s + u * c};
        double w[3] = {q[0] - src[0], q[1] - src[1], q[2] - src[2]};
        double L = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        w[0] /= L; w[1] /= L; w[2] /= L;
        double acc = 0.0;
        for (int e = 0; e < ne; e++) acc += chord3(src, w, E + 16 * e);
        proj[((long)kk * nv + iv) * nu + iu] = (float)acc;
      }
    }
  return 0;
}

// Density of an ellipse / ellipsoid set at pixel / voxel centres.
int orc_rasterize_ellipses(const double* E, int ne, int nx, int nz, double pix, double* img) {
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < nz; iz++)
    for (int ix = 0; ix < nx; ix++) {
      double x = (ix + 0.5 - nx / 2.0) * pix, z = (iz + 0.5 - nz / 2.0) * pix, acc = 0.0;
      for (int e = 0; e < ne; e++) {
        const double* p = E + 6 * e;
        double c = std::cos(p[5]), s = std::sin(p[5]);
        double px = x - p[3], pz = z - p[4];
        double qx = (px * c + pz * s) / p[1], qz = (-px * s + pz * c) / p[2];
        if (qx * qx + qz * qz <= 1.0) acc += p[0];
      }
      img[(long)iz * nx + ix] = acc;
    }
  return 0;
}

int orc_rasterize_ellipsoids(const double* E, int ne, int nx, int ny, int nz, double vox,
                             double* vol) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < ny; iy++)
      for (int ix = 0; ix < nx; ix++) {
        double P[3] = {(ix + 0.5 - nx / 2.0) * vox, (iy + 0.5 - ny / 2.0) * vox,
                       (iz + 0.5 - nz / 2.0) * vox};
        double acc = 0.0;
        for (int e = 0; e < ne; e++) {
          const double* p = E + 16 * e;
          const double* R = p + 7;
          double d[3] = {P[0] - p[4], P[1] - p[5], P[2] - p[6]}, r2 = 0.0;
          for (int i = 0; i < 3; i++) {
            double q = (d[0] * R[0 * 3 + i] + d[1] * R[1 * 3 + i] + d[2] * R[2 * 3 + i]) / p[1 + i];
            r2 += q * q;
          }
          if (r2 <= 1.0) acc += p[0];
        }
        vol[((long)iz * ny + iy) * nx + ix] = acc;
      }
  return 0;
}

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_num_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"

// ---------------------------------------------------------------------------
// FP32 CPU restatement of the cone backprojector, written for speed (OpenMP
// over voxel columns along the rotation axis, the per-view detector column
// and weights hoisted out of the y loop). It is the timed CPU baseline for
// the backprojection stage, labelled "CPU restatement, not reference code":
// the reference ships no CPU backprojector. q holds the filtered images of
// the listed views (q[s] is view views[s] of nviews); the sums over those
// views for y-slices [y0, y1) are added into the slab vol[iz][iy - y0][ix].
extern "C" int orc_bp_cone_f32(const float* q, const int* views, int nsel, int nu, int nv, int nviews,
                               double sod, double sdd, double du, double dv, double span, double offset,
                               int nx, int ny, int nz, double vox, int y0, int y1, float* vol) {
  std::vector<float> cs(nsel), sn(nsel);
  for (int s = 0; s < nsel; s++) {
    double th = offset + span * views[s] / nviews;
    cs[s] = (float)std::cos(th);
    sn[s] = (float)std::sin(th);
  }
  const float fsod = (float)sod, fsdd = (float)sdd;
  const float rdu = (float)(1.0 / du), rdv = (float)(1.0 / dv);
  const float cu = nu / 2.0f - 0.5f, cv = nv / 2.0f - 0.5f;
  const float scale = (float)(kPiExact / nviews * sdd / (sod * du));
  const long vsz = (long)nu * nv;
  const int sy = y1 - y0;
#pragma omp parallel
  {
    std::vector<float> acc(std::max(0, sy));
#pragma omp for collapse(2) schedule(dynamic, 8)
    for (int iz = 0; iz < nz; iz++)
      for (int ix = 0; ix < nx; ix++) {
        const float X = (float)((ix + 0.5 - nx / 2.0) * vox), Z = (float)((iz + 0.5 - nz / 2.0) * vox);
        std::fill(acc.begin(), acc.end(), 0.0f);
        for (int k = 0; k < nsel; k++) {
          float L = fsod + X * cs[k] + Z * sn[k];
          float s = -X * sn[k] + Z * cs[k];
          float rL = 1.0f / L;
          float ui = fsdd * s * rL * rdu + cu;
          float w = fsod * rL;
          w *= w;
          float fu = std::floor(ui);
          int iu = (int)fu;
          float au = ui - fu;
          if (iu < -1 || iu >= nu) continue;
          const float* img = q + k * vsz;
          const float g = fsdd * rL * rdv;
          for (int iy = y0; iy < y1; iy++) {
            float Y = (float)((iy + 0.5 - ny / 2.0) * vox);
            float vi = Y * g + cv;
            float fv = std::floor(vi);
            int iv = (int)fv;
            float av = vi - fv;
            if (iv < -1 || iv >= nv) continue;
            float p00 = 0, p01 = 0, p10 = 0, p11 = 0;
            if (iv >= 0) {
              if (iu >= 0) p00 = img[(long)iv * nu + iu];
              if (iu + 1 < nu) p01 = img[(long)iv * nu + iu + 1];
            }
            if (iv + 1 < nv) {
              if (iu >= 0) p10 = img[(long)(iv + 1) * nu + iu];
              if (iu + 1 < nu) p11 = img[(long)(iv + 1) * nu + iu + 1];
            }
            float r0 = p00 + au * (p01 - p00), r1 = p10 + au * (p11 - p10);
            acc[iy - y0] += w * (r0 + av * (r1 - r0));
          }
        }
        for (int iy = y0; iy < y1; iy++)
          vol[((long)iz * sy + (iy - y0)) * nx + ix] += acc[iy - y0] * scale;
      }
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Forward projection (ray-driven), FBP3D::project_forward_cone_to_projections /
// project_forward_parallel_to_projections (Source/FilteredBackProjection/
// FBP3D.cpp:212-330) and FBP2D::project_forward (FBP2D.cpp:54-94). The
// reference's shaders are absent; the library defines the transform as: in
// the backprojector's conventions, the ray of detector pixel (iu, iv) at view
// k (cone: from the source -SOD d through the pixel centre on the flat
// detector at (SDD - SOD) d + u e_u + v y; parallel: along d through
// u e_u + v y) is clipped to the volume box; its length L is cut into
// n = ceil(L / (vox / 2)) equal steps; the volume, trilinearly interpolated
// between voxel centres (zero outside), is summed at the step midpoints and
// times the step. Restated here in FP64 with the same n.
extern "C" int orc_forward_project(const double* vol, int nx, int ny, int nz, double vox, int cone, double sod,
                                   double sdd, double du, double dv, int nu, int nv, int nviews, double span,
                                   double offset, double* out /* [view][v][u] */) {
  const double hx = 0.5 * nx * vox, hy = 0.5 * ny * vox, hz = 0.5 * nz * vox;
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
  for (int k = 0; k < nviews; ++k)
    for (int iv = 0; iv < nv; ++iv) {
      const double th = offset + span * k / nviews, c = std::cos(th), s = std::sin(th);
      for (int iu = 0; iu < nu; ++iu) {
        const double u = (iu + 0.5 - 0.5 * nu) * du, v = (iv + 0.5 - 0.5 * nv) * dv;
        double S[3], D[3];
        if (cone) {
          S[0] = -sod * c; S[1] = 0.0; S[2] = -sod * s;
          const double P[3] = {(sdd - sod) * c - u * s, v, (sdd - sod) * s + u * c};
          for (int a = 0; a < 3; ++a) D[a] = P[a] - S[a];
        } else {
          const double R = 2.0 * (hx + hy + hz);  // start well outside the box
          S[0] = -R * c - u * s; S[1] = v; S[2] = -R * s + u * c;
          D[0] = c; D[1] = 0.0; D[2] = s;
        }
        const double len = std::sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
        for (int a = 0; a < 3; ++a) D[a] /= len;
        double t0 = -1e300, t1 = 1e300;
        const double h[3] = {hx, hy, hz};
        bool miss = false;
        for (int a = 0; a < 3; ++a) {
          if (std::fabs(D[a]) < 1e-300) {
            if (S[a] <= -h[a] || S[a] >= h[a]) miss = true;
            continue;
          }
          double ta = (-h[a] - S[a]) / D[a], tb = (h[a] - S[a]) / D[a];
          if (ta > tb) std::swap(ta, tb);
          t0 = std::max(t0, ta);
          t1 = std::min(t1, tb);
        }
        double acc = 0.0;
        if (!miss && t1 > t0) {
          const long n = (long)std::ceil((t1 - t0) / (0.5 * vox));
          const double step = (t1 - t0) / n;
          for (long q = 0; q < n; ++q) {
            const double t = t0 + (q + 0.5) * step;
            const double f[3] = {(S[0] + t * D[0]) / vox + 0.5 * nx - 0.5, (S[1] + t * D[1]) / vox + 0.5 * ny - 0.5,
                                 (S[2] + t * D[2]) / vox + 0.5 * nz - 0.5};
            const long i0 = (long)std::floor(f[0]), j0 = (long)std::floor(f[1]), l0 = (long)std::floor(f[2]);
            const double wx = f[0] - i0, wy = f[1] - j0, wz = f[2] - l0;
            double val = 0.0;
            for (int dz = 0; dz < 2; ++dz)
              for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                  const long i = i0 + dx, j = j0 + dy, l = l0 + dz;
                  if (i < 0 || i >= nx || j < 0 || j >= ny || l < 0 || l >= nz) continue;
                  const double w = (dx ? wx : 1 - wx) * (dy ? wy : 1 - wy) * (dz ? wz : 1 - wz);
                  val += w * vol[(l * ny + j) * nx + i];
                }
            acc += val;
          }
          acc *= step;
        }
        out[((long)k * nv + iv) * nu + iu] = acc;
      }
    }
  return 0;
}
