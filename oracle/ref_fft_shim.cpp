// C-callable shim around the reference's own CPU FFT (namespace FFT in
// Source/FastFourierTransformCPU/FastFourierTransform.cpp), compiled together
// with that unmodified source file by oracle/Makefile into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY: it pins the oracle's FFT restatement and is the
// reference arm of the bench (row filtering with the reference's FFT).
// Nothing in the product library links it.
#include <vector>
#include <cmath>
#include <omp.h>
#include "FastFourierTransformCPU/FastFourierTransform.h"

extern "C" {

double ref_pi(void) { return FFT::PI; }

// In-place FFT::fft_radix2 / FFT::inverse_fft_radix2 on one vector.
int ref_fft(double* re, double* im, int n, int inverse) {
  std::vector<FFT::complex> v(n);
  for (int i = 0; i < n; i++) v[i] = FFT::complex(re[i], im[i]);
  try {
    if (inverse) FFT::inverse_fft_radix2(v); else FFT::fft_radix2(v);
  } catch (...) {
    return -1;
  }
  for (int i = 0; i < n; i++) { re[i] = v[i].r; im[i] = v[i].i; }
  return 0;
}

int ref_fft_shift(double* re, double* im, int n, int inverse) {
  std::vector<FFT::complex> v(n);
  for (int i = 0; i < n; i++) v[i] = FFT::complex(re[i], im[i]);
  if (inverse) FFT::inverse_fft_shift(v); else FFT::fft_shift(v);
  for (int i = 0; i < n; i++) { re[i] = v[i].r; im[i] = v[i].i; }
  return 0;
}

// Filter float rows the way FBP3D::apply_filter_to_projections does
// (FBP3D.cpp:399-413) with the reference's FFT: pad to n, fft_radix2,
// fft_shift, multiply by the shifted response Hs, inverse_fft_shift,
// inverse_fft_radix2, real part of the first m samples. OpenMP over rows.
int ref_filter_rows(const float* in, float* out, long rows, int m, int n, const double* Hs,
                    int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  int bad = 0;
#pragma omp parallel
  {
    std::vector<FFT::complex> v(n);
#pragma omp for schedule(static)
    for (long r = 0; r < rows; r++) {
      for (int i = 0; i < n; i++) v[i] = FFT::complex(i < m ? in[r * m + i] : 0.0, 0.0);
      try {
        FFT::fft_radix2(v);
        FFT::fft_shift(v);
        for (int i = 0; i < n; i++) v[i] = FFT::mult(Hs[i], v[i]);
        FFT::inverse_fft_shift(v);
        FFT::inverse_fft_radix2(v);
      } catch (...) {
        bad = 1;
      }
      for (int i = 0; i < m; i++) out[r * m + i] = (float)v[i].r;
    }
  }
  return bad ? -1 : 0;
}

}  // extern "C"
