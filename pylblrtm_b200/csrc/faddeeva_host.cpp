// Host build of the engine's Faddeeva routines (faddeeva.cuh) for CPU-side
// accuracy checks against scipy.special.wofz. Diagnostics only: the engine never
// calls this library; it exists so the algorithm can be verified without a GPU.
#include "faddeeva.cuh"

extern "C" {

void lbl_host_faddeeva_f64(const double* x, const double* y, long long n, double* re, double* im) {
  for (long long i = 0; i < n; ++i) {
    const lbl::cpx<double> w = lbl::faddeeva<double>(x[i], y[i]);
    re[i] = w.re;
    im[i] = w.im;
  }
}

void lbl_host_faddeeva_f32(const float* x, const float* y, long long n, float* re, float* im, int mode) {
  for (long long i = 0; i < n; ++i) {
    if (mode == 1) {
      re[i] = lbl::faddeeva_re_f32(x[i], y[i]);
      continue;
    }
    const lbl::cpx<float> w = lbl::faddeeva<float>(x[i], y[i]);
    re[i] = w.re;
    im[i] = w.im;
  }
}
}
