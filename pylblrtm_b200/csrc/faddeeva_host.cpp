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

// Re w by Weideman's approximation with the 36-term set (terms = 36) or the 28-term
// set of the float32 multi-level engine's near zone (terms = 28).
int lbl_host_weideman_re(const double* x, const double* y, long long n, int terms, double* re) {
  if (terms != 36 && terms != 28) return -1;
  for (long long i = 0; i < n; ++i)
    re[i] = terms == 36 ? lbl::weideman_re(x[i], y[i]) : lbl::weideman_re_f32(x[i], y[i]);
  return 0;
}

void lbl_host_faddeeva_f32(const float* x, const float* y, long long n, float* re, float* im, int mode) {
  for (long long i = 0; i < n; ++i) {
    if (mode == 1) {
      re[i] = lbl::faddeeva_re_f32(x[i], y[i]);
      continue;
    }
    if (mode == 2) {                       // the near-zone tails' eight-term series (36 <= |z|^2 < 64)
      re[i] = lbl::re_w_asym8(y[i], x[i] * x[i] + y[i] * y[i]);
      continue;
    }
    const lbl::cpx<float> w = lbl::faddeeva<float>(x[i], y[i]);
    re[i] = w.re;
    im[i] = w.im;
  }
}
}
