// Faddeeva function w(z) = exp(-z^2) erfc(-iz) for the Voigt line shape.
//
// The reference evaluates Re w with scipy.special.wofz (pylblrtm/forward.py:51-62).
// This file implements published methods independently:
//
//  * Gautschi, W. (1970) "Efficient computation of the complex error function",
//    SIAM J. Numer. Anal. 7(1):187-198, in the region split used by Poppe & Wijers
//    (1990) ACM TOMS 16(1):38-46: the Maclaurin series of erfc near the origin, a
//    Taylor expansion about z + ih whose coefficients come from the Laplace
//    continued fraction in the intermediate region, and the continued fraction
//    alone outside the ellipse (x/5.33)^2 + (y/4.29)^2 = 1.
//  * The large-|z| asymptotic expansion w(z) ~ (i/sqrt(pi)) sum (2n-1)!!/(2^n z^(2n+1)),
//    truncated after two terms, for the far wings (|z|^2 >= FAR_Z2) that make up
//    almost every evaluation of a 25 cm^-1 line cut-off.
//
// All functions take x = Re z and y = Im z and handle every quadrant through
// w(-conj z) = conj w(z) and, for y < 0, w(z) = 2 exp(-z^2) - w(-z).
// Accuracy (tests/test_faddeeva*.py, against scipy.special.wofz):
//   double: |w - w_ref| <= ~1e-11 |w_ref| everywhere tested; Re w relative error
//           <= ~1e-8 for y >= 1e-3.
//   float : Re w relative error <= ~1e-6 for the arguments the engine produces.
#pragma once

#ifndef LBL_HD
#ifdef __CUDACC__
#define LBL_HD __host__ __device__ __forceinline__
#else
#define LBL_HD inline
#endif
#endif

#include <math.h>

#include "weideman_coeffs.h"

namespace lbl {

// |z|^2 above which the two-term asymptotic real part is used (relative error <= 6e-7).
constexpr float FAR_Z2 = 2500.0f;

constexpr double INV_SQRT_PI = 0.56418958354775628695;   // 1/sqrt(pi)
constexpr double TWO_INV_SQRT_PI = 1.1283791670955125739; // 2/sqrt(pi)

template <typename T> struct cpx { T re, im; };

template <typename T> LBL_HD T fexp(T v);
template <> LBL_HD double fexp<double>(double v) { return exp(v); }
template <> LBL_HD float fexp<float>(float v) { return expf(v); }
template <typename T> LBL_HD T fcos(T v);
template <> LBL_HD double fcos<double>(double v) { return cos(v); }
template <> LBL_HD float fcos<float>(float v) { return cosf(v); }
template <typename T> LBL_HD T fsin(T v);
template <> LBL_HD double fsin<double>(double v) { return sin(v); }
template <> LBL_HD float fsin<float>(float v) { return sinf(v); }
template <typename T> LBL_HD T fsqrt(T v);
template <> LBL_HD double fsqrt<double>(double v) { return sqrt(v); }
template <> LBL_HD float fsqrt<float>(float v) { return sqrtf(v); }

// Region parameters of the Taylor/continued-fraction method per precision:
// h = HK*s, N = NA + NB*s Taylor terms, NU = NUA + NUB*s fraction depth.
template <typename T> struct GautschiParams;
template <> struct GautschiParams<double> {
  static constexpr double HK = 1.88, NA = 7, NB = 34, NUA = 16, NUB = 26, SERIES_K = 72;
  static constexpr int SERIES_EXTRA = 12;
};
template <> struct GautschiParams<float> {
  static constexpr float HK = 1.6f, NA = 6, NB = 23, NUA = 9, NUB = 21, SERIES_K = 40;
  static constexpr int SERIES_EXTRA = 6;
};

// Continued-fraction depth for the outer region, as a function of |z|^2.
template <typename T> LBL_HD int cf_depth(T rho2);
template <> LBL_HD int cf_depth<double>(double q) {
  // q = (x/5.33)^2 + (y/4.29)^2 >= 1; depth shrinks with distance (~1e-13).
  double rho = sqrt(q);
  return 3 + (int)(1442.0 / (26.0 * rho + 77.0));
}
template <> LBL_HD int cf_depth<float>(float z2) {
  // measured depths for Re w relative error <= 3e-8 (double arithmetic).
  return z2 >= 400.f ? 4 : z2 >= 144.f ? 5 : z2 >= 64.f ? 6 : z2 >= 36.f ? 7 : 10;
}

// w(z) for x >= 0, y >= 0.
template <typename T>
LBL_HD cpx<T> faddeeva_q1(T x, T y) {
  using P = GautschiParams<T>;
  const T xs = x / T(5.33), ys = y / T(4.29);
  const T q = xs * xs + ys * ys;
  cpx<T> w;
  if (q < T(0.085264)) {
    // Maclaurin series: w = exp(-z^2) (1 + (2i/sqrt(pi)) z sum_n z^(2n) / (n! (2n+1))).
    const T ur = x * x - y * y, ui = T(2) * x * y;  // u = z^2
    const int n_terms = (int)(T(6) + P::SERIES_K * fsqrt(q)) + P::SERIES_EXTRA;
    T sr = T(1) / T(2 * n_terms + 1), si = T(0);
    for (int n = n_terms; n >= 1; --n) {
      const T inv_n = T(1) / T(n);
      const T tr = (sr * ur - si * ui) * inv_n;
      const T ti = (sr * ui + si * ur) * inv_n;
      sr = tr + T(1) / T(2 * n - 1);
      si = ti;
    }
    // a = 1 + (2i/sqrt(pi)) z S
    const T zr = sr * x - si * y, zi = sr * y + si * x;       // z*S
    const T ar = T(1) - T(TWO_INV_SQRT_PI) * zi, ai = T(TWO_INV_SQRT_PI) * zr;
    const T e = fexp<T>(-ur);
    const T er = e * fcos<T>(ui), ei = -e * fsin<T>(ui);       // exp(-u)
    w.re = er * ar - ei * ai;
    w.im = er * ai + ei * ar;
    return w;
  }
  T h = T(0);
  int n_taylor = 0, depth;
  if (q < T(1)) {
    const T s = (T(1) - y / T(4.29)) * fsqrt(T(1) - q);
    h = P::HK * s;
    n_taylor = (int)(P::NA + P::NB * s);
    depth = (int)(P::NUA + P::NUB * s);
  } else {
    if constexpr (sizeof(T) == 8) depth = cf_depth<T>(q);
    else depth = cf_depth<T>(x * x + y * y);
  }
  // r_{n-1} = (1/2) / (h - i z + n r_n), r_depth = 0, with h - iz = (y + h) - i x.
  // Taylor sum s = sum_{n<=N} (2h)^n prod_{k<=n} r_k accumulated by Horner while
  // the fraction is unwound (Gautschi 1970, eqs. 3.4-3.6).
  const T tr0 = y + h, ti0 = -x;
  T rr = T(0), ri = T(0);
  T sr = T(0), si = T(0);
  const T two_h = T(2) * h;
  T lam = T(1);
  if (h > T(0)) {
    for (int n = 0; n < n_taylor; ++n) lam *= two_h;   // (2h)^N
  }
  for (int n = depth - 1; n >= 0; --n) {
    const T cr = tr0 + T(n + 1) * rr;
    const T ci = ti0 + T(n + 1) * ri;
    const T inv = T(0.5) / (cr * cr + ci * ci);
    rr = cr * inv;
    ri = -ci * inv;
    if (h > T(0) && n <= n_taylor) {
      const T ar = lam + sr, ai = si;
      sr = rr * ar - ri * ai;
      si = rr * ai + ri * ar;
      lam /= two_h;
    }
  }
  if (h > T(0)) {
    w.re = T(TWO_INV_SQRT_PI) * sr;
    w.im = T(TWO_INV_SQRT_PI) * si;
  } else {
    w.re = T(TWO_INV_SQRT_PI) * rr;
    w.im = T(TWO_INV_SQRT_PI) * ri;
    // A finite fraction omits the exponentially small exp(-z^2) term, which is
    // the whole real part on and near the real axis.
    if (y < T(0.1)) w.re += fexp<T>(y * y - x * x) * fcos<T>(T(2) * x * y);
  }
  return w;
}

// w(z) for any z.
template <typename T>
LBL_HD cpx<T> faddeeva(T x, T y) {
  const T ax = x < T(0) ? -x : x;
  if (y >= T(0)) {
    cpx<T> w = faddeeva_q1<T>(ax, y);
    if (x < T(0)) w.im = -w.im;
    return w;
  }
  // w(z) = 2 exp(-z^2) - w(-z); -z = -x - i y lies in the upper half plane.
  cpx<T> wm = faddeeva_q1<T>(ax, -y);
  if (-x < T(0)) wm.im = -wm.im;   // w(-x + i|y|) from w(|x| + i|y|)
  const T ur = x * x - y * y, ui = T(2) * x * y;
  const T e = T(2) * fexp<T>(-ur);
  cpx<T> w;
  w.re = e * fcos<T>(ui) - wm.re;
  w.im = -e * fsin<T>(ui) - wm.im;
  return w;
}

// w(z) by Weideman's (1994) rational approximation with N terms for Im z >= 0
// (weideman_re reflects w(z) = 2 exp(-z^2) - w(-z) below the real axis). Fixed cost
// and no data-dependent loop. N = 36: |w| relative error <= 2e-14 for |z| <= 6
// against scipy.special.wofz; N = 28 below (coefficients: gen_weideman.py).
template <int N, bool HORNER = false>
LBL_HD cpx<double> weideman_upper_n(double x, double y) {
  static_assert(N == LBL_WEIDEMAN_N || N == LBL_WEIDEMAN28_N, "coefficient set");
  constexpr double L = N == LBL_WEIDEMAN_N ? LBL_WEIDEMAN_L : LBL_WEIDEMAN28_L;
  const double dr = L + y, di = -x;             // L - i z
  const double nr = L - y, ni = x;              // L + i z
  const double inv = 1.0 / (dr * dr + di * di);
  const double zr = (nr * dr + ni * di) * inv, zi = (ni * dr - nr * di) * inv;   // Z
  double a[N];                                   // folded into immediates when unrolled
  if constexpr (N == LBL_WEIDEMAN_N) {
    const double c[N] = {LBL_WEIDEMAN_COEFFS};
    for (int k = 0; k < N; ++k) a[k] = c[k];
  } else {
    const double c[N] = {LBL_WEIDEMAN28_COEFFS};
    for (int k = 0; k < N; ++k) a[k] = c[k];
  }
  // p(Z) = sum a_k Z^k with real a_k: dividing p by the real quadratic (Z - Z0)(Z - conj Z0)
  // leaves a linear remainder, which equals p at Z0; its recurrence
  // b_k = a_k + 2 Re(Z) b_{k+1} - |Z|^2 b_{k+2} costs 2 multiply-adds per coefficient where
  // complex Horner costs 4 (as accurate here: the error is the approximation's own).
  // HORNER selects complex Horner instead (4 per term, fewer live registers).
  double pr, pi;
  if constexpr (HORNER) {
    pr = a[N - 1];
    pi = 0.0;
#pragma unroll
    for (int k = N - 2; k >= 0; --k) {
      const double tr = pr * zr - pi * zi + a[k];
      pi = pr * zi + pi * zr;
      pr = tr;
    }
  } else {
    const double t2 = 2.0 * zr, s2 = zr * zr + zi * zi;
    double b1 = 0.0, b2 = 0.0;
#pragma unroll
    for (int k = N - 1; k >= 1; --k) {
      const double b0 = fma(-s2, b2, fma(t2, b1, a[k]));
      b2 = b1;
      b1 = b0;
    }
    pr = fma(zr, b1, fma(-s2, b2, a[0]));
    pi = zi * b1;
  }
  const double er = dr * inv, ei = -di * inv;           // 1 / (L - iz)
  const double e2r = er * er - ei * ei, e2i = 2.0 * er * ei;
  cpx<double> w;
  w.re = 2.0 * (pr * e2r - pi * e2i) + INV_SQRT_PI * er;
  w.im = 2.0 * (pr * e2i + pi * e2r) + INV_SQRT_PI * ei;
  return w;
}

LBL_HD cpx<double> weideman_upper(double x, double y) { return weideman_upper_n<LBL_WEIDEMAN_N>(x, y); }

template <int N = LBL_WEIDEMAN_N, bool HORNER = false>
LBL_HD double weideman_re(double x, double y) {
  if (y >= 0.0) return weideman_upper_n<N, HORNER>(x, y).re;
  const cpx<double> wm = weideman_upper_n<N, HORNER>(-x, -y);
  return 2.0 * exp(y * y - x * x) * cos(2.0 * x * y) - wm.re;
}

// Re w inside |z|^2 < CORE_Z2 for the float32 multi-level engine: the 28-term set
// (Re w relative error <= 7e-7 for y >= 1e-4, <= 1e-8 for y >= 0.01), a quarter
// fewer float64 steps than the 36-term set.
LBL_HD double weideman_re_f32(double x, double y) { return weideman_re<LBL_WEIDEMAN28_N>(x, y); }
// The same by complex Horner, for rarely taken paths of kernels at their register limit.
LBL_HD double weideman_re_f32_compact(double x, double y) { return weideman_re<LBL_WEIDEMAN28_N, true>(x, y); }

// |z|^2 below which the engine evaluates Re w in double precision (Weideman's
// approximation): inside it a float complex evaluation loses relative accuracy
// in the real part for small y.
constexpr float CORE_Z2 = 36.0f;
// |z|^2 above which five asymptotic terms suffice (relative error <= 4e-7).
constexpr float MID_Z2 = 64.0f;

// Re w by the asymptotic series, two terms: (y/sqrt(pi)) r (1 + 1.5 r - 2 y^2 r^2)
// with r = 1/|z|^2 (valid for |z|^2 >= FAR_Z2).
LBL_HD float re_w_asym2(float y, float y2, float r) {
  return float(INV_SQRT_PI) * y * r * (1.0f + r * (1.5f - 2.0f * y2 * r));
}

// Bracket S of the five-term asymptotic real part, Re w = (y/sqrt(pi)) r S, with
// r = 1/|z|^2 and q = y^2 r (valid for |z|^2 >= MID_Z2). Term k of
// (i/sqrt(pi)) sum (2k-1)!!/2^k z^-(2k+1) contributes r^k A_k(q) with
//   A_1 = 1.5 - 2q, A_2 = 3.75 - 15q + 12q^2, A_3 = 13.125 - 105q + 210q^2 - 120q^3,
//   A_4 = 59.0625 - 787.5q + 2835q^2 - 3780q^3 + 1680q^4
// (from Im z^(2k+1) / |z|^(4k+2) written in |z|^2 and y^2).
LBL_HD float asym5_bracket(float y2, float r) {
  const float q = y2 * r;
  const float a4 = (((1680.0f * q - 3780.0f) * q + 2835.0f) * q - 787.5f) * q + 59.0625f;
  const float a3 = ((-120.0f * q + 210.0f) * q - 105.0f) * q + 13.125f;
  const float a2 = (12.0f * q - 15.0f) * q + 3.75f;
  const float a1 = 1.5f - 2.0f * q;
  return 1.0f + r * (a1 + r * (a2 + r * (a3 + r * a4)));
}

LBL_HD float re_w_asym5(float y, float y2, float r) {
  return float(INV_SQRT_PI) * y * r * asym5_bracket(y2, r);
}

LBL_HD float approx_div(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fdividef(a, b);
#else
  return a / b;
#endif
}

// Re w by eight terms of the asymptotic series in its real-part form,
//   Re w = (y/sqrt(pi)) r (1 + sum_{k=1..7} r^k A_k(q)),  r = 1/|z|^2, q = y^2 r,
//   A_k(q) = (2k-1)!!/2^k sum_j C(2k+1, 2j+1) (-1)^j (1-q)^(k-j) q^j
// (term k of (i/sqrt(pi)) sum (2k-1)!!/2^k z^-(2k+1), its real part written in |z|^2 and
// y^2; A_1..A_4 are those of asym5_bracket). For CORE_Z2 <= |z|^2 < MID_Z2 the first omitted
// term is below 6.3e-8 of Re w (against scipy.special.wofz) and every term carries the factor
// y, so Re w keeps its relative accuracy for small y; exp(-x^2) (below 2.3e-16 of |w| there)
// is left out. Float32 evaluation stays within 3.6e-7, as the float continued fraction below.
// No divisions but one reciprocal, so it costs a third of the continued fraction.
LBL_HD float re_w_asym8(float y, float z2) {
  const float r = approx_div(1.0f, z2), q = y * y * r;
  const float a7 = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-17297280.0f, q, 64864800.0f), q, -97297200.0f), q, 74324250.0f),
                                      q, -30405375.0f), q, 6385128.75f), q, -591215.625f), q, 15836.1328125f);
  const float a6 = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(665280.0f, q, -2162160.0f), q, 2702700.0f), q, -1621620.0f), q,
                                 472972.5f), q, -59121.5625f), q, 2111.484375f);
  const float a5 = fmaf(fmaf(fmaf(fmaf(fmaf(-30240.0f, q, 83160.0f), q, -83160.0f), q, 36382.5f), q, -6496.875f), q,
                        324.84375f);
  const float a4 = fmaf(fmaf(fmaf(fmaf(1680.0f, q, -3780.0f), q, 2835.0f), q, -787.5f), q, 59.0625f);
  const float a3 = fmaf(fmaf(fmaf(-120.0f, q, 210.0f), q, -105.0f), q, 13.125f);
  const float a2 = fmaf(fmaf(12.0f, q, -15.0f), q, 3.75f);
  const float a1 = fmaf(-2.0f, q, 1.5f);
  float s = fmaf(a7, r, a6);
  s = fmaf(s, r, a5);
  s = fmaf(s, r, a4);
  s = fmaf(s, r, a3);
  s = fmaf(s, r, a2);
  s = fmaf(s, r, a1);
  s = fmaf(s, r, 1.0f);
  return float(INV_SQRT_PI) * y * r * s;
}

// Re w by the Laplace continued fraction in float (valid for |z|^2 >= CORE_Z2,
// y >= 0); its real parts never cancel, so Re w keeps relative accuracy.
LBL_HD float re_w_cf32(float x, float y, float z2) {
  const int depth = cf_depth<float>(z2);
  float rr = 0.0f, ri = 0.0f;
  for (int n = depth - 1; n >= 0; --n) {
    const float cr = y + float(n + 1) * rr;
    const float ci = -x + float(n + 1) * ri;
    const float inv = approx_div(0.5f, cr * cr + ci * ci);
    rr = cr * inv;
    ri = -ci * inv;
  }
  float re = float(TWO_INV_SQRT_PI) * rr;
  if (y < 0.1f) re += fexp<float>(fminf(y * y - x * x, 0.0f)) * fcos<float>(2.0f * x * y);
  return re;
}

// Real part of w as the float32 engine computes it, for y >= 0 (the engine's
// Lorentz parameter is never negative for physical inputs; y < 0 goes through
// the general double routine).
LBL_HD float faddeeva_re_f32(float x, float y) {
  const float y2 = y * y;
  const float z2 = x * x + y2;
  if (y < 0.0f || z2 < CORE_Z2) return (float)weideman_re((double)x, (double)y);
  if (z2 >= FAR_Z2) return re_w_asym2(y, y2, 1.0f / z2);
  if (z2 >= MID_Z2) return re_w_asym5(y, y2, 1.0f / z2);
  return re_w_cf32(x, y, z2);
}

}  // namespace lbl
