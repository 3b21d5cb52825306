// Layer Jacobians by the multi-level summation (no reference counterpart: the
// retrieval adjoint).
//
// For every (row = profile-layer, grid point) it accumulates three sums over the
// lines admitted by the reference tile window (pylblrtm/forward.py:295-301):
//   od       = sum amp u
//   d/dT     = sum jT_u u - jT_x x u_x - jT_y u_y
//   d/dlnVMR = sum jv_u u + jv_y u_y - jv_x u_x
// with u = Re w, u_x = Re w', u_y = -Im w' (coefficients: lbl_line_prep_jac), and
// writes od R, d(od R)/dT = R_T od + R dT and R d/dlnVMR. Because a layer's
// temperature and mixing ratio enter only that layer's optical depth, these are
// the full per-layer Jacobians of tau = sum_k od_k; Voigt values are recomputed,
// never stored. With a loss gradient g(nu) the epilogue contracts instead
// (vector-Jacobian product), so backward passes need no Jacobian storage.
//
// The distance split is the one of tau_ml_kernel (voigt_ml.cu) with 4 points per
// lane: Chebyshev nodes for lines far from the chunk (level 1, a line-per-thread
// kernel of its own, jac_far_kernel) or from a warp's 128-point sub-chunk (level 2),
// and a branch-free clamped loop plus a CTA-wide near-zone correction for the rest
// (level 3). The far field uses the asymptotic series of w and its termwise
// derivative for w' (five terms; two where |z|^2 >= FAR_Z2); forming
// w' = -2zw + 2i/sqrt(pi) there would cancel catastrophically.
#include <math.h>

#include "cheb_tables.h"
#include "faddeeva.cuh"
#include "lbl_common.cuh"
#include "sum_common.cuh"

namespace lbl {

constexpr int MJ_P = 4;
constexpr int MJ_WARP_PTS = 32 * MJ_P;
constexpr int MJ_THREADS = 256;
constexpr int MJ_CHUNK = MJ_THREADS * MJ_P;       // 1024 points
constexpr int MJ_K = 16;
constexpr float MJ_MIN_H1 = 32.f;
constexpr float MJ_MIN_H2 = 16.f;
constexpr int MJ_NBW = 128;                        // near items buffered per warp (bit-reproducible mode)

// Chebyshev node offsets (fractions of the half-width) and DCT weights, row-major [k][j]
static __constant__ float c_jnode16[MJ_K] = {LBL_CHEB16_NODES};
static __constant__ double c_jdct16[MJ_K * MJ_K] = {LBL_DCT16};
constexpr int MJ_KF = 8;                           // nodes for level-1 lines beyond four half-widths
constexpr float MJ_FAR1 = 3.f;                     // "far": more than (1 + MJ_FAR1) half-widths from the centre
constexpr int MJ_NCOEF = 3 * (MJ_K + MJ_KF);       // level-1 coefficients per (chunk, row)
constexpr int MJF_THREADS = 256;                   // lines per round of jac_far_kernel
constexpr int MJF_STAGES = 2;                      // rounds of line records in flight per thread
constexpr int MJF_FLUSH = 32;                      // rounds summed in float before the double sums
static __constant__ float c_jnode8[MJ_KF] = {LBL_CHEB8_NODES};
static __constant__ double c_jdct8[MJ_KF * MJ_KF] = {LBL_DCT8};
static_assert(MJ_K == 16 && MJ_KF == 8, "tables of cheb_tables.h");

struct JLine {
  float4 g;   // jf (or C1 - jf for level 1), a, b, amp
  float4 h;   // y, y^2, jT_u, jT_x
  float4 k;   // jT_y, jv_u, jv_y, jv_x
};

struct U3 { float u, ux, uy; };

// u, u_x, u_y from the five-term series with a given r (1/|z|^2, or 1/max(|z|^2, c)):
//   w  = (i/sqrt(pi)) q (1 + p/2 + 3p^2/4 + 15p^3/8 + 105p^4/16),
//   w' = -(i/sqrt(pi)) p (1 + 3p/2 + 15p^2/4 + 105p^3/8 + 945p^4/16),
// q = conj(z) r (= 1/z unclamped), p = q^2.
__device__ __forceinline__ U3 series5(float x, float y, float r) {
  const float qr = x * r, qi = -y * r;
  const float pr = qr * qr - qi * qi, pi_ = 2.f * qr * qi;
  float ar = 6.5625f, ai = 0.f, tr;
  tr = ar * pr - ai * pi_ + 1.875f; ai = ar * pi_ + ai * pr; ar = tr;
  tr = ar * pr - ai * pi_ + 0.75f;  ai = ar * pi_ + ai * pr; ar = tr;
  tr = ar * pr - ai * pi_ + 0.5f;   ai = ar * pi_ + ai * pr; ar = tr;
  tr = ar * pr - ai * pi_ + 1.0f;   ai = ar * pi_ + ai * pr; ar = tr;
  float br = 59.0625f, bi = 0.f;
  tr = br * pr - bi * pi_ + 13.125f; bi = br * pi_ + bi * pr; br = tr;
  tr = br * pr - bi * pi_ + 3.75f;   bi = br * pi_ + bi * pr; br = tr;
  tr = br * pr - bi * pi_ + 1.5f;    bi = br * pi_ + bi * pr; br = tr;
  tr = br * pr - bi * pi_ + 1.0f;    bi = br * pi_ + bi * pr; br = tr;
  const float xi = qr * ai + qi * ar;           // Im(q P1)
  const float yr = pr * br - pi_ * bi;          // Re(p P2)
  const float yi = pr * bi + pi_ * br;          // Im(p P2)
  const float k = float(INV_SQRT_PI);
  U3 o;
  o.u = -k * xi;      // Re w  = -Im(q P1) / sqrt(pi)
  o.ux = k * yi;      // Re w' =  Im(p P2) / sqrt(pi)
  o.uy = k * yr;      // -Im w' = Re(p P2) / sqrt(pi)
  return o;
}

// The same series cut after two terms, for |z|^2 >= FAR_Z2 (|p| <= 4e-4; against
// scipy.special.wofz and w' = -2zw + 2i/sqrt(pi): 1.2e-7 of |w|, 6e-7 of |w'|):
// w = (i/sqrt(pi)) q (1 + p/2), w' = -(i/sqrt(pi)) p (1 + 3p/2).
__device__ __forceinline__ U3 series2(float x, float y, float r) {
  const float qr = x * r, qi = -y * r;
  const float pr = qr * qr - qi * qi, pi_ = 2.f * qr * qi;
  const float ar = fmaf(0.5f, pr, 1.0f), ai = 0.5f * pi_;
  const float br = fmaf(1.5f, pr, 1.0f), bi = 1.5f * pi_;
  const float k = float(INV_SQRT_PI);
  U3 o;
  o.u = -k * (qr * ai + qi * ar);
  o.ux = k * (pr * bi + pi_ * br);
  o.uy = k * (pr * br - pi_ * bi);
  return o;
}

// The series cut after three terms, for |z|^2 >= TIER3_Z2 (|p| <= 1/400; measured as
// above: 3e-8 of |w|, 2.1e-7 of |w'|): P1 = 1 + p/2 + 3p^2/4, P2 = 1 + 3p/2 + 15p^2/4.
constexpr float TIER3_Z2 = 400.0f;
__device__ __forceinline__ U3 series3(float x, float y, float r) {
  const float qr = x * r, qi = -y * r;
  const float pr = qr * qr - qi * qi, pi_ = 2.f * qr * qi;
  const float ar = fmaf(0.75f, pr, 0.5f), ai = 0.75f * pi_;            // 1/2 + 3p/4
  const float a1r = fmaf(ar, pr, -ai * pi_ + 1.0f), a1i = fmaf(ar, pi_, ai * pr);
  const float br = fmaf(3.75f, pr, 1.5f), bi = 3.75f * pi_;            // 3/2 + 15p/4
  const float b1r = fmaf(br, pr, -bi * pi_ + 1.0f), b1i = fmaf(br, pi_, bi * pr);
  const float k = float(INV_SQRT_PI);
  U3 o;
  o.u = -k * (qr * a1i + qi * a1r);
  o.ux = k * (pr * b1i + pi_ * b1r);
  o.uy = k * (pr * b1r - pi_ * b1i);
  return o;
}

// u, u_x, u_y from eight terms of the asymptotic series in its real-part form (as re_w_asym8
// in faddeeva.cuh): u = (y/sqrt(pi)) r S with S = 1 + sum_{k=1..7} r^k A_k(q), r = 1/|z|^2,
// q = y^2 r, and by Cauchy-Riemann (u_x = Re w', u_y = -Im w' are the x and y derivatives of u)
//   u_x = -(2xy/sqrt(pi)) r^2 (S + r S_r + q S_q),
//   u_y = (r/sqrt(pi)) (S - 2q S - 2q r S_r + 2q (1 - q) S_q),
// with S_r, S_q the partial derivatives of S. For CORE_Z2 <= |z|^2 < MID_Z2 all three stay within
// 6.3e-8 of |w| and |w'| (float64 evaluation, against scipy.special.wofz). Forming w' =
// -2zw + 2i/sqrt(pi) from the float continued fraction's w there cancels ~70x of w's rounding.
__device__ __forceinline__ U3 asym8_u3(float x, float y, float z2) {
  const float r = __fdividef(1.0f, z2), q = y * y * r;
  const float a1 = fmaf(-2.0f, q, 1.5f);
  const float d1 = -2.0f;
  const float a2 = fmaf(fmaf(12.0f, q, -15.0f), q, 3.75f);
  const float d2 = fmaf(24.0f, q, -15.0f);
  const float a3 = fmaf(fmaf(fmaf(-120.0f, q, 210.0f), q, -105.0f), q, 13.125f);
  const float d3 = fmaf(fmaf(-360.0f, q, 420.0f), q, -105.0f);
  const float a4 = fmaf(fmaf(fmaf(fmaf(1680.0f, q, -3780.0f), q, 2835.0f), q, -787.5f), q, 59.0625f);
  const float d4 = fmaf(fmaf(fmaf(6720.0f, q, -11340.0f), q, 5670.0f), q, -787.5f);
  const float a5 = fmaf(fmaf(fmaf(fmaf(fmaf(-30240.0f, q, 83160.0f), q, -83160.0f), q, 36382.5f), q, -6496.875f), q, 324.84375f);
  const float d5 = fmaf(fmaf(fmaf(fmaf(-151200.0f, q, 332640.0f), q, -249480.0f), q, 72765.0f), q, -6496.875f);
  const float a6 = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(665280.0f, q, -2162160.0f), q, 2702700.0f), q, -1621620.0f), q, 472972.5f), q, -59121.5625f), q, 2111.484375f);
  const float d6 = fmaf(fmaf(fmaf(fmaf(fmaf(3991680.0f, q, -10810800.0f), q, 10810800.0f), q, -4864860.0f), q, 945945.0f), q, -59121.5625f);
  const float a7 = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-17297280.0f, q, 64864800.0f), q, -97297200.0f), q, 74324250.0f), q, -30405375.0f), q, 6385128.75f), q, -591215.625f), q, 15836.1328125f);
  const float d7 = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-121080960.0f, q, 389188800.0f), q, -486486000.0f), q, 297297000.0f), q, -91216125.0f), q, 12770257.5f), q, -591215.625f);
  const float s = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(a7, r, a6), r, a5), r, a4), r, a3), r, a2), r, a1) * r + 1.0f;
  const float sr = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(7.0f * a7, r, 6.0f * a6), r, 5.0f * a5), r, 4.0f * a4), r, 3.0f * a3), r,
                        2.0f * a2), r, a1);
  const float sq = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(d7, r, d6), r, d5), r, d4), r, d3), r, d2), r, d1) * r;
  const float k = float(INV_SQRT_PI);
  U3 o;
  o.u = k * y * r * s;
  o.ux = -2.0f * k * x * y * r * r * fmaf(q, sq, fmaf(r, sr, s));
  o.uy = k * r * fmaf(2.0f * q * (1.0f - q), sq, fmaf(-2.0f * q * r, sr, fmaf(-2.0f * q, s, s)));
  return o;
}

// Accurate u, u_x, u_y for |z|^2 < MID_Z2 (the eight-term series above CORE_Z2, Weideman
// below). With core set, Weideman's float64 form at any |z|^2 (the 28-term set stays within
// 8e-8 of Re w up to MID_Z2), so the items of a zone's middle never branch off.
__device__ __noinline__ U3 near3(float x, float y, float z2, bool core = false) {
  double wr, wi;
  if (!core && z2 >= CORE_Z2 && y >= 0.f) return asym8_u3(x, y, z2);
  if (y >= 0.f) {
    const cpx<double> w = weideman_upper_n<LBL_WEIDEMAN28_N>(x, y);
    wr = w.re;
    wi = w.im;
  } else {
    const cpx<double> wm = weideman_upper_n<LBL_WEIDEMAN28_N>(-(double)x, -(double)y);
    const double e = 2.0 * exp((double)y * y - (double)x * x);
    wr = e * cos(2.0 * x * y) - wm.re;
    wi = -e * sin(2.0 * x * y) - wm.im;
  }
  const double dr = -2.0 * (x * wr - y * wi);                         // w' = -2 z w + 2i/sqrt(pi)
  const double di = -2.0 * (x * wi + y * wr) + TWO_INV_SQRT_PI;
  U3 o;
  o.u = (float)wr;
  o.ux = (float)dr;
  o.uy = (float)(-di);
  return o;
}

__device__ __forceinline__ U3 value3(float x, const JLine& L) {
  const float z2 = fmaf(x, x, L.h.y);
  if (z2 >= FAR_Z2) return series2(x, L.h.x, rcp_approx(z2));
  if (z2 >= MID_Z2) return series5(x, L.h.x, rcp_approx(z2));
  return near3(x, L.h.x, z2);
}

__device__ __forceinline__ void add3(float* a, const U3& v, float x, const JLine& L) {
  a[0] = fmaf(L.g.w, v.u, a[0]);
  a[1] = fmaf(L.h.z, v.u, fmaf(-L.h.w * x, v.ux, fmaf(-L.k.x, v.uy, a[1])));
  a[2] = fmaf(L.k.y, v.u, fmaf(L.k.z, v.uy, fmaf(-L.k.w, v.ux, a[2])));
}

__device__ __forceinline__ void kahan3(float* sum, float* comp, const float* v) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const float yk = v[q] - comp[q];
    const float t = sum[q] + yk;
    comp[q] = (t - sum[q]) - yk;
    sum[q] = t;
  }
}

template <int K = MJ_K>
__device__ __forceinline__ float clenshaw_k(const float* c, float t) {
  float b1 = 0.f, b2 = 0.f;
  const float t2 = 2.f * t;
#pragma unroll
  for (int k = K - 1; k >= 1; --k) {
    const float b0 = fmaf(t2, b1, c[k] - b2);
    b2 = b1;
    b1 = b0;
  }
  return fmaf(t, b1, 0.5f * c[0] - b2);
}

// ---------------------------------------------------------------------------
// Level 1 of the Jacobian sums as its own kernel (as tau_far_kernel for the optical
// depth): one thread takes one level-1 line and evaluates u, u_x, u_y at all of the
// chunk's Chebyshev nodes (16; 8 beyond four half-widths), adding the three weighted sums
// in registers. It writes the chunk's 3 x (16 + 8) Chebyshev coefficients to l1_coef
// ([row][chunk of the launch][MJ_NCOEF]), which jac_ml_kernel reads.
struct JFarLine {
  LineF32 l;
  LineJac j;
};

static __device__ __noinline__ U3 jac_node_general(float x, float y, float y2) {
  const float z2 = fmaf(x, x, y2);
  if (z2 >= FAR_Z2) return series2(x, y, rcp_approx(z2));
  if (z2 >= MID_Z2) return series5(x, y, rcp_approx(z2));
  return near3(x, y, z2);
}

// The three sums of add3 for one line at one node.
__device__ __forceinline__ void add3_line(float& s0, float& s1, float& s2, const U3& v, float x, const LineF32& L,
                                          const LineJac& J) {
  s0 = fmaf(L.amp, v.u, s0);
  s1 = fmaf(J.jT_u, v.u, fmaf(-J.jT_x * x, v.ux, fmaf(-J.jT_y, v.uy, s1)));
  s2 = fmaf(J.jv_u, v.u, fmaf(J.jv_y, v.uy, fmaf(-J.jv_x, v.ux, s2)));
}

// Node sums of one level-1 line: nodes k and K-1-k sit at +xs[k] and -xs[k] from the chunk centre.
template <int K>
__device__ __forceinline__ void jfar_line(float (&f)[3][K], const float (&xs)[K / 2], const LineF32& L,
                                          const LineJac& J, float xc, float y2, bool fast) {
  if (fast) {
#pragma unroll
    for (int k = 0; k < K / 2; ++k) {
      const float xp = fmaf(xs[k], L.a, xc), xm = fmaf(-xs[k], L.a, xc);
      add3_line(f[0][k], f[1][k], f[2][k], series2(xp, L.y, rcp_approx(fmaf(xp, xp, y2))), xp, L, J);
      add3_line(f[0][K - 1 - k], f[1][K - 1 - k], f[2][K - 1 - k],
                series2(xm, L.y, rcp_approx(fmaf(xm, xm, y2))), xm, L, J);
    }
  } else {
#pragma unroll
    for (int k = 0; k < K / 2; ++k) {
      const float xp = fmaf(xs[k], L.a, xc), xm = fmaf(-xs[k], L.a, xc);
      add3_line(f[0][k], f[1][k], f[2][k], jac_node_general(xp, L.y, y2), xp, L, J);
      add3_line(f[0][K - 1 - k], f[1][K - 1 - k], f[2][K - 1 - k], jac_node_general(xm, L.y, y2), xm, L, J);
    }
  }
}

// One pass of jac_far_kernel over the tile's candidate lines for the lines of one node
// class (K = MJ_K: level-1 lines within four half-widths; K = MJ_KF: beyond); the warp's
// float64 sums of that class go to row[q * K + k]. Two passes keep 3 K accumulators live
// instead of 3 (MJ_K + MJ_KF).
template <int K>
__device__ __forceinline__ void jfar_pass(float4 (*s_line)[4][MJF_THREADS], const LineF32* lp, const LineJac* jp,
                                          int2 rng, double wlo, double whi, long long c0, float H1,
                                          const float (&xs)[K / 2], double* row) {
  const int tid = threadIdx.x, lane = tid & 31;
  const float C1 = H1;
  float f[3][K];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int k = 0; k < K; ++k) f[q][k] = 0.f;
  // records of round r (line rng.x + r * MJF_THREADS + tid) go to stage r % 2, one round
  // ahead; each thread copies into and reads only its own slots
  const int n_rounds = rng.y > rng.x ? (rng.y - rng.x + MJF_THREADS - 1) / MJF_THREADS : 0;
  auto issue = [&](int r, int stage) {
    const int li = rng.x + r * MJF_THREADS + tid;
    if (li < rng.y) {   // 32-B records in 256-B aligned allocations
      const float4* g = reinterpret_cast<const float4*>(lp + li);
      const float4* h = reinterpret_cast<const float4*>(jp + li);
      cp_async16(&s_line[stage][0][tid], g);
      cp_async16(&s_line[stage][1][tid], g + 1);
      cp_async16(&s_line[stage][2][tid], h);
      cp_async16(&s_line[stage][3][tid], h + 1);
    }
    cp_async_commit();
  };
  issue(0, 0);
  int rounds = 0;
  for (int r = 0; r < n_rounds; ++r) {
    const int stage = r & 1;
    issue(r + 1, stage ^ 1);                                // the stage read last round
    cp_async_wait<1>();
    const bool have = rng.x + r * MJF_THREADS + tid < rng.y;
    JFarLine R;
    if (have) {
      R.l = line_f32_from_planes(s_line[stage][0][tid], s_line[stage][1][tid]);
      R.j = line_jac_from_planes(s_line[stage][2][tid], s_line[stage][3][tid]);
    }
    // the level-1 test of jac_ml_kernel, expression for expression, then the node class
    const bool pass = have && (R.l.nuc >= wlo) && (R.l.nuc <= whi);
    const float jf = (float)((long long)R.l.j0 - c0);
    const float dd = fabsf(jf - C1) - H1;
    const bool far8 = dd > MJ_FAR1 * H1;
    if (pass && dd > H1 + 1.f && far8 == (K == MJ_KF)) {
      const float xc = fmaf(C1 - jf, R.l.a, -R.l.b);
      const float y2 = R.l.y * R.l.y;
      const float xm = fmaf(-H1 * c_jnode16[0], R.l.a, fabsf(xc));   // nearest node, as in tau_far_kernel
      jfar_line<K>(f, xs, R.l, R.j, xc, y2, fmaf(xm, xm, y2) >= FAR_Z2);
    }
    if (++rounds == MJF_FLUSH) {
      rounds = 0;
#pragma unroll
      for (int q = 0; q < 3; ++q) flush_nodes(f[q], row + q * K, lane);
    }
  }
  cp_async_wait<0>();                                      // only empty groups remain
#pragma unroll
  for (int q = 0; q < 3; ++q) flush_nodes(f[q], row + q * K, lane);
}

__global__ void __launch_bounds__(MJF_THREADS, 2)
jac_far_kernel(const LineF32* __restrict__ prep, const LineJac* __restrict__ jprep, int n_lines,
               const int2* __restrict__ ranges, const int2* __restrict__ near_ranges, double nu_min, double step,
               long long n_nu, int tile_samples, int chunks_per_tile, int chunk_pts, double cutoff,
               float* __restrict__ l1_coef) {
  __shared__ __align__(16) float4 s_line[MJF_STAGES][4][MJF_THREADS];  // 64-B records as four 16-B planes
  __shared__ double s_part[MJF_THREADS / 32][MJ_NCOEF];                 // [q][16] then [q][8] per warp

  const int row = blockIdx.y;
  const int tile = blockIdx.x / chunks_per_tile, chunk = blockIdx.x % chunks_per_tile;
  const long long t0 = (long long)tile * tile_samples;
  const long long t1 = min(t0 + (long long)tile_samples, n_nu);
  long long c0;
  int n_c;
  if (!tile_chunk(t0, t1, chunk, chunk_pts, c0, n_c)) return;
  const float H1 = 0.5f * (float)(n_c - 1);               // same chunk geometry as jac_ml_kernel
  if (!(H1 >= MJ_MIN_H1)) return;                         // no level 1: jac_ml_kernel takes every line
  const double wlo = __dsub_rn(grid_nu(nu_min, step, t0), cutoff);
  const double whi = __dadd_rn(grid_nu(nu_min, step, t1 - 1), cutoff);
  const int2 rng = ranges[tile];
  const LineF32* lp = prep + (long long)row * n_lines;
  const LineJac* jp = jprep + (long long)row * n_lines;
  const int tid = threadIdx.x, warp = tid >> 5;
  if ((tid & 31) == 0)
    for (int k = 0; k < MJ_NCOEF; ++k) s_part[warp][k] = 0.0;

  float xa[MJ_K / 2], xb[MJ_KF / 2];
#pragma unroll
  for (int k = 0; k < MJ_K / 2; ++k) xa[k] = H1 * c_jnode16[k];
#pragma unroll
  for (int k = 0; k < MJ_KF / 2; ++k) xb[k] = H1 * c_jnode8[k];
  // the 16-node class lies within four half-widths of the chunk: its pass reads only the
  // tile's near range (lbl_jac_near_ranges) when one is given
  int2 rng16 = rng;
  if (near_ranges) {
    const int2 q = near_ranges[tile];
    rng16 = make_int2(max(rng.x, q.x), min(rng.y, q.y));
  }
  jfar_pass<MJ_K>(s_line, lp, jp, rng16, wlo, whi, c0, H1, xa, s_part[warp]);
  jfar_pass<MJ_KF>(s_line, lp, jp, rng, wlo, whi, c0, H1, xb, s_part[warp] + 3 * MJ_K);
  __syncthreads();
  if (tid < MJ_NCOEF) {                                    // column tid: only this thread touches it
    double v = 0.0;
    for (int w = 0; w < MJF_THREADS / 32; ++w) v += s_part[w][tid];
    s_part[0][tid] = v;
  }
  __syncthreads();
  if (tid < MJ_NCOEF) {                                    // Chebyshev coefficients (DCT)
    double c = 0.0;
    if (tid < 3 * MJ_K) {
      const int q = tid / MJ_K, k = tid % MJ_K;
      for (int j = 0; j < MJ_K; ++j) c += s_part[0][q * MJ_K + j] * c_jdct16[k * MJ_K + j];
      c *= 2.0 / MJ_K;
    } else {
      const int q = (tid - 3 * MJ_K) / MJ_KF, k = (tid - 3 * MJ_K) % MJ_KF;
      for (int j = 0; j < MJ_KF; ++j) c += s_part[0][3 * MJ_K + q * MJ_KF + j] * c_jdct8[k * MJ_KF + j];
      c *= 2.0 / MJ_KF;
    }
    l1_coef[((long long)row * gridDim.x + blockIdx.x) * MJ_NCOEF + tid] = (float)c;
  }
}

template <bool DET>
__global__ void __launch_bounds__(MJ_THREADS, 3)
jac_ml_kernel(const LineF32* __restrict__ prep, const LineJac* __restrict__ jprep, int n_lines,
              const int2* __restrict__ ranges, const int2* __restrict__ inner_ranges,
              const double* __restrict__ t_layer, double nu_min, double step, long long n_nu, int tile_samples,
              int chunks_per_tile, double cutoff, const float* __restrict__ l1_coef, float* __restrict__ od,
              float* __restrict__ d_t, float* __restrict__ d_v, int n_lay, const double* __restrict__ g_tau,
              double* __restrict__ vjp_t, double* __restrict__ vjp_v) {
  constexpr int P = MJ_P;
  __shared__ JLine s2[MJ_THREADS];
  __shared__ unsigned char s_l2[MJ_THREADS / 32][MJ_THREADS];
  __shared__ unsigned char s_l3[MJ_THREADS / 32][MJ_THREADS];
  __shared__ int s_cnt[MJ_THREADS / 32];
  __shared__ short4 s_nr[MJ_THREADS];                // near range (lo, n) and its middle (lo, n), chunk points
  __shared__ float s_core[3][MJ_CHUNK];              // near corrections (each warp owns its points)
  extern __shared__ float s_nbuf_dyn[];              // bit-reproducible mode: [warp][3][MJ_NBW] near-item values
  __shared__ float s_c1[MJ_NCOEF];                  // level-1 coefficients from jac_far_kernel
  __shared__ float s_c2[MJ_THREADS / 32][3][MJ_K];   // merged series of levels 1 and 2 per warp
  __shared__ double s_vjp[2][MJ_THREADS / 32];

  const int row = blockIdx.y;
  const int tile = blockIdx.x / chunks_per_tile, chunk = blockIdx.x % chunks_per_tile;
  const long long t0 = (long long)tile * tile_samples;
  const long long t1 = min(t0 + (long long)tile_samples, n_nu);
  long long c0;
  int n_c;
  if (!tile_chunk(t0, t1, chunk, blockDim.x * P, c0, n_c)) return;
  const double wlo = __dsub_rn(grid_nu(nu_min, step, t0), cutoff);
  const double whi = __dadd_rn(grid_nu(nu_min, step, t1 - 1), cutoff);
  const LineF32* lp = prep + (long long)row * n_lines;
  const LineJac* jp = jprep + (long long)row * n_lines;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, n_warps = blockDim.x >> 5;
  const float H1 = 0.5f * (float)(n_c - 1), C1 = H1;
  const bool use_l1 = H1 >= MJ_MIN_H1;
  // with level 1 (jac_far_kernel) only the inner range can hold inner lines of this chunk
  int2 rng = ranges[tile];
  if (use_l1 && inner_ranges) {
    const int2 q = inner_ranges[tile];
    rng = make_int2(max(rng.x, q.x), min(rng.y, q.y));
  }
  if (use_l1 && tid < MJ_NCOEF) s_c1[tid] = l1_coef[((long long)row * gridDim.x + blockIdx.x) * MJ_NCOEF + tid];
  const int w0 = warp * MJ_WARP_PTS;
  const int n_w = max(0, min(MJ_WARP_PTS, n_c - w0));
  const float H2 = 0.5f * (float)(n_w - 1), C2w = (float)w0 + H2;
  const bool use_l2 = H2 >= MJ_MIN_H2;
  const float xn2 = H2 * c_jnode16[lane & 15];
  const float xn2f = H2 * c_jnode8[lane & 7];
  const float pf = (float)(w0 + lane * P);

  for (int i = tid; i < 3 * MJ_CHUNK; i += blockDim.x) (&s_core[0][0])[i] = 0.f;

  float acc[3][P];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int m = 0; m < P; ++m) acc[q][m] = 0.f;
  float sum2[3] = {0.f, 0.f, 0.f}, comp2[3] = {0.f, 0.f, 0.f}, sum2f[3] = {0.f, 0.f, 0.f};

  // round r takes lines rng.x + k * n_rounds + r (k = thread): an even sample of the inner
  // range per round, so the warps' level-3 and near-zone shares stay balanced round by round
  const int n_in = max(0, rng.y - rng.x);
  const int n_rounds = (n_in + (int)blockDim.x - 1) / (int)blockDim.x;
  for (int r = 0; r < n_rounds; ++r) {
    const int k = tid * n_rounds + r;
    const int li = rng.x + k;
    const bool have = k < n_in;
    LineF32 L;
    LineJac J;
    if (have) {
      L = lp[li];
      J = jp[li];
    }
    const bool pass = have && (L.nuc >= wlo) && (L.nuc <= whi);
    const float jf = (float)((long long)L.j0 - c0);
    const bool lev1 = pass && use_l1 && (fabsf(jf - C1) - H1 > H1 + 1.f);   // jac_far_kernel's line
    const bool inner = pass && !lev1;
    const float y2 = L.y * L.y;
    bool any3 = false;
    if (inner) {
      for (int w = 0; w < n_warps; ++w) {              // same test as the per-warp split below
        const int nw = min(MJ_WARP_PTS, n_c - w * MJ_WARP_PTS);
        if (nw <= 0) break;
        const float h2 = 0.5f * (float)(nw - 1);
        any3 |= !(h2 >= MJ_MIN_H2 && fabsf(jf - ((float)(w * MJ_WARP_PTS) + h2)) - h2 > h2 + 1.f);
      }
    }
    // near range (points with possibly |z|^2 < MID_Z2) clipped to the chunk, and its middle
    // (|z|^2 possibly < CORE_Z2), one point of margin each
    int near_lo = 0, near_n = 0, mid_lo = 0, mid_n = 0;
    if (inner && any3 && !(y2 >= MID_Z2 && L.y >= 0.f)) {
      const float hw = sqrtf(fmaxf(MID_Z2 - y2, 0.f)) / L.a + 1.0f;
      const float q = jf + L.b / L.a;
      const float lo_f = fmaxf(ceilf(q - hw), 0.f);
      const float hi_f = fminf(floorf(q + hw), (float)(n_c - 1));
      if (lo_f <= hi_f) {
        near_lo = (int)lo_f;
        near_n = (int)hi_f - near_lo + 1;
        if (y2 < CORE_Z2 && L.y >= 0.f) {
          const float hw36 = sqrtf(CORE_Z2 - y2) / L.a + 1.0f;
          const float a0 = fmaxf(ceilf(q - hw36), (float)near_lo);
          const float a1 = fminf(floorf(q + hw36), (float)(near_lo + near_n - 1));
          if (a0 <= a1) {
            mid_lo = (int)a0;
            mid_n = (int)a1 - mid_lo + 1;
          }
        }
      }
    }
    const unsigned b2 = __ballot_sync(0xffffffffu, inner);
    if (lane == 0) s_cnt[warp] = __popc(b2);
    __syncthreads();
    int off2 = 0, n2 = 0;
    for (int w = 0; w < n_warps; ++w) {
      const int a2 = s_cnt[w];
      off2 += (w < warp) ? a2 : 0;
      n2 += a2;
    }
    if (inner) {
      JLine r;
      r.g = make_float4(jf, L.a, L.b, L.amp);
      r.h = make_float4(L.y, y2, J.jT_u, J.jT_x);
      r.k = make_float4(J.jT_y, J.jv_u, J.jv_y, J.jv_x);
      const int slot = off2 + __popc(b2 & ((1u << lane) - 1u));
      s2[slot] = r;
      s_nr[slot] = make_short4((short)near_lo, (short)near_n, (short)mid_lo, (short)mid_n);
    }
    __syncthreads();

    // per-warp split of the inner lines into level 2 (16 nodes; 8 beyond four sub-chunk
    // half-widths, listed from the back of s_l2) and level 3
    int n2w = 0, n2fw = 0, n3w = 0;
    for (int k = 0; k < n2; k += 32) {
      const int l = k + lane;
      bool is2 = false, is2f = false, is3 = false;
      if (l < n2) {
        const float d = fabsf(s2[l].g.x - C2w) - H2;
        const bool lev2 = use_l2 && d > H2 + 1.f;
        is2f = lev2 && d > MJ_FAR1 * H2;
        is2 = lev2 && !is2f;
        is3 = !lev2 && n_w > 0;
      }
      const unsigned q2 = __ballot_sync(0xffffffffu, is2), q3 = __ballot_sync(0xffffffffu, is3);
      const unsigned q2f = __ballot_sync(0xffffffffu, is2f);
      const unsigned lt = (1u << lane) - 1u;
      if (is2) s_l2[warp][n2w + __popc(q2 & lt)] = (unsigned char)l;
      if (is2f) s_l2[warp][MJ_THREADS - 1 - (n2fw + __popc(q2f & lt))] = (unsigned char)l;
      if (is3) s_l3[warp][n3w + __popc(q3 & lt)] = (unsigned char)l;
      n2w += __popc(q2);
      n2fw += __popc(q2f);
      n3w += __popc(q3);
    }
    __syncwarp();
    // level 2: half-warps take one line each, lane (& 15) = node
    {
      float a[3] = {0.f, 0.f, 0.f};
      for (int i = lane >> 4; i < n2w; i += 2) {
        const JLine R = s2[s_l2[warp][i]];
        const float x = fmaf(xn2 + (C2w - R.g.x), R.g.y, -R.g.z);
        add3(a, value3(x, R), x, R);
      }
      kahan3(sum2, comp2, a);
      // far level-2 lines: quarter-warps take one line each, lane (& 7) = node
      for (int i = lane >> 3; i < n2fw; i += 4) {
        const JLine R = s2[s_l2[warp][MJ_THREADS - 1 - i]];
        const float x = fmaf(xn2f + (C2w - R.g.x), R.g.y, -R.g.z);
        add3(sum2f, value3(x, R), x, R);
      }
    }
    // level 3, clamped loop (branch-free per line). A line whose nearest point of the
    // warp's sub-chunk has |z|^2 >= TIER3_Z2 (no near point here) takes the three-term
    // series at every point; the choice is uniform across the warp. A sub-chunk of at most
    // P points (the one-point tile at the end of a grid) lets each lane take its own lines
    // at lane 0's points; the lanes' sums are added after the last round.
    auto level3_line = [&](int i, float pl0) {
      const JLine R = s2[s_l3[warp][i]];
      const float x0 = fmaf(pl0 - R.g.x, R.g.y, -R.g.z);
      const float xl = fmaf((float)w0 - R.g.x, R.g.y, -R.g.z);       // x at the sub-chunk's first point
      const float xh = fmaf((float)(n_w - 1), R.g.y, xl);            // and at its last (x grows with p)
      const float xmin = xl > 0.f ? xl : (xh < 0.f ? -xh : 0.f);
      if (fmaf(xmin, xmin, R.h.y) >= TIER3_Z2) {
#pragma unroll
        for (int m = 0; m < P; ++m) {
          const float x = fmaf((float)m, R.g.y, x0);
          const U3 v = series3(x, R.h.x, rcp_approx(fmaf(x, x, R.h.y)));
          float a3[3] = {acc[0][m], acc[1][m], acc[2][m]};
          add3(a3, v, x, R);
          acc[0][m] = a3[0];
          acc[1][m] = a3[1];
          acc[2][m] = a3[2];
        }
      } else {
#pragma unroll
        for (int m = 0; m < P; ++m) {
          const float x = fmaf((float)m, R.g.y, x0);
          const U3 v = series5(x, R.h.x, rcp_approx(fmaxf(fmaf(x, x, R.h.y), MID_Z2)));
          float a3[3] = {acc[0][m], acc[1][m], acc[2][m]};
          add3(a3, v, x, R);
          acc[0][m] = a3[0];
          acc[1][m] = a3[1];
          acc[2][m] = a3[2];
        }
      }
    };
    {
      const bool few = n_w <= P;                      // warp-uniform
      const float pl0 = few ? (float)w0 : pf;
      for (int i = few ? lane : 0; i < n3w; i += few ? 32 : 1) level3_line(i, pl0);
    }
    // level 3, near correction (accurate - clamped) of the warp's level-3 lines at the near
    // points inside its sub-chunk, 32 lines at a time: the middles (float64 core), then the
    // tails, as item spaces; lanes take consecutive items and find their line by a shuffle
    // search. x is formed exactly as in the loop above, so the clamped values cancel.
    for (int j0 = 0; j0 < n3w; j0 += 32) {
      const int j = j0 + lane;
      int slot = 0, lo = 0, mlo = 0, mhi = 0, mn = 0, tn = 0, ln = 0;
      if (j < n3w) {
        slot = s_l3[warp][j];
        const short4 nr = s_nr[slot];
        const int a0 = max((int)nr.x, w0), a1 = min((int)nr.x + (int)nr.y, w0 + n_w);
        if (a1 > a0) {
          lo = a0;
          mlo = max((int)nr.z, a0);
          mhi = min((int)nr.z + (int)nr.w, a1);
          mn = max(0, mhi - mlo);
          if (mn == 0) mlo = mhi = a1;                  // no middle here: all of it is the left tail
          tn = (a1 - a0) - mn;
          ln = mlo - a0;                                // left tail [a0, mlo), right tail [mhi, a1)
        }
      }
      int mo = mn, to = tn;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, mo, o), w = __shfl_up_sync(0xffffffffu, to, o);
        if (lane >= o) {
          mo += u;
          to += w;
        }
      }
      const int M = __shfl_sync(0xffffffffu, mo, 31), T = __shfl_sync(0xffffffffu, to, 31);
      mo -= mn;
      to -= tn;
      // item t of a space lies in the run of the last lane whose offset is <= t
      auto owner = [&](int off, int t) {
        int o = 0;
#pragma unroll
        for (int st = 16; st >= 1; st >>= 1)
          if (__shfl_sync(0xffffffffu, off, o + st) <= t) o += st;
        return o;
      };
      auto locate = [&](bool mid, int t, int& p, int& sl) {
        const int off = mid ? mo : to;
        const int o = owner(off, t);
        const int k = t - __shfl_sync(0xffffffffu, off, o);
        const int m_lo = __shfl_sync(0xffffffffu, mlo, o), t_lo = __shfl_sync(0xffffffffu, lo, o);
        const int t_ln = __shfl_sync(0xffffffffu, ln, o), t_hi = __shfl_sync(0xffffffffu, mhi, o);
        sl = __shfl_sync(0xffffffffu, slot, o);
        p = mid ? m_lo + k : (k < t_ln ? t_lo + k : t_hi + (k - t_ln));
      };
      auto correction = [&](bool mid, int p, int sl, float (&d)[3]) {
        d[0] = d[1] = d[2] = 0.f;
        const JLine R = s2[sl];
        const float x0 = fmaf((float)(p & ~(P - 1)) - R.g.x, R.g.y, -R.g.z);
        const float x = fmaf((float)(p & (P - 1)), R.g.y, x0);
        const float z2 = fmaf(x, x, R.h.y);
        if (z2 >= MID_Z2) return;
        const U3 good = near3(x, R.h.x, z2, mid);
        const U3 clamped = series5(x, R.h.x, rcp_approx(fmaxf(z2, MID_Z2)));
        float a[3] = {0.f, 0.f, 0.f}, b[3] = {0.f, 0.f, 0.f};
        add3(a, good, x, R);
        add3(b, clamped, x, R);
        d[0] = a[0] - b[0];
        d[1] = a[1] - b[1];
        d[2] = a[2] - b[2];
      };
      for (int pass_mid = 1; pass_mid >= 0; --pass_mid) {
        const bool mid = pass_mid;
        const int total = mid ? M : T;
        if constexpr (!DET) {
          // shared-memory atomics: overlapping near zones of two lines in one 32-item step
          // meet at a point in an order the hardware picks (~1e-9 relative)
          for (int it0 = 0; it0 < total; it0 += 32) {
            const int t = min(it0 + lane, total - 1);
            int p, sl;
            locate(mid, t, p, sl);
            if (it0 + lane < total) {
              float d[3];
              correction(mid, p, sl, d);
              if (d[0] != 0.f || d[1] != 0.f || d[2] != 0.f) {
                atomicAdd(&s_core[0][p], d[0]);
                atomicAdd(&s_core[1][p], d[1]);
                atomicAdd(&s_core[2][p], d[2]);
              }
            }
          }
        } else {
          // bit-reproducible: values into the warp's buffer, then added line by line in list
          // order, each line's points spread over the lanes
          float* buf = s_nbuf_dyn + warp * 3 * MJ_NBW;
          for (int b0 = 0; b0 < total; b0 += MJ_NBW) {
            const int b1 = min(total, b0 + MJ_NBW);
            for (int it0 = b0; it0 < b1; it0 += 32) {
              const int t = min(it0 + lane, b1 - 1);
              int p, sl;
              locate(mid, t, p, sl);
              if (it0 + lane < b1) {
                float d[3];
                correction(mid, p, sl, d);
                buf[t - b0] = d[0];
                buf[MJ_NBW + t - b0] = d[1];
                buf[2 * MJ_NBW + t - b0] = d[2];
              }
            }
            __syncwarp();
            // only the lines whose items fall in [b0, b1): from the owner of b0 to that of b1 - 1
            const int j_hi = owner(mid ? mo : to, b1 - 1);
            for (int jl = owner(mid ? mo : to, b0); jl <= j_hi; ++jl) {
              const int st = __shfl_sync(0xffffffffu, mid ? mo : to, jl);
              const int n = __shfl_sync(0xffffffffu, mid ? mn : tn, jl);
              const int m_lo = __shfl_sync(0xffffffffu, mlo, jl), t_lo = __shfl_sync(0xffffffffu, lo, jl);
              const int t_ln = __shfl_sync(0xffffffffu, ln, jl), t_hi = __shfl_sync(0xffffffffu, mhi, jl);
              const int ia = max(st, b0), ib = min(st + n, b1);
              for (int it = ia + lane; it < ib; it += 32) {
                const int k = it - st;
                const int p = mid ? m_lo + k : (k < t_ln ? t_lo + k : t_hi + (k - t_ln));
                s_core[0][p] += buf[it - b0];
                s_core[1][p] += buf[MJ_NBW + it - b0];
                s_core[2][p] += buf[2 * MJ_NBW + it - b0];
              }
              __syncwarp();
            }
          }
        }
      }
    }
    // No barrier here: the next round writes the staging arrays only after its first
    // barrier, which every warp reaches after finishing this round.
  }
  __syncthreads();
  if (n_w <= P) {                                   // lanes' level-3 sums at lane 0's points
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int m = 0; m < P; ++m)
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) acc[q][m] += __shfl_xor_sync(0xffffffffu, acc[q][m], o);
  }

  // One Chebyshev series per sum and sub-chunk: the level-2 node sums (lanes j and j+16
  // hold halves of node j), the 8-node interpolant and the level-1 series evaluated at the
  // 16 nodes, transformed back to coefficients; each point then evaluates one series per sum.
  const float inv_h1 = use_l1 ? 1.0f / H1 : 0.f, inv_h2 = use_l2 ? 1.0f / H2 : 0.f;
  if (use_l2) {
    const int jn = lane & 15;
    const float tj = c_jnode16[jn];
    const float t1 = fmaf(H2, tj, C2w - C1) * inv_h1;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float f2 = sum2[q] - comp2[q];
      f2 += __shfl_xor_sync(0xffffffffu, f2, 16);
      float g2 = sum2f[q];                                    // lanes j, j+8, j+16, j+24: quarters of node j
      g2 += __shfl_xor_sync(0xffffffffu, g2, 16);
      g2 += __shfl_xor_sync(0xffffffffu, g2, 8);
      double cf = 0.0;
      for (int j = 0; j < MJ_KF; ++j) cf += (double)__shfl_sync(0xffffffffu, g2, j) * c_jdct8[(lane & 7) * MJ_KF + j];
      float c8f[MJ_KF];
#pragma unroll
      for (int k = 0; k < MJ_KF; ++k) c8f[k] = (float)(__shfl_sync(0xffffffffu, cf, k) * (2.0 / MJ_KF));
      double fj = (double)f2 + (double)clenshaw_k<MJ_KF>(c8f, tj);
      if (use_l1)
        fj += (double)(clenshaw_k(s_c1 + q * MJ_K, t1) + clenshaw_k<MJ_KF>(s_c1 + 3 * MJ_K + q * MJ_KF, t1));
      double ck = 0.0;
      for (int j = 0; j < MJ_K; ++j) ck += __shfl_sync(0xffffffffu, fj, j) * c_jdct16[jn * MJ_K + j];
      if (lane < MJ_K) s_c2[warp][q][lane] = (float)(ck * (2.0 / MJ_K));
    }
  }
  __syncwarp();

  const double T = t_layer[row];
  const float half_c2_t = (float)(0.5 * C2 / T), inv_t = (float)(1.0 / T);
  const double* g = g_tau ? g_tau + (long long)(row / n_lay) * n_nu : nullptr;
  double pt = 0.0, pv = 0.0;
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const int pl = w0 + lane * P + m;
    if (pl >= n_c) continue;
    float v[3];
    const float t1 = ((float)pl - C1) * inv_h1, t2 = ((float)pl - C2w) * inv_h2;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float s = s_core[q][pl];
      if (use_l2) s += clenshaw_k(s_c2[warp][q], t2);
      else if (use_l1) s += clenshaw_k(s_c1 + q * MJ_K, t1) + clenshaw_k<MJ_KF>(s_c1 + 3 * MJ_K + q * MJ_KF, t1);
      v[q] = acc[q][m] + s;
    }
    const long long p = c0 + pl;
    const float nu = (float)grid_nu(nu_min, step, p);
    const float hv = nu * half_c2_t;                          // c2 nu / 2T
    const float R = nu * tanhf(hv);                           // R(nu, T)
    const float ch = coshf(hv);
    const float R_T = -nu * (hv * inv_t) / (ch * ch);         // dR/dT
    const float jt = R_T * v[0] + R * v[1], jv = R * v[2];
    if (g) {                      // vector-Jacobian product with d loss / d tau
      pt += g[p] * (double)jt;
      pv += g[p] * (double)jv;
    } else {
      const long long o = (long long)row * n_nu + p;
      od[o] = v[0] * R;
      d_t[o] = jt;
      d_v[o] = jv;
    }
  }
  if (g) {
    for (int o = 16; o > 0; o >>= 1) {
      pt += __shfl_xor_sync(0xffffffffu, pt, o);
      pv += __shfl_xor_sync(0xffffffffu, pv, o);
    }
    if (lane == 0) {
      s_vjp[0][warp] = pt;
      s_vjp[1][warp] = pv;
    }
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < n_warps; ++w) {
        a += s_vjp[0][w];
        b += s_vjp[1][w];
      }
      atomicAdd(&vjp_t[row], a);
      atomicAdd(&vjp_v[row], b);
    }
  }
}

}  // namespace lbl

using namespace lbl;

static void jac_geometry(int tile_samples, long long n_nu, int* threads, int* cp, long long* n_tiles,
                         long long* chunks) {
  const int per_tile = tile_samples < MJ_CHUNK ? tile_samples : MJ_CHUNK;
  *threads = 32 * ((per_tile + MJ_WARP_PTS - 1) / MJ_WARP_PTS);
  *cp = *threads * MJ_P;
  *n_tiles = (n_nu + tile_samples - 1) / tile_samples;
  *chunks = (tile_samples + *cp - 1) / *cp;
}

extern "C" long long lbl_jacobian_ml_work_floats(int n_rows, long long n_nu, int tile_samples) {
  if (n_rows < 1 || n_nu < 1 || tile_samples < 1) return -1;
  int threads, cp;
  long long n_tiles, chunks;
  jac_geometry(tile_samples, n_nu, &threads, &cp, &n_tiles, &chunks);
  return (long long)n_rows * n_tiles * chunks * MJ_NCOEF;
}

extern "C" int lbl_jac_near_ranges(const LineIn* lines, const int* n_kept, double nu_min, double step, long long n_nu,
                                   int tile_samples, double pad, int n_tiles, int* near, void* stream) {
  if (tile_samples < 1 || !(step > 0) || n_nu < 1)
    return lbl_set_error(LBL_EINVAL, "lbl_jac_near_ranges: bad arguments");
  // A 16-node level-1 line of a chunk (half-width H) has |j0 - centre| <= (1 + MJ_FAR1) H, so
  // its centre lies within MJ_FAR1 H + 1.5 grid steps of the chunk; chunks lie inside their tile
  // and have at most min(tile_samples, chunk size) points. Two further steps absorb rounding.
  int threads, cp;
  long long n_all, chunks;
  jac_geometry(tile_samples, n_nu, &threads, &cp, &n_all, &chunks);
  const int n_c_max = tile_samples < cp ? tile_samples : cp;
  const double reach = (0.5 * MJ_FAR1 * (n_c_max - 1) + 3.5) * step;
  return lbl_tile_ranges(lines, n_kept, nu_min, step, n_nu, tile_samples, reach, pad, n_tiles, near, stream);
}

extern "C" int lbl_jacobian_ml_f32(const LineF32* prep, const LineJac* jprep, int n_lines, const int* ranges,
                                   const int* inner, const int* near, const double* t_layer, int n_rows, int n_lay, double nu_min,
                                   double step, long long n_nu, int tile_samples, double cutoff, float* l1_work,
                                   float* od, float* d_t, float* d_v, const double* g_tau, double* vjp_t,
                                   double* vjp_v, int flags, void* stream) {
  const bool vjp = g_tau != nullptr;
  if (!prep || !jprep || !ranges || !t_layer || !l1_work || n_lines < 1 || n_rows < 1 || n_lay < 1 ||
      n_rows % n_lay || n_rows > 65535 || n_nu < 1 || tile_samples < 1 || !(step > 0) || !(cutoff >= 0) ||
      (vjp ? (!vjp_t || !vjp_v) : (!od || !d_t || !d_v)))
    return lbl_set_error(LBL_EINVAL, "lbl_jacobian_ml_f32: bad arguments");
  int threads, cp;
  long long n_tiles, chunks;
  jac_geometry(tile_samples, n_nu, &threads, &cp, &n_tiles, &chunks);
  if (n_tiles * chunks > 0x7fffffffLL) return lbl_set_error(LBL_EINVAL, "lbl_jacobian_ml_f32: grid too large");
  dim3 grid((unsigned)(n_tiles * chunks), (unsigned)n_rows);
  cudaStream_t st = (cudaStream_t)stream;
  jac_far_kernel<<<grid, MJF_THREADS, 0, st>>>(prep, jprep, n_lines, (const int2*)ranges, (const int2*)near, nu_min,
                                               step, n_nu, tile_samples, (int)chunks, cp, cutoff, l1_work);
  if (flags & LBL_DETERMINISTIC) {
    constexpr int dyn_bytes = (MJ_THREADS / 32) * 3 * MJ_NBW * (int)sizeof(float);   // near-item buffers
    int dev = 0;
    cudaGetDevice(&dev);
    static int attr_set[64] = {0};
    if (dev < 0 || dev >= 64) return lbl_set_error(LBL_EINVAL, "lbl_jacobian_ml_f32: device index out of range");
    if (!attr_set[dev]) {
      if (cudaFuncSetAttribute(jac_ml_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_bytes) !=
          cudaSuccess)
        return lbl_check_launch("lbl_jacobian_ml_f32 (shared memory attribute)");
      attr_set[dev] = 1;
    }
    jac_ml_kernel<true><<<grid, threads, dyn_bytes, st>>>(
        prep, jprep, n_lines, (const int2*)ranges, (const int2*)inner, t_layer, nu_min, step, n_nu, tile_samples,
        (int)chunks, cutoff, l1_work, od, d_t, d_v, n_lay, g_tau, vjp_t, vjp_v);
  } else {
    jac_ml_kernel<false><<<grid, threads, 0, st>>>(
        prep, jprep, n_lines, (const int2*)ranges, (const int2*)inner, t_layer, nu_min, step, n_nu, tile_samples,
        (int)chunks, cutoff, l1_work, od, d_t, d_v, n_lay, g_tau, vjp_t, vjp_v);
  }
  return lbl_check_launch("lbl_jacobian_ml_f32");
}
