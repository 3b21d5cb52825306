// Multi-level float32 Voigt summation (the default float32 engine).
//
// Same result contract as tau_f32_kernel (voigt.cu): od[row, p] = R(nu_p, T_row) *
// sum over the lines admitted by the reference's tile window (forward.py:295-301)
// of S * phi(nu_p). The sum is split by distance so that most lines are
// evaluated at a handful of points instead of every grid point:
//
//  level 1  lines farther than one chunk half-width from the CTA's chunk
//           (<= 2048 points of one reference tile): their summed profile is
//           analytic on a Bernstein ellipse with rho >= 2 + sqrt(3) around the
//           chunk, so it is evaluated at K1 = 16 Chebyshev nodes and interpolated
//           (interpolation error ~rho^-16 ~ 1e-9 of the level-1 sum; lines more than
//           four half-widths out use 8 nodes, rho >= 7.87: ~7e-8 of their sum). A
//           separate kernel (tau_far_kernel) computes this level and hands its
//           coefficients over through a workspace;
//  level 2  the other lines farther than one sub-chunk half-width from a warp's
//           256-point sub-chunk: 16 Chebyshev nodes per sub-chunk, same geometry
//           (8 beyond four sub-chunk half-widths);
//  level 3  the remaining lines: direct evaluation at every point. The warp's
//           loop is branch-free: it evaluates the five-term asymptotic form with
//           |z|^2 clamped to >= MID_Z2 = 64, so every point inside a line's near
//           zone receives the same constant. A CTA-wide near pass then gives each
//           near point (accurate value - that constant): eight terms of the float
//           asymptotic series for 36 <= |z|^2 < 64, Weideman's float64 approximation below.
//
// Inside a reference tile the set of lines is fixed, so every level-1/2 sum is
// smooth over its interval; the window test keeps the reference's truncation.
// tau_ml_kernel reads only the lines that can be inner for its chunk (a range per
// tile from lbl_ml_inner_ranges), applies the same level-1 test and skips the
// level-1 lines among them.
#include <math.h>

#include "cheb_tables.h"
#include "faddeeva.cuh"
#include "lbl_common.cuh"
#include "sum_common.cuh"

namespace lbl {

constexpr int ML_P = 8;                        // points per lane (level 3)
constexpr int ML_WARP_PTS = 32 * ML_P;         // points per warp sub-chunk
constexpr int ML_THREADS = 256;                // max threads per CTA = lines staged per round
constexpr int ML_CHUNK = ML_THREADS * ML_P;    // max points per CTA
constexpr int ML_K = 16;                       // Chebyshev nodes per level
constexpr int ML_KF = 8;                       // nodes for level-1 lines far from the chunk
constexpr float ML_FAR1 = 3.f;                 // "far": more than (1 + ML_FAR1) half-widths from the centre
constexpr float ML_MIN_H1 = 32.f;              // smallest chunk half-width (points) using level 1
constexpr float ML_MIN_H2 = 16.f;              // smallest sub-chunk half-width using level 2

// Chebyshev node offsets (fractions of the half-width) and DCT weights, row-major [k][j]
static __constant__ float c_node16[ML_K] = {LBL_CHEB16_NODES};
static __constant__ float c_node8[ML_KF] = {LBL_CHEB8_NODES};
static __constant__ double c_dct16[ML_K * ML_K] = {LBL_DCT16};
static __constant__ double c_dct8[ML_KF * ML_KF] = {LBL_DCT8};
static_assert(ML_K == 16 && ML_KF == 8, "tables of cheb_tables.h");

struct MlLine {
  float4 g;   // jf (centre index relative to the chunk start), a, b, amp_far
  float4 h;   // y, y^2, amp, value the clamped far-wing loop adds inside the near zone
  float4 p;   // amp_far * (B_1, B_2, B_3, B_4)
  float4 q;   // amp_far * (B_5, B_6, B_7, B_8)
};

// Re w times the line amplitude at one point, any distance (fast far wing first).
__device__ __forceinline__ float line_value(float x, const MlLine& L) {
  const float z2 = fmaf(x, x, L.h.y);
  if (z2 >= FAR_Z2 && L.h.x >= 0.f) {
    const float r = rcp_approx(z2);
    return L.g.w * r * fmaf(fmaf(-2.0f * L.h.y, r, 1.5f), r, 1.0f);
  }
  if (z2 >= CORE_Z2 && L.h.x >= 0.f) return L.h.z * re_w_f32_mid(x, L.h.x, L.h.y, z2);
  return (float)((double)L.h.z * weideman_re_f32((double)x, (double)L.h.x));
}

// Five-term asymptotic real part regrouped by powers of r = 1/|z|^2 for one line:
// with s = y^2 (fixed per line) and q = s r, 1 + sum_k r^k A_k(q) = sum_m B_m(s) r^m,
//   B_0 = 1, B_1 = 1.5, B_2 = 3.75 - 2s, B_3 = 13.125 - 15s, B_4 = 59.0625 - 105s + 12s^2,
//   B_5 = -787.5s + 210s^2, B_6 = 2835s^2 - 120s^3, B_7 = -3780s^3, B_8 = 1680s^4
// (A_k from asym5_bracket). For s >= 4096, |z|^2 >= s gives r <= 1/4096 and the
// r^5..r^8 terms stay below 1e-8 of the sum, so they are dropped (which also keeps
// the coefficients far from float overflow). Float32 evaluation by Horner's rule
// agrees with the grouped form to 6e-8 relative for s <= 1e4 and clamped r.
__device__ __forceinline__ void asym5_line_coeffs(float s, float amp_far, float4& p, float4& q) {
  const float b2 = fmaf(-2.0f, s, 3.75f), b3 = fmaf(-15.0f, s, 13.125f);
  const float b4 = fmaf(fmaf(12.0f, s, -105.0f), s, 59.0625f);
  p = make_float4(amp_far * 1.5f, amp_far * b2, amp_far * b3, amp_far * b4);
  if (s < 4096.0f) {
    const float s2 = s * s;
    q = make_float4(amp_far * (fmaf(210.0f, s, -787.5f) * s), amp_far * (fmaf(-120.0f, s, 2835.0f) * s2),
                    amp_far * (-3780.0f * s2 * s), amp_far * (1680.0f * s2 * s2));
  } else {
    q = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// amp_far * S at r (the level-3 loop body without the final r factor).
__device__ __forceinline__ float asym5_scaled(float r, const MlLine& R) {
  float v = fmaf(R.q.w, r, R.q.z);
  v = fmaf(v, r, R.q.y);
  v = fmaf(v, r, R.q.x);
  v = fmaf(v, r, R.p.w);
  v = fmaf(v, r, R.p.z);
  v = fmaf(v, r, R.p.y);
  v = fmaf(v, r, R.p.x);
  return fmaf(v, r, R.g.w);
}

// r = 1/|z|^2 with |z|^2 clamped to >= MID_Z2: inside the near zone the loop adds the
// constant r_c * asym5_scaled(r_c), r_c = rcp(MID_Z2).
__device__ __forceinline__ float clamped_r(float x, float y2) {
  return rcp_approx(fmaxf(fmaf(x, x, y2), MID_Z2));
}

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float v) {
  const float yk = v - comp;
  const float t = sum + yk;
  comp = (t - sum) - yk;
  sum = t;
}

// p(t) = c0/2 + sum_{k>=1} c_k T_k(t) by Clenshaw's recurrence (K coefficients).
template <int K = ML_K>
__device__ __forceinline__ float clenshaw16(const float* c, float t) {
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
// Level 1 as its own kernel. Nine in ten lines of a chunk's window are level-1
// lines; each contributes only through the chunk's Chebyshev nodes, so one thread
// takes one line and evaluates it at all nodes from registers (each thread copies its
// own records through a cp.async ring; no barriers). The kernel leaves the chunk's
// 16 + 8 Chebyshev coefficients in l1_work ([row][chunk of the launch][24]), which
// tau_ml_kernel reads.
constexpr int MF_THREADS = 256;                // lines per round
constexpr int MF_FLUSH = 32;                   // rounds summed in float before the double sums

constexpr int MF_STAGES = 3;                   // rounds of line records in flight per thread

// amp * Re w by the far-wing form (amp_far = amp y / sqrt(pi)), added to f (|z|^2 >= FAR_Z2, y >= 0).
__device__ __forceinline__ void far_wing_add(float& f, float x, float y2, float ny2, float amp_far) {
  const float r = rcp_approx(fmaf(x, x, y2));
  f = fmaf(amp_far * r, fmaf(fmaf(ny2, r, 1.5f), r, 1.0f), f);
}

// amp * Re w at one node for a level-1 line that is not in the far-wing regime at
// every node (broad lines, coarse geometry): the engine's full float32 algorithm.
static __device__ __noinline__ float far_node_general(float x, float y, float y2, float amp, float amp_far) {
  const float z2 = fmaf(x, x, y2);
  if (z2 >= FAR_Z2 && y >= 0.f) {
    const float r = rcp_approx(z2);
    return amp_far * r * fmaf(fmaf(-2.0f * y2, r, 1.5f), r, 1.0f);
  }
  if (z2 >= CORE_Z2 && y >= 0.f) return amp * re_w_f32_mid(x, y, y2, z2);
  return (float)((double)amp * weideman_re_f32_compact((double)x, (double)y));
}

// Node sums of one level-1 line: nodes k and K-1-k sit at +xs[k] and -xs[k] from the chunk centre.
template <int K>
__device__ __forceinline__ void far_line_nodes(float (&f)[K], const float (&xs)[K / 2], const LineF32& L, float xc,
                                               float y2, bool fast) {
  if (fast) {
    const float ny2 = -2.0f * y2, na = -L.a;
#pragma unroll
    for (int k = 0; k < K / 2; ++k) {
      far_wing_add(f[k], fmaf(xs[k], L.a, xc), y2, ny2, L.amp_far);
      far_wing_add(f[K - 1 - k], fmaf(xs[k], na, xc), y2, ny2, L.amp_far);
    }
  } else {
#pragma unroll
    for (int k = 0; k < K / 2; ++k) {
      f[k] += far_node_general(fmaf(xs[k], L.a, xc), L.y, y2, L.amp, L.amp_far);
      f[K - 1 - k] += far_node_general(fmaf(xs[k], -L.a, xc), L.y, y2, L.amp, L.amp_far);
    }
  }
}

__global__ void __launch_bounds__(MF_THREADS, 4)
tau_far_kernel(const LineF32* __restrict__ prep, int n_lines, const int2* __restrict__ ranges, double nu_min,
               double step, long long n_nu, int tile_samples, int chunks_per_tile, int chunk_pts, double cutoff,
               float* __restrict__ l1_work, unsigned long long* evals, unsigned long long* work, int tile_first) {
  // Whole 32-B records: read back by their own thread they meet 2-way bank conflicts, but
  // the 16-B planes that jac_far_kernel stages its records in (no conflicts) made this
  // kernel slower (summation call 10.40 -> 11.06 ms, with more spilled registers).
  __shared__ __align__(16) LineF32 s_line[MF_STAGES][MF_THREADS];   // records are 32 B, 16-B aligned
  __shared__ double s_part[MF_THREADS / 32][ML_K + ML_KF];
  __shared__ float s_coef[ML_K + ML_KF];
  __shared__ unsigned s_cnt[2];

  const int row = blockIdx.y;
  const int tile = tile_first + (int)(blockIdx.x / chunks_per_tile), chunk = blockIdx.x % chunks_per_tile;
  const long long t0 = (long long)tile * tile_samples;
  const long long t1 = min(t0 + (long long)tile_samples, n_nu);
  long long c0;
  int n_c;
  if (!tile_chunk(t0, t1, chunk, chunk_pts, c0, n_c)) return;
  const float H1 = 0.5f * (float)(n_c - 1), C1 = H1;      // same chunk geometry as tau_ml_kernel
  if (!(H1 >= ML_MIN_H1)) return;                         // no level 1: tau_ml_kernel takes every line
  const int c0i = (int)c0;
  const double wlo = __dsub_rn(grid_nu(nu_min, step, t0), cutoff);
  const double whi = __dadd_rn(grid_nu(nu_min, step, t1 - 1), cutoff);
  const int2 rng = ranges[tile];
  const LineF32* lp = prep + (long long)row * n_lines;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < 2) s_cnt[tid] = 0u;
  if (lane == 0)                                           // this warp's node sums: lane 0 alone
    for (int k = 0; k < ML_K + ML_KF; ++k) s_part[warp][k] = 0.0;   // writes and reads them

  float xa[ML_K / 2], xb[ML_KF / 2];                      // node offsets, as tau_ml_kernel places them
#pragma unroll
  for (int k = 0; k < ML_K / 2; ++k) xa[k] = H1 * c_node16[k];
#pragma unroll
  for (int k = 0; k < ML_KF / 2; ++k) xb[k] = H1 * c_node8[k];

  float f1[ML_K], ff[ML_KF];
#pragma unroll
  for (int k = 0; k < ML_K; ++k) f1[k] = 0.f;
#pragma unroll
  for (int k = 0; k < ML_KF; ++k) ff[k] = 0.f;
  unsigned n1 = 0, nf = 0;

  // line records of round r (line rng.x + r * MF_THREADS + tid) go to stage r % MF_STAGES,
  // MF_STAGES - 1 rounds ahead; every round commits one group (empty past the end), so
  // waiting for all but the newest MF_STAGES - 1 groups completes the current round's copy
  const int n_rounds = rng.y > rng.x ? (rng.y - rng.x + MF_THREADS - 1) / MF_THREADS : 0;
  auto issue = [&](int r, int stage) {
    const int li = rng.x + r * MF_THREADS + tid;
    if (li < rng.y) {   // prep records: 32 B each in a 256-B aligned allocation
      const float4* g = reinterpret_cast<const float4*>(lp + li);
      float4* d = reinterpret_cast<float4*>(&s_line[stage][tid]);
      cp_async16(d, g);
      cp_async16(d + 1, g + 1);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int r = 0; r < MF_STAGES - 1; ++r) issue(r, r);
  int rounds = 0, stage = 0;
  for (int r = 0; r < n_rounds; ++r) {
    issue(r + MF_STAGES - 1, stage == 0 ? MF_STAGES - 1 : stage - 1);   // the stage read last round
    cp_async_wait<MF_STAGES - 1>();
    const bool have = rng.x + r * MF_THREADS + tid < rng.y;
    LineF32 L;
    if (have) L = s_line[stage][tid];
    stage = stage + 1 == MF_STAGES ? 0 : stage + 1;
    // the level-1 test of tau_ml_kernel, expression for expression
    const bool pass = have && (L.nuc >= wlo) && (L.nuc <= whi);
    const float jf = (float)(L.j0 - c0i);
    const float dd = fabsf(jf - C1) - H1;
    if (pass && dd > H1 + 1.f) {
      const float xc = fmaf(C1 - jf, L.a, -L.b);         // line centre -> chunk centre, in x units
      const float y2 = L.y * L.y;
      // every node lies on one side of the line; the nearest is xa[0] in from the centre
      const float xm = fmaf(-xa[0], L.a, fabsf(xc));
      const bool fast = fmaf(xm, xm, y2) >= FAR_Z2 && L.y >= 0.f;
      if (dd > ML_FAR1 * H1) {
        far_line_nodes<ML_KF>(ff, xb, L, xc, y2, fast);
        ++nf;
      } else {
        far_line_nodes<ML_K>(f1, xa, L, xc, y2, fast);
        ++n1;
      }
    }
    if (++rounds == MF_FLUSH) {                            // warp-uniform: every lane runs every round
      rounds = 0;
      flush_nodes(f1, s_part[warp], lane);
      flush_nodes(ff, s_part[warp] + ML_K, lane);
    }
  }
  cp_async_wait<0>();                                      // only empty groups remain
  // node sums over the CTA in double: warps, then across warps
  flush_nodes(f1, s_part[warp], lane);
  flush_nodes(ff, s_part[warp] + ML_K, lane);
  n1 = __reduce_add_sync(0xffffffffu, n1);
  nf = __reduce_add_sync(0xffffffffu, nf);
  __syncthreads();                                         // s_cnt zeroed, s_part written
  if (lane == 0) {
    atomicAdd(&s_cnt[0], n1);
    atomicAdd(&s_cnt[1], nf);
  }
  if (tid < ML_K + ML_KF) {                                // column tid: only this thread touches it
    double s = 0.0;
    for (int w = 0; w < MF_THREADS / 32; ++w) s += s_part[w][tid];
    s_part[0][tid] = s;
  }
  __syncthreads();
  // Chebyshev coefficients (DCT of the node values)
  if (tid < ML_K) {
    double c = 0.0;
    for (int j = 0; j < ML_K; ++j) c += s_part[0][j] * c_dct16[tid * ML_K + j];
    s_coef[tid] = (float)(c * (2.0 / ML_K));
  } else if (tid < ML_K + ML_KF) {
    const int k = tid - ML_K;
    double c = 0.0;
    for (int j = 0; j < ML_KF; ++j)
      c += s_part[0][ML_K + j] * c_dct8[k * ML_KF + j];
    s_coef[tid] = (float)(c * (2.0 / ML_KF));
  }
  if (tid < ML_K + ML_KF) l1_work[((long long)row * gridDim.x + blockIdx.x) * (ML_K + ML_KF) + tid] = s_coef[tid];
  if (tid == 0) {
    const unsigned long long a = s_cnt[0], b = s_cnt[1];
    if (evals && a + b) atomicAdd(evals, (a + b) * (unsigned long long)n_c);
    if (work && a + b) atomicAdd(&work[0], a * ML_K + b * ML_KF);
  }
}

// ---------------------------------------------------------------------------
// Levels 2 and 3 (tau_ml_kernel). Each round stages up to 256 candidate lines; the
// inner ones (not level-1 lines of tau_far_kernel) go to shared memory as
// structure-of-arrays records, with a 2-bit class per warp (none, level 3, level 2
// with 16 nodes, level 2 with 8 nodes). Then each warp works alone on its own
// 256-point sub-chunk, with no CTA barrier until the next round:
//  * level 2, one lane per line: the lane evaluates its line at every node of the
//    sub-chunk from registers (node offsets are constant operands); the lanes' node
//    sums are reduced once per round (transposed warp reduction) and added to the
//    warp's float64 node sums;
//  * level 3: each lane evaluates the line at its own 8 points, by the clamped
//    five-term form, or by the two-term form when the line is far from every point of
//    the sub-chunk (|z|^2 >= FAR_Z2 there);
//  * near zones: the near points of the warp's level-3 lines inside its sub-chunk form
//    an item space (middles, where the float64 core may apply, then tails); lanes take
//    consecutive items, find their line by a shuffle search over a group of 32 lines
//    and add (accurate value - clamped loop value) into the warp's part of s_core.
// The epilogue folds the level-1 series and both level-2 interpolants into one
// 16-term Chebyshev series per sub-chunk, so each point evaluates one series.
constexpr int ML_NBW = 128;                    // near items buffered per warp (bit-reproducible mode)
constexpr unsigned FULL_MASK = 0xffffffffu;

// Sum over the 32 lanes of f[16], transposed: afterwards lanes 2j and 2j+1 hold the
// total of node j (j = (lane >> 1) & 15); 16 shuffles for the 16 sums.
__device__ __forceinline__ float reduce16_transposed(const float (&f)[ML_K], int lane) {
  float g[8], h[4], u[2];
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
#pragma unroll
  for (int k = 0; k < 8; ++k) g[k] = (b4 ? f[k + 8] : f[k]) + __shfl_xor_sync(FULL_MASK, b4 ? f[k] : f[k + 8], 16);
#pragma unroll
  for (int k = 0; k < 4; ++k) h[k] = (b3 ? g[k + 4] : g[k]) + __shfl_xor_sync(FULL_MASK, b3 ? g[k] : g[k + 4], 8);
#pragma unroll
  for (int k = 0; k < 2; ++k) u[k] = (b2 ? h[k + 2] : h[k]) + __shfl_xor_sync(FULL_MASK, b2 ? h[k] : h[k + 2], 4);
  float v = (b1 ? u[1] : u[0]) + __shfl_xor_sync(FULL_MASK, b1 ? u[0] : u[1], 2);
  return v + __shfl_xor_sync(FULL_MASK, v, 1);
}

// The same for f[8]: afterwards lanes 4j .. 4j+3 hold the total of node j = (lane >> 2) & 7.
__device__ __forceinline__ float reduce8_transposed(const float (&f)[ML_KF], int lane) {
  float g[4], h[2];
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
  for (int k = 0; k < 4; ++k) g[k] = (b4 ? f[k + 4] : f[k]) + __shfl_xor_sync(FULL_MASK, b4 ? f[k] : f[k + 4], 16);
#pragma unroll
  for (int k = 0; k < 2; ++k) h[k] = (b3 ? g[k + 2] : g[k]) + __shfl_xor_sync(FULL_MASK, b3 ? g[k] : g[k + 2], 8);
  float v = (b2 ? h[1] : h[0]) + __shfl_xor_sync(FULL_MASK, b2 ? h[0] : h[1], 4);
  v += __shfl_xor_sync(FULL_MASK, v, 2);
  return v + __shfl_xor_sync(FULL_MASK, v, 1);
}

// amp_far * (1 + B_1 r + ... + B_8 r^8) of one line by Horner's rule (see asym5_line_coeffs).
__device__ __forceinline__ float asym5_poly(float r, float amp_far, const float4& p, const float4& q) {
  float v = fmaf(q.w, r, q.z);
  v = fmaf(v, r, q.y);
  v = fmaf(v, r, q.x);
  v = fmaf(v, r, p.w);
  v = fmaf(v, r, p.z);
  v = fmaf(v, r, p.y);
  v = fmaf(v, r, p.x);
  return fmaf(v, r, amp_far);
}

// Level 2, one lane per line: lane i of each 32-line step takes line list[stride * i]
// and adds its values at the K nodes offset (node_k * H2) from the sub-chunk centre C2w
// into f. Nodes k and K-1-k are mirror images, so each pair shares one offset. Three
// warp-uniform paths: two-term far-wing form when every lane's line has |z|^2 >=
// FAR_Z2 at every node, five-term form when |z|^2 >= MID_Z2 everywhere, else the full
// algorithm per node.
template <int K>
__device__ __forceinline__ void level2_lines(float (&f)[K], const unsigned char* list, int stride, int n,
                                             const float4* __restrict__ s_g, const float4* __restrict__ s_h,
                                             const float4* __restrict__ s_p, const float4* __restrict__ s_q,
                                             float C2w, float H2, int lane) {
  const float* nodes = K == ML_K ? c_node16 : c_node8;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    const bool act = i < n;
    int l = 0;
    float4 g = make_float4(C2w, 0.f, -1.0e4f, 0.f), h = make_float4(1.f, 1.f, 0.f, 0.f);   // idle lane: adds 0
    if (act) {
      l = list[stride * i];
      g = s_g[l];
      h = s_h[l];
    }
    const float xc = fmaf(C2w - g.x, g.y, -g.z);          // x at the sub-chunk centre
    const float ha = H2 * g.y;                            // sub-chunk half-width in x units
    const float xm = fmaf(-nodes[0], ha, fabsf(xc));      // |x| at the node nearest the line
    const float zm = fmaf(xm, xm, h.y);
    int path = 0;
    if (act && !(h.x >= 0.f && zm >= FAR_Z2)) path = (h.x >= 0.f && xm > 0.f && zm >= MID_Z2) ? 1 : 2;
    const int wpath = __reduce_max_sync(FULL_MASK, path);
    if (wpath == 0) {
      const float ny2 = -2.0f * h.y;
#pragma unroll
      for (int k = 0; k < K / 2; ++k) {
        far_wing_add(f[k], fmaf(nodes[k], ha, xc), h.y, ny2, g.w);
        far_wing_add(f[K - 1 - k], fmaf(-nodes[k], ha, xc), h.y, ny2, g.w);
      }
    } else if (wpath == 1) {
      float4 p = make_float4(0.f, 0.f, 0.f, 0.f), q = p;
      if (act) {
        p = s_p[l];
        q = s_q[l];
      }
#pragma unroll
      for (int k = 0; k < K / 2; ++k) {
        const float xa = fmaf(nodes[k], ha, xc), xb = fmaf(-nodes[k], ha, xc);
        const float ra = rcp_approx(fmaf(xa, xa, h.y)), rb = rcp_approx(fmaf(xb, xb, h.y));
        f[k] = fmaf(ra, asym5_poly(ra, g.w, p, q), f[k]);
        f[K - 1 - k] = fmaf(rb, asym5_poly(rb, g.w, p, q), f[K - 1 - k]);
      }
    } else {
#pragma unroll 1
      for (int k = 0; k < K / 2; ++k) {
        f[k] += far_node_general(fmaf(nodes[k], ha, xc), h.x, h.y, h.z, g.w);
        f[K - 1 - k] += far_node_general(fmaf(-nodes[k], ha, xc), h.x, h.y, h.z, g.w);
      }
    }
  }
}

// (accurate value - clamped loop value) of a level-3 line at chunk point p; x is
// formed exactly as in the level-3 loop, so the clamped constant h.w cancels. Items of
// a zone's middle (MID) take the float64 core at every point, the margin points with
// |z|^2 >= CORE_Z2 included (28-term set: Re w within 8e-8 there too), so no lane of a
// warp branches off to another form; tail items take the eight-term asymptotic series.
template <bool MID>
__device__ __forceinline__ float near_correction(int p, const float4& g, const float4& h) {
  const float x0 = fmaf((float)(p & ~(ML_P - 1)) - g.x, g.y, -g.z);
  const float x = fmaf((float)(p & (ML_P - 1)), g.y, x0);
  const float z2 = fmaf(x, x, h.y);
  if (z2 >= MID_Z2) return 0.f;
  float v;
  if (MID) v = (float)((double)h.z * weideman_re_f32((double)x, (double)h.x));
  else if (z2 >= CORE_Z2 && h.x >= 0.f) v = h.z * re_w_asym8(h.x, z2);
  else v = (float)((double)h.z * weideman_re_f32_compact((double)x, (double)h.x));
  return v - h.w;
}

// One round's staged inner lines (slot = thread), in dynamic shared memory, two rounds deep.
struct MlStage {
  float4 g[ML_THREADS];            // jf, a, b, amp_far
  float4 h[ML_THREADS];            // y, y^2, amp, clamped-loop value inside the near zone
  float4 p[ML_THREADS];            // amp_far * (B_1 .. B_4)
  float4 q[ML_THREADS];            // amp_far * (B_5 .. B_8)
  short4 nr[ML_THREADS];           // near range (lo, n) and its middle (lo, n), chunk points
  unsigned short cls[ML_THREADS];  // 2-bit class per warp: 0 -, 1 level 3, 2/3 level 2 (16/8)
};
constexpr size_t ML_STAGE_BYTES = 2 * sizeof(MlStage);

#ifndef LBL_ML_CTA_SUBS
#define LBL_ML_CTA_SUBS 8
#endif
constexpr int ML_CTA_SUBS = LBL_ML_CTA_SUBS;    // 256-point sub-chunks (warps) per CTA of tau_ml_kernel

template <bool DET>
__global__ void __launch_bounds__(32 * ML_CTA_SUBS, 4 * 8 / ML_CTA_SUBS)
tau_ml_kernel(const LineF32* __restrict__ prep, int n_lines, const int2* __restrict__ ranges,
              const int2* __restrict__ inner_ranges, const float* __restrict__ l1_work,
              const double* __restrict__ t_layer, double nu_min,
              double step, long long n_nu, int tile_samples, int chunks_per_tile, int chunk_pts, double cutoff,
              int n_grp, float* __restrict__ od, int* err, unsigned long long* evals, unsigned long long* work,
              int tile_first, long long out_first, long long out_stride) {
  constexpr int P = ML_P;
  constexpr int NW = ML_CTA_SUBS;
  constexpr int ST = 32 * NW;                       // lines staged per round (one per thread)
  extern __shared__ __align__(16) unsigned char s_dyn[];
  MlStage* const s_stage = reinterpret_cast<MlStage*>(s_dyn);   // two rounds' staging buffers
  __shared__ unsigned char s_l2[NW][ST];    // per-warp level-2 slots (16 nodes from the front, 8 from the back)
  __shared__ unsigned char s_l3[NW][ST];    // per-warp level-3 slots
  __shared__ float s_core[NW * ML_WARP_PTS];        // near-zone corrections (each warp owns its points)
  __shared__ double s_n2[NW][ML_K + ML_KF];         // level-2 node sums per warp
  __shared__ float s_c1[ML_K + ML_KF];              // level-1 coefficients from tau_far_kernel
  __shared__ float s_nbuf[DET ? NW : 1][DET ? ML_NBW : 1];   // near-item values (bit-reproducible mode)

  const int row = blockIdx.y;
  // a chunk's sub-chunks are split over `parts` CTAs of up to NW warps each
  const int parts = (chunk_pts / ML_WARP_PTS + NW - 1) / NW;
  const int chunk_id = blockIdx.x / parts, part = blockIdx.x % parts;
  const int tile = tile_first + chunk_id / chunks_per_tile, chunk = chunk_id % chunks_per_tile;
  const long long t0 = (long long)tile * tile_samples;
  const long long t1 = min(t0 + (long long)tile_samples, n_nu);
  long long c0;
  int n_c;
  if (!tile_chunk(t0, t1, chunk, chunk_pts, c0, n_c)) return;
  const int first_sub = part * NW, p0 = first_sub * ML_WARP_PTS;   // this CTA's first sub-chunk and point
  if (p0 >= n_c) return;
  const int c0i = (int)c0;
  const double wlo = __dsub_rn(grid_nu(nu_min, step, t0), cutoff);
  const double whi = __dadd_rn(grid_nu(nu_min, step, t1 - 1), cutoff);
  const LineF32* lp = prep + (long long)row * n_lines;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, n_warps = blockDim.x >> 5;
  // chunk geometry (points relative to c0)
  const float H1 = 0.5f * (float)(n_c - 1), C1 = H1;
  const bool use_l1 = H1 >= ML_MIN_H1;
  // With level 1 (done by tau_far_kernel) only lines inside the tile's inner range
  // can be inner lines of this chunk; without it every line of the window is.
  int2 rng = ranges[tile];
  if (use_l1 && inner_ranges) {
    const int2 q = inner_ranges[tile];
    rng = make_int2(max(rng.x, q.x), min(rng.y, q.y));
  }
  // this warp's sub-chunk
  const int w0 = (first_sub + warp) * ML_WARP_PTS;
  const int n_w = max(0, min(ML_WARP_PTS, n_c - w0));
  const float H2 = 0.5f * (float)(n_w - 1), C2w = (float)w0 + H2;
  const bool use_l2 = H2 >= ML_MIN_H2;
  const float pf = (float)(w0 + lane * P);                   // this lane's first point

  for (int i = lane; i < ML_WARP_PTS; i += 32) s_core[w0 - p0 + i] = 0.f;
  if (lane < ML_K + ML_KF) s_n2[warp][lane] = 0.0;
  if (use_l1 && tid < ML_K + ML_KF)
    s_c1[tid] = l1_work[((long long)row * (gridDim.x / parts) + chunk_id) * (ML_K + ML_KF) + tid];

  // level-3 sums hold only the lines within ~2 sub-chunk widths (tens of terms), so
  // plain float accumulation suffices
  float acc[P];
#pragma unroll
  for (int m = 0; m < P; ++m) acc[m] = 0.f;
  unsigned long long n_pass = 0, n_nodes = 0, n_l3 = 0, n_near_items = 0;

  // register prefetch of the next round's line records
  // Round r stages lines rng.x + k * n_rounds + r (k = thread): every round is an even
  // sample of the whole inner range, so each warp's sub-chunk gets about the same share of
  // level-3 and near-zone work in every round. With consecutive lines per round, the lines
  // of a round lie next to one or two sub-chunks and the other warps wait at the barrier.
  const int n_in = max(0, rng.y - rng.x);
  const int n_rounds = (n_in + (int)blockDim.x - 1) / (int)blockDim.x;
  LineF32 nxt;
  if (tid * n_rounds < n_in) nxt = lp[rng.x + tid * n_rounds];

  for (int r = 0; r < n_rounds; ++r) {
    MlStage& S = s_stage[r & 1];
    float4* const s_g = S.g;
    float4* const s_h = S.h;
    float4* const s_p = S.p;
    float4* const s_q = S.q;
    short4* const s_nr = S.nr;
    unsigned short* const s_cls = S.cls;
    const LineF32 L = nxt;
    const int k = tid * n_rounds + r;
    const bool have = k < n_in;
    if (r + 1 < n_rounds && k + 1 < n_in) nxt = lp[rng.x + k + 1];
    const bool pass = have && (L.nuc >= wlo) && (L.nuc <= whi);
    const float jf = (float)(L.j0 - c0i);           // |j0 - c0| < 1.5e9 (grid index span check)
    const float d1 = fabsf(jf - C1) - H1;
    const bool lev1 = pass && use_l1 && (d1 > H1 + 1.f);   // tau_far_kernel's line
    const bool inner = pass && !lev1;
    // class of the line for every warp's sub-chunk
    unsigned cls = 0u;
    bool any3 = false;
    if (inner) {
      for (int w = 0; w < n_warps; ++w) {
        const int nw = min(ML_WARP_PTS, n_c - (first_sub + w) * ML_WARP_PTS);
        if (nw <= 0) break;
        const float h2 = 0.5f * (float)(nw - 1);
        const float d = fabsf(jf - ((float)((first_sub + w) * ML_WARP_PTS) + h2)) - h2;
        unsigned c = 1u;
        if (h2 >= ML_MIN_H2 && d > h2 + 1.f) c = d > ML_FAR1 * h2 ? 3u : 2u;
        any3 |= c == 1u;
        cls |= c << (2 * w);
      }
    }
    // near range (points with possibly |z|^2 < MID_Z2) of an inner line, clipped to the
    // chunk, and its middle, where |z|^2 may be below CORE_Z2 (one point of margin each;
    // every item still picks its formula from its own |z|^2)
    const float y2 = L.y * L.y;
    int near_lo = 0, near_n = 0, mid_lo = 0, mid_n = 0;
    if (inner && any3 && !(y2 >= MID_Z2 && L.y >= 0.f)) {
      const float hw = sqrtf(fmaxf(MID_Z2 - y2, 0.f)) / L.a + 1.0f;
      const float q = jf + L.b / L.a;                       // centre in points
      const float lo_f = fmaxf(ceilf(q - hw), 0.f);
      const float hi_f = fminf(floorf(q + hw), (float)(n_c - 1));
      if (lo_f <= hi_f) {
        near_lo = (int)lo_f;
        near_n = (int)hi_f - near_lo + 1;
        if (y2 < CORE_Z2 && L.y >= 0.f) {
          const float hw36 = sqrtf(CORE_Z2 - y2) / L.a + 1.0f;
          const float a0 = fmaxf(ceilf(q - hw36), (float)near_lo);           // clamped before the
          const float a1 = fminf(floorf(q + hw36), (float)(near_lo + near_n - 1));   // int conversion
          if (a0 <= a1) {
            mid_lo = (int)a0;
            mid_n = (int)a1 - mid_lo + 1;
          }
        }
      }
    }
    // every thread owns slot tid of this round's buffer; a line that is not inner leaves
    // class 0 there, so no warp lists it
    const int n2 = blockDim.x;
    s_cls[tid] = inner ? (unsigned short)cls : (unsigned short)0;
    if (inner) {
      const int slot = tid;
      float4 p, q;
      asym5_line_coeffs(y2, L.amp_far, p, q);
      const float rc = clamped_r(0.f, y2);                      // = rcp(MID_Z2) when y2 < MID_Z2
      s_g[slot] = make_float4(jf, L.a, L.b, L.amp_far);
      s_h[slot] = make_float4(L.y, y2, L.amp, rc * asym5_poly(rc, L.amp_far, p, q));
      s_p[slot] = p;
      s_q[slot] = q;
      s_nr[slot] = make_short4((short)near_lo, (short)near_n, (short)mid_lo, (short)mid_n);
    }
    // One barrier per round: this round's buffer was last read two rounds ago, and every
    // warp finished that round before it reached the previous round's barrier.
    __syncthreads();
    n_pass += (unsigned long long)__popc(__ballot_sync(FULL_MASK, inner));   // this warp's lines

    // ---- this warp's lists: level 2 (16 nodes from the front, 8 from the back), level 3
    int n2w = 0, n2fw = 0, n3w = 0;
    for (int k = 0; k < n2; k += 32) {
      const int l = k + lane;
      const unsigned c = l < n2 ? ((unsigned)s_cls[l] >> (2 * warp)) & 3u : 0u;
      const unsigned q3 = __ballot_sync(FULL_MASK, c == 1u), q2 = __ballot_sync(FULL_MASK, c == 2u);
      const unsigned q2f = __ballot_sync(FULL_MASK, c == 3u);
      const unsigned lt = (1u << lane) - 1u;
      if (c == 2u) s_l2[warp][n2w + __popc(q2 & lt)] = (unsigned char)l;
      if (c == 3u) s_l2[warp][ST - 1 - (n2fw + __popc(q2f & lt))] = (unsigned char)l;
      if (c == 1u) s_l3[warp][n3w + __popc(q3 & lt)] = (unsigned char)l;
      n2w += __popc(q2);
      n2fw += __popc(q2f);
      n3w += __popc(q3);
    }
    __syncwarp();

    // ---- level 2, one lane per line; node sums reduced once per round
    if (n2w > 0) {
      float f[ML_K];
#pragma unroll
      for (int k = 0; k < ML_K; ++k) f[k] = 0.f;
      level2_lines<ML_K>(f, s_l2[warp], 1, n2w, s_g, s_h, s_p, s_q, C2w, H2, lane);
      const float v = reduce16_transposed(f, lane);
      if (!(lane & 1)) s_n2[warp][(lane >> 1) & 15] += (double)v;
    }
    if (n2fw > 0) {
      float f[ML_KF];
#pragma unroll
      for (int k = 0; k < ML_KF; ++k) f[k] = 0.f;
      level2_lines<ML_KF>(f, &s_l2[warp][ST - 1], -1, n2fw, s_g, s_h, s_p, s_q, C2w, H2, lane);
      const float v = reduce8_transposed(f, lane);
      if (!(lane & 3)) s_n2[warp][ML_K + ((lane >> 2) & 7)] += (double)v;
    }
    if (lane == 0) n_nodes += (unsigned long long)n2w * ML_K + (unsigned long long)n2fw * ML_KF;

    // ---- level 3: every point of the warp. A sub-chunk of at most P points (the one-point
    // tile at the end of a grid) lets each lane take its own lines at lane 0's points
    // instead; the lanes' sums are added after the last round.
    const float xw_lo = (float)w0, xw_hi = (float)(w0 + n_w - 1);
    auto level3_line = [&](int i, float pl0) {
      const int l = s_l3[warp][i];
      const float4 g = s_g[l], h = s_h[l];
      const float x0 = fmaf(pl0 - g.x, g.y, -g.z);
      // |x| at the sub-chunk point nearest to the line centre (0 if it lies inside)
      const float xmin = fmaxf(fmaxf(fmaf(xw_lo - g.x, g.y, -g.z), -fmaf(xw_hi - g.x, g.y, -g.z)), 0.f);
      if (h.x >= 0.f && fmaf(xmin, xmin, h.y) >= FAR_Z2) {        // far from every point: two terms
        const float ny2 = -2.0f * h.y;
#pragma unroll
        for (int m = 0; m < P; ++m) far_wing_add(acc[m], fmaf((float)m, g.y, x0), h.y, ny2, g.w);
      } else {                                                    // |z|^2 clamped to >= MID_Z2
        const float4 p = s_p[l], q = s_q[l];
#pragma unroll
        for (int m = 0; m < P; ++m) {
          const float r = clamped_r(fmaf((float)m, g.y, x0), h.y);
          acc[m] = fmaf(r, asym5_poly(r, g.w, p, q), acc[m]);
        }
      }
    };
    {
      const bool few = n_w <= P;                      // warp-uniform
      const float pl0 = few ? (float)w0 : pf;
      for (int i = few ? lane : 0; i < n3w; i += few ? 32 : 1) level3_line(i, pl0);
    }
    if (lane == 0) n_l3 += (unsigned long long)n3w * n_w;

    // ---- near zones of the warp's level-3 lines inside its points, 32 lines at a time
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
      int mo = mn, to = tn;                             // inclusive scans, then exclusive offsets
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(FULL_MASK, mo, o), w = __shfl_up_sync(FULL_MASK, to, o);
        if (lane >= o) {
          mo += u;
          to += w;
        }
      }
      const int M = __shfl_sync(FULL_MASK, mo, 31), T = __shfl_sync(FULL_MASK, to, 31);
      mo -= mn;
      to -= tn;
      // item t of a space lies in the run of the last lane whose offset is <= t
      auto owner = [&](int off, int t) {
        int o = 0;
#pragma unroll
        for (int s = 16; s >= 1; s >>= 1)
          if (__shfl_sync(FULL_MASK, off, o + s) <= t) o += s;
        return o;
      };
      // point of item t of the middles (mid) or tails space, and the item's line slot
      auto locate = [&](bool mid, int t, int& p, int& sl) {
        const int o = owner(mid ? mo : to, t);
        const int k = t - __shfl_sync(FULL_MASK, mid ? mo : to, o);
        const int m_lo = __shfl_sync(FULL_MASK, mlo, o), t_lo = __shfl_sync(FULL_MASK, lo, o);
        const int t_ln = __shfl_sync(FULL_MASK, ln, o), t_hi = __shfl_sync(FULL_MASK, mhi, o);
        sl = __shfl_sync(FULL_MASK, slot, o);
        p = mid ? m_lo + k : (k < t_ln ? t_lo + k : t_hi + (k - t_ln));
      };
      if constexpr (!DET) {
        // values added by shared-memory atomics: overlapping near zones of two lines in one
        // 32-item step meet at a point in an order the hardware picks (~1e-9 relative)
        for (int pass_mid = 1; pass_mid >= 0; --pass_mid) {
          const bool mid = pass_mid;
          const int total = mid ? M : T;
          for (int it0 = 0; it0 < total; it0 += 32) {
            const int t = min(it0 + lane, total - 1);
            int p, sl;
            locate(mid, t, p, sl);
            if (it0 + lane < total) {
              const float v = mid ? near_correction<true>(p, s_g[sl], s_h[sl])
                                  : near_correction<false>(p, s_g[sl], s_h[sl]);
              if (v != 0.f) atomicAdd(&s_core[p - p0], v);
            }
          }
        }
      } else {
        // bit-reproducible: values go through a buffer; then the lines add theirs in
        // list order, middles before tails, each line's points spread over the lanes
        for (int pass_mid = 1; pass_mid >= 0; --pass_mid) {
          const bool mid = pass_mid;
          const int total = mid ? M : T;
          for (int b0 = 0; b0 < total; b0 += ML_NBW) {
            const int b1 = min(total, b0 + ML_NBW);
            for (int it0 = b0; it0 < b1; it0 += 32) {
              const int t = min(it0 + lane, b1 - 1);
              int p, sl;
              locate(mid, t, p, sl);
              if (it0 + lane < b1)
                s_nbuf[warp][t - b0] = mid ? near_correction<true>(p, s_g[sl], s_h[sl])
                                           : near_correction<false>(p, s_g[sl], s_h[sl]);
            }
            __syncwarp();
            // only the lines whose items fall in [b0, b1): from the owner of b0 to that of b1 - 1
            const int j_hi = owner(mid ? mo : to, b1 - 1);
            for (int jl = owner(mid ? mo : to, b0); jl <= j_hi; ++jl) {
              const int st = __shfl_sync(FULL_MASK, mid ? mo : to, jl), n = __shfl_sync(FULL_MASK, mid ? mn : tn, jl);
              const int m_lo = __shfl_sync(FULL_MASK, mlo, jl), t_lo = __shfl_sync(FULL_MASK, lo, jl);
              const int t_ln = __shfl_sync(FULL_MASK, ln, jl), t_hi = __shfl_sync(FULL_MASK, mhi, jl);
              const int ia = max(st, b0), ib = min(st + n, b1);
              for (int it = ia + lane; it < ib; it += 32) {
                const int k = it - st;
                const int p = mid ? m_lo + k : (k < t_ln ? t_lo + k : t_hi + (k - t_ln));
                s_core[p - p0] += s_nbuf[warp][it - b0];
              }
              __syncwarp();
            }
          }
        }
      }
      if (lane == 0) n_near_items += (unsigned long long)(M + T);
    }
    // No barrier here: the next round stages into the other buffer.
  }
  __syncthreads();                                  // s_c1 visible even when no round ran
  if (n_w <= P) {                                   // lanes' level-3 sums at lane 0's points
#pragma unroll
    for (int m = 0; m < P; ++m)
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) acc[m] += __shfl_xor_sync(FULL_MASK, acc[m], o);
  }

  // ---- one Chebyshev series per sub-chunk: level-2 node sums + the 8-node interpolant
  // + the level-1 series, at the 16 nodes, transformed back to coefficients
  const float inv_h1 = use_l1 ? 1.0f / H1 : 0.f, inv_h2 = use_l2 ? 1.0f / H2 : 0.f;
  float cw[ML_K];
#pragma unroll
  for (int k = 0; k < ML_K; ++k) cw[k] = 0.f;
  if (use_l2) {
    double c8 = 0.0;
    if (lane < ML_KF) {
      for (int j = 0; j < ML_KF; ++j) c8 += s_n2[warp][ML_K + j] * c_dct8[lane * ML_KF + j];
      c8 *= 2.0 / ML_KF;
    }
    float c8f[ML_KF];
#pragma unroll
    for (int k = 0; k < ML_KF; ++k) c8f[k] = (float)__shfl_sync(FULL_MASK, c8, k);
    const int jn = lane & 15;
    const float tj = c_node16[jn];
    double fj = s_n2[warp][jn] + (double)clenshaw16<ML_KF>(c8f, tj);
    if (use_l1) {
      const float t1 = fmaf(H2, tj, C2w - C1) * inv_h1;
      fj += (double)(clenshaw16(s_c1, t1) + clenshaw16<ML_KF>(s_c1 + ML_K, t1));
    }
    double ck = 0.0;
#pragma unroll
    for (int j = 0; j < ML_K; ++j) ck += __shfl_sync(FULL_MASK, fj, j) * c_dct16[jn * ML_K + j];
    ck *= 2.0 / ML_K;
#pragma unroll
    for (int k = 0; k < ML_K; ++k) cw[k] = (float)__shfl_sync(FULL_MASK, ck, k);
  }
  __syncwarp();

  const double T = t_layer[row];
  const float half_c2_t = (float)(0.5 * C2 / T);
  float* out = od + (long long)row * out_stride;   // points [out_first, out_first + out_stride) of the grid
  bool bad = false;
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const int pl = w0 + lane * P + m;
    if (pl < n_c) {
      const long long p = c0 + pl;
      float v = s_core[pl - p0];
      if (use_l2) {
        v += clenshaw16(cw, ((float)pl - C2w) * inv_h2);
      } else if (use_l1) {
        const float t1 = ((float)pl - C1) * inv_h1;
        v += clenshaw16(s_c1, t1) + clenshaw16<ML_KF>(s_c1 + ML_K, t1);
      }
      const float nu = (float)grid_nu(nu_min, step, p);
      const float o = (acc[m] + v) * (nu * tanhf(nu * half_c2_t));   // R(nu, T) = nu tanh(c2 nu / 2T)
      bad |= !isfinite(o);
      out[p - out_first] = o;
    }
  }
  if (bad) flag_error(err, row * (n_grp + 1) + n_grp);
  if (lane == 0 && evals && n_pass)
    atomicAdd(evals, n_pass * (unsigned long long)(min(n_c, p0 + n_warps * ML_WARP_PTS) - p0));
  if (work) {   // work[0]: node evaluations, work[1]: level-3 loop evaluations, work[2]: near items
    if (n_nodes) atomicAdd(&work[0], n_nodes);
    if (n_l3) atomicAdd(&work[1], n_l3);
    if (n_near_items) atomicAdd(&work[2], n_near_items);
  }
}

}  // namespace lbl

using namespace lbl;

extern "C" int lbl_ml_inner_ranges(const LineIn* lines, const int* n_kept, double nu_min, double step, long long n_nu,
                                   int tile_samples, double pad, int n_tiles, int* inner, void* stream) {
  if (tile_samples < 1 || !(step > 0))
    return lbl_set_error(LBL_EINVAL, "lbl_ml_inner_ranges: bad arguments");
  // A line is inner for a chunk of n_c points (half-width H = (n_c - 1) / 2) when its
  // grid index j0 = rint((nuc - nu_min) / step) lies within H + 1 points of the chunk,
  // so nuc lies within (H + 1.5) steps of it; chunks lie inside their tile and have at
  // most min(tile_samples, chunk size) points. Two further steps absorb rounding.
  const int per_tile = tile_samples < ML_CHUNK ? tile_samples : ML_CHUNK;
  const int cp = 32 * ((per_tile + ML_WARP_PTS - 1) / ML_WARP_PTS) * ML_P;
  const int n_c_max = tile_samples < cp ? tile_samples : cp;
  const double reach = (0.5 * (n_c_max - 1) + 3.5) * step;
  return lbl_tile_ranges(lines, n_kept, nu_min, step, n_nu, tile_samples, reach, pad, n_tiles, inner, stream);
}

static void ml_geometry(int tile_samples, int* threads, int* cp, long long* chunks) {
  const int per_tile = tile_samples < ML_CHUNK ? tile_samples : ML_CHUNK;
  *threads = 32 * ((per_tile + ML_WARP_PTS - 1) / ML_WARP_PTS);
  *cp = *threads * ML_P;
  *chunks = (tile_samples + *cp - 1) / *cp;
}

extern "C" long long lbl_ml_work_floats(int n_rows, int tile_samples, int tile_count) {
  if (n_rows < 1 || tile_samples < 1 || tile_count < 1) return -1;
  int threads, cp;
  long long chunks;
  ml_geometry(tile_samples, &threads, &cp, &chunks);
  return (long long)n_rows * tile_count * chunks * (ML_K + ML_KF);
}

extern "C" int lbl_tau_tiles_ml_f32(const LineF32* prep, int n_lines, const int* ranges, const int* inner,
                                    float* l1_work, const double* t_layer, int n_rows, double nu_min, double step,
                                    long long n_nu, int tile_samples, double cutoff, int n_grp, float* od, int* err,
                                    unsigned long long* evals, unsigned long long* work, int tile_first,
                                    int tile_count, int flags, void* stream) {
  if (!prep || !ranges || !t_layer || !od || !l1_work || n_lines < 1 || n_rows < 1 || n_rows > 65535 || n_nu < 1 ||
      n_nu > 1500000000LL || tile_samples < 1 || !(step > 0) || !(cutoff >= 0) || n_grp < 1)
    return lbl_set_error(LBL_EINVAL, "lbl_tau_tiles_ml_f32: bad arguments");
  const long long n_all = (n_nu + tile_samples - 1) / tile_samples;
  if (tile_first < 0 || tile_count < 1 || (long long)tile_first + tile_count > n_all)
    return lbl_set_error(LBL_EINVAL, "lbl_tau_tiles_ml_f32: tile range outside the grid");
  const long long out_first = (long long)tile_first * tile_samples;
  const long long out_end = (long long)(tile_first + tile_count) * tile_samples < n_nu
                                ? (long long)(tile_first + tile_count) * tile_samples : n_nu;
  int threads, cp;
  long long chunks;
  ml_geometry(tile_samples, &threads, &cp, &chunks);
  const long long n_tiles = tile_count;
  const int subs = threads / 32, parts = (subs + ML_CTA_SUBS - 1) / ML_CTA_SUBS;
  const int cta_threads = 32 * (subs < ML_CTA_SUBS ? subs : ML_CTA_SUBS);
  if (n_tiles * chunks * parts > 0x7fffffffLL) return lbl_set_error(LBL_EINVAL, "lbl_tau_tiles_ml_f32: grid too large");
  dim3 grid_far((unsigned)(n_tiles * chunks), (unsigned)n_rows);
  cudaStream_t st = (cudaStream_t)stream;
  tau_far_kernel<<<grid_far, MF_THREADS, 0, st>>>(prep, n_lines, (const int2*)ranges, nu_min, step, n_nu, tile_samples,
                                                   (int)chunks, cp, cutoff, l1_work, evals, work, tile_first);
  dim3 grid((unsigned)(n_tiles * chunks * parts), (unsigned)n_rows);
  // the staging buffers take the kernel past 48 KB of shared memory: opt in (per call, so
  // that every device and context the caller uses gets it; a host-side attribute write)
  {
    const void* fn = (flags & LBL_DETERMINISTIC) ? (const void*)tau_ml_kernel<true> : (const void*)tau_ml_kernel<false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ML_STAGE_BYTES);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return lbl_set_error(LBL_ECUDA, "lbl_tau_tiles_ml_f32 (shared-memory attributes): %s", cudaGetErrorString(e));
    }
  }
  if (flags & LBL_DETERMINISTIC)
    tau_ml_kernel<true><<<grid, cta_threads, ML_STAGE_BYTES, st>>>(prep, n_lines, (const int2*)ranges, (const int2*)inner, l1_work,
                                                      t_layer, nu_min, step, n_nu, tile_samples, (int)chunks, cp,
                                                      cutoff, n_grp, od, err, evals, work, tile_first, out_first,
                                                      out_end - out_first);
  else
    tau_ml_kernel<false><<<grid, cta_threads, ML_STAGE_BYTES, st>>>(prep, n_lines, (const int2*)ranges, (const int2*)inner, l1_work,
                                                       t_layer, nu_min, step, n_nu, tile_samples, (int)chunks, cp,
                                                       cutoff, n_grp, od, err, evals, work, tile_first, out_first,
                                                       out_end - out_first);
  return lbl_check_launch("lbl_tau_tiles_ml_f32");
}
