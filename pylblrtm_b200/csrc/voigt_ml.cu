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
//           six half-widths out use 8 nodes). A separate kernel (tau_far_kernel)
//           computes this level and hands its coefficients over through od;
//  level 2  the other lines farther than one sub-chunk half-width from a warp's
//           256-point sub-chunk: 16 Chebyshev nodes per sub-chunk, same geometry
//           (8 beyond six sub-chunk half-widths);
//  level 3  the remaining lines: direct evaluation at every point. The warp's
//           loop is branch-free: it evaluates the five-term asymptotic form with
//           |z|^2 clamped to >= MID_Z2 = 64, so every point inside a line's near
//           zone receives the same constant. A CTA-wide near pass then gives each
//           near point (accurate value - that constant): float continued fraction
//           for 36 <= |z|^2 < 64, Weideman's float64 approximation below.
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
constexpr float ML_FAR1 = 5.f;                 // "far": more than (1 + ML_FAR1) half-widths from the centre
constexpr float ML_MIN_H1 = 32.f;              // smallest chunk half-width (points) using level 1
constexpr float ML_MIN_H2 = 16.f;              // smallest sub-chunk half-width using level 2
constexpr int ML_NB = 2048;                    // near items buffered per batch

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
// takes one line and evaluates it at all nodes from registers (no shared-memory
// staging, no barriers). The kernel leaves the chunk's 16 + 8 Chebyshev coefficients
// in the first 24 floats of the chunk's own od slice (level 1 needs >= 65 points);
// tau_ml_kernel reads them before it writes the slice.
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
               float* __restrict__ od, unsigned long long* evals, unsigned long long* work, int tile_first,
               long long out_first, long long out_stride) {
  __shared__ __align__(16) LineF32 s_line[MF_STAGES][MF_THREADS];   // records are 32 B, 16-B aligned
  __shared__ double s_part[MF_THREADS / 32][ML_K + ML_KF];
  __shared__ float s_coef[ML_K + ML_KF];
  __shared__ unsigned s_cnt[2];

  const int row = blockIdx.y;
  const int tile = tile_first + (int)(blockIdx.x / chunks_per_tile), chunk = blockIdx.x % chunks_per_tile;
  const long long t0 = (long long)tile * tile_samples;
  const long long t1 = min(t0 + (long long)tile_samples, n_nu);
  const long long c0 = t0 + (long long)chunk * chunk_pts;
  if (c0 >= t1) return;
  const int n_c = (int)(min(c0 + (long long)chunk_pts, t1) - c0);
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
  if (tid < ML_K + ML_KF) od[(long long)row * out_stride + (c0 - out_first) + tid] = s_coef[tid];
  if (tid == 0) {
    const unsigned long long a = s_cnt[0], b = s_cnt[1];
    if (evals && a + b) atomicAdd(evals, (a + b) * (unsigned long long)n_c);
    if (work && a + b) atomicAdd(&work[0], a * ML_K + b * ML_KF);
  }
}

template <bool DET>
__global__ void __launch_bounds__(ML_THREADS, 4)
tau_ml_kernel(const LineF32* __restrict__ prep, int n_lines, const int2* __restrict__ ranges,
              const int2* __restrict__ inner_ranges, const double* __restrict__ t_layer, double nu_min,
              double step, long long n_nu, int tile_samples, int chunks_per_tile, double cutoff, int n_grp,
              float* __restrict__ od, int* err, unsigned long long* evals, unsigned long long* work,
              int tile_first, long long out_first, long long out_stride) {
  constexpr int P = ML_P;
  __shared__ MlLine s2[ML_THREADS];                 // inner lines of the round
  __shared__ unsigned char s_l2[ML_THREADS / 32][ML_THREADS];   // per-warp level-2 slots
  __shared__ unsigned char s_l3[ML_THREADS / 32][ML_THREADS];   // per-warp level-3 slots
  __shared__ unsigned char s_nl[ML_THREADS / 32][ML_THREADS];   // per-warp slots with near points in it
  __shared__ int s_cnt[3][ML_THREADS / 32];
  __shared__ int s_seg_start[ML_THREADS + 1];       // near-item prefix per inner slot (default: middles)
  __shared__ short s_seg_lo[ML_THREADS];            // first near point per inner slot (default: of the middle)
  // default mode: the near zone of a slot is split into its middle (|z|^2 < CORE_Z2, the
  // float64 core) and its two tails (the float continued fraction), each kind in an item
  // space of its own, so that a warp's consecutive items take the same branch
  __shared__ int s_segc_start[ML_THREADS + 1];      // tail-item prefix per inner slot
  __shared__ short s_segc_lo[ML_THREADS];           // first point of the left tail
  __shared__ short s_segc_nl[ML_THREADS];           // points in the left tail
  __shared__ short s_segc_rlo[ML_THREADS];          // first point of the right tail
  __shared__ unsigned char s_seg_mask[ML_THREADS];  // warps treating the inner line directly (level 3)
  __shared__ float s_core[ML_CHUNK];               // near-zone corrections (each point owned by one thread)
  __shared__ float s_nbuf[ML_NB];                   // near-item values of one batch
  __shared__ float s_c1[ML_K + ML_KF];              // level-1 coefficients from tau_far_kernel
  __shared__ float s_c2[ML_THREADS / 32][ML_K];
  __shared__ float s_c2f[ML_THREADS / 32][ML_KF];

  const int row = blockIdx.y;
  const int tile = tile_first + (int)(blockIdx.x / chunks_per_tile), chunk = blockIdx.x % chunks_per_tile;
  const long long t0 = (long long)tile * tile_samples;
  const long long t1 = min(t0 + (long long)tile_samples, n_nu);
  const long long c0 = t0 + (long long)chunk * (blockDim.x * P);
  if (c0 >= t1) return;
  const int n_c = (int)(min(c0 + (long long)(blockDim.x * P), t1) - c0);
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
  const int w0 = warp * ML_WARP_PTS;
  const int n_w = max(0, min(ML_WARP_PTS, n_c - w0));
  const float H2 = 0.5f * (float)(n_w - 1), C2w = (float)w0 + H2;
  const bool use_l2 = H2 >= ML_MIN_H2;
  // level-2 Chebyshev nodes owned by this lane: (lane & 15), and (lane & 7) of the 8-node set
  const float xn2 = H2 * c_node16[lane & 15];
  const float xn2f = H2 * c_node8[lane & 7];
  const float pf = (float)(w0 + lane * P);                   // this lane's first point

  for (int i = tid; i < ML_CHUNK; i += blockDim.x) s_core[i] = 0.f;
  // read before the first barrier; this CTA writes the slice only after the last one
  if (use_l1 && tid < ML_K + ML_KF) s_c1[tid] = od[(long long)row * out_stride + (c0 - out_first) + tid];

  // level-3 sums hold only the lines within ~2 sub-chunk widths (tens of terms), so
  // plain float accumulation suffices; the 16-node level-2 sums are Kahan-compensated
  // across rounds, the 8-node ones (far lines, smaller terms) are plain float.
  float acc[P];
#pragma unroll
  for (int m = 0; m < P; ++m) acc[m] = 0.f;
  float sum2 = 0.f, comp2 = 0.f, sum2f = 0.f;
  unsigned long long n_pass = 0, n_nodes = 0, n_l3 = 0, n_near_items = 0;

  // register prefetch of the next round's line records
  LineF32 nxt;
  int li = rng.x + tid;
  if (li < rng.y) nxt = lp[li];

  for (int base = rng.x; base < rng.y; base += blockDim.x) {
    const LineF32 L = nxt;
    const bool have = base + tid < rng.y;
    if (base + blockDim.x + tid < rng.y) nxt = lp[base + blockDim.x + tid];
    const bool pass = have && (L.nuc >= wlo) && (L.nuc <= whi);
    const float jf = (float)(L.j0 - c0i);           // |j0 - c0| < 1.5e9 (grid index span check)
    const float d1 = fabsf(jf - C1) - H1;
    const bool lev1 = pass && use_l1 && (d1 > H1 + 1.f);   // tau_far_kernel's line
    const bool inner = pass && !lev1;
    // near range (points with possibly |z|^2 < MID_Z2) of an inner line, clipped to the chunk
    const float y2 = L.y * L.y;
    float hw = -1.0f;                               // near half-width in points (inner lines only)
    if (inner && !(y2 >= MID_Z2 && L.y >= 0.f)) hw = sqrtf(fmaxf(MID_Z2 - y2, 0.f)) / L.a + 1.0f;
    int near_lo = 0, near_n = 0;
    unsigned l3mask = 0;
    if (inner) {
      for (int w = 0; w < n_warps; ++w) {             // same test as the per-warp split below
        const int nw = min(ML_WARP_PTS, n_c - w * ML_WARP_PTS);
        if (nw <= 0) break;
        const float h2 = 0.5f * (float)(nw - 1);
        const bool l2 = h2 >= ML_MIN_H2 && fabsf(jf - ((float)(w * ML_WARP_PTS) + h2)) - h2 > h2 + 1.f;
        if (!l2) l3mask |= 1u << w;
      }
    }
    if (inner && hw >= 0.f && l3mask) {
      const float q = jf + L.b / L.a;                       // centre in points
      const float lo_f = fmaxf(ceilf(q - hw), 0.f);
      const float hi_f = fminf(floorf(q + hw), (float)(n_c - 1));
      if (lo_f <= hi_f) {
        near_lo = (int)lo_f;
        near_n = (int)hi_f - near_lo + 1;
      }
    }
    // default mode: the middle [mid_lo, mid_lo + mid_n) of the near range, where |z|^2 may be
    // below CORE_Z2 (one point of margin; each item still picks its formula from its own |z|^2)
    int mid_lo = near_lo, mid_n = 0;
    if constexpr (!DET) {
      if (near_n > 0 && y2 < CORE_Z2 && L.y >= 0.f) {
        const float hw36 = sqrtf(CORE_Z2 - y2) / L.a + 1.0f;
        const float q = jf + L.b / L.a;
        const float a0 = fmaxf(ceilf(q - hw36), (float)near_lo);           // clamped before the
        const float a1 = fminf(floorf(q + hw36), (float)(near_lo + near_n - 1));   // int conversion
        if (a0 <= a1) {
          mid_lo = (int)a0;
          mid_n = (int)a1 - mid_lo + 1;
        }
      }
    }
    const int tail_n = near_n - mid_n;
    // inclusive warp scans: DET the whole near range; default the middles and the tails
    int near_scan = DET ? near_n : mid_n, tail_scan = tail_n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, near_scan, o);
      const int u = __shfl_up_sync(0xffffffffu, tail_scan, o);
      if (lane >= o) {
        near_scan += t;
        tail_scan += u;
      }
    }
    const unsigned b2 = __ballot_sync(0xffffffffu, inner);
    if (lane == 0) s_cnt[0][warp] = __popc(b2);
    if (lane == 31) {
      s_cnt[1][warp] = near_scan;
      s_cnt[2][warp] = tail_scan;
    }
    __syncthreads();
    int off2 = 0, off3 = 0, offc = 0, n2 = 0, n_near = 0, n_tail = 0;
    for (int w = 0; w < n_warps; ++w) {
      const int a2 = s_cnt[0][w], a3 = s_cnt[1][w], a4 = s_cnt[2][w];
      off2 += (w < warp) ? a2 : 0;
      off3 += (w < warp) ? a3 : 0;
      offc += (w < warp) ? a4 : 0;
      n2 += a2;
      n_near += a3;
      n_tail += a4;
    }
    if (inner) {
      MlLine r;
      r.g = make_float4(jf, L.a, L.b, L.amp_far);
      asym5_line_coeffs(y2, L.amp_far, r.p, r.q);
      const float rc = clamped_r(0.f, y2);                      // = rcp(MID_Z2) when y2 < MID_Z2
      r.h = make_float4(L.y, y2, L.amp, rc * asym5_scaled(rc, r));
      const int slot = off2 + __popc(b2 & ((1u << lane) - 1u));
      s2[slot] = r;
      s_seg_mask[slot] = (unsigned char)l3mask;
      if constexpr (DET) {
        s_seg_start[slot] = off3 + near_scan - near_n;       // exclusive prefix in slot order
        s_seg_lo[slot] = (short)near_lo;
      } else {
        s_seg_start[slot] = off3 + near_scan - mid_n;
        s_seg_lo[slot] = (short)mid_lo;
        s_segc_start[slot] = offc + tail_scan - tail_n;
        s_segc_lo[slot] = (short)near_lo;
        s_segc_nl[slot] = (short)(mid_n > 0 ? mid_lo - near_lo : tail_n);
        s_segc_rlo[slot] = (short)(mid_lo + mid_n);
      }
    }
    if (tid == 0) {
      s_seg_start[n2] = n_near;
      if constexpr (!DET) s_segc_start[n2] = n_tail;
    }
    __syncthreads();
    n_pass += (unsigned long long)n2;

    // ---- per-warp split of the inner lines into level 2 (16 nodes; 8 beyond six
    // sub-chunk half-widths, listed from the back of s_l2) and level 3
    int n2w = 0, n2fw = 0, n3w = 0, nnw = 0;
    for (int k = 0; k < n2; k += 32) {
      const int l = k + lane;
      bool is2 = false, is2f = false, is3 = false, nz = false;
      if (l < n2) {
        const float d = fabsf(s2[l].g.x - C2w) - H2;
        const bool lev2 = use_l2 && d > H2 + 1.f;
        is2f = lev2 && d > ML_FAR1 * H2;
        is2 = lev2 && !is2f;
        is3 = !lev2 && n_w > 0;
        if constexpr (DET) {   // near points of slot l inside this warp's sub-chunk (level 3 here)
          const int st = s_seg_start[l], len = s_seg_start[l + 1] - st, lo = s_seg_lo[l];
          nz = len > 0 && ((s_seg_mask[l] >> warp) & 1u) && lo < w0 + n_w && lo + len > w0;
        }
      }
      const unsigned q2 = __ballot_sync(0xffffffffu, is2), q3 = __ballot_sync(0xffffffffu, is3);
      const unsigned q2f = __ballot_sync(0xffffffffu, is2f);
      const unsigned lt = (1u << lane) - 1u;
      if (is2) s_l2[warp][n2w + __popc(q2 & lt)] = (unsigned char)l;
      if (is2f) s_l2[warp][ML_THREADS - 1 - (n2fw + __popc(q2f & lt))] = (unsigned char)l;
      if (is3) s_l3[warp][n3w + __popc(q3 & lt)] = (unsigned char)l;
      n2w += __popc(q2);
      n2fw += __popc(q2f);
      n3w += __popc(q3);
      if constexpr (DET) {
        const unsigned qn = __ballot_sync(0xffffffffu, nz);
        if (nz) s_nl[warp][nnw + __popc(qn & lt)] = (unsigned char)l;
        nnw += __popc(qn);
      }
    }
    __syncwarp();

    // ---- level 2: half-warps take one line each, lane (& 15) = node
    {
      float a2 = 0.f;
      for (int i = lane >> 4; i < n2w; i += 2) {
        const MlLine R = s2[s_l2[warp][i]];
        const float e = C2w - R.g.x;                          // exact: half-integer minus integer
        const float x = fmaf(xn2 + e, R.g.y, -R.g.z);
        a2 += line_value(x, R);
      }
      kahan_add(sum2, comp2, a2);
      // far level-2 lines: quarter-warps take one line each, lane (& 7) = node
      for (int i = lane >> 3; i < n2fw; i += 4) {
        const MlLine R = s2[s_l2[warp][ML_THREADS - 1 - i]];
        const float x = fmaf(xn2f + (C2w - R.g.x), R.g.y, -R.g.z);
        sum2f += line_value(x, R);
      }
      if (lane == 0) n_nodes += (unsigned long long)n2w * ML_K + (unsigned long long)n2fw * ML_KF;
    }

    // ---- level 3, far part: every point of the warp, |z|^2 clamped (branch-free)
    for (int i = 0; i < n3w; ++i) {
      const MlLine R = s2[s_l3[warp][i]];
      const float x0 = fmaf(pf - R.g.x, R.g.y, -R.g.z);
#pragma unroll
      for (int m = 0; m < P; ++m) {
        const float r = clamped_r(fmaf((float)m, R.g.y, x0), R.h.y);
        acc[m] = fmaf(r, asym5_scaled(r, R), acc[m]);
      }
    }
    if (lane == 0) n_l3 += (unsigned long long)n3w * n_w;
    // ---- level 3, near part, spread over the CTA: near item i is point
    // s_seg_lo[l] + (i - s_seg_start[l]) of inner line l. It gets (accurate value -
    // clamped loop value) if the line is level 3 for the warp owning the point and
    // |z|^2 < MID_Z2 there; x is formed exactly as in the loop, so the clamped value
    // cancels. Consecutive threads take consecutive points of a line. Where near
    // zones of several lines overlap, the shared-memory atomics add in scheduling
    // order (results reproducible to rounding, ~1e-9 relative).
    if constexpr (!DET) {
      auto near_item = [&](int l, int p) {
        if (!((s_seg_mask[l] >> (p >> 8)) & 1u)) return;   // level 2 for the owning warp
        const MlLine R = s2[l];
        const float x0 = fmaf((float)(p & ~(P - 1)) - R.g.x, R.g.y, -R.g.z);
        const float x = fmaf((float)(p & (P - 1)), R.g.y, x0);
        const float z2 = fmaf(x, x, R.h.y);
        if (z2 >= MID_Z2) return;
        float v;
        if (z2 >= CORE_Z2 && R.h.x >= 0.f) v = R.h.z * re_w_cf32(x, R.h.x, z2);
        else v = (float)((double)R.h.z * weideman_re_f32((double)x, (double)R.h.x));
        atomicAdd(&s_core[p], v - R.h.w);
      };
      // the middles (float64 core), then the tails (continued fraction)
      for (int i = tid; i < n_near; i += blockDim.x) {
        int l = 0, hi = n2;                               // largest l with s_seg_start[l] <= i
        while (hi - l > 1) {
          const int mid = (l + hi) >> 1;
          if (s_seg_start[mid] <= i) l = mid; else hi = mid;
        }
        near_item(l, s_seg_lo[l] + (i - s_seg_start[l]));
      }
      for (int i = tid; i < n_tail; i += blockDim.x) {
        int l = 0, hi = n2;                               // largest l with s_segc_start[l] <= i
        while (hi - l > 1) {
          const int mid = (l + hi) >> 1;
          if (s_segc_start[mid] <= i) l = mid; else hi = mid;
        }
        const int k = i - s_segc_start[l], nl = s_segc_nl[l];
        near_item(l, k < nl ? s_segc_lo[l] + k : s_segc_rlo[l] + (k - nl));
      }
    } else {
      // Bit-reproducible variant, in two phases so that the sums do not depend on thread
      // scheduling. Phase 1 spreads the near items over the CTA: item i is point
      // s_seg_lo[l] + (i - s_seg_start[l]) of inner line l; its value is (accurate value -
      // clamped loop value) if the line is level 3 for the warp owning the point and
      // |z|^2 < MID_Z2 there (x is formed exactly as in the loop, so the clamped value
      // cancels), else 0. Phase 2: every thread adds the values of its own points in slot
      // order. Items go through a buffer of ML_NB at a time.
      for (int nb0 = 0; nb0 < n_near; nb0 += ML_NB) {
        const int nb1 = min(n_near, nb0 + ML_NB);
        for (int i = nb0 + tid; i < nb1; i += blockDim.x) {
          int l = 0, hi = n2;                               // largest l with s_seg_start[l] <= i
          while (hi - l > 1) {
            const int mid = (l + hi) >> 1;
            if (s_seg_start[mid] <= i) l = mid; else hi = mid;
          }
          const int p = s_seg_lo[l] + (i - s_seg_start[l]);
          float v = 0.f;
          if ((s_seg_mask[l] >> (p >> 8)) & 1u) {            // level 3 for the owning warp
            const MlLine R = s2[l];
            const float x0 = fmaf((float)(p & ~(P - 1)) - R.g.x, R.g.y, -R.g.z);
            const float x = fmaf((float)(p & (P - 1)), R.g.y, x0);
            const float z2 = fmaf(x, x, R.h.y);
            if (z2 < MID_Z2) {
              if (z2 >= CORE_Z2 && R.h.x >= 0.f) v = R.h.z * re_w_cf32(x, R.h.x, z2);
              else v = (float)((double)R.h.z * weideman_re_f32((double)x, (double)R.h.x));
              v -= R.h.w;
            }
          }
          s_nbuf[i - nb0] = v;
        }
        __syncthreads();
        const int q0 = w0 + lane * P;                       // this thread's points [q0, q0 + P)
        for (int j = 0; j < nnw; ++j) {                     // slots with near points in this warp, in order
          const int l = s_nl[warp][j];
          const int st = s_seg_start[l], en = s_seg_start[l + 1];
          if (en <= nb0 || st >= nb1) continue;
          const int lo = s_seg_lo[l];
          const int pa = max(q0, lo + (max(st, nb0) - st)), pb = min(q0 + P, lo + (min(en, nb1) - st));
          for (int p = pa; p < pb; ++p) s_core[p] += s_nbuf[st + (p - lo) - nb0];
        }
        if (nb1 < n_near) __syncthreads();                  // the buffer is refilled
      }
    }
    if (tid == 0) n_near_items += (unsigned long long)(DET ? n_near : n_near + n_tail);
    // No barrier here: the next round writes the staging arrays only after its first
    // barrier, which every warp reaches after finishing this round.
  }
  __syncthreads();

  // ---- level-2 node values of this warp: lanes j and j+16 hold halves of node j
  {
    float f2 = sum2 - comp2;
    f2 += __shfl_xor_sync(0xffffffffu, f2, 16);
    double c = 0.0;
    for (int j = 0; j < ML_K; ++j) {
      const float fj = __shfl_sync(0xffffffffu, f2, j);
      c += (double)fj * c_dct16[(lane & 15) * ML_K + j];
    }
    if (lane < ML_K) s_c2[warp][lane] = use_l2 ? (float)(c * (2.0 / ML_K)) : 0.f;
    // 8-node set: lanes j, j+8, j+16, j+24 hold quarters of node j
    float g2 = sum2f;
    g2 += __shfl_xor_sync(0xffffffffu, g2, 16);
    g2 += __shfl_xor_sync(0xffffffffu, g2, 8);
    double cf = 0.0;
    for (int j = 0; j < ML_KF; ++j) {
      const float gj = __shfl_sync(0xffffffffu, g2, j);
      cf += (double)gj * c_dct8[(lane & 7) * ML_KF + j];
    }
    if (lane < ML_KF) s_c2f[warp][lane] = use_l2 ? (float)(cf * (2.0 / ML_KF)) : 0.f;
  }
  __syncthreads();

  const double T = t_layer[row];
  float* out = od + (long long)row * out_stride;   // points [out_first, out_first + out_stride) of the grid
  float c2[ML_K];
#pragma unroll
  for (int k = 0; k < ML_K; ++k) c2[k] = s_c2[warp][k];
  const float inv_h1 = use_l1 ? 1.0f / H1 : 0.f, inv_h2 = use_l2 ? 1.0f / H2 : 0.f;
  bool bad = false;
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const int pl = w0 + lane * P + m;
    if (pl < n_c) {
      const long long p = c0 + pl;
      float v = s_core[pl];
      if (use_l1) {
        const float t1 = ((float)pl - C1) * inv_h1;
        v += clenshaw16(s_c1, t1) + clenshaw16<ML_KF>(s_c1 + ML_K, t1);
      }
      if (use_l2) {
        const float t2 = ((float)pl - C2w) * inv_h2;
        v += clenshaw16(c2, t2) + clenshaw16<ML_KF>(s_c2f[warp], t2);
      }
      const double nu = grid_nu(nu_min, step, p);
      const float o = (float)(((double)acc[m] + (double)v) * radiation_term_grid(nu, T));
      bad |= !isfinite(o);
      out[p - out_first] = o;
    }
  }
  if (bad) flag_error(err, row * (n_grp + 1) + n_grp);
  if (tid == 0 && evals && n_pass) atomicAdd(evals, n_pass * (unsigned long long)n_c);
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

extern "C" int lbl_tau_tiles_ml_f32(const LineF32* prep, int n_lines, const int* ranges, const int* inner,
                                    const double* t_layer, int n_rows, double nu_min, double step, long long n_nu,
                                    int tile_samples, double cutoff, int n_grp, float* od, int* err,
                                    unsigned long long* evals, unsigned long long* work, int tile_first,
                                    int tile_count, int flags, void* stream) {
  if (!prep || !ranges || !t_layer || !od || n_lines < 1 || n_rows < 1 || n_rows > 65535 || n_nu < 1 ||
      n_nu > 1500000000LL || tile_samples < 1 || !(step > 0) || !(cutoff >= 0) || n_grp < 1)
    return lbl_set_error(LBL_EINVAL, "lbl_tau_tiles_ml_f32: bad arguments");
  const long long n_all = (n_nu + tile_samples - 1) / tile_samples;
  if (tile_first < 0 || tile_count < 1 || (long long)tile_first + tile_count > n_all)
    return lbl_set_error(LBL_EINVAL, "lbl_tau_tiles_ml_f32: tile range outside the grid");
  const long long out_first = (long long)tile_first * tile_samples;
  const long long out_end = (long long)(tile_first + tile_count) * tile_samples < n_nu
                                ? (long long)(tile_first + tile_count) * tile_samples : n_nu;
  const int per_tile = tile_samples < ML_CHUNK ? tile_samples : ML_CHUNK;
  const int threads = 32 * ((per_tile + ML_WARP_PTS - 1) / ML_WARP_PTS);
  const int cp = threads * ML_P;
  const long long n_tiles = tile_count;
  const long long chunks = (tile_samples + cp - 1) / cp;
  if (n_tiles * chunks > 0x7fffffffLL) return lbl_set_error(LBL_EINVAL, "lbl_tau_tiles_ml_f32: grid too large");
  dim3 grid((unsigned)(n_tiles * chunks), (unsigned)n_rows);
  cudaStream_t st = (cudaStream_t)stream;
  tau_far_kernel<<<grid, MF_THREADS, 0, st>>>(prep, n_lines, (const int2*)ranges, nu_min, step, n_nu, tile_samples,
                                               (int)chunks, cp, cutoff, od, evals, work, tile_first, out_first,
                                               out_end - out_first);
  if (flags & LBL_DETERMINISTIC)
    tau_ml_kernel<true><<<grid, threads, 0, st>>>(prep, n_lines, (const int2*)ranges, (const int2*)inner, t_layer,
                                                  nu_min, step, n_nu, tile_samples, (int)chunks, cutoff, n_grp, od,
                                                  err, evals, work, tile_first, out_first, out_end - out_first);
  else
    tau_ml_kernel<false><<<grid, threads, 0, st>>>(prep, n_lines, (const int2*)ranges, (const int2*)inner, t_layer,
                                                   nu_min, step, n_nu, tile_samples, (int)chunks, cutoff, n_grp, od,
                                                   err, evals, work, tile_first, out_first, out_end - out_first);
  return lbl_check_launch("lbl_tau_tiles_ml_f32");
}
