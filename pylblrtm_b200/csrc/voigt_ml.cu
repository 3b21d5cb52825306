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
//           (interpolation error ~rho^-16 ~ 1e-9 of the level-1 sum);
//  level 2  the other lines farther than one sub-chunk half-width from a warp's
//           256-point sub-chunk: 16 Chebyshev nodes per sub-chunk, same geometry;
//  level 3  the remaining lines: direct evaluation at every point. The warp's
//           loop is branch-free: it evaluates the five-term asymptotic form with
//           |z|^2 clamped to >= MID_Z2 = 64, so every point inside a line's near
//           zone receives the same constant. A CTA-wide near pass then gives each
//           near point (accurate value - that constant): float continued fraction
//           for 36 <= |z|^2 < 64, Weideman's float64 approximation below. Its values
//           are added per point in a fixed order, so results are bit-reproducible.
//
// Inside a reference tile the set of lines is fixed, so every level-1/2 sum is
// smooth over its interval; the window test keeps the reference's truncation.
#include <math.h>

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

struct MlLine {
  float4 g;   // jf (centre index relative to the chunk start), a, b, amp_far
  float4 h;   // y, y^2, amp, value the clamped far-wing loop adds inside the near zone
};

// Re w times the line amplitude at one point, any distance (fast far wing first).
__device__ __forceinline__ float line_value(float x, const MlLine& L) {
  const float z2 = fmaf(x, x, L.h.y);
  if (z2 >= FAR_Z2 && L.h.x >= 0.f) {
    const float r = rcp_approx(z2);
    return L.g.w * r * fmaf(fmaf(-2.0f * L.h.y, r, 1.5f), r, 1.0f);
  }
  if (z2 >= CORE_Z2 && L.h.x >= 0.f) return L.h.z * re_w_f32_mid(x, L.h.x, L.h.y, z2);
  return (float)((double)L.h.z * weideman_re((double)x, (double)L.h.x));
}

// Five-term asymptotic form with |z|^2 clamped to >= MID_Z2 (the level-3 loop
// body, times amp_far); inside the near zone it is the constant rc S(rc), rc = 1/MID_Z2.
__device__ __forceinline__ float mid_clamped_term(float x, float y2) {
  const float r = rcp_approx(fmaxf(fmaf(x, x, y2), MID_Z2));
  return r * asym5_bracket(y2, r);
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

template <bool DET>
__global__ void __launch_bounds__(ML_THREADS, 4)
tau_ml_kernel(const LineF32* __restrict__ prep, int n_lines, const int2* __restrict__ ranges,
              const double* __restrict__ t_layer, double nu_min, double step, long long n_nu,
              int tile_samples, int chunks_per_tile, double cutoff, int n_grp, float* __restrict__ od,
              int* err, unsigned long long* evals, unsigned long long* work, int tile_first,
              long long out_first, long long out_stride) {
  constexpr int P = ML_P;
  __shared__ MlLine s1[ML_THREADS];                 // level-1 lines of the round
  __shared__ MlLine s2[ML_THREADS];                 // inner lines of the round
  __shared__ unsigned char s_l2[ML_THREADS / 32][ML_THREADS];   // per-warp level-2 slots
  __shared__ unsigned char s_l3[ML_THREADS / 32][ML_THREADS];   // per-warp level-3 slots
  __shared__ unsigned char s_nl[ML_THREADS / 32][ML_THREADS];   // per-warp slots with near points in it
  __shared__ int s_cnt[4][ML_THREADS / 32];
  __shared__ int s_seg_start[ML_THREADS + 1];       // near-item prefix per inner slot
  __shared__ short s_seg_lo[ML_THREADS];            // first near point per inner slot
  __shared__ unsigned char s_seg_mask[ML_THREADS];  // warps treating the inner line directly (level 3)
  __shared__ float s_core[ML_CHUNK];               // near-zone corrections (each point owned by one thread)
  __shared__ float s_nbuf[ML_NB];                   // near-item values of one batch
  __shared__ double s_red[ML_THREADS];
  __shared__ double s_redf[ML_THREADS];
  __shared__ float s_c1[ML_K];
  __shared__ float s_c1f[ML_KF];
  __shared__ float s_c2[ML_THREADS / 32][ML_K];

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
  const int2 rng = ranges[tile];
  const LineF32* lp = prep + (long long)row * n_lines;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, n_warps = blockDim.x >> 5;
  // chunk geometry (points relative to c0)
  const float H1 = 0.5f * (float)(n_c - 1), C1 = H1;
  const bool use_l1 = H1 >= ML_MIN_H1;
  // this warp's sub-chunk
  const int w0 = warp * ML_WARP_PTS;
  const int n_w = max(0, min(ML_WARP_PTS, n_c - w0));
  const float H2 = 0.5f * (float)(n_w - 1), C2w = (float)w0 + H2;
  const bool use_l2 = H2 >= ML_MIN_H2;
  // Chebyshev node offsets owned by this thread: level 1 node (tid & 15), level 2 node (lane & 15)
  const float xn1 = H1 * (float)cospi((2.0 * (tid & 15) + 1.0) / (2.0 * ML_K));
  const float xn1f = H1 * (float)cospi((2.0 * (tid & 7) + 1.0) / (2.0 * ML_KF));
  const float xn2 = H2 * (float)cospi((2.0 * (lane & 15) + 1.0) / (2.0 * ML_K));
  const float pf = (float)(w0 + lane * P);                   // this lane's first point

  for (int i = tid; i < ML_CHUNK; i += blockDim.x) s_core[i] = 0.f;

  // level-3 sums hold only the lines within ~2 sub-chunk widths (tens of terms), so
  // plain float accumulation suffices; the long node sums use Kahan compensation.
  float acc[P];
#pragma unroll
  for (int m = 0; m < P; ++m) acc[m] = 0.f;
  float sum1 = 0.f, comp1 = 0.f, sumf = 0.f, compf = 0.f, sum2 = 0.f, comp2 = 0.f;
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
    const bool lev1 = pass && use_l1 && (d1 > H1 + 1.f);
    const bool lev1f = lev1 && (d1 > ML_FAR1 * H1);     // far: 8 nodes suffice
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
    int near_scan = near_n;                                  // inclusive warp scan
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, near_scan, o);
      if (lane >= o) near_scan += t;
    }
    const unsigned b1 = __ballot_sync(0xffffffffu, lev1 && !lev1f), bf = __ballot_sync(0xffffffffu, lev1f);
    const unsigned b2 = __ballot_sync(0xffffffffu, inner);
    if (lane == 0) { s_cnt[0][warp] = __popc(b1); s_cnt[1][warp] = __popc(b2); s_cnt[3][warp] = __popc(bf); }
    if (lane == 31) s_cnt[2][warp] = near_scan;
    __syncthreads();
    int off1 = 0, offf = 0, off2 = 0, off3 = 0, n1 = 0, nf = 0, n2 = 0, n_near = 0;
    for (int w = 0; w < n_warps; ++w) {
      const int a1 = s_cnt[0][w], a2 = s_cnt[1][w], a3 = s_cnt[2][w], af = s_cnt[3][w];
      off1 += (w < warp) ? a1 : 0;
      offf += (w < warp) ? af : 0;
      off2 += (w < warp) ? a2 : 0;
      off3 += (w < warp) ? a3 : 0;
      n1 += a1;
      nf += af;
      n2 += a2;
      n_near += a3;
    }
    if (pass) {
      MlLine r;
      r.g = make_float4(lev1 ? C1 - jf : jf, L.a, L.b, L.amp_far);
      float clamp_val = 0.f;                          // used by level 3 only
      if (!lev1) clamp_val = L.amp_far * mid_clamped_term(0.f, y2);   // r = 1/MID_Z2 when y2 < MID_Z2
      r.h = make_float4(L.y, y2, L.amp, clamp_val);
      const unsigned lt = (1u << lane) - 1u;
      if (lev1f) {
        s1[n1 + offf + __popc(bf & lt)] = r;              // far level-1 lines after the others
      } else if (lev1) {
        s1[off1 + __popc(b1 & lt)] = r;
      } else {
        const int slot = off2 + __popc(b2 & lt);
        s2[slot] = r;
        s_seg_start[slot] = off3 + near_scan - near_n;       // exclusive prefix in slot order
        s_seg_lo[slot] = (short)near_lo;
        s_seg_mask[slot] = (unsigned char)l3mask;
      }
    }
    if (tid == 0) s_seg_start[n2] = n_near;
    __syncthreads();
    n_pass += (unsigned long long)(n1 + nf + n2);

    // ---- level 1: thread (tid & 15) evaluates its node for lines tid>>4, +16, ...
    {
      float a1 = 0.f;
      const int stride = blockDim.x >> 4;
      for (int l = tid >> 4; l < n1; l += stride) {
        const MlLine R = s1[l];
        const float x = fmaf(xn1 + R.g.x, R.g.y, -R.g.z);     // (node - centre) * s
        a1 += line_value(x, R);
      }
      kahan_add(sum1, comp1, a1);
      // far lines: thread (tid & 7) evaluates its node for far lines tid>>3, +32, ...
      float af = 0.f;
      for (int l = tid >> 3; l < nf; l += (int)(blockDim.x >> 3)) {
        const MlLine R = s1[n1 + l];
        const float x = fmaf(xn1f + R.g.x, R.g.y, -R.g.z);
        af += line_value(x, R);
      }
      kahan_add(sumf, compf, af);
      if (tid == 0) n_nodes += (unsigned long long)n1 * ML_K + (unsigned long long)nf * ML_KF;
    }

    // ---- per-warp split of the inner lines into level 2 and level 3
    int n2w = 0, n3w = 0, nnw = 0;
    for (int k = 0; k < n2; k += 32) {
      const int l = k + lane;
      bool is2 = false, is3 = false, nz = false;
      if (l < n2) {
        const float d = fabsf(s2[l].g.x - C2w) - H2;
        is2 = use_l2 && d > H2 + 1.f;
        is3 = !is2 && n_w > 0;
        if constexpr (DET) {   // near points of slot l inside this warp's sub-chunk (level 3 here)
          const int st = s_seg_start[l], len = s_seg_start[l + 1] - st, lo = s_seg_lo[l];
          nz = len > 0 && ((s_seg_mask[l] >> warp) & 1u) && lo < w0 + n_w && lo + len > w0;
        }
      }
      const unsigned q2 = __ballot_sync(0xffffffffu, is2), q3 = __ballot_sync(0xffffffffu, is3);
      const unsigned lt = (1u << lane) - 1u;
      if (is2) s_l2[warp][n2w + __popc(q2 & lt)] = (unsigned char)l;
      if (is3) s_l3[warp][n3w + __popc(q3 & lt)] = (unsigned char)l;
      n2w += __popc(q2);
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
      if (lane == 0) n_nodes += (unsigned long long)n2w * ML_K;
    }

    // ---- level 3, far part: every point of the warp, |z|^2 clamped (branch-free)
    for (int i = 0; i < n3w; ++i) {
      const MlLine R = s2[s_l3[warp][i]];
      const float x0 = fmaf(pf - R.g.x, R.g.y, -R.g.z);
#pragma unroll
      for (int m = 0; m < P; ++m) acc[m] = fmaf(R.g.w, mid_clamped_term(fmaf((float)m, R.g.y, x0), R.h.y), acc[m]);
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
      for (int i = tid; i < n_near; i += blockDim.x) {
        int l = 0, hi = n2;                               // largest l with s_seg_start[l] <= i
        while (hi - l > 1) {
          const int mid = (l + hi) >> 1;
          if (s_seg_start[mid] <= i) l = mid; else hi = mid;
        }
        const int p = s_seg_lo[l] + (i - s_seg_start[l]);
        if (!((s_seg_mask[l] >> (p >> 8)) & 1u)) continue;   // level 2 for the owning warp
        const MlLine R = s2[l];
        const float x0 = fmaf((float)(p & ~(P - 1)) - R.g.x, R.g.y, -R.g.z);
        const float x = fmaf((float)(p & (P - 1)), R.g.y, x0);
        const float z2 = fmaf(x, x, R.h.y);
        if (z2 >= MID_Z2) continue;
        float v;
        if (z2 >= CORE_Z2 && R.h.x >= 0.f) v = R.h.z * re_w_cf32(x, R.h.x, z2);
        else v = (float)((double)R.h.z * weideman_re((double)x, (double)R.h.x));
        atomicAdd(&s_core[p], v - R.h.w);
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
              else v = (float)((double)R.h.z * weideman_re((double)x, (double)R.h.x));
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
    if (tid == 0) n_near_items += (unsigned long long)n_near;
    // No barrier here: the next round writes the staging arrays only after its first
    // barrier, which every warp reaches after finishing this round.
  }
  __syncthreads();

  // ---- level-1 node values: reduce the 16-thread groups, then Chebyshev coefficients
  s_red[tid] = (double)sum1 - (double)comp1;
  s_redf[tid] = (double)sumf - (double)compf;
  __syncthreads();
  if (tid < ML_K) {
    double f = 0.0;
    for (int i = tid; i < (int)blockDim.x; i += ML_K) f += s_red[i];
    s_red[tid] = f;      // only read back after the barrier below
  } else if (tid < ML_K + ML_KF) {
    const int j = tid - ML_K;
    double f = 0.0;
    for (int i = j; i < (int)blockDim.x; i += ML_KF) f += s_redf[i];
    s_redf[j] = f;
  }
  __syncthreads();
  if (tid < ML_K) {
    double c = 0.0;
    for (int j = 0; j < ML_K; ++j) c += s_red[j] * cospi((double)tid * (2.0 * j + 1.0) / (2.0 * ML_K));
    s_c1[tid] = use_l1 ? (float)(c * (2.0 / ML_K)) : 0.f;
  } else if (tid < ML_K + ML_KF) {
    const int k = tid - ML_K;
    double c = 0.0;
    for (int j = 0; j < ML_KF; ++j) c += s_redf[j] * cospi((double)k * (2.0 * j + 1.0) / (2.0 * ML_KF));
    s_c1f[k] = use_l1 ? (float)(c * (2.0 / ML_KF)) : 0.f;
  }
  // ---- level-2 node values of this warp: lanes j and j+16 hold halves of node j
  {
    float f2 = sum2 - comp2;
    f2 += __shfl_xor_sync(0xffffffffu, f2, 16);
    double c = 0.0;
    for (int j = 0; j < ML_K; ++j) {
      const float fj = __shfl_sync(0xffffffffu, f2, j);
      c += (double)fj * cospi((double)(lane & 15) * (2.0 * j + 1.0) / (2.0 * ML_K));
    }
    if (lane < ML_K) s_c2[warp][lane] = use_l2 ? (float)(c * (2.0 / ML_K)) : 0.f;
  }
  __syncthreads();

  const double T = t_layer[row];
  float* out = od + (long long)row * out_stride;   // points [out_first, out_first + out_stride) of the grid
  float c1[ML_K], c2[ML_K];
#pragma unroll
  for (int k = 0; k < ML_K; ++k) { c1[k] = s_c1[k]; c2[k] = s_c2[warp][k]; }
  const float inv_h1 = use_l1 ? 1.0f / H1 : 0.f, inv_h2 = use_l2 ? 1.0f / H2 : 0.f;
  bool bad = false;
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const int pl = w0 + lane * P + m;
    if (pl < n_c) {
      float v = s_core[pl];
      if (use_l1) {
        const float t1 = ((float)pl - C1) * inv_h1;
        v += clenshaw16(c1, t1) + clenshaw16<ML_KF>(s_c1f, t1);
      }
      if (use_l2) v += clenshaw16(c2, ((float)pl - C2w) * inv_h2);
      const long long p = c0 + pl;
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

extern "C" int lbl_tau_tiles_ml_f32(const LineF32* prep, int n_lines, const int* ranges, const double* t_layer,
                                    int n_rows, double nu_min, double step, long long n_nu, int tile_samples,
                                    double cutoff, int n_grp, float* od, int* err, unsigned long long* evals,
                                    unsigned long long* work, int tile_first, int tile_count, int flags,
                                    void* stream) {
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
  if (flags & LBL_DETERMINISTIC)
    tau_ml_kernel<true><<<grid, threads, 0, (cudaStream_t)stream>>>(prep, n_lines, (const int2*)ranges, t_layer,
                                                                   nu_min, step, n_nu, tile_samples, (int)chunks,
                                                                   cutoff, n_grp, od, err, evals, work,
                                                                   tile_first, out_first, out_end - out_first);
  else
    tau_ml_kernel<false><<<grid, threads, 0, (cudaStream_t)stream>>>(prep, n_lines, (const int2*)ranges, t_layer,
                                                                    nu_min, step, n_nu, tile_samples, (int)chunks,
                                                                    cutoff, n_grp, od, err, evals, work,
                                                                    tile_first, out_first, out_end - out_first);
  return lbl_check_launch("lbl_tau_tiles_ml_f32");
}
