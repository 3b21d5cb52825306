// Device helpers shared by the summation kernels (voigt.cu, voigt_ml.cu, voigt_ml_jac.cu).
#pragma once

#include <stddef.h>

#include "faddeeva.cuh"
#include "lbl_common.cuh"

namespace lbl {

// Points [c0, c0 + n_c) of chunk `chunk` of the tile [t0, t1): a tile of n points is cut
// into ceil(n / chunk_max) chunks of near-equal size, none longer than chunk_max, so no
// chunk is a sliver too short for the far-field levels (a 1,050-point tile gives 525 + 525,
// not 1,024 + 26). Returns false for a chunk index the tile does not have.
__device__ __forceinline__ bool tile_chunk(long long t0, long long t1, int chunk, int chunk_max, long long& c0,
                                           int& n_c) {
  const long long n = t1 - t0;
  const long long nch = (n + chunk_max - 1) / chunk_max;
  if (chunk >= nch) return false;
  c0 = t0 + chunk * n / nch;
  n_c = (int)(t0 + (chunk + 1) * n / nch - c0);
  return true;
}

__device__ __forceinline__ float rcp_approx(float v) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

// Out-of-line general evaluations keep the register allocation of the hot
// far-wing loop independent of the (rarely executed) full algorithm.
static __device__ __noinline__ double re_w_f64(double x, double y) { return faddeeva<double>(x, y).re; }

__device__ __forceinline__ double radiation_term_grid(double nu, double T) {
  return __dmul_rn(nu, tanh(__ddiv_rn(__dmul_rn(0.5 * C2, nu), T)));
}

// Stages one round of candidate lines; returns the number that passed the window
// test. Compaction keeps the candidate order (warp ballot + per-warp offsets).
template <typename Rec, typename Emit>
__device__ __forceinline__ int stage_round(const Rec* __restrict__ lp, int li, int hi, double wlo, double whi,
                                           int* warp_cnt, Emit emit) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, n_warps = blockDim.x >> 5;
  bool pass = false;
  Rec L;
  if (li < hi) {
    L = lp[li];
    pass = (L.nuc >= wlo) && (L.nuc <= whi);       // NaN (inactive) fails
  }
  const unsigned ballot = __ballot_sync(0xffffffffu, pass);
  if (lane == 0) warp_cnt[warp] = __popc(ballot);
  __syncthreads();
  int off = 0, total = 0;
  for (int w = 0; w < n_warps; ++w) {
    const int c = warp_cnt[w];
    off += (w < warp) ? c : 0;
    total += c;
  }
  if (pass) emit(off + __popc(ballot & ((1u << lane) - 1u)), L);
  __syncthreads();
  return total;
}

// Asynchronous 16-byte global -> shared copies (cp.async, L2 only); a thread that
// copies into and later reads only its own slots is ordered by its own wait_group.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Line records staged in shared memory as 16-byte planes, plane[k][slot] holding bytes
// 16k..16k+15 of slot's record: a thread reading its own slot then reads 16 consecutive
// bytes per thread per plane, so the eight threads of each quarter-warp phase of a
// 128-bit load hit eight different 16-byte bank groups (a 32- or 64-byte record read
// whole from an array of records puts them on 4 or 2 groups). The records are put
// back together field by field (little-endian byte order of the device).
static_assert(sizeof(LineF32) == 32 && sizeof(LineJac) == 32, "line records are two 16-byte planes");
static_assert(offsetof(LineF32, nuc) == 0 && offsetof(LineF32, j0) == 8 && offsetof(LineF32, b) == 12 &&
                  offsetof(LineF32, a) == 16 && offsetof(LineF32, y) == 20 && offsetof(LineF32, amp) == 24 &&
                  offsetof(LineF32, amp_far) == 28,
              "LineF32 field offsets assumed by line_f32_from_planes");
static_assert(offsetof(LineJac, jT_u) == 0 && offsetof(LineJac, jv_u) == 12 && offsetof(LineJac, jv_y) == 16 &&
                  offsetof(LineJac, pad1) == 28,
              "LineJac field offsets assumed by line_jac_from_planes");
__device__ __forceinline__ LineF32 line_f32_from_planes(const float4& p0, const float4& p1) {
  LineF32 L;
  L.nuc = __hiloint2double(__float_as_int(p0.y), __float_as_int(p0.x));   // bytes 0-7
  L.j0 = __float_as_int(p0.z);                                             // bytes 8-11
  L.b = p0.w;
  L.a = p1.x;
  L.y = p1.y;
  L.amp = p1.z;
  L.amp_far = p1.w;
  return L;
}
__device__ __forceinline__ LineJac line_jac_from_planes(const float4& p0, const float4& p1) {
  LineJac J;
  J.jT_u = p0.x;
  J.jT_x = p0.y;
  J.jT_y = p0.z;
  J.jv_u = p0.w;
  J.jv_y = p1.x;
  J.jv_x = p1.y;
  J.pad0 = p1.z;
  J.pad1 = p1.w;
  return J;
}

// Adds the lanes' float node sums into the warp's float64 sums (lane 0 owns the row)
// and clears them; every lane of the warp calls it.
template <int K>
__device__ __forceinline__ void flush_nodes(float (&f)[K], double* row, int lane) {
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double v = (double)f[k];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) row[k] += v;
    f[k] = 0.f;
  }
}

static __device__ __noinline__ float re_w_f32_mid(float x, float y, float y2, float z2) {
  if (z2 >= MID_Z2) return re_w_asym5(y, y2, 1.0f / z2);
  return re_w_cf32(x, y, z2);
}

}  // namespace lbl
