// Device helpers shared by the summation kernels (voigt.cu, voigt_ml.cu).
#pragma once

#include "faddeeva.cuh"
#include "lbl_common.cuh"

namespace lbl {

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

static __device__ __noinline__ float re_w_f32_mid(float x, float y, float y2, float z2) {
  if (z2 >= MID_Z2) return re_w_asym5(y, y2, 1.0f / z2);
  return re_w_cf32(x, y, z2);
}

}  // namespace lbl
