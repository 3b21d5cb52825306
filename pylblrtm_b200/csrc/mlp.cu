// BF16 tensor-core GEMM (tcgen05 + TMA + tensor memory) with fused epilogues, and the
// small kernels of the surrogate network's training and gated inference. The surrogate
// has no reference counterpart: it maps a layer profile to channel-mean transmittance
// and is trained on spectra produced by this library's own engine.
//
// D[M, N] = A[M, K] . B[N, K]^T, A and B bf16 row-major with K contiguous ("K-major"),
// accumulated in float32 in tensor memory. The kernel is persistent (one CTA per SM,
// each looping over 128 x BN output tiles, BN = 256 or 128) and warp-specialised:
//   warp 0, lane 0   streams 128 x 64 tiles of A and BN x 64 tiles of B into a 4-stage
//                    shared-memory ring with TMA (128-byte swizzle, no multicast);
//                    each stage completes a "full" mbarrier;
//   warp 1, lane 0   issues tcgen05.mma (M = 128, N = BN, K = 16) four times per stage
//                    into one of two tensor-memory accumulators and frees the stage
//                    with tcgen05.commit on its "empty" mbarrier; a finished tile is
//                    signalled on the accumulator's "tmem_full" mbarrier;
//   warps 2-9        (the epilogue, two per SM sub-partition) each read 32 accumulator
//                    rows x half the columns with tcgen05.ld, apply the epilogue, store,
//                    and release the accumulator ("tmem_empty", one arrival per warp), so
//                    the epilogue of one tile overlaps the main loop of the next.
// Split-K (n_split > 1) is offered for the float32 mode only: split z writes its partial
// sum to out_f32 + z * split_stride and the consumer adds the partials in a fixed order
// (deterministic).
//
// Every mbarrier wait is bounded by wall-clock time (globaltimer); a wait that runs out
// marks the CTA failed, every role leaves its loop, the MMA warp drains its own
// outstanding MMAs, tensor memory is always freed and the caller's error word is raised.
#include <cuda.h>
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "lbl_common.cuh"

namespace lbl {

constexpr int GM = 128, GK = 64, GSTAGES = 4;
constexpr int G_A_BYTES = GM * GK * 2;                             // 16 KiB A tile per stage
constexpr int G_EPI_WARPS = 8;                                     // 2 per SM sub-partition
constexpr int G_EPI_GROUPS = G_EPI_WARPS / 4;                      // column groups of a tile
constexpr int G_THREADS = 64 + 32 * G_EPI_WARPS;                   // TMA warp, MMA warp, epilogue
constexpr unsigned long long G_WAIT_NS = 2000000000ull;            // 2 s per wait at most

template <int BN>
struct GemmCfg {
  static constexpr int B_BYTES = BN * GK * 2;
  static constexpr int STAGE_BYTES = G_A_BYTES + B_BYTES;
  static constexpr int TMEM_COLS = 2 * BN;                         // two float32 accumulators
  static constexpr int SMEM = GSTAGES * STAGE_BYTES + 1024 + 256;  // ring + alignment + barriers
  // kind::f16: D f32 (bits 4-5 = 1), A and B bf16 (bits 7-9, 10-12 = 1), both K-major
  // (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24.
  static constexpr uint32_t IDESC =
      (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(GM >> 4) << 24);
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait for the phase of the given parity; false when G_WAIT_NS elapsed first.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > G_WAIT_NS) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"((uint64_t)map), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle: 128-byte
// rows (64 bf16), 8-row groups 1024 B apart (stride byte offset), descriptor version 1,
// layout type 2 (SWIZZLE_128B). The tile base is 1024-byte aligned (base offset 0);
// the K = 16 slices inside a 64-wide tile start 32 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// GELU (erf form) and its derivative.
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * __expf(-0.5f * z * z);
}

// 16 consecutive bf16 of one row: two 16-byte stores.
__device__ __forceinline__ void store_row16(__nv_bfloat16* dst, const float* v) {
  uint32_t p[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    p[i] = *reinterpret_cast<uint32_t*>(&h);
  }
  uint4* d = reinterpret_cast<uint4*>(dst);
  d[0] = make_uint4(p[0], p[1], p[2], p[3]);
  d[1] = make_uint4(p[4], p[5], p[6], p[7]);
}

// 16 bf16 of one row from memory (z_in of the GELU' epilogue).
__device__ __forceinline__ void load_row16(const __nv_bfloat16* src, float* v) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  const uint4 a = s[0], b = s[1];
  const uint32_t p[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&p[i]);
    float2 f = __bfloat1622float2(h);
    v[2 * i] = f.x;
    v[2 * i + 1] = f.y;
  }
}

// Epilogue of one 16-column slice of one accumulator row (row, col = first column).
__device__ __forceinline__ void epilogue16(const LblGemmEpilogue& ep, int split, int row, int col, float* v,
                                           float& loss) {
  if (ep.mode == LBL_GEMM_F32) {
    float4* d = reinterpret_cast<float4*>(ep.out_f32 + (long long)split * ep.split_stride +
                                          (long long)row * ep.ld_f32 + col);
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    return;
  }
  float bias[16];
  if (ep.mode == LBL_GEMM_BIAS_GELU || ep.mode == LBL_GEMM_BIAS_SIGMOID) {   // four 16-byte loads (broadcast)
    const float4* b4 = reinterpret_cast<const float4*>(ep.bias + col);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float4 t = __ldg(b4 + i);
      bias[4 * i] = t.x;
      bias[4 * i + 1] = t.y;
      bias[4 * i + 2] = t.z;
      bias[4 * i + 3] = t.w;
    }
  }
  if (ep.mode == LBL_GEMM_BIAS_GELU) {
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] += bias[i];
    if (ep.z_out) store_row16((__nv_bfloat16*)ep.z_out + (long long)row * ep.ld_z + col, v);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = gelu(v[i]);
  } else if (ep.mode == LBL_GEMM_BIAS_SIGMOID) {
    float p[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) p[i] = __fdividef(1.0f, 1.0f + __expf(-(v[i] + bias[i])));
    if (ep.out_f32) {
      float4* d = reinterpret_cast<float4*>(ep.out_f32 + (long long)row * ep.ld_f32 + col);
#pragma unroll
      for (int i = 0; i < 4; ++i) d[i] = make_float4(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
    }
    if (!ep.target) return;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      if (col + i < ep.n_valid) {
        const float d = p[i] - ep.target[(long long)row * ep.ld_target + col + i];
        loss += d * d;
        v[i] = ep.grad_scale * 2.0f * d * p[i] * (1.0f - p[i]);
      } else {
        v[i] = 0.0f;                               // padded outputs carry no gradient
      }
    }
  } else {                                         // LBL_GEMM_DGELU
    float z[16];
    load_row16((const __nv_bfloat16*)ep.z_in + (long long)row * ep.ld_zin + col, z);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] *= gelu_grad(z[i]);
  }
  if (ep.y) store_row16((__nv_bfloat16*)ep.y + (long long)row * ep.ld_y + col, v);
  if (ep.y_t) {
    __nv_bfloat16* yt = (__nv_bfloat16*)ep.y_t;
#pragma unroll
    for (int i = 0; i < 16; ++i) yt[(long long)(col + i) * ep.ld_yt + row] = __float2bfloat16(v[i]);
  }
}

// Work unit u -> (split, m tile, n tile); n varies fastest so concurrent CTAs share A.
struct GemmGrid {
  int n_m, n_n, kt_per;
  __device__ __forceinline__ void unit(int u, int& split, int& m0, int& n0, int bn) const {
    split = u / (n_m * n_n);
    const int r = u - split * n_m * n_n;
    m0 = (r / n_n) * GM;
    n0 = (r % n_n) * bn;
  }
};

template <int BN>
__global__ void __launch_bounds__(G_THREADS, 1)
gemm_bf16_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                 GemmGrid gg, int units, LblGemmEpilogue ep, int* err) {
  using Cfg = GemmCfg<BN>;
  extern __shared__ unsigned char g_smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)g_smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + GSTAGES * Cfg::STAGE_BYTES);
  uint64_t* full = bars;                       // [GSTAGES], one producer arrival + TMA bytes
  uint64_t* empty = bars + GSTAGES;            // [GSTAGES], one tcgen05.commit
  uint64_t* tfull = bars + 2 * GSTAGES;        // [2], one tcgen05.commit
  uint64_t* tempty = bars + 2 * GSTAGES + 2;   // [2], one arrival per epilogue warp
  uint64_t* drain = bars + 2 * GSTAGES + 4;    // MMA warp's final commit
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * GSTAGES + 5);
  volatile int* fail = (volatile int*)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    *fail = 0;
    for (int i = 0; i < GSTAGES; ++i) {
      mbar_init(smem_u32(&full[i]), 1);
      mbar_init(smem_u32(&empty[i]), 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(smem_u32(&tfull[i]), 1);
      mbar_init(smem_u32(&tempty[i]), G_EPI_WARPS);
    }
    mbar_init(smem_u32(drain), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(Cfg::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  float loss = 0.0f;

  if (warp == 0) {
    if (lane == 0) {                           // TMA producer
      int g = 0;
      for (int u = blockIdx.x; u < units && !*fail; u += gridDim.x) {
        int split, m0, n0;
        gg.unit(u, split, m0, n0, BN);
        const int k0 = split * gg.kt_per;
        for (int kt = 0; kt < gg.kt_per; ++kt, ++g) {
          const int s = g % GSTAGES;
          if (g >= GSTAGES && !mbar_wait(smem_u32(&empty[s]), ((g / GSTAGES) - 1) & 1)) {
            *fail = 1;
            break;
          }
          if (*fail) break;
          unsigned char* st = smem + s * Cfg::STAGE_BYTES;
          const uint32_t fb = smem_u32(&full[s]);
          mbar_expect_tx(fb, Cfg::STAGE_BYTES);
          tma_load_2d(smem_u32(st), &map_a, fb, (k0 + kt) * GK, m0);
#pragma unroll
          for (int h = 0; h < BN / 128; ++h)
            tma_load_2d(smem_u32(st + G_A_BYTES + h * 128 * GK * 2), &map_b, fb, (k0 + kt) * GK, n0 + 128 * h);
        }
      }
      // no copy may still be writing shared memory when the CTA ends (bounded wait)
      for (int j = g > GSTAGES ? g - GSTAGES : 0; j < g; ++j)
        if (!mbar_wait(smem_u32(&full[j % GSTAGES]), (j / GSTAGES) & 1)) *fail = 1;
    }
  } else if (warp == 1) {
    if (lane == 0) {                           // MMA issuer
      int g = 0, i = 0;
      for (int u = blockIdx.x; u < units && !*fail; u += gridDim.x, ++i) {
        const int b = i & 1;
        if (i >= 2 && !mbar_wait(smem_u32(&tempty[b]), ((i >> 1) - 1) & 1)) {
          *fail = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(b * BN);
        bool ok = true;
        for (int kt = 0; kt < gg.kt_per; ++kt, ++g) {
          const int s = g % GSTAGES;
          if (!mbar_wait(smem_u32(&full[s]), (g / GSTAGES) & 1)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(smem + s * Cfg::STAGE_BYTES), b0 = a0 + G_A_BYTES;
#pragma unroll
          for (int kk = 0; kk < GK / 16; ++kk)
            umma_bf16(acc, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32), Cfg::IDESC,
                      (kt > 0 || kk > 0) ? 1u : 0u);
          umma_commit(smem_u32(&empty[s]));
        }
        if (!ok) {
          *fail = 1;
          break;
        }
        umma_commit(smem_u32(&tfull[b]));
      }
      umma_commit(smem_u32(drain));            // arrives once every MMA issued above has finished
      if (!mbar_wait(smem_u32(drain), 0)) *fail = 1;
    }
  } else {  // epilogue warps: tensor-memory lanes 32 * (warp % 4), column group (warp - 2) / 4
    const int q = warp & 3;
    const int cg = (warp - 2) >> 2;
    constexpr int CW = BN / G_EPI_GROUPS;      // columns per group
    int i = 0;
    for (int u = blockIdx.x; u < units; u += gridDim.x, ++i) {
      const int b = i & 1;
      bool ok = !*fail && mbar_wait(smem_u32(&tfull[b]), (i >> 1) & 1);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) {
        if (lane == 0) *fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int split, m0, n0;
      gg.unit(u, split, m0, n0, BN);
      const int row = m0 + q * 32 + lane;
      const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN);
#pragma unroll 1
      for (int c0 = cg * CW; c0 < (cg + 1) * CW; c0 += 16) {
        float v[16];
        tmem_ld16(base + (uint32_t)c0, v);
        epilogue16(ep, split, row, n0 + c0, v, loss);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&tempty[b]));
    }
    if (ep.loss && ep.mode == LBL_GEMM_BIAS_SIGMOID && ep.target) {
      double l = loss;
      for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
      if (lane == 0 && l != 0.0) atomicAdd(ep.loss, l);
    }
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (threadIdx.x == 0 && *fail && err) atomicMax(err, 1);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS));
}

// ---------------------------------------------------------------------------
// Small kernels of the training step and of the gate.

// Adam on float32 master weights [rows, cols] (row stride ld) with the gradient summed
// over n_split partials (stride split_stride, added in order); refreshes the bf16 copy
// [rows, ld] and its transpose [cols, ld_t] when given.
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, int n_split, long long split_stride, int rows, int cols,
                            int ld, float lr, float b1, float b2, float eps, float c1, float c2,
                            __nv_bfloat16* __restrict__ w_bf, __nv_bfloat16* __restrict__ wt_bf, int ld_t) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)rows * cols) return;
  const int r = (int)(i / cols), c = (int)(i % cols);
  const long long o = (long long)r * ld + c;
  float gi = g[o];
  for (int s = 1; s < n_split; ++s) gi += g[s * split_stride + o];
  const float mi = b1 * m[o] + (1.0f - b1) * gi;
  const float vi = b2 * v[o] + (1.0f - b2) * gi * gi;
  m[o] = mi;
  v[o] = vi;
  const float wi = w[o] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  w[o] = wi;
  if (w_bf) w_bf[o] = __float2bfloat16(wi);
  if (wt_bf) wt_bf[(long long)c * ld_t + r] = __float2bfloat16(wi);
}

// out[r] = sum_c x[r, c] over a bf16 matrix (bias gradients from dZ^T).
__global__ void rowsum_bf16_kernel(const __nv_bfloat16* __restrict__ x, int rows, int cols, int ld,
                                   float* __restrict__ out) {
  const int r = blockIdx.x;
  float s = 0.f;
  for (int c = threadIdx.x; c < cols; c += blockDim.x) s += __bfloat162float(x[(long long)r * ld + c]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    out[r] = t;
  }
}

// x[b, c] = (raw[b, c] - mean[c]) * inv_std[c] as bf16, zero beyond cols up to ld; the
// transposed copy x_t[c, b] (row stride ld_t) when given.
__global__ void pack_inputs_kernel(const float* __restrict__ raw, int rows, int cols, const float* __restrict__ mean,
                                   const float* __restrict__ inv_std, __nv_bfloat16* __restrict__ x, int ld,
                                   __nv_bfloat16* __restrict__ x_t, int ld_t) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)rows * ld) return;
  const int r = (int)(i / ld), c = (int)(i % ld);
  const float v = c < cols ? (raw[(long long)r * cols + c] - mean[c]) * inv_std[c] : 0.0f;
  const __nv_bfloat16 b = __float2bfloat16(v);
  x[(long long)r * ld + c] = b;
  if (x_t) x_t[(long long)c * ld_t + r] = b;
}

// Ensemble statistics of one sample per CTA: mean over the members of pred[m, b, c]
// and the error estimate est[b] = max over channels of the members' standard deviation
// (population form); flag[b] = (scale * est[b] > gate).
__global__ void ensemble_gate_kernel(const float* __restrict__ pred, int n_mem, long long member_stride, int ld,
                                     int n_ch, const float* __restrict__ ch_scale, float scale, float gate,
                                     float* __restrict__ mean, float* __restrict__ est, int* __restrict__ flag) {
  const int b = blockIdx.x;
  float worst = 0.0f;
  for (int c = threadIdx.x; c < n_ch; c += blockDim.x) {
    const float* col = pred + (long long)b * ld + c;
    float s = 0.f;
    for (int m = 0; m < n_mem; ++m) s += col[m * member_stride];
    const float mu = s / n_mem;
    float s2 = 0.f;                                  // second pass: deviations (no cancellation)
    for (int m = 0; m < n_mem; ++m) {
      const float d = col[m * member_stride] - mu;
      s2 += d * d;
    }
    mean[(long long)b * n_ch + c] = mu;
    const float sd = sqrtf(s2 / n_mem);
    worst = fmaxf(worst, ch_scale ? ch_scale[c] * sd : sd);
  }
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = worst;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmaxf(t, part[w]);
    est[b] = t;
    flag[b] = (scale * t > gate) ? 1 : 0;
  }
}

}  // namespace lbl

using namespace lbl;

// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

extern "C" size_t lbl_tensor_map_bytes(void) { return sizeof(CUtensorMap); }

extern "C" int lbl_tensor_map_bf16(void* map_out, const void* base, long long rows, long long cols, long long ld) {
  if (!map_out || !base || rows < GM || rows % GM || cols < GK || cols % GK || ld < cols || ld % 8 ||
      ((uintptr_t)base) % 16)
    return lbl_set_error(LBL_EINVAL,
                         "lbl_tensor_map_bf16: rows must be a multiple of 128, cols of 64, ld a multiple of 8 "
                         ">= cols and the base 16-byte aligned");
  EncodeTiledFn fn = encode_fn();
  if (!fn) return lbl_set_error(LBL_ECUDA, "lbl_tensor_map_bf16: cuTensorMapEncodeTiled unavailable");
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {GK, GM};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn((CUtensorMap*)map_out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return lbl_set_error(LBL_ECUDA, "lbl_tensor_map_bf16: encode failed (%d)", (int)r);
  return LBL_OK;
}

template <int BN>
static int launch_gemm(const CUtensorMap& a, const CUtensorMap& b, int M, int N, int K, int n_split,
                       const LblGemmEpilogue* ep, int* err, cudaStream_t stream) {
  int dev = 0;
  cudaGetDevice(&dev);
  static int attr_set[64] = {0};
  static int n_sm[64] = {0};
  if (dev < 0 || dev >= 64) return lbl_set_error(LBL_EINVAL, "lbl_gemm_bf16: device index out of range");
  if (!attr_set[dev]) {
    if (cudaFuncSetAttribute(gemm_bf16_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             GemmCfg<BN>::SMEM) != cudaSuccess)
      return lbl_check_launch("lbl_gemm_bf16 (shared memory attribute)");
    cudaDeviceGetAttribute(&n_sm[dev], cudaDevAttrMultiProcessorCount, dev);
    attr_set[dev] = 1;
  }
  GemmGrid gg;
  gg.n_m = M / GM;
  gg.n_n = N / BN;
  gg.kt_per = K / GK / n_split;
  const long long units = (long long)gg.n_m * gg.n_n * n_split;
  if (units > 0x7fffffffLL) return lbl_set_error(LBL_EINVAL, "lbl_gemm_bf16: too many tiles");
  const int grid = (int)(units < n_sm[dev] ? units : n_sm[dev]);
  gemm_bf16_kernel<BN><<<grid, G_THREADS, GemmCfg<BN>::SMEM, stream>>>(a, b, gg, (int)units, *ep, err);
  return lbl_check_launch("lbl_gemm_bf16");
}

extern "C" int lbl_gemm_bf16(const void* map_a, const void* map_b, int M, int N, int K, int n_split,
                             const LblGemmEpilogue* ep, int* err, void* stream) {
  if (!map_a || !map_b || !ep || M < GM || N < 128 || K < GK || M % GM || N % 128 || K % GK || n_split < 1 ||
      (K / GK) % n_split || ep->mode < LBL_GEMM_F32 || ep->mode > LBL_GEMM_DGELU)
    return lbl_set_error(LBL_EINVAL, "lbl_gemm_bf16: M, N must be multiples of 128, K of 64 * n_split");
  if (n_split > 1 && ep->mode != LBL_GEMM_F32)
    return lbl_set_error(LBL_EINVAL, "lbl_gemm_bf16: split-K needs the float32 epilogue");
  const bool needs_f32 = ep->mode == LBL_GEMM_F32;
  if ((needs_f32 && (!ep->out_f32 || ep->ld_f32 < N || ep->ld_f32 % 4 ||
                     (n_split > 1 && ep->split_stride < (long long)M * ep->ld_f32))) ||
      (ep->mode != LBL_GEMM_F32 && ep->mode != LBL_GEMM_DGELU && (!ep->bias || ((uintptr_t)ep->bias) % 16)) ||
      (ep->mode == LBL_GEMM_DGELU && (!ep->z_in || ep->ld_zin < N || ep->ld_zin % 8)) ||
      (ep->z_out && (ep->ld_z < N || ep->ld_z % 8)) || (ep->y && (ep->ld_y < N || ep->ld_y % 8)) ||
      (ep->y_t && ep->ld_yt < M) || (ep->mode == LBL_GEMM_BIAS_SIGMOID && ep->out_f32 && ep->ld_f32 % 4) ||
      (ep->mode == LBL_GEMM_BIAS_SIGMOID && ep->target && ep->ld_target < ep->n_valid))
    return lbl_set_error(LBL_EINVAL, "lbl_gemm_bf16: epilogue buffers missing or strides too small/unaligned");
  CUtensorMap a, b;
  memcpy(&a, map_a, sizeof(a));
  memcpy(&b, map_b, sizeof(b));
  if (N % 256 == 0) return launch_gemm<256>(a, b, M, N, K, n_split, ep, err, (cudaStream_t)stream);
  return launch_gemm<128>(a, b, M, N, K, n_split, ep, err, (cudaStream_t)stream);
}

extern "C" int lbl_adam_step(float* w, float* m, float* v, const float* g, int n_split, long long split_stride,
                             int rows, int cols, int ld, float lr, float b1, float b2, float eps, int step,
                             void* w_bf16, void* wt_bf16, int ld_t, void* stream) {
  if (!w || !m || !v || !g || rows < 1 || cols < 1 || ld < cols || step < 1 || n_split < 1 ||
      (n_split > 1 && split_stride < (long long)rows * ld) || (wt_bf16 && ld_t < rows))
    return lbl_set_error(LBL_EINVAL, "lbl_adam_step: bad arguments");
  const float c1 = (float)(1.0 / (1.0 - pow((double)b1, step))), c2 = (float)(1.0 / (1.0 - pow((double)b2, step)));
  const long long n = (long long)rows * cols;
  adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      w, m, v, g, n_split, split_stride, rows, cols, ld, lr, b1, b2, eps, c1, c2, (__nv_bfloat16*)w_bf16,
      (__nv_bfloat16*)wt_bf16, ld_t);
  return lbl_check_launch("lbl_adam_step");
}

extern "C" int lbl_rowsum_bf16(const void* x, int rows, int cols, int ld, float* out, void* stream) {
  if (!x || !out || rows < 1 || cols < 1 || ld < cols)
    return lbl_set_error(LBL_EINVAL, "lbl_rowsum_bf16: bad arguments");
  rowsum_bf16_kernel<<<rows, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)x, rows, cols, ld, out);
  return lbl_check_launch("lbl_rowsum_bf16");
}

extern "C" int lbl_pack_inputs_bf16(const float* raw, int rows, int cols, const float* mean, const float* inv_std,
                                    void* x, int ld, void* x_t, int ld_t, void* stream) {
  if (!raw || !mean || !inv_std || !x || rows < 1 || cols < 1 || ld < cols || (x_t && ld_t < rows))
    return lbl_set_error(LBL_EINVAL, "lbl_pack_inputs_bf16: bad arguments");
  const long long n = (long long)rows * ld;
  pack_inputs_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      raw, rows, cols, mean, inv_std, (__nv_bfloat16*)x, ld, (__nv_bfloat16*)x_t, ld_t);
  return lbl_check_launch("lbl_pack_inputs_bf16");
}

extern "C" int lbl_ensemble_gate(const float* pred, int n_mem, long long member_stride, int n_samples, int ld,
                                 int n_ch, const float* ch_scale, float scale, float gate, float* mean, float* est,
                                 int* flag, void* stream) {
  if (!pred || !mean || !est || !flag || n_mem < 1 || n_samples < 1 || n_ch < 1 || ld < n_ch ||
      (n_mem > 1 && member_stride < (long long)n_samples * ld))
    return lbl_set_error(LBL_EINVAL, "lbl_ensemble_gate: bad arguments");
  ensemble_gate_kernel<<<n_samples, 256, 0, (cudaStream_t)stream>>>(pred, n_mem, member_stride, ld, n_ch, ch_scale,
                                                                     scale, gate, mean, est, flag);
  return lbl_check_launch("lbl_ensemble_gate");
}
