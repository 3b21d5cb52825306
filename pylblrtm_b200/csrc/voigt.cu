// Voigt summation over reference tiles (pylblrtm/forward.py:295-315).
//
// One CTA handles one chunk of grid points inside one reference tile of one
// profile-layer row. The lines of the tile's candidate range are staged into
// shared memory in rounds of blockDim lines; each line passes the reference's
// exact window test (shifted centre within [nu_first - cutoff, nu_last + cutoff]
// of the tile, forward.py:298-301) before it is compacted into the round.
// Every thread owns P consecutive grid points and loops over the staged lines
// reading them as shared-memory broadcasts.
#include <math.h>

#include "faddeeva.cuh"
#include "lbl_common.cuh"
#include "sum_common.cuh"

namespace lbl {

constexpr int F32_P = 8;          // grid points per thread (float32 kernel)
constexpr int F64_P = 4;          // grid points per thread (float64 kernel)
constexpr int MAX_THREADS = 128;  // threads per CTA (and lines staged per round)

struct StagedF32 {
  float4 g;   // jf (line index relative to chunk start), a, b, amp_far
  float4 h;   // y, warp far-test threshold, amp, unused
};

// Shared-memory queue of (staged line, point) pairs with |z|^2 < CORE_Z2. They
// are evaluated in double precision by the whole CTA after each round, so the
// few core points of a line do not serialise a warp.
constexpr int CORE_QCAP = 2048;

__global__ void __launch_bounds__(MAX_THREADS)
tau_f32_kernel(const LineF32* __restrict__ prep, int n_lines, const int2* __restrict__ ranges,
               const double* __restrict__ t_layer, double nu_min, double step, long long n_nu,
               int tile_samples, int chunks_per_tile, double cutoff, int n_grp, float* __restrict__ od,
               int* err, unsigned long long* evals) {
  constexpr int P = F32_P;
  __shared__ float4 s_g[MAX_THREADS];
  __shared__ float4 s_h[MAX_THREADS];
  __shared__ int warp_cnt[MAX_THREADS / 32];
  __shared__ int s_q[CORE_QCAP];
  __shared__ int s_qn;
  __shared__ float s_core[MAX_THREADS * P];

  const int row = blockIdx.y;
  const int tile = blockIdx.x / chunks_per_tile, chunk = blockIdx.x % chunks_per_tile;
  const long long t0 = (long long)tile * tile_samples;
  const long long t1 = min(t0 + (long long)tile_samples, n_nu);
  const long long c0 = t0 + (long long)chunk * (blockDim.x * P);
  if (c0 >= t1) return;
  const long long c1 = min(c0 + (long long)(blockDim.x * P), t1);
  const double wlo = __dsub_rn(grid_nu(nu_min, step, t0), cutoff);
  const double whi = __dadd_rn(grid_nu(nu_min, step, t1 - 1), cutoff);
  const int2 rng = ranges[tile];
  const LineF32* lp = prep + (long long)row * n_lines;

  const int tid = threadIdx.x;
  const float pf = (float)(tid * P);
  constexpr float WHW = 0.5f * (32 * P - 1);            // half-width of a warp's points
  const float wc = (float)((tid >> 5) * 32 * P) + WHW;  // centre of this warp's points

  for (int i = tid; i < MAX_THREADS * P; i += blockDim.x) s_core[i] = 0.f;
  if (tid == 0) s_qn = 0;

  float sum[P], comp[P], acc[P];
#pragma unroll
  for (int m = 0; m < P; ++m) sum[m] = comp[m] = acc[m] = 0.f;
  unsigned long long n_pass = 0;

  for (int base = rng.x; base < rng.y; base += blockDim.x) {
    const int total = stage_round<LineF32>(
        lp, base + tid, rng.y, wlo, whi, warp_cnt, [&](int slot, const LineF32& L) {
          const float jf = (float)((long long)L.j0 - c0);
          const float y2 = L.y * L.y;
          // points within hw of the centre may have |z|^2 < FAR_Z2
          const float hw = sqrtf(fmaxf(FAR_Z2 - y2, 0.f)) / L.a + 1.0f;
          const float thr = (y2 >= FAR_Z2 && L.y >= 0.f) ? -1.0f : hw + WHW;
          s_g[slot] = make_float4(jf, L.a, L.b, L.amp_far);
          s_h[slot] = make_float4(L.y, thr, L.amp, 0.f);
        });
    n_pass += (unsigned long long)total;
    for (int l = 0; l < total; ++l) {
      const float4 g = s_g[l];
      const float4 h = s_h[l];
      const float x0 = fmaf(pf - g.x, g.y, -g.z);         // x at this thread's first point
      const float y2 = h.x * h.x;
      if (fabsf(g.x - wc) > h.y) {
        // every point of the warp is in the far wing: two-term asymptotic
        // Re w = y/sqrt(pi) r (1 + 1.5 r - 2 y^2 r^2), r = 1/|z|^2
        const float n2y2 = -2.0f * y2;
#pragma unroll
        for (int m = 0; m < P; ++m) {
          const float x = fmaf((float)m, g.y, x0);
          const float r = rcp_approx(fmaf(x, x, y2));
          const float v = fmaf(fmaf(n2y2, r, 1.5f), r, 1.0f);
          acc[m] = fmaf(g.w, r * v, acc[m]);
        }
      } else {
#pragma unroll
        for (int m = 0; m < P; ++m) {
          const float x = fmaf((float)m, g.y, x0);
          const float z2 = fmaf(x, x, y2);
          if (z2 >= FAR_Z2 && h.x >= 0.f) {
            const float r = rcp_approx(z2);
            const float v = fmaf(fmaf(-2.0f * y2, r, 1.5f), r, 1.0f);
            acc[m] = fmaf(g.w, r * v, acc[m]);
          } else if (z2 >= CORE_Z2 && h.x >= 0.f) {
            acc[m] = fmaf(h.z, re_w_f32_mid(x, h.x, y2, z2), acc[m]);
          } else {
            const int qi = atomicAdd(&s_qn, 1);
            if (qi < CORE_QCAP) {
              s_q[qi] = (l << 10) | (tid * P + m);
            } else {   // queue full: evaluate in place
              acc[m] = fmaf(h.z, (float)re_w_f64((double)x, (double)h.x), acc[m]);
            }
          }
        }
      }
    }
    __syncthreads();
    // the round's core points, in double precision, spread over the CTA
    const int nq = min(s_qn, CORE_QCAP);
    for (int i = tid; i < nq; i += blockDim.x) {
      const int item = s_q[i];
      const int l = item >> 10, p = item & 1023;
      const float4 g = s_g[l];
      const float4 h = s_h[l];
      const double x = ((double)p - (double)g.x) * (double)g.y - (double)g.z;
      atomicAdd(&s_core[p], (float)((double)h.z * re_w_f64(x, (double)h.x)));
    }
    __syncthreads();
    if (tid == 0) s_qn = 0;
    // compensated (Kahan) merge of this round's partial sums
#pragma unroll
    for (int m = 0; m < P; ++m) {
      const float yk = acc[m] - comp[m];
      const float t = sum[m] + yk;
      comp[m] = (t - sum[m]) - yk;
      sum[m] = t;
      acc[m] = 0.f;
    }
  }
  __syncthreads();

  const double T = t_layer[row];
  float* out = od + (long long)row * n_nu;
  bool bad = false;
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const long long p = c0 + tid * P + m;
    if (p < c1) {
      const double nu = grid_nu(nu_min, step, p);
      const double tot = (double)sum[m] - (double)comp[m] + (double)s_core[tid * P + m];
      const float v = (float)(tot * radiation_term_grid(nu, T));
      bad |= !isfinite(v);
      out[p] = v;
    }
  }
  if (bad) flag_error(err, row * (n_grp + 1) + n_grp);
  if (evals && tid == 0 && n_pass) atomicAdd(evals, n_pass * (unsigned long long)(c1 - c0));
}

struct StagedF64 {
  double nuc, inv_ad, y, amp;
};

__global__ void __launch_bounds__(MAX_THREADS)
tau_f64_kernel(const LineF64* __restrict__ prep, int n_lines, const int2* __restrict__ ranges,
               const double* __restrict__ t_layer, double nu_min, double step, long long n_nu,
               int tile_samples, int chunks_per_tile, double cutoff, int n_grp, double* __restrict__ od,
               int* err, unsigned long long* evals) {
  constexpr int P = F64_P;
  __shared__ StagedF64 s_l[MAX_THREADS];
  __shared__ int warp_cnt[MAX_THREADS / 32];

  const int row = blockIdx.y;
  const int tile = blockIdx.x / chunks_per_tile, chunk = blockIdx.x % chunks_per_tile;
  const long long t0 = (long long)tile * tile_samples;
  const long long t1 = min(t0 + (long long)tile_samples, n_nu);
  const long long c0 = t0 + (long long)chunk * (blockDim.x * P);
  if (c0 >= t1) return;
  const long long c1 = min(c0 + (long long)(blockDim.x * P), t1);
  const double wlo = __dsub_rn(grid_nu(nu_min, step, t0), cutoff);
  const double whi = __dadd_rn(grid_nu(nu_min, step, t1 - 1), cutoff);
  const int2 rng = ranges[tile];
  const LineF64* lp = prep + (long long)row * n_lines;
  const int tid = threadIdx.x;

  double nu[P], acc[P];
#pragma unroll
  for (int m = 0; m < P; ++m) {
    nu[m] = grid_nu(nu_min, step, min(c0 + tid * P + m, c1 - 1));
    acc[m] = 0.0;
  }
  unsigned long long n_pass = 0;
  for (int base = rng.x; base < rng.y; base += blockDim.x) {
    const int total = stage_round<LineF64>(
        lp, base + tid, rng.y, wlo, whi, warp_cnt, [&](int slot, const LineF64& L) {
          s_l[slot] = StagedF64{L.nuc, L.inv_ad, L.y, L.amp};
        });
    n_pass += (unsigned long long)total;
    for (int l = 0; l < total; ++l) {
      const StagedF64 L = s_l[l];
#pragma unroll
      for (int m = 0; m < P; ++m) {
        const double x = (nu[m] - L.nuc) * L.inv_ad;
        acc[m] = fma(L.amp, re_w_f64(x, L.y), acc[m]);
      }
    }
  }
  const double T = t_layer[row];
  double* out = od + (long long)row * n_nu;
  bool bad = false;
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const long long p = c0 + tid * P + m;
    if (p < c1) {
      const double v = __dmul_rn(acc[m], radiation_term_grid(nu[m], T));
      bad |= !isfinite(v);
      out[p] = v;
    }
  }
  if (bad) flag_error(err, row * (n_grp + 1) + n_grp);
  if (evals && tid == 0 && n_pass) atomicAdd(evals, n_pass * (unsigned long long)(c1 - c0));
}

// Threads per CTA for a reference tile: enough warps for the tile, at most 128.
static int tile_threads(int tile_samples, int points_per_thread) {
  int warps = (tile_samples + 32 * points_per_thread - 1) / (32 * points_per_thread);
  if (warps > MAX_THREADS / 32) warps = MAX_THREADS / 32;
  return 32 * warps;
}

template <typename Rec, typename Out, typename K>
static int launch_tau(K kernel, int P, const Rec* prep, int n_lines, const int* ranges, const double* t_layer,
                      int n_rows, double nu_min, double step, long long n_nu, int tile_samples, double cutoff,
                      int n_grp, Out* od, int* err, unsigned long long* evals, void* stream, const char* name) {
  if (!prep || !ranges || !t_layer || !od || n_lines < 1 || n_rows < 1 || n_rows > 65535 || n_nu < 1 ||
      tile_samples < 1 || !(step > 0) || !(cutoff >= 0) || n_grp < 1)
    return lbl_set_error(LBL_EINVAL, "%s: bad arguments", name);
  const int threads = tile_threads(tile_samples, P);
  const int cp = threads * P;
  const long long n_tiles = (n_nu + tile_samples - 1) / tile_samples;
  const long long chunks = (tile_samples + cp - 1) / cp;
  if (n_tiles * chunks > 0x7fffffffLL) return lbl_set_error(LBL_EINVAL, "%s: grid too large", name);
  dim3 grid((unsigned)(n_tiles * chunks), (unsigned)n_rows);
  kernel<<<grid, threads, 0, (cudaStream_t)stream>>>(prep, n_lines, (const int2*)ranges, t_layer, nu_min, step,
                                                      n_nu, tile_samples, (int)chunks, cutoff, n_grp, od, err,
                                                      evals);
  return lbl_check_launch(name);
}

// ---------------------------------------------------------------------------
// Layer sums and transmittance (pylblrtm/forward.py:151, config.py:266-270).
template <typename T>
__global__ void layer_sum_exp_kernel(const T* __restrict__ od, int n_prof, int n_lay, long long n_nu,
                                     const double* __restrict__ mu, double* __restrict__ trans,
                                     double* __restrict__ tau) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_prof * n_nu) return;
  const long long b = idx / n_nu, i = idx % n_nu;
  const T* p = od + b * n_lay * n_nu + i;
  double s = 0.0;
  for (int k = 0; k < n_lay; ++k) s = __dadd_rn(s, (double)p[(long long)k * n_nu]);
  if (tau) tau[idx] = s;
  if (trans) trans[idx] = exp(__ddiv_rn(-s, mu[b]));
}

// ---------------------------------------------------------------------------
__global__ void faddeeva_f64_kernel(const double* x, const double* y, long long n, double* re, double* im) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const cpx<double> w = faddeeva<double>(x[i], y[i]);
  re[i] = w.re;
  if (im) im[i] = w.im;
}

__global__ void faddeeva_f32_kernel(const float* x, const float* y, long long n, float* re, float* im,
                                    int mode) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mode == 1) {
    re[i] = faddeeva_re_f32(x[i], y[i]);
    return;
  }
  const cpx<float> w = faddeeva<float>(x[i], y[i]);
  re[i] = w.re;
  if (im) im[i] = w.im;
}

}  // namespace lbl

using namespace lbl;

extern "C" int lbl_tau_tiles_f32(const LineF32* prep, int n_lines, const int* ranges, const double* t_layer,
                                 int n_rows, double nu_min, double step, long long n_nu, int tile_samples,
                                 double cutoff, int n_grp, float* od, int* err, unsigned long long* evals,
                                 void* stream) {
  return launch_tau(tau_f32_kernel, F32_P, prep, n_lines, ranges, t_layer, n_rows, nu_min, step, n_nu,
                    tile_samples, cutoff, n_grp, od, err, evals, stream, "lbl_tau_tiles_f32");
}

extern "C" int lbl_tau_tiles_f64(const LineF64* prep, int n_lines, const int* ranges, const double* t_layer,
                                 int n_rows, double nu_min, double step, long long n_nu, int tile_samples,
                                 double cutoff, int n_grp, double* od, int* err, unsigned long long* evals,
                                 void* stream) {
  return launch_tau(tau_f64_kernel, F64_P, prep, n_lines, ranges, t_layer, n_rows, nu_min, step, n_nu,
                    tile_samples, cutoff, n_grp, od, err, evals, stream, "lbl_tau_tiles_f64");
}

template <typename T>
static int launch_sum_exp(const T* od, int n_prof, int n_lay, long long n_nu, const double* mu, double* trans,
                          double* tau, void* stream, const char* name) {
  if (!od || n_prof < 1 || n_lay < 0 || n_nu < 1 || (!trans && !tau) || (trans && !mu))
    return lbl_set_error(LBL_EINVAL, "%s: bad arguments", name);
  const long long n = (long long)n_prof * n_nu;
  layer_sum_exp_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(od, n_prof, n_lay, n_nu,
                                                                                         mu, trans, tau);
  return lbl_check_launch(name);
}

extern "C" int lbl_layer_sum_exp_f32(const float* od, int n_prof, int n_lay, long long n_nu, const double* mu,
                                     double* trans, double* tau, void* stream) {
  return launch_sum_exp(od, n_prof, n_lay, n_nu, mu, trans, tau, stream, "lbl_layer_sum_exp_f32");
}

extern "C" int lbl_layer_sum_exp_f64(const double* od, int n_prof, int n_lay, long long n_nu, const double* mu,
                                     double* trans, double* tau, void* stream) {
  return launch_sum_exp(od, n_prof, n_lay, n_nu, mu, trans, tau, stream, "lbl_layer_sum_exp_f64");
}

extern "C" int lbl_faddeeva_f64(const double* x, const double* y, long long n, double* re, double* im,
                                void* stream) {
  if (!x || !y || !re || n < 0) return lbl_set_error(LBL_EINVAL, "lbl_faddeeva_f64: bad arguments");
  if (n == 0) return LBL_OK;
  faddeeva_f64_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(x, y, n, re, im);
  return lbl_check_launch("lbl_faddeeva_f64");
}

extern "C" int lbl_faddeeva_f32(const float* x, const float* y, long long n, float* re, float* im, int mode,
                                void* stream) {
  if (!x || !y || !re || n < 0 || mode < 0 || mode > 1)
    return lbl_set_error(LBL_EINVAL, "lbl_faddeeva_f32: bad arguments");
  if (n == 0) return LBL_OK;
  faddeeva_f32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(x, y, n, re, im, mode);
  return lbl_check_launch("lbl_faddeeva_f32");
}

// ---------------------------------------------------------------------------
// Measurement probe: sustained float32 FMA throughput of this device, used as
// the denominator of the summation kernel's roofline fraction. Each thread runs
// 8 independent dependency chains of `iters` FMAs (16 flops per chain step).
__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float seed) {
  float a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + 0.001f * (threadIdx.x + i);
  const float m = 0.9999f, c = 1e-4f;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = fmaf(a[i], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  if (s == 12345.678f) out[0] = s;   // keeps the chains live
}

extern "C" int lbl_probe_fma_f32(float* out, int iters, int blocks, void* stream) {
  if (!out || iters < 1 || blocks < 1) return lbl_set_error(LBL_EINVAL, "lbl_probe_fma_f32: bad arguments");
  fma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters, 1.0f);
  return lbl_check_launch("lbl_probe_fma_f32");
}

// ---------------------------------------------------------------------------
// Fused column sum, transmittance and channel box-average: channel c of profile b
// is the mean of exp(-sum_k od[b,k,p] / mu[b]) over the half-open point range
// [first + c*width, first + (c+1)*width). One CTA per (channel, profile); the
// per-point transmittance never goes to memory.
template <typename T>
__global__ void __launch_bounds__(256)
channel_mean_kernel(const T* __restrict__ od, int n_lay, long long n_nu, const double* __restrict__ mu,
                    long long first, int width, int n_ch, double* __restrict__ out) {
  __shared__ double s_part[8];
  const int c = blockIdx.x, b = blockIdx.y;
  const T* base = od + (long long)b * n_lay * n_nu;
  const double inv_mu = 1.0 / mu[b];
  double acc = 0.0;
  for (int t = threadIdx.x; t < width; t += blockDim.x) {
    const long long p = first + (long long)c * width + t;
    double s = 0.0;
    for (int k = 0; k < n_lay; ++k) s = __dadd_rn(s, (double)base[(long long)k * n_nu + p]);
    acc += exp(-s * inv_mu);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[w];
    out[(long long)b * n_ch + c] = t / width;
  }
}

template <typename T>
static int launch_channel_mean(const T* od, int n_prof, int n_lay, long long n_nu, const double* mu, long long first,
                               int width, int n_ch, double* out, void* stream, const char* name) {
  if (!od || !mu || !out || n_prof < 1 || n_prof > 65535 || n_lay < 0 || width < 1 || n_ch < 1 || first < 0 ||
      first + (long long)width * n_ch > n_nu)
    return lbl_set_error(LBL_EINVAL, "%s: bad arguments", name);
  dim3 grid((unsigned)n_ch, (unsigned)n_prof);
  channel_mean_kernel<T><<<grid, 256, 0, (cudaStream_t)stream>>>(od, n_lay, n_nu, mu, first, width, n_ch, out);
  return lbl_check_launch(name);
}

extern "C" int lbl_channel_mean_f32(const float* od, int n_prof, int n_lay, long long n_nu, const double* mu,
                                    long long first, int width, int n_ch, double* out, void* stream) {
  return launch_channel_mean(od, n_prof, n_lay, n_nu, mu, first, width, n_ch, out, stream, "lbl_channel_mean_f32");
}

extern "C" int lbl_channel_mean_f64(const double* od, int n_prof, int n_lay, long long n_nu, const double* mu,
                                    long long first, int width, int n_ch, double* out, void* stream) {
  return launch_channel_mean(od, n_prof, n_lay, n_nu, mu, first, width, n_ch, out, stream, "lbl_channel_mean_f64");
}
