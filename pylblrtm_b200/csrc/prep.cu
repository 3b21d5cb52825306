// Preparation kernels: hydrostatic layers, per-(layer, group) quantities with the
// partition-sum interpolation, candidate-line sort, tile windows and the per
// (layer, line) HITRAN scaling ("line prep").
#include <float.h>
#include <limits.h>
#include <math.h>

#include "faddeeva.cuh"
#include "lbl_common.cuh"

namespace lbl {

// ---------------------------------------------------------------------------
// Layers from levels (pylblrtm/atmosphere.py:117-141), same operation order so
// the result matches the host NumPy version bit for bit.
__global__ void build_layers_kernel(const double* __restrict__ p_hpa, const double* __restrict__ t_k,
                                    const double* __restrict__ vmr, int n_prof, int n_lev, int n_gas,
                                    double col_factor, double* __restrict__ p_atm,
                                    double* __restrict__ t_layer, double* __restrict__ vmr_layer,
                                    double* __restrict__ col) {
  const int n_lay = n_lev - 1;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_prof * n_lay) return;
  const int b = (int)(idx / n_lay), k = (int)(idx % n_lay);
  const double p0 = p_hpa[(long long)b * n_lev + k], p1 = p_hpa[(long long)b * n_lev + k + 1];
  p_atm[idx] = __ddiv_rn(__dsqrt_rn(__dmul_rn(p0, p1)), P_STD_HPA);
  const double t0 = t_k[(long long)b * n_lev + k], t1 = t_k[(long long)b * n_lev + k + 1];
  t_layer[idx] = __dmul_rn(0.5, __dadd_rn(t0, t1));
  const double dp_pa = __dmul_rn(fabs(__dsub_rn(p1, p0)), 100.0);
  const double air = __ddiv_rn(__dmul_rn(col_factor, dp_pa), 1e4);
  for (int g = 0; g < n_gas; ++g) {
    const double* v = vmr + ((long long)b * n_gas + g) * n_lev;
    const double vl = __dmul_rn(0.5, __dadd_rn(v[k], v[k + 1]));
    const long long o = ((long long)b * n_gas + g) * n_lay + k;
    vmr_layer[o] = vl;
    col[o] = __dmul_rn(vl, air);
  }
}

// np.interp(x, xp, fp) for increasing xp, clamped at both ends
// (pylblrtm/spectral_data.py:52 calls np.interp).
__device__ double interp_clamped(double x, const double* __restrict__ xp, const double* __restrict__ fp,
                                 int n) {
  if (isnan(x)) return x;
  if (x >= xp[n - 1]) return fp[n - 1];
  if (x < xp[0]) return fp[0];
  int lo = 0, hi = n - 1;            // invariant xp[lo] <= x < xp[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (xp[mid] <= x) lo = mid; else hi = mid;
  }
  if (x == xp[lo]) return fp[lo];
  const double slope = __ddiv_rn(__dsub_rn(fp[lo + 1], fp[lo]), __dsub_rn(xp[lo + 1], xp[lo]));
  double r = __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[lo])), fp[lo]);
  if (isnan(r)) {
    r = __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[lo + 1])), fp[lo + 1]);
    if (isnan(r) && fp[lo] == fp[lo + 1]) r = fp[lo];
  }
  return r;
}

// Per (profile, layer, group): partial pressures, column, Q(296)/Q(T) and
// sqrt(T/M) (pylblrtm/forward.py:236-240, 249-259, 292).
__global__ void layer_groups_kernel(const double* __restrict__ t_layer, const double* __restrict__ p_atm,
                                    const double* __restrict__ vmr_layer, const double* __restrict__ col,
                                    int n_rows, int n_lay, int n_gas, int n_grp,
                                    const int* __restrict__ grp_gas, const double* __restrict__ grp_mass,
                                    const int* __restrict__ tips_off, const int* __restrict__ tips_len,
                                    const double* __restrict__ tips_t, const double* __restrict__ tips_q,
                                    LayerGroup* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_rows * n_grp) return;
  const int row = (int)(idx / n_grp), g = (int)(idx % n_grp);
  const int b = row / n_lay, k = row % n_lay;
  const int gas = grp_gas[g];
  const double T = t_layer[row], P = p_atm[row];
  const long long gi = ((long long)b * n_gas + gas) * n_lay + k;
  const double v = vmr_layer[gi];
  LayerGroup lg;
  lg.T = T;
  lg.p_self = __dmul_rn(v, P);
  lg.p_air = __dsub_rn(P, lg.p_self);
  lg.col = col[gi];
  const double* xt = tips_t + tips_off[g];
  const double* xq = tips_q + tips_off[g];
  const int n = tips_len[g];
  const double q_ref = interp_clamped(T_REF, xt, xq, n);
  lg.q_ratio = __ddiv_rn(q_ref, interp_clamped(T, xt, xq, n));
  lg.dop = __dsqrt_rn(__ddiv_rn(T, grp_mass[g]));
  out[idx] = lg;
}

// ---------------------------------------------------------------------------
// Candidate-line sort. Keys are nu0 of the lines the reference masks in
// (pylblrtm/forward.py:215-220) and +inf otherwise; ties break on the input
// index so the order, and every sum built on it, is deterministic.
constexpr int SORT_BLOCK = 2048;   // elements sorted per CTA in shared memory

__global__ void sort_keys_kernel(const double* __restrict__ nu0, const double* __restrict__ shift,
                                 const int* __restrict__ gid, int n_lines, int n_pad, double mask_lo,
                                 double mask_hi, double p_max, double* __restrict__ keys,
                                 int* __restrict__ vals, int* __restrict__ n_kept, double* __restrict__ max_sb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pad) return;
  double key = CUDART_INF;
  if (i < n_lines && gid[i] >= 0) {
    const double sb = __dmul_rn(fabs(shift[i]), p_max);      // forward.py:191
    const double v = nu0[i];
    // a non-finite centre never lies in a tile window, so it can be dropped here
    if (isfinite(v) && v >= __dsub_rn(mask_lo, sb) && v <= __dadd_rn(mask_hi, sb)) {
      key = v;
      atomicAdd(n_kept, 1);
      // shift bound of a kept line (non-negative doubles order like their bits)
      atomicMax((unsigned long long*)max_sb, (unsigned long long)__double_as_longlong(sb));
    }
  }
  keys[i] = key;
  vals[i] = i;
}

__device__ __forceinline__ bool key_greater(double ka, int va, double kb, int vb) {
  return ka > kb || (ka == kb && va > vb);
}

// Sort stages whose stride is below SORT_BLOCK, in shared memory. With
// k_first = 2 the kernel sorts every block fully; otherwise it finishes the
// merge of bitonic size k (strides SORT_BLOCK/2 .. 1).
__global__ void __launch_bounds__(SORT_BLOCK / 2)
bitonic_smem_kernel(double* __restrict__ keys, int* __restrict__ vals, int k_first, int k_last) {
  __shared__ double sk[SORT_BLOCK];
  __shared__ int sv[SORT_BLOCK];
  const int base = blockIdx.x * SORT_BLOCK;
  for (int i = threadIdx.x; i < SORT_BLOCK; i += blockDim.x) {
    sk[i] = keys[base + i];
    sv[i] = vals[base + i];
  }
  __syncthreads();
  for (int k = k_first; k <= k_last; k <<= 1) {
    for (int j = (k == k_first && k_first > SORT_BLOCK) ? SORT_BLOCK / 2 : k >> 1; j > 0; j >>= 1) {
      const int t = threadIdx.x;
      const int i = 2 * t - (t & (j - 1));
      const int p = i + j;
      const bool asc = (((base + i) & k) == 0);
      const double ka = sk[i], kb = sk[p];
      const int va = sv[i], vb = sv[p];
      if (key_greater(ka, va, kb, vb) == asc) {
        sk[i] = kb; sk[p] = ka; sv[i] = vb; sv[p] = va;
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < SORT_BLOCK; i += blockDim.x) {
    keys[base + i] = sk[i];
    vals[base + i] = sv[i];
  }
}

__global__ void bitonic_global_kernel(double* __restrict__ keys, int* __restrict__ vals, int n_pad, int k,
                                      int j) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_pad / 2) return;
  const int i = 2 * t - (t & (j - 1));
  const int p = i + j;
  const bool asc = ((i & k) == 0);
  const double ka = keys[i], kb = keys[p];
  const int va = vals[i], vb = vals[p];
  if (key_greater(ka, va, kb, vb) == asc) {
    keys[i] = kb; keys[p] = ka; vals[i] = vb; vals[p] = va;
  }
}

// Sorted structure-of-records copy of the kept lines. Slots past the device's kept
// count (the caller may size the output for an upper bound it knows on the host)
// get an inactive record: nu0 = NaN, group 0, src = -1.
__global__ void gather_lines_kernel(const double* __restrict__ nu0, const double* __restrict__ sref,
                                    const double* __restrict__ g_air, const double* __restrict__ g_self,
                                    const double* __restrict__ elow, const double* __restrict__ n_air,
                                    const double* __restrict__ shift, const int* __restrict__ gid,
                                    const int* __restrict__ order, const int* __restrict__ n_kept,
                                    int n_lines, LineIn* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_lines) return;
  LineIn r;
  if (j >= *n_kept) {
    r.nu0 = CUDART_NAN; r.sref = 0.0; r.g_air = 0.0; r.g_self = 0.0;
    r.elow = 0.0; r.n_air = 0.0; r.shift = 0.0; r.gid = 0; r.src = -1;
    out[j] = r;
    return;
  }
  const int i = order[j];
  r.nu0 = nu0[i]; r.sref = sref[i]; r.g_air = g_air[i]; r.g_self = g_self[i];
  r.elow = elow[i]; r.n_air = n_air[i]; r.shift = shift[i]; r.gid = gid[i]; r.src = i;
  out[j] = r;
}

// Candidate range of each reference tile (pylblrtm/forward.py:295-301): the
// sorted lines whose unshifted centre lies within the tile window widened by
// the largest pressure shift. The exact test on the shifted centre is applied
// per layer inside the summation kernels.
__global__ void tile_ranges_kernel(const LineIn* __restrict__ lines, const int* __restrict__ n_kept,
                                   double nu_min, double step, long long n_nu, int tile_samples,
                                   double cutoff, double pad, int n_tiles, int2* __restrict__ ranges) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tiles) return;
  const long long i0 = (long long)t * tile_samples;
  const long long i1 = min(i0 + tile_samples, n_nu) - 1;
  const double lo_nu = __dsub_rn(__dsub_rn(grid_nu(nu_min, step, i0), cutoff), pad);
  const double hi_nu = __dadd_rn(__dadd_rn(grid_nu(nu_min, step, i1), cutoff), pad);
  const int n = *n_kept;
  int a = 0, b = n;               // first index with nu0 >= lo_nu
  while (a < b) { const int m = (a + b) >> 1; if (lines[m].nu0 < lo_nu) a = m + 1; else b = m; }
  int c = a, d = n;               // first index with nu0 > hi_nu
  while (c < d) { const int m = (c + d) >> 1; if (lines[m].nu0 <= hi_nu) c = m + 1; else d = m; }
  ranges[t] = make_int2(a, c);
}

// ---------------------------------------------------------------------------
// Line prep (pylblrtm/forward.py:257-292): shifted centre, temperature-scaled
// strength with column and 1/R(nuc, T), Lorentz and Doppler widths.
struct ScaledLine {
  double nuc, S, gamma, alpha;
  bool active;
};

__device__ __forceinline__ double radiation_term(double nu, double T) {
  // nu * tanh(c2 nu / 2T), evaluated as ((0.5 c2) nu) / T like forward.py:48
  return __dmul_rn(nu, tanh(__ddiv_rn(__dmul_rn(0.5 * C2, nu), T)));
}

__device__ __forceinline__ ScaledLine scale_line(const LineIn& L, const LayerGroup& G, int* err,
                                                 int err_key) {
  ScaledLine s;
  s.active = G.col != 0.0;                                      // forward.py:253-255
  if (!s.active) return s;
  const double T = G.T;
  s.nuc = __dadd_rn(L.nu0, __dmul_rn(L.shift, G.p_air));        // forward.py:263
  double S = __dmul_rn(L.sref, G.q_ratio);
  S = __dmul_rn(S, exp(__dmul_rn(__dmul_rn(-C2, L.elow), __dsub_rn(__ddiv_rn(1.0, T), 1.0 / T_REF))));
  S = __dmul_rn(S, -expm1(__ddiv_rn(__dmul_rn(-C2, L.nu0), T)));
  S = __ddiv_rn(S, -expm1(__ddiv_rn(__dmul_rn(-C2, L.nu0), T_REF)));
  S = __dmul_rn(S, G.col);
  S = __ddiv_rn(S, radiation_term(s.nuc, T));                   // forward.py:270-278
  if (!isfinite(S) || S < 0.0) flag_error(err, err_key);        // forward.py:280-283
  s.S = S;
  s.gamma = __dmul_rn(pow(__ddiv_rn(T_REF, T), L.n_air),
                      __dadd_rn(__dmul_rn(L.g_air, G.p_air), __dmul_rn(L.g_self, G.p_self)));
  s.alpha = __dmul_rn(__dmul_rn(L.nu0, DOPPLER), G.dop);        // forward.py:292
  return s;
}

__global__ void line_prep_f64_kernel(const LineIn* __restrict__ lines, const int* __restrict__ n_kept,
                                     int n_lines, const LayerGroup* __restrict__ lg, int n_rows, int n_grp,
                                     LineF64* __restrict__ out, int* err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (j >= n_lines || row >= n_rows) return;
  LineF64 r;
  r.nuc = CUDART_NAN; r.inv_ad = 0.0; r.y = 0.0; r.amp = 0.0;
  if (j < *n_kept) {
    const LineIn L = lines[j];
    const ScaledLine s = scale_line(L, lg[(long long)row * n_grp + L.gid], err, row * (n_grp + 1) + L.gid);
    if (s.active) {
      r.nuc = s.nuc;
      r.inv_ad = __ddiv_rn(SQRT_LN2, s.alpha);
      r.y = __ddiv_rn(__dmul_rn(SQRT_LN2, s.gamma), s.alpha);
      r.amp = __dmul_rn(__ddiv_rn(VOIGT_K, s.alpha), s.S);
    }
  }
  out[(long long)row * n_lines + j] = r;
}

// Float32-engine line prep: one thread per line over PREP_ROWS rows (profile-layers), so
// a line's record is read once and its layer-independent factors are formed once: the
// stimulated-emission denominator -expm1(-c2 nu0 / 296), c2 E'' and 1/(nu0 * 3.581e-7).
// Per (row, group) the CTA stages 1/T, 1/T - 1/296, 0.5 c2 / T, ln(296/T) and 1/sqrt(T/M)
// in shared memory. The Boltzmann factor stays float64 (exp), the strength is divided by
// R(nuc, T) in float64 as in forward.py:277 (through expm1); the stimulated-emission
// factor (expm1f) and the Lorentz width's (296/T)^n_air (expf) are float, at the float
// record's precision. Same records and error word as before; the float64 engine's prep
// (line_prep_f64_kernel) keeps the reference's operation order.
#ifndef LBL_PREP_ROWS
#define LBL_PREP_ROWS 8
#endif
constexpr int PREP_ROWS = LBL_PREP_ROWS;                       // rows (profile-layers) per thread
constexpr int PREP_THREADS = 128;

struct RowGroupF32 {
  double p_self, p_air, col_q, dinv, minus_c2_inv_t, half_c2_inv_t, inv_dop;
  float log_t296;
  int active;
};

__global__ void __launch_bounds__(PREP_THREADS)
line_prep_f32_kernel(const LineIn* __restrict__ lines, const int* __restrict__ n_kept, int n_lines,
                     const LayerGroup* __restrict__ lg, int n_rows, int n_grp, double nu_min, double step,
                     LineF32* __restrict__ out, int* err) {
  extern __shared__ RowGroupF32 s_rg[];                         // [PREP_ROWS][n_grp]
  const int r0 = blockIdx.y * PREP_ROWS;
  const int nr = min(PREP_ROWS, n_rows - r0);
  for (int i = threadIdx.x; i < nr * n_grp; i += blockDim.x) {
    const LayerGroup G = lg[(long long)r0 * n_grp + i];
    const double inv_t = 1.0 / G.T;
    RowGroupF32 q;
    q.p_self = G.p_self;
    q.p_air = G.p_air;
    q.col_q = G.q_ratio * G.col;
    q.dinv = inv_t - 1.0 / T_REF;
    q.minus_c2_inv_t = -C2 * inv_t;
    q.half_c2_inv_t = 0.5 * C2 * inv_t;
    q.inv_dop = 1.0 / G.dop;
    q.log_t296 = (float)log(T_REF * inv_t);
    q.active = G.col != 0.0;                                    // forward.py:253-255
    s_rg[i] = q;
  }
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_lines) return;
  LineF32 r;
  r.nuc = CUDART_NAN; r.j0 = 0; r.b = 0.f; r.a = 0.f; r.y = 0.f; r.amp = 0.f; r.amp_far = 0.f;
  if (j >= *n_kept) {
    for (int k = 0; k < nr; ++k) out[(long long)(r0 + k) * n_lines + j] = r;
    return;
  }
  const LineIn L = lines[j];
  const double stim296 = -expm1(-C2 * L.nu0 / T_REF);
  const double sref_stim = L.sref / stim296;
  const double c2_elow = -C2 * L.elow;
  const double inv_nd = 1.0 / (L.nu0 * DOPPLER);
  const double inv_step = 1.0 / step;
  const float n_air = (float)L.n_air;
#pragma unroll 2
  for (int k = 0; k < nr; ++k) {
    const int row = r0 + k;
    const RowGroupF32& G = s_rg[k * n_grp + L.gid];
    LineF32 o = r;
    if (G.active) {
      const double nuc = L.nu0 + L.shift * G.p_air;             // forward.py:263
      // Boltzmann factor in float64 (its argument reaches +-20 for large E''); the
      // stimulated-emission factor 1 - exp(-c2 nu0 / T) by expm1f keeps float32 relative
      // accuracy (no cancellation at any argument), which the float32 record needs
      const double stim = -(double)expm1f((float)(G.minus_c2_inv_t * L.nu0));
      double S = sref_stim * G.col_q * exp(c2_elow * G.dinv) * stim;
      // / R(nuc, T) = nuc tanh(v), v = c2 nuc / 2T (forward.py:277): with e = expm1(-2v),
      // tanh(v) = -e / (2 + e), so S / R = S (2 + e) / (-nuc e): one expm1, no tanh
      const double e = expm1(G.minus_c2_inv_t * nuc);
      S = S * (2.0 + e) / (-nuc * e);
      if (!isfinite(S) || S < 0.0) flag_error(err, row * (n_grp + 1) + L.gid);   // forward.py:280-283
      const double gamma = (double)expf(n_air * G.log_t296) * (L.g_air * G.p_air + L.g_self * G.p_self);
      const double sc = SQRT_LN2 * inv_nd * G.inv_dop;           // sqrt(ln 2) / alpha_D, forward.py:292
      double jd = rint((nuc - nu_min) * inv_step);
      jd = fmin(fmax(jd, -2.0e9), 2.0e9);     // host guarantees |j0| < 2^31 for kept lines
      const int j0 = (int)jd;
      const double rem = nuc - grid_nu(nu_min, step, j0);
      const double y = sc * gamma;
      const double amp = VOIGT_K * inv_nd * G.inv_dop * S;
      o.nuc = nuc;
      o.j0 = j0;
      o.b = (float)(rem * sc);
      o.a = (float)(step * sc);
      o.y = (float)y;
      o.amp = (float)amp;
      o.amp_far = (float)(amp * y * INV_SQRT_PI);
    }
    out[(long long)row * n_lines + j] = o;
  }
}

}  // namespace lbl

using namespace lbl;

static inline unsigned grid1(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

extern "C" int lbl_build_layers(const double* p_hpa, const double* t_k, const double* vmr, int n_prof,
                                int n_lev, int n_gas, double col_factor, double* p_atm, double* t_layer,
                                double* vmr_layer, double* col, void* stream) {
  if (n_prof < 1 || n_lev < 2 || n_gas < 0 || !p_hpa || !t_k || !p_atm || !t_layer ||
      (n_gas > 0 && (!vmr || !vmr_layer || !col)))
    return lbl_set_error(LBL_EINVAL, "lbl_build_layers: bad arguments");
  const long long n = (long long)n_prof * (n_lev - 1);
  build_layers_kernel<<<grid1(n, 128), 128, 0, (cudaStream_t)stream>>>(
      p_hpa, t_k, vmr, n_prof, n_lev, n_gas, col_factor, p_atm, t_layer, vmr_layer, col);
  return lbl_check_launch("lbl_build_layers");
}

extern "C" int lbl_layer_groups(const double* t_layer, const double* p_atm, const double* vmr_layer,
                                const double* col, int n_prof, int n_lay, int n_gas, int n_grp,
                                const int* grp_gas, const double* grp_mass, const int* tips_off,
                                const int* tips_len, const double* tips_t, const double* tips_q,
                                LayerGroup* out, void* stream) {
  if (n_prof < 1 || n_lay < 1 || n_grp < 1 || n_gas < 1 || !out)
    return lbl_set_error(LBL_EINVAL, "lbl_layer_groups: bad arguments");
  const long long n = (long long)n_prof * n_lay * n_grp;
  layer_groups_kernel<<<grid1(n, 128), 128, 0, (cudaStream_t)stream>>>(
      t_layer, p_atm, vmr_layer, col, n_prof * n_lay, n_lay, n_gas, n_grp, grp_gas, grp_mass, tips_off,
      tips_len, tips_t, tips_q, out);
  return lbl_check_launch("lbl_layer_groups");
}

static int pad_pow2(int n) {
  int p = SORT_BLOCK;
  while (p < n) p <<= 1;
  return p;
}

extern "C" size_t lbl_sort_workspace_bytes(int n_lines) {
  if (n_lines < 0) return 0;
  const size_t n_pad = (size_t)pad_pow2(n_lines);
  return n_pad * (sizeof(double) + sizeof(int));
}

extern "C" int lbl_sort_lines(const double* nu0, const double* shift, const int* gid, int n_lines,
                              double mask_lo, double mask_hi, double p_max, void* workspace,
                              size_t workspace_bytes, int* order, int* n_kept, double* max_shift_bound,
                              void* stream) {
  if (n_lines < 1 || n_lines > (1 << 30) || !nu0 || !shift || !gid || !workspace || !order || !n_kept ||
      !max_shift_bound)
    return lbl_set_error(LBL_EINVAL, "lbl_sort_lines: bad arguments");
  if (workspace_bytes < lbl_sort_workspace_bytes(n_lines))
    return lbl_set_error(LBL_EINVAL, "lbl_sort_lines: workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  const int n_pad = pad_pow2(n_lines);
  double* keys = (double*)workspace;
  int* vals = (int*)(keys + n_pad);
  cudaMemsetAsync(n_kept, 0, sizeof(int), s);
  cudaMemsetAsync(max_shift_bound, 0, sizeof(double), s);
  sort_keys_kernel<<<grid1(n_pad, 256), 256, 0, s>>>(nu0, shift, gid, n_lines, n_pad, mask_lo, mask_hi,
                                                     p_max, keys, vals, n_kept, max_shift_bound);
  const int n_blk = n_pad / SORT_BLOCK;
  bitonic_smem_kernel<<<n_blk, SORT_BLOCK / 2, 0, s>>>(keys, vals, 2, SORT_BLOCK);
  for (int k = 2 * SORT_BLOCK; k <= n_pad; k <<= 1) {
    for (int j = k >> 1; j >= SORT_BLOCK; j >>= 1)
      bitonic_global_kernel<<<grid1(n_pad / 2, 256), 256, 0, s>>>(keys, vals, n_pad, k, j);
    bitonic_smem_kernel<<<n_blk, SORT_BLOCK / 2, 0, s>>>(keys, vals, k, k);
  }
  cudaMemcpyAsync(order, vals, sizeof(int) * (size_t)n_lines, cudaMemcpyDeviceToDevice, s);
  return lbl_check_launch("lbl_sort_lines");
}

extern "C" int lbl_gather_lines(const double* nu0, const double* sref, const double* g_air,
                                const double* g_self, const double* elow, const double* n_air,
                                const double* shift, const int* gid, const int* order, const int* n_kept,
                                int n_lines, LineIn* out, void* stream) {
  if (n_lines < 1 || !order || !n_kept || !out)
    return lbl_set_error(LBL_EINVAL, "lbl_gather_lines: bad arguments");
  gather_lines_kernel<<<grid1(n_lines, 256), 256, 0, (cudaStream_t)stream>>>(
      nu0, sref, g_air, g_self, elow, n_air, shift, gid, order, n_kept, n_lines, out);
  return lbl_check_launch("lbl_gather_lines");
}

extern "C" int lbl_tile_ranges(const LineIn* lines, const int* n_kept, double nu_min, double step,
                               long long n_nu, int tile_samples, double cutoff, double pad, int n_tiles,
                               int* ranges, void* stream) {
  if (n_nu < 1 || tile_samples < 1 || n_tiles < 1 || !lines || !n_kept || !ranges)
    return lbl_set_error(LBL_EINVAL, "lbl_tile_ranges: bad arguments");
  tile_ranges_kernel<<<grid1(n_tiles, 128), 128, 0, (cudaStream_t)stream>>>(
      lines, n_kept, nu_min, step, n_nu, tile_samples, cutoff, pad, n_tiles, (int2*)ranges);
  return lbl_check_launch("lbl_tile_ranges");
}

extern "C" int lbl_line_prep_f64(const LineIn* lines, const int* n_kept, int n_lines, const LayerGroup* lg,
                                 int n_rows, int n_grp, LineF64* out, int* err, void* stream) {
  if (n_lines < 1 || n_rows < 1 || n_rows > 65535 || n_grp < 1 || !lines || !lg || !out)
    return lbl_set_error(LBL_EINVAL, "lbl_line_prep_f64: bad arguments");
  dim3 grid(grid1(n_lines, 128), n_rows);
  line_prep_f64_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(lines, n_kept, n_lines, lg, n_rows, n_grp,
                                                               out, err);
  return lbl_check_launch("lbl_line_prep_f64");
}

extern "C" int lbl_line_prep_f32(const LineIn* lines, const int* n_kept, int n_lines, const LayerGroup* lg,
                                 int n_rows, int n_grp, double nu_min, double step, LineF32* out, int* err,
                                 void* stream) {
  if (n_lines < 1 || n_rows < 1 || n_rows > 65535 || n_grp < 1 || !lines || !lg || !out || !(step > 0))
    return lbl_set_error(LBL_EINVAL, "lbl_line_prep_f32: bad arguments");
  dim3 grid(grid1(n_lines, PREP_THREADS), (unsigned)((n_rows + PREP_ROWS - 1) / PREP_ROWS));
  const size_t smem = sizeof(RowGroupF32) * PREP_ROWS * (size_t)n_grp;
  if (smem > 48 * 1024) return lbl_set_error(LBL_EINVAL, "lbl_line_prep_f32: too many line groups");
  line_prep_f32_kernel<<<grid, PREP_THREADS, smem, (cudaStream_t)stream>>>(lines, n_kept, n_lines, lg, n_rows,
                                                                           n_grp, nu_min, step, out, err);
  return lbl_check_launch("lbl_line_prep_f32");
}

// ---------------------------------------------------------------------------
// Allocation-free variant of lbl_sort_lines.
//
// Some callers cannot allocate device memory at the time they sort lines: host
// programs that hand all GPU memory to their own pool or allocator at start-up
// and forbid later cudaMalloc calls, or plugins running inside such a host. For
// them the sort scratch (keys and values of the bitonic sort) lives in the
// static array below, which every GPU that loads this library holds until the
// process exits.
constexpr int NOALLOC_MAX_LINES = 1 << 18;                                   // 262,144 lines
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)NOALLOC_MAX_LINES * (sizeof(double) + sizeof(int));  // 3 MiB
static __device__ __align__(256) unsigned char g_sort_scratch[NOALLOC_SCRATCH_BYTES];

#include <cuda.h>   // CUcontext / CUresult types only; the two driver calls are resolved at run time

#include <mutex>
static std::mutex g_scratch_mutex;
constexpr int NOALLOC_MAX_CONTEXTS = 64;
struct ScratchAddr {
  unsigned long long ctx_id;   // process-unique id of the CUDA context (cuCtxGetId), 0 = empty slot
  void* addr;
};
static ScratchAddr g_scratch_addr[NOALLOC_MAX_CONTEXTS] = {};
static int g_scratch_next = 0;   // next slot to (re)use once the table is full

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// Process-unique id of the calling thread's current CUDA context, or 0 when the
// driver offers no such query (the caller then looks the address up every time).
// The id of a context is never reused, so an address cached under it cannot go
// stale: after cudaDeviceReset, or when a host application makes a context of its
// own current, the id differs and the address is looked up again.
static unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {                                   // under g_scratch_mutex
    resolved = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (CtxGetIdFn)f;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_sort_scratch in the current context. The name is only a
// host-side stand-in; the real address comes from cudaGetSymbolAddress, called
// with the device current the first time a context uses this entry point and then
// cached under the context's unique id.
static int sort_scratch_address(void** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  void* p = nullptr;
  unsigned long long id = current_context_id();
  if (id != 0) {
    for (const ScratchAddr& s : g_scratch_addr)
      if (s.ctx_id == id) {
        *out = s.addr;
        return LBL_OK;
      }
  }
  // first use in this context (the lookup also binds the runtime's primary context
  // when the thread has none current yet, so read the id again afterwards)
  cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
  if (e != cudaSuccess || !p)
    return lbl_set_error(LBL_ECUDA, "lbl_sort_lines_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
  if (id == 0) id = current_context_id();
  if (id != 0) {
    g_scratch_addr[g_scratch_next] = ScratchAddr{id, p};
    g_scratch_next = (g_scratch_next + 1) % NOALLOC_MAX_CONTEXTS;
  }
  *out = p;
  return LBL_OK;
}

extern "C" int lbl_sort_lines_noalloc(const double* nu0, const double* shift, const int* gid, int n_lines,
                                      double mask_lo, double mask_hi, double p_max, int* order, int* n_kept,
                                      double* max_shift_bound, void* stream) {
  if (n_lines > NOALLOC_MAX_LINES)
    return lbl_set_error(LBL_EINVAL,
                         "lbl_sort_lines_noalloc: %d lines exceed the static scratch limit of %d lines; "
                         "use lbl_sort_lines with caller-provided workspace",
                         n_lines, NOALLOC_MAX_LINES);
  void* scratch = nullptr;
  const int st = sort_scratch_address(&scratch);
  if (st != LBL_OK) return st;
  // Every entry of the scratch that the sort reads is written first by
  // sort_keys_kernel, so the previous call's contents never leak into this one.
  return lbl_sort_lines(nu0, shift, gid, n_lines, mask_lo, mask_hi, p_max, scratch, NOALLOC_SCRATCH_BYTES,
                        order, n_kept, max_shift_bound, stream);
}

// ---------------------------------------------------------------------------
// Jacobian coefficients (no reference counterpart; the retrieval adjoint).
//
// With u = Re w(z), u_x = Re w'(z), u_y = -Im w'(z) (w' = -2 z w + 2i/sqrt(pi)) and
// amp = S sqrt(ln2/pi)/alpha_D, one line's contribution to a layer's optical depth
// (before the radiation factor R(nu, T)) is amp * u and its derivatives are
//   d/dT      = jT_u u - jT_x x u_x - jT_y u_y
//   d/dlnVMR  = jv_u u + jv_y u_y - jv_x u_x        (lines of the chosen gas only)
// with, per (layer, line),
//   jT_u = amp (dlnS/dT - 1/(2T)),  jT_x = amp/(2T),  jT_y = amp y (1/(2T) + n_air/T),
//   jv_u = amp (1 - dlnR(nuc)/dnuc * c_v),  jv_y = amp s dgamma/dlnVMR,  jv_x = amp s c_v,
// where s = sqrt(ln2)/alpha_D, c_v = dnuc/dlnVMR = -shift p_self,
//   dgamma/dlnVMR = (296/T)^n_air (g_self - g_air) p_self,
//   dlnS/dT = -Q'(T)/Q(T) + c2 E''/T^2 - (c2 nu0/T^2)/(exp(c2 nu0/T) - 1) + (2v/T)/sinh(2v),
//   v = c2 nuc/(2T)  (the last term is -dlnR(nuc, T)/dT), dlnR(nu)/dnu = 1/nu + (c2/T)/sinh(2v).
// They follow from differentiating the expressions of pylblrtm/forward.py:257-292
// (alpha_D scales as sqrt(T), gamma as T^-n_air, the column as the VMR).

// d ln Q / dT of np.interp's piecewise-linear table (0 where clamped).
__device__ double interp_dlog(double x, const double* __restrict__ xp, const double* __restrict__ fp, int n) {
  if (isnan(x) || n < 2 || x >= xp[n - 1] || x < xp[0]) return 0.0;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (xp[mid] <= x) lo = mid; else hi = mid;
  }
  const double slope = (fp[lo + 1] - fp[lo]) / (xp[lo + 1] - xp[lo]);
  return slope / interp_clamped(x, xp, fp, n);
}

__global__ void layer_groups_dlnq_kernel(const LayerGroup* __restrict__ lg, int n_rows, int n_grp,
                                         const int* __restrict__ tips_off, const int* __restrict__ tips_len,
                                         const double* __restrict__ tips_t, const double* __restrict__ tips_q,
                                         double* __restrict__ dlnq) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_rows * n_grp) return;
  const int g = (int)(idx % n_grp);
  dlnq[idx] = interp_dlog(lg[idx].T, tips_t + tips_off[g], tips_q + tips_off[g], tips_len[g]);
}

__global__ void line_prep_jac_kernel(const LineIn* __restrict__ lines, int n_lines, const LayerGroup* __restrict__ lg,
                                     const double* __restrict__ dlnq, int n_rows, int n_grp, int jac_grp_mask,
                                     LineJac* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (j >= n_lines || row >= n_rows) return;
  const LineIn L = lines[j];
  LineJac r = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (L.src < 0) {                                   // inactive slot of lbl_gather_lines
    out[(long long)row * n_lines + j] = r;
    return;
  }
  const long long gi = (long long)row * n_grp + L.gid;
  const LayerGroup G = lg[gi];
  const ScaledLine s = scale_line(L, G, nullptr, 0);
  if (s.active) {
    const double T = G.T;
    const double amp = VOIGT_K / s.alpha * s.S;
    const double sc = SQRT_LN2 / s.alpha;
    const double y = sc * s.gamma;
    const double a = C2 * L.nu0 / T;
    const double v = 0.5 * C2 * s.nuc / T;
    const double dlnS = -dlnq[gi] + C2 * L.elow / (T * T) - (a / T) / expm1(a) + (2.0 * v / T) / sinh(2.0 * v);
    r.jT_u = (float)(amp * (dlnS - 0.5 / T));
    r.jT_x = (float)(amp * 0.5 / T);
    r.jT_y = (float)(amp * y * (0.5 / T + L.n_air / T));
    if ((jac_grp_mask >> L.gid) & 1) {
      const double c_v = -L.shift * G.p_self;
      const double dlnR_dnu = 1.0 / s.nuc + (C2 / T) / sinh(2.0 * v);
      const double dgamma = pow(T_REF / T, L.n_air) * (L.g_self - L.g_air) * G.p_self;
      r.jv_u = (float)(amp * (1.0 - dlnR_dnu * c_v));
      r.jv_y = (float)(amp * sc * dgamma);
      r.jv_x = (float)(amp * sc * c_v);
    }
  }
  out[(long long)row * n_lines + j] = r;
}

extern "C" int lbl_line_prep_jac(const LineIn* lines, int n_lines, const LayerGroup* lg, int n_rows, int n_grp,
                                 const int* tips_off, const int* tips_len, const double* tips_t,
                                 const double* tips_q, int jac_grp_mask, double* dlnq_scratch, LineJac* out,
                                 void* stream) {
  if (n_lines < 1 || n_rows < 1 || n_rows > 65535 || n_grp < 1 || n_grp > 31 || !lines || !lg || !out ||
      !dlnq_scratch || !tips_off || !tips_len || !tips_t || !tips_q)
    return lbl_set_error(LBL_EINVAL, "lbl_line_prep_jac: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)n_rows * n_grp;
  layer_groups_dlnq_kernel<<<grid1(n, 128), 128, 0, st>>>(lg, n_rows, n_grp, tips_off, tips_len, tips_t, tips_q,
                                                           dlnq_scratch);
  dim3 grid(grid1(n_lines, 128), n_rows);
  line_prep_jac_kernel<<<grid, 128, 0, st>>>(lines, n_lines, lg, dlnq_scratch, n_rows, n_grp, jac_grp_mask, out);
  return lbl_check_launch("lbl_line_prep_jac");
}
