/*
 * lblgpu.h — C ABI of the B200 line-by-line transmittance engine (liblblgpu.so).
 *
 * Every entry point takes DEVICE pointers (except where noted), sizes, scalars
 * and a cudaStream_t passed as void*, enqueues its kernels on that stream and
 * returns a status code; nothing allocates and nothing synchronises. Buffers
 * written by one call are read by the next on the same stream. Errors found by
 * kernels (non-finite or negative line strengths, non-finite optical depth) are
 * reported through an int error word in device memory that the caller
 * initialises to INT_MAX and reads after synchronising: it receives the
 * smallest key  row * (n_grp + 1) + g  (g = group index, g = n_grp for the
 * optical-depth check), i.e. the first failure in the reference's loop order.
 *
 * The reference (PyLBLRTM 0.1.2) is pure Python; each entry point names the
 * reference code it replaces. The Python host layer (pylblrtm_b200) binds these
 * symbols with ctypes and keeps the reference's public API on top.
 */
#ifndef LBLGPU_H
#define LBLGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* flags of the multi-level summation and Jacobian kernels */
#define LBL_DETERMINISTIC 1   /* bit-reproducible near-zone sums (fixed order; ~10-15 % slower) */

/* status codes */
#define LBL_OK 0
#define LBL_EINVAL 1    /* bad argument (message in lbl_last_error) */
#define LBL_ECUDA 2     /* CUDA launch / runtime error */

/* ---- records exchanged between the stages (layouts fixed, 8-byte aligned) ---- */

/* Per (profile-layer, line group): forward.py:236-259, 292. */
typedef struct {
  double T, p_self, p_air, col, q_ratio, dop; /* dop = sqrt(T / molar_mass) */
} LayerGroup;

/* One line after the candidate sort (input parameters + group + input index). */
typedef struct {
  double nu0, sref, g_air, g_self, elow, n_air, shift;
  int gid, src;
} LineIn;

/* Prepared line for the float64 summation. nuc = NaN marks an inactive line. */
typedef struct {
  double nuc, inv_ad, y, amp;
} LineF64;

/* Prepared line for the float32 summation (integer grid index + remainder). */
typedef struct {
  double nuc;
  int j0;
  float b, a, y, amp, amp_far;
} LineF32;

/* Jacobian coefficients of one prepared line (see lbl_line_prep_jac). */
typedef struct {
  float jT_u, jT_x, jT_y, jv_u, jv_y, jv_x, pad0, pad1;
} LineJac;

/* Last error message of the calling thread ("" if none). */
const char* lbl_last_error(void);
/* ABI version of this library. */
int lbl_abi_version(void);

/* Layers from levels; replaces pylblrtm/atmosphere.py:110-141
 * (AtmosphericProfile.build_layers) for a batch of profiles.
 * p_hpa, t_k: [n_prof, n_lev]; vmr: [n_prof, n_gas, n_lev];
 * p_atm, t_layer: [n_prof, n_lev-1]; vmr_layer, col: [n_prof, n_gas, n_lev-1].
 * col_factor = AVOGADRO / (GRAVITY * M_DRY_AIR) (atmosphere.py:134). */
int lbl_build_layers(const double* p_hpa, const double* t_k, const double* vmr, int n_prof, int n_lev,
                     int n_gas, double col_factor, double* p_atm, double* t_layer, double* vmr_layer,
                     double* col, void* stream);

/* Per (profile, layer, group) quantities with Q(296)/Q(T) interpolated from the
 * TIPS tables; replaces pylblrtm/forward.py:236-240 (with SpectralData.Q,
 * spectral_data.py:43-52) and forward.py:249-259. out: [n_prof*n_lay, n_grp].
 * grp_gas[g] indexes the gas axis of vmr_layer/col; tips_t/tips_q hold every
 * group's table back to back at tips_off[g], length tips_len[g]. */
int lbl_layer_groups(const double* t_layer, const double* p_atm, const double* vmr_layer, const double* col,
                     int n_prof, int n_lay, int n_gas, int n_grp, const int* grp_gas, const double* grp_mass,
                     const int* tips_off, const int* tips_len, const double* tips_t, const double* tips_q,
                     LayerGroup* out, void* stream);

/* Workspace bytes for lbl_sort_lines. */
size_t lbl_sort_workspace_bytes(int n_lines);

/* Selects the lines the reference masks in (forward.py:189-220: valid group,
 * nu0 in [mask_lo - |shift| p_max, mask_hi + |shift| p_max] with
 * mask_lo = nu[0] - cutoff, mask_hi = nu[-1] + cutoff) and sorts them by nu0
 * (ties by input index). gid[i] < 0 drops line i. Writes the input indices in
 * sorted order to order[0 .. *n_kept), the count to *n_kept and the largest
 * |shift| p_max of a kept line to *max_shift_bound (all device memory). */
int lbl_sort_lines(const double* nu0, const double* shift, const int* gid, int n_lines, double mask_lo,
                   double mask_hi, double p_max, void* workspace, size_t workspace_bytes, int* order,
                   int* n_kept, double* max_shift_bound, void* stream);

/* Same as lbl_sort_lines without caller-provided workspace, for callers that
 * cannot allocate device memory when they run (for example a host application
 * whose memory pool owns the whole GPU and forbids further cudaMalloc calls).
 * No counterpart in the reference. The scratch is a static device array inside
 * the library (3 MiB on every GPU that loads it, held until the process exits),
 * so n_lines may not exceed 262,144 (LBL_EINVAL otherwise). The first call in a
 * CUDA context looks up the array's device address (cudaGetSymbolAddress) with
 * that context's device current and caches it under the context's unique id
 * (cuCtxGetId), so a cudaDeviceReset or another context current on the thread
 * gets a fresh lookup instead of a stale address; make the first call in each
 * context before any stream capture. All calls
 * share the one array: calls that overlap on the GPU (different streams, or
 * threads on one device) race and must be serialised by the caller. Allocates
 * nothing; same outputs as lbl_sort_lines. */
int lbl_sort_lines_noalloc(const double* nu0, const double* shift, const int* gid, int n_lines, double mask_lo,
                           double mask_hi, double p_max, int* order, int* n_kept, double* max_shift_bound,
                           void* stream);

/* Gathers the sorted lines into LineIn records (out[0 .. *n_kept)). n_lines is the
 * record count of out and may exceed the device count *n_kept (a bound the caller
 * knows on the host, so nothing waits for the count): slots *n_kept .. n_lines-1
 * receive inactive records (nu0 = NaN, gid = 0, src = -1) that no tile range holds. */
int lbl_gather_lines(const double* nu0, const double* sref, const double* g_air, const double* g_self,
                     const double* elow, const double* n_air, const double* shift, const int* gid,
                     const int* order, const int* n_kept, int n_lines, LineIn* out, void* stream);

/* Candidate line range [ranges[2t], ranges[2t+1]) of each reference tile of
 * tile_samples grid points: lines whose unshifted centre is within
 * cutoff + pad of the tile (pad >= the largest pressure shift). The exact
 * window test of forward.py:295-301 runs inside the summation kernels. */
int lbl_tile_ranges(const LineIn* lines, const int* n_kept, double nu_min, double step, long long n_nu,
                    int tile_samples, double cutoff, double pad, int n_tiles, int* ranges, void* stream);

/* Per (row = profile-layer, sorted line) HITRAN scaling; replaces
 * pylblrtm/forward.py:257-292 (strength with column and 1/R(nuc), Lorentz and
 * Doppler widths, pressure shift). out: [n_rows, n_lines]. */
int lbl_line_prep_f64(const LineIn* lines, const int* n_kept, int n_lines, const LayerGroup* lg, int n_rows,
                      int n_grp, LineF64* out, int* err, void* stream);
int lbl_line_prep_f32(const LineIn* lines, const int* n_kept, int n_lines, const LayerGroup* lg, int n_rows,
                      int n_grp, double nu_min, double step, LineF32* out, int* err, void* stream);

/* Per (row, sorted line) coefficients of the layer Jacobians d od / dT_layer and
 * d od / d ln VMR_layer (no reference counterpart: the retrieval adjoint). They
 * differentiate the expressions of pylblrtm/forward.py:257-292. jac_grp_mask has
 * bit g set for the groups of the gas whose VMR is differentiated; dlnq_scratch
 * holds n_rows * n_grp doubles (d ln Q / dT). */
int lbl_line_prep_jac(const LineIn* lines, int n_lines, const LayerGroup* lg, int n_rows, int n_grp,
                      const int* tips_off, const int* tips_len, const double* tips_t, const double* tips_q,
                      int jac_grp_mask, double* dlnq_scratch, LineJac* out, void* stream);

/* Optical depth of every (row, grid point): the Voigt sum over the lines of
 * the point's reference tile window, times R(nu, T_row); replaces
 * pylblrtm/forward.py:295-315 (tile loop, _voigt, phi @ S, radiation term and
 * its finiteness check). od: [n_rows, n_nu]. evals (nullable, u64) receives
 * the number of (row, point, line) evaluations admitted by the tile rule.
 * _f64: float64 throughout (Gautschi-type Faddeeva). _f32: float32 Faddeeva
 * with the asymptotic far-wing branch and compensated sums. */
int lbl_tau_tiles_f64(const LineF64* prep, int n_lines, const int* ranges, const double* t_layer, int n_rows,
                      double nu_min, double step, long long n_nu, int tile_samples, double cutoff, int n_grp,
                      double* od, int* err, unsigned long long* evals, void* stream);
int lbl_tau_tiles_f32(const LineF32* prep, int n_lines, const int* ranges, const double* t_layer, int n_rows,
                      double nu_min, double step, long long n_nu, int tile_samples, double cutoff, int n_grp,
                      float* od, int* err, unsigned long long* evals, void* stream);

/* Inner-line range [inner[2t], inner[2t+1]) of each reference tile for
 * lbl_tau_tiles_ml_f32: the lines that can lie within one chunk half-width of a
 * chunk of the tile (same candidate search as lbl_tile_ranges, narrower reach;
 * pad as there). No reference counterpart: an index of the summation. */
int lbl_ml_inner_ranges(const LineIn* lines, const int* n_kept, double nu_min, double step, long long n_nu,
                        int tile_samples, double pad, int n_tiles, int* inner, void* stream);

/* Same contract as lbl_tau_tiles_f32, multi-level float32 summation (the
 * default float32 engine): per chunk (<= 2048 points of one reference tile),
 * lines farther than a chunk half-width contribute through 16 Chebyshev nodes over
 * the chunk (8 beyond four half-widths; a line-per-thread kernel that runs first and
 * leaves the chunk's coefficients in l1_work), the remaining lines farther than a
 * 256-point sub-chunk half-width through 16 nodes over that sub-chunk, the rest
 * directly; one warp per sub-chunk does levels 2 and 3. inner (nullable; from
 * lbl_ml_inner_ranges with the ranges' lines and pad) limits the second kernel to the
 * lines that can be inner; NULL scans every candidate of the tile (same results,
 * slower). l1_work: lbl_ml_work_floats floats of device memory (required). evals
 * counts reference-rule evaluations; work (nullable, 3 x u64) receives the
 * evaluations actually performed: [0] Chebyshev-node evaluations, [1] level-3
 * loop evaluations, [2] near-zone points. flags: LBL_DETERMINISTIC adds the
 * near-zone corrections in a fixed order (bit-reproducible across launches and
 * batchings); without it overlapping near zones are summed by shared-memory
 * atomics (reproducible to ~1e-9 relative). n_nu <= 1.5e9. Only the reference
 * tiles [tile_first, tile_first + tile_count) of the grid are computed (all of
 * them: 0 and ceil(n_nu / tile_samples)); od is then [n_rows, n_local] with the
 * tiles' n_local points, grid values staying nu_min + i*step of the full grid (a
 * wavenumber shard gives bit-identical results). Replaces pylblrtm/forward.py:295-315. */
int lbl_tau_tiles_ml_f32(const LineF32* prep, int n_lines, const int* ranges, const int* inner, float* l1_work,
                         const double* t_layer, int n_rows, double nu_min, double step, long long n_nu,
                         int tile_samples, double cutoff, int n_grp, float* od, int* err, unsigned long long* evals,
                         unsigned long long* work, int tile_first, int tile_count, int flags, void* stream);

/* Floats of the l1_work buffer of lbl_tau_tiles_ml_f32 for tile_count reference tiles
 * (16 + 8 level-1 coefficients per chunk and row); -1 for bad arguments. No reference
 * counterpart: a workspace of the summation. */
long long lbl_ml_work_floats(int n_rows, int tile_samples, int tile_count);

/* Layer Jacobians by the multi-level float32 summation (no reference
 * counterpart; the retrieval adjoint): writes od (as lbl_tau_tiles_ml_f32),
 * d_t = d od / dT_layer and d_v = d od / d ln VMR_layer of the gas chosen in
 * lbl_line_prep_jac, all [n_rows, n_nu] (rows = n_prof * n_lay). Since layer k's
 * T and VMR enter only od_k, these are the full per-layer Jacobians of
 * tau = sum_k od_k. With g_tau ([n_prof, n_nu] float64, d loss / d tau) the
 * kernel writes nothing per point and instead adds sum_p g_tau * d_t (d_v) into
 * vjp_t[row] (vjp_v[row]) (caller zeroes them): the vector-Jacobian product,
 * recomputing every Voigt value instead of storing the Jacobian (its per-row
 * sums use global atomics). flags: LBL_DETERMINISTIC as for lbl_tau_tiles_ml_f32.
 * Level 1 runs first as a line-per-thread kernel that leaves its Chebyshev
 * coefficients in l1_work (lbl_jacobian_ml_work_floats floats, required); inner
 * (nullable) are the ranges of lbl_ml_inner_ranges for the same grid, a superset of
 * the inner lines of this kernel's smaller chunks; near (nullable) those of
 * lbl_jac_near_ranges, which limit the level-1 pass over lines within four chunk
 * half-widths. NULL scans every candidate (same results, slower). */
int lbl_jacobian_ml_f32(const LineF32* prep, const LineJac* jprep, int n_lines, const int* ranges, const int* inner,
                        const int* near, const double* t_layer, int n_rows, int n_lay, double nu_min, double step, long long n_nu,
                        int tile_samples, double cutoff, float* l1_work, float* od, float* d_t, float* d_v,
                        const double* g_tau, double* vjp_t, double* vjp_v, int flags, void* stream);

/* Per-tile candidate range [near[2t], near[2t+1]) of the level-1 lines of
 * lbl_jacobian_ml_f32 that lie within four chunk half-widths of a chunk (same search as
 * lbl_tile_ranges, pad as there). No reference counterpart: an index of the summation. */
int lbl_jac_near_ranges(const LineIn* lines, const int* n_kept, double nu_min, double step, long long n_nu,
                        int tile_samples, double pad, int n_tiles, int* near, void* stream);

/* Floats of the l1_work buffer lbl_jacobian_ml_f32 needs (level-1 Chebyshev
 * coefficients per chunk and row); -1 for bad arguments. */
long long lbl_jacobian_ml_work_floats(int n_rows, long long n_nu, int tile_samples);

/* Column sums over layers and transmittance exp(-tau / mu); replaces
 * pylblrtm/forward.py:151 and config.py:266-270. od: [n_prof, n_lay, n_nu]
 * (float32 or float64); trans, tau (each nullable): [n_prof, n_nu] float64;
 * mu: [n_prof] device array of view cosines (mu_view). */
int lbl_layer_sum_exp_f32(const float* od, int n_prof, int n_lay, long long n_nu, const double* mu,
                          double* trans, double* tau, void* stream);
int lbl_layer_sum_exp_f64(const double* od, int n_prof, int n_lay, long long n_nu, const double* mu,
                          double* trans, double* tau, void* stream);

/* Channel box-average of the transmittance (no reference counterpart; serves
 * channel-averaged retrievals and the surrogate's training targets): out[b, c] =
 * mean over p in [first + c*width, first + (c+1)*width) of
 * exp(-sum_k od[b, k, p] / mu[b]); od [n_prof, n_lay, n_nu], mu [n_prof] and
 * out [n_prof, n_ch] in device memory. */
int lbl_channel_mean_f32(const float* od, int n_prof, int n_lay, long long n_nu, const double* mu, long long first,
                         int width, int n_ch, double* out, void* stream);
int lbl_channel_mean_f64(const double* od, int n_prof, int n_lay, long long n_nu, const double* mu, long long first,
                         int width, int n_ch, double* out, void* stream);

/* Faddeeva function on arrays (diagnostics; replaces the scipy.special.wofz call
 * at forward.py:62). mode 0: general algorithm; mode 1 (f32 only): the
 * engine's real part with the far-wing branch (im not written). */
int lbl_faddeeva_f64(const double* x, const double* y, long long n, double* re, double* im, void* stream);
int lbl_faddeeva_f32(const float* x, const float* y, long long n, float* re, float* im, int mode,
                     void* stream);

/* ---- surrogate network (no reference counterpart) ----
 * The channel-transmittance surrogate (an MLP trained on this engine's own spectra)
 * runs on one BF16 tensor-core GEMM, D[M, N] = A[M, K] . B[N, K]^T with A and B
 * row-major bf16 (K contiguous) and float32 accumulation, whose epilogue is one of: */
#define LBL_GEMM_F32 0          /* out_f32[z][m, n] = D (split z of n_split; partials summed by the consumer) */
#define LBL_GEMM_BIAS_GELU 1    /* z = D + bias -> z_out (bf16); gelu(z) -> y and y_t (bf16) */
#define LBL_GEMM_BIAS_SIGMOID 2 /* p = sigmoid(D + bias) -> out_f32; with target: dz = grad_scale * 2 (p - t) p (1 - p)
                                   -> y and y_t (bf16, zero for n >= n_valid) and sum (p - t)^2 -> *loss */
#define LBL_GEMM_DGELU 3        /* dz = D * gelu'(z_in) -> y and y_t (bf16) */

/* Epilogue operands of lbl_gemm_bf16 (device pointers; NULL skips an optional output).
 * Leading dimensions are in elements; y_t is written transposed ([N, M] row-major). */
typedef struct {
  int mode;
  int n_valid;                  /* SIGMOID: columns >= n_valid are padding */
  const float* bias;            /* [N], 16-byte aligned */
  float* out_f32;               /* [M, ld_f32] (per split for LBL_GEMM_F32) */
  long long ld_f32;
  long long split_stride;       /* elements between split partials */
  void* z_out;                  /* bf16 [M, ld_z] */
  long long ld_z;
  const void* z_in;             /* bf16 [M, ld_zin] */
  long long ld_zin;
  void* y;                      /* bf16 [M, ld_y] */
  long long ld_y;
  void* y_t;                    /* bf16 [N, ld_yt] */
  long long ld_yt;
  const float* target;          /* [M, ld_target] */
  long long ld_target;
  float grad_scale;
  int pad0;
  double* loss;                 /* accumulated sum of squared errors */
} LblGemmEpilogue;

/* Size of the opaque TMA descriptor (a CUtensorMap, 128 bytes). */
size_t lbl_tensor_map_bytes(void);
/* Encode (host call, no stream work) the TMA descriptor of a bf16 matrix [rows, cols]
 * with row stride ld elements, for use as operand A or B of lbl_gemm_bf16. map_out is
 * HOST memory of lbl_tensor_map_bytes(); base is device memory. rows must be a multiple
 * of 128 and cols of 64. */
int lbl_tensor_map_bf16(void* map_out, const void* base, long long rows, long long cols, long long ld);
/* D = A . B^T through the maps (host memory) of A [M, K] and B [N, K]; M and N
 * multiples of 128, K a multiple of 64 * n_split. err: device int raised to 1 if a
 * pipeline wait timed out (the CTA's tile is then not written). */
int lbl_gemm_bf16(const void* map_a, const void* map_b, int M, int N, int K, int n_split,
                  const LblGemmEpilogue* ep, int* err, void* stream);
/* Adam (bias-corrected, step >= 1) on float32 master weights w [rows, cols] (row stride
 * ld) with moments m, v; the gradient is the in-order sum of n_split partials of g.
 * Refreshes the bf16 copy w_bf16 [rows, ld] and its transpose wt_bf16 [cols, ld_t]
 * when non-NULL. */
int lbl_adam_step(float* w, float* m, float* v, const float* g, int n_split, long long split_stride, int rows,
                  int cols, int ld, float lr, float b1, float b2, float eps, int step, void* w_bf16, void* wt_bf16,
                  int ld_t, void* stream);
/* out[r] = sum_c x[r, c] of a bf16 matrix (bias gradients). */
int lbl_rowsum_bf16(const void* x, int rows, int cols, int ld, float* out, void* stream);
/* Standardised bf16 network inputs: x[b, c] = (raw[b, c] - mean[c]) * inv_std[c] for
 * c < cols, zero up to ld; the transposed copy x_t [ld, ld_t] when non-NULL. */
int lbl_pack_inputs_bf16(const float* raw, int rows, int cols, const float* mean, const float* inv_std, void* x,
                         int ld, void* x_t, int ld_t, void* stream);
/* Ensemble gate: for each sample b, mean[b, c] over the n_mem members' predictions
 * pred[m * member_stride + b * ld + c], est[b] = max_c of their standard deviation,
 * weighted by ch_scale[c] when ch_scale (device, [n_ch]) is not NULL, and
 * flag[b] = (scale * est[b] > gate). The weights and the gate come from a calibration
 * split (pylblrtm_b200.surrogate.calibrate_gate). */
int lbl_ensemble_gate(const float* pred, int n_mem, long long member_stride, int n_samples, int ld, int n_ch,
                      const float* ch_scale, float scale, float gate, float* mean, float* est, int* flag,
                      void* stream);

/* Measurement probe (no reference counterpart): `blocks` CTAs of 256 threads
 * each run 8 chains of `iters` dependent float32 FMAs, i.e.
 * blocks * 256 * 8 * iters * 2 flops; the caller times the launch. */
int lbl_probe_fma_f32(float* out, int iters, int blocks, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LBLGPU_H */
