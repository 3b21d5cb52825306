/*
 * lblio.h — C ABI of the host-side helpers (liblblio.so; no CUDA): the HITRAN text
 * reader and the line-list group scan.
 *
 * Replaces the line loop of pylblrtm/hitran_manager.py:816-872 (par_to_dict) with the
 * same semantics (see pylblrtm_b200/csrc/hitran_par.cpp); the Python layer
 * (pylblrtm_b200/hitran_io.py) assembles the reference's columns, warnings and errors.
 * All pointers are HOST memory.
 */
#ifndef LBLIO_H
#define LBLIO_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef LBL_OK
#define LBL_OK 0
#endif
#ifndef LBL_EINVAL
#define LBL_EINVAL 1
#endif

/* per-line status values besides 0..9 (= number of fields converted, in the order
 * mol_id, iso_id, nu0, Sref, g_air, g_self, Elow, n_air, shift) */
#define LBL_PAR_SHORT (-1)     /* fewer than 155 characters: skipped */
#define LBL_PAR_NONASCII (-2)  /* contains a byte >= 0x80: the caller decodes and parses it */

/* Number of lines of `text` under Python's universal-newline rule (\r\n, \r, \n). */
long long lbl_par_count_lines(const char* text, long long len);

/* Parse every line: values [n, 7] (nu0, Sref, g_air, g_self, Elow, n_air, shift),
 * ids [n, 2] (mol_id, iso_id), status [n]; cap must equal lbl_par_count_lines. */
int lbl_par_parse(const char* text, long long len, long long cap, double* values, int* ids,
                  signed char* status);

/* Group scan of the line list (replaces the pair discovery and band-mask counts of
 * pylblrtm/forward.py:189-245): distinct (mol, iso) pairs in first-seen order
 * (pair_mol, pair_iso [max_pairs]), the number of lines of each inside the band
 * mask nu0 in [(nu_first - cutoff) - |shift| p_max, (nu_last + cutoff) + |shift| p_max]
 * with lo_edge = nu_first - cutoff and hi_edge = nu_last + cutoff (pair_band), their
 * count (n_pairs), every line's pair (pair_index [n]) and the largest finite |shift|
 * (*max_abs_shift; -1 when there is none). LBL_EINVAL when more than max_pairs pairs
 * occur. */
int lbl_line_pairs(const int* mol, const int* iso, const double* nu0, const double* shift, long long n,
                   double lo_edge, double hi_edge, double p_max, int max_pairs, int* pair_mol, int* pair_iso,
                   long long* pair_band, int* n_pairs, int* pair_index, double* max_abs_shift);

/* out[i] = lut[index[i]] for i < n (the group index of every line from its pair index
 * and the pair -> group table of the group selection); LBL_EINVAL for an index outside
 * [0, n_lut). */
int lbl_map_index(const int* index, long long n, const int* lut, int n_lut, int* out);

/* Number of lines that lbl_sort_lines (lblgpu.h) keeps for these band edges: gid >= 0
 * and finite nu0 in [lo_edge - |shift| p_max, hi_edge + |shift| p_max], compared in the
 * same order as the device (the same count). No reference counterpart: it sizes the
 * buffers of a wavenumber shard, whose band edges are narrowed to the shard's lines,
 * before the device has counted. -1 for bad arguments. */
long long lbl_count_band(const double* nu0, const double* shift, const int* gid, long long n, double lo_edge,
                         double hi_edge, double p_max);

#ifdef __cplusplus
}
#endif

#endif /* LBLIO_H */
