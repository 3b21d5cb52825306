// One host pass over the line list for the group selection of pylblrtm/forward.py:189-245
// (liblblio.so): the distinct (mol_id, iso_id) pairs, how many lines of each fall inside
// the band mask of forward.py:190-191, and the pair index of every line. The band test
// is evaluated in the reference's operation order,
//     sb = |shift| * p_max;  in = (nu0 >= (nu_first - cutoff) - sb) & (nu0 <= (nu_last + cutoff) + sb)
// and this file is compiled with floating-point contraction off, so every comparison
// sees the same doubles as NumPy's.
#include <math.h>

#include "../../include/lblio.h"

extern "C" int lbl_line_pairs(const int* mol, const int* iso, const double* nu0, const double* shift, long long n,
                              double lo_edge, double hi_edge, double p_max, int max_pairs, int* pair_mol,
                              int* pair_iso, long long* pair_band, int* n_pairs, int* pair_index,
                              double* max_abs_shift) {
  if (n < 0 || max_pairs < 1 || !n_pairs || (n > 0 && (!mol || !iso || !nu0 || !shift || !pair_index)) ||
      !pair_mol || !pair_iso || !pair_band || !max_abs_shift)
    return LBL_EINVAL;
  int np_ = 0, last = -1;
  double smax = -1.0;                               // largest finite |shift| (-1: none)
  for (long long i = 0; i < n; ++i) {
    const int m = mol[i], s = iso[i];
    int k = last;
    if (k < 0 || pair_mol[k] != m || pair_iso[k] != s) {
      k = -1;
      for (int j = 0; j < np_; ++j)
        if (pair_mol[j] == m && pair_iso[j] == s) {
          k = j;
          break;
        }
      if (k < 0) {
        if (np_ >= max_pairs) return LBL_EINVAL;
        k = np_++;
        pair_mol[k] = m;
        pair_iso[k] = s;
        pair_band[k] = 0;
      }
      last = k;
    }
    pair_index[i] = k;
    const double as = fabs(shift[i]);
    if (isfinite(as) && as > smax) smax = as;
    const double sb = as * p_max;
    const double v = nu0[i];
    if ((v >= lo_edge - sb) & (v <= hi_edge + sb)) ++pair_band[k];
  }
  *n_pairs = np_;
  *max_abs_shift = smax;
  return LBL_OK;
}

extern "C" int lbl_map_index(const int* index, long long n, const int* lut, int n_lut, int* out) {
  if (n < 0 || n_lut < 0 || (n > 0 && (!index || !lut || !out))) return LBL_EINVAL;
  unsigned bad = 0;
  for (long long i = 0; i < n; ++i) {
    const int k = index[i];
    const bool ok = k >= 0 && k < n_lut;
    bad |= !ok;
    out[i] = lut[ok ? k : 0];
  }
  return bad ? LBL_EINVAL : LBL_OK;
}

// Host count of the lines the device sort keeps (lbl_sort_lines): gid >= 0, finite nu0
// inside [lo_edge - |shift| p_max, hi_edge + |shift| p_max], the same comparisons in the
// same order, so the count equals the device's. Sizes a wavenumber shard's buffers when
// the band edges are narrowed to the shard's line window.
extern "C" long long lbl_count_band(const double* nu0, const double* shift, const int* gid, long long n,
                                    double lo_edge, double hi_edge, double p_max) {
  if (n < 0 || (n > 0 && (!nu0 || !shift || !gid))) return -1;
  long long c = 0;
  for (long long i = 0; i < n; ++i) {
    if (gid[i] < 0) continue;
    const double sb = fabs(shift[i]) * p_max;
    const double v = nu0[i];
    c += isfinite(v) && (v >= lo_edge - sb) && (v <= hi_edge + sb);
  }
  return c;
}
