/*
 * lblio.h — C ABI of the host-side HITRAN text reader (liblblio.so; no CUDA).
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

#ifdef __cplusplus
}
#endif

#endif /* LBLIO_H */
