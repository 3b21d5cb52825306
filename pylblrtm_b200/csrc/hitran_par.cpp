// Host parser of HITRAN-2004 .par text (liblblio.so) with the semantics of the
// reference's reader, pylblrtm/hitran_manager.py:816-872 (par_to_dict):
//   * the text is split into lines like Python's universal newlines (\r\n, \r, \n);
//   * a line shorter than 155 characters is skipped;
//   * fields are taken by character position: mol_id [0,2) and iso_id [2,3) as Python
//     int(), nu0 [3,15), Sref [15,25), g_air [35,40), g_self [40,45), Elow [45,55),
//     n_air [55,59), shift [59,67) as Python float(), in that order; the first field
//     that does not convert stops the line (the reference has appended the fields
//     before it, so its columns can differ in length).
// Number syntax is Python's for ASCII text: surrounding whitespace (space, \t, \n, \v,
// \f, \r), an optional sign, digits with single underscores between digits,
// an optional fraction and exponent, or inf / infinity / nan in any case. Conversion
// is correctly rounded (glibc strtod on the validated digits). A line with a byte
// >= 0x80 is reported as LBL_PAR_NONASCII and left to the caller, because Python
// counts and slices such a line by decoded characters.
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/lblio.h"

namespace {

inline bool py_space(unsigned char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

inline bool is_digit(unsigned char c) { return c >= '0' && c <= '9'; }

// Trim Python whitespace; returns false for an empty result.
inline bool trim(const char*& s, const char*& e) {
  while (s < e && py_space((unsigned char)*s)) ++s;
  while (e > s && py_space((unsigned char)e[-1])) --e;
  return s < e;
}

// Copies digits of a digit run allowing single underscores between digits; returns the
// position after the run or nullptr on a misplaced underscore. Requires >= 1 digit.
inline const char* digit_run(const char* p, const char* e, char*& out, int& n_digits) {
  n_digits = 0;
  bool prev_digit = false;
  while (p < e) {
    const unsigned char c = (unsigned char)*p;
    if (is_digit(c)) {
      *out++ = (char)c;
      ++n_digits;
      prev_digit = true;
      ++p;
    } else if (c == '_') {
      if (!prev_digit || p + 1 >= e || !is_digit((unsigned char)p[1])) return nullptr;
      prev_digit = false;
      ++p;
    } else {
      break;
    }
  }
  return p;
}

inline bool ieq(const char* s, const char* e, const char* word) {
  const size_t n = strlen(word);
  if ((size_t)(e - s) != n) return false;
  for (size_t i = 0; i < n; ++i) {
    char c = s[i];
    if (c >= 'A' && c <= 'Z') c = (char)(c - 'A' + 'a');
    if (c != word[i]) return false;
  }
  return true;
}

bool py_float(const char* s, const char* e, double* out) {
  if (!trim(s, e)) return false;
  char buf[96];
  if (e - s > 80) return false;   // fields here are at most 12 characters
  char* o = buf;
  const char* p = s;
  if (*p == '+' || *p == '-') *o++ = *p++;
  if (p < e && !is_digit((unsigned char)*p) && *p != '.') {
    // inf / infinity / nan
    if (ieq(p, e, "inf") || ieq(p, e, "infinity")) {
      *out = (buf[0] == '-') ? -HUGE_VAL : HUGE_VAL;
      return true;
    }
    if (ieq(p, e, "nan")) {
      *out = (buf[0] == '-') ? -NAN : NAN;
      return true;
    }
    return false;
  }
  int nd_int = 0, nd_frac = 0;
  if (p < e && is_digit((unsigned char)*p)) {
    p = digit_run(p, e, o, nd_int);
    if (!p) return false;
  }
  if (p < e && *p == '.') {
    *o++ = *p++;
    if (p < e && is_digit((unsigned char)*p)) {
      p = digit_run(p, e, o, nd_frac);
      if (!p) return false;
    }
  }
  if (nd_int + nd_frac == 0) return false;
  if (p < e && (*p == 'e' || *p == 'E')) {
    *o++ = 'e';
    ++p;
    if (p < e && (*p == '+' || *p == '-')) *o++ = *p++;
    int nd_exp = 0;
    if (p >= e || !is_digit((unsigned char)*p)) return false;
    p = digit_run(p, e, o, nd_exp);
    if (!p) return false;
  }
  if (p != e) return false;
  *o = '\0';
  *out = strtod(buf, nullptr);
  return true;
}

bool py_int(const char* s, const char* e, int* out) {
  if (!trim(s, e)) return false;
  bool neg = false;
  if (*s == '+' || *s == '-') {
    neg = *s == '-';
    ++s;
  }
  if (s >= e || !is_digit((unsigned char)*s)) return false;
  char buf[32];
  char* o = buf;
  int nd = 0;
  if (e - s > 20) return false;
  const char* p = digit_run(s, e, o, nd);
  if (!p || p != e) return false;
  *o = '\0';
  const long long v = strtoll(buf, nullptr, 10);
  if (v > 2147483647LL) return false;
  *out = neg ? (int)-v : (int)v;
  return true;
}

// Next line [s, e) of the text and the start of the following one.
inline const char* next_line(const char* p, const char* end, const char** line_end) {
  const char* q = p;
  while (q < end && *q != '\n' && *q != '\r') ++q;
  *line_end = q;
  if (q < end && *q == '\r' && q + 1 < end && q[1] == '\n') return q + 2;
  return q < end ? q + 1 : q;
}

}  // namespace

extern "C" long long lbl_par_count_lines(const char* text, long long len) {
  if (!text || len <= 0) return 0;
  const char* p = text;
  const char* end = text + len;
  long long n = 0;
  while (p < end) {
    const char* le;
    p = next_line(p, end, &le);
    ++n;
  }
  return n;
}

extern "C" int lbl_par_parse(const char* text, long long len, long long cap, double* values, int* ids,
                             signed char* status) {
  if (!text || len < 0 || cap < 0 || (cap > 0 && (!values || !ids || !status))) return LBL_EINVAL;
  const char* p = text;
  const char* end = text + len;
  long long i = 0;
  static const int F_START[7] = {3, 15, 35, 40, 45, 55, 59};
  static const int F_END[7] = {15, 25, 40, 45, 55, 59, 67};
  while (p < end) {
    if (i >= cap) return LBL_EINVAL;
    const char* le;
    const char* s = p;
    p = next_line(p, end, &le);
    const long long n = le - s;
    bool ascii = true;
    for (const char* c = s; c < le; ++c)
      if ((unsigned char)*c >= 0x80) {
        ascii = false;
        break;
      }
    double* v = values + 7 * i;
    int* id = ids + 2 * i;
    if (!ascii) {
      status[i++] = LBL_PAR_NONASCII;
      continue;
    }
    if (n < 155) {
      status[i++] = LBL_PAR_SHORT;
      continue;
    }
    int k = 0;
    if (py_int(s, s + 2, &id[0])) {
      k = 1;
      if (py_int(s + 2, s + 3, &id[1])) {
        k = 2;
        for (int f = 0; f < 7; ++f) {
          if (!py_float(s + F_START[f], s + F_END[f], &v[f])) break;
          ++k;
        }
      }
    }
    status[i++] = (signed char)k;
  }
  return i == cap ? LBL_OK : LBL_EINVAL;
}
