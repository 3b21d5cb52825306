// Status plumbing of the C ABI: a per-thread last-error message.
#include <stdarg.h>
#include <stdio.h>

#include "lbl_common.cuh"

static thread_local char g_last_error[512] = "";

int lbl_set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int lbl_check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lbl_set_error(LBL_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return LBL_OK;
}

extern "C" const char* lbl_last_error(void) { return g_last_error; }

extern "C" int lbl_abi_version(void) { return 1; }
