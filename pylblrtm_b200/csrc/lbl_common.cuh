// Shared constants, record layouts and launch helpers of the line-by-line engine.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../include/lblgpu.h"

namespace lbl {

// Physical constants of the reference forward model (pylblrtm/forward.py:32-36).
constexpr double T_REF = 296.0;
constexpr double C2 = 1.4387752;            // second radiation constant [cm K]
constexpr double DOPPLER = 3.5810e-7;       // Doppler HWHM factor
constexpr double SQRT_LN2 = 0.83255461115769775635;   // sqrt(ln 2)
constexpr double VOIGT_K = 0.46971863934982566689;    // sqrt(ln 2 / pi)
// Hydrostatic constants (pylblrtm/atmosphere.py:15-18).
constexpr double P_STD_HPA = 1013.25;

// Grid point nu_i = nu_min + i * step, rounded exactly like the reference's
// nu_min + np.arange(n) * step (pylblrtm/forward.py:141-142).
__device__ __forceinline__ double grid_nu(double nu_min, double step, long long i) {
  return __dadd_rn(nu_min, __dmul_rn((double)i, step));
}

// Record the first failing (layer, group) position in reference loop order.
__device__ __forceinline__ void flag_error(int* err, int key) {
  if (err) atomicMin(err, key);
}

}  // namespace lbl

// Status plumbing of the C ABI (capi.cu).
int lbl_set_error(int code, const char* fmt, ...);
int lbl_check_launch(const char* what);
