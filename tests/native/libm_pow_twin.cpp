// Host build of the library's device pow (mycel_b200/csrc/libm_pow.h) for the CPU tests: the same operation
// sequence compiled for the CPU, compared there with the C library's pow.
#include <stdint.h>

#include "../../mycel_b200/csrc/libm_pow.h"

extern "C" void twin_pow(int64_t n, const double* x, const double* y, int64_t y_len, double* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = mycel::libm_pow::pow(x[i], y[y_len == 1 ? 0 : i]);
}
