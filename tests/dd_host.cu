// Host entry points over the double-word routines of gbskernels_b200/csrc/gbs_common.cuh
// (the same __host__ __device__ source the kernels inline), for the CPU test of
// their error bounds (tests/test_dd_bounds.py).  Each takes arrays of n operands,
// a double-word as (hi, lo) pairs, a complex double-word as (re.hi, re.lo, im.hi,
// im.lo).
#include "gbs_common.cuh"

using namespace gbsb;

extern "C" {
void t_dd_add(int n, const double* a, const double* b, double* out) {
  for (int i = 0; i < n; ++i) {
    const dd r = dd_add(dd{a[2 * i], a[2 * i + 1]}, dd{b[2 * i], b[2 * i + 1]});
    out[2 * i] = r.hi;
    out[2 * i + 1] = r.lo;
  }
}
void t_dd_add_d(int n, const double* a, const double* b, double* out) {
  for (int i = 0; i < n; ++i) {
    const dd r = dd_add_d(dd{a[2 * i], a[2 * i + 1]}, b[i]);
    out[2 * i] = r.hi;
    out[2 * i + 1] = r.lo;
  }
}
void t_dd_mul(int n, const double* a, const double* b, double* out) {
  for (int i = 0; i < n; ++i) {
    const dd r = dd_mul(dd{a[2 * i], a[2 * i + 1]}, dd{b[2 * i], b[2 * i + 1]});
    out[2 * i] = r.hi;
    out[2 * i + 1] = r.lo;
  }
}
// x / j as the certified Newton recurrence divides (per component): the quotient
// q = dd_div_d(x, j), the computed product q j and the computed residual x - q j;
// out holds (q, qj, r) as three double-words per operand.
void t_dd_div_resid(int n, const double* a, const double* j, double* out) {
  for (int i = 0; i < n; ++i) {
    const dd x{a[2 * i], a[2 * i + 1]};
    const dd q = dd_div_d(x, j[i]);
    const dd qj = dd_mul_d(q, j[i]);
    const dd r = dd_sub(x, qj);
    double* o = out + 6 * i;
    o[0] = q.hi; o[1] = q.lo; o[2] = qj.hi; o[3] = qj.lo; o[4] = r.hi; o[5] = r.lo;
  }
}
void t_ddc_mul(int n, const double* a, const double* b, double* out) {
  for (int i = 0; i < n; ++i) {
    const double* x = a + 4 * i;
    const double* y = b + 4 * i;
    const ddc r = ddc_mul(ddc{dd{x[0], x[1]}, dd{x[2], x[3]}}, ddc{dd{y[0], y[1]}, dd{y[2], y[3]}});
    out[4 * i] = r.re.hi;
    out[4 * i + 1] = r.re.lo;
    out[4 * i + 2] = r.im.hi;
    out[4 * i + 3] = r.im.lo;
  }
}
}
