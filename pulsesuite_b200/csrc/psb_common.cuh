// psb_common.cuh -- shared device helpers of the pulsesuite_b200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pulsesuite_b200.h"

namespace psb {

constexpr double kPi = 3.14159265358979323846;
constexpr double kEuler = 0.5772156649015329;

// Sets the thread-local error message (capi.cu) and returns `code`.
int set_error(int code, const char* fmt, ...);
// Checks the last CUDA launch/runtime error; returns PSB_OK or PSB_ERR_CUDA.
int check_cuda(const char* what);

// ---------------------------------------------------------------------------
// Bessel K0 as the reference evaluates it.
//
// The reference's K03 runs cik01 (Zhang & Jin) on numpy complex scalars with
// zero imaginary part; numpy divides such values as a * (1/b) and raises them
// to integer powers by binary exponentiation.  The functions below restate
// the method with that arithmetic (pulsesuite/PSTD3D/usefulsubs.py:1669-1820).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double np_div(double a, double b) { return a * (1.0 / b); }

__device__ __forceinline__ double np_powi(double a, int n) {
  if (n == 1) return a;
  if (n == 2) return a * a;
  if (n == 3) return a * (a * a);
  double aa = 1.0, p = a;
  int mask = 1;
  for (;;) {
    if (n & mask) aa = aa * p;
    mask <<= 1;
    if (n < mask) break;
    p = p * p;
  }
  return aa;
}

// I0(x), x > 0: power series up to 18, Hankel asymptotic series above with
// a_k = ((2k-1)!!)^2 / (k! 8^k) generated from the formula.
__device__ inline double bessel_i0(double x) {
  if (x <= 18.0) {
    double z2 = x * x, s = 1.0, cr = 1.0;
    for (int k = 1; k <= 50; ++k) {
      cr = np_div(__dmul_rn(__dmul_rn(0.25, cr), z2), (double)(k * k));
      s = __dadd_rn(s, cr);
      if (fabs(np_div(cr, s)) < 1e-15) break;
    }
    return s;
  }
  int k0 = x < 35.0 ? 12 : (x < 50.0 ? 9 : 7);
  double ca = np_div(exp(x), sqrt(2.0 * kPi * x));
  double zr = np_div(1.0, x), s = 1.0, ak = 1.0;
  for (int k = 1; k <= k0; ++k) {
    double odd = (double)(2 * k - 1);
    ak = ak * odd * odd / ((double)k * 8.0);
    s = __dadd_rn(s, __dmul_rn(ak, np_powi(zr, k)));
  }
  return ca * s;
}

// K0(x) of the reference's K03: series with harmonic weights up to 9, the
// I0*K0 asymptotic product above (b_k = [(2k-1)!!/(2k)!!] ((2k-1)!!)^2/4^k),
// 0 past 100.  __dmul_rn/__dadd_rn keep the compiler from fusing the
// products into FMAs, which would change the rounding the series amplifies.
__device__ inline double bessel_k0(double x) {
  if (x > 100.0) return 0.0;
  if (x <= 0.0) return 1e30;
  if (x <= 9.0) {
    double z2 = x * x;
    double ct = -log(0.5 * x) - kEuler;
    double w0 = 0.0, cr = 1.0, cs = 0.0, cw = 0.0;
    for (int k = 1; k <= 50; ++k) {
      w0 = w0 + 1.0 / (double)k;
      cr = __dmul_rn(np_div(__dmul_rn(0.25, cr), (double)(k * k)), z2);
      cs = __dadd_rn(cs, __dmul_rn(cr, w0 + ct));
      if (fabs(np_div(cs - cw, cs)) < 1e-15) break;
      cw = cs;
    }
    return ct + cs;
  }
  double cb = np_div(0.5, x);
  double zr2 = np_div(1.0, x * x), s = 1.0, ratio = 1.0, dfac = 1.0;
  for (int k = 1; k <= 10; ++k) {
    double odd = (double)(2 * k - 1);
    ratio = ratio * odd / (double)(2 * k);
    dfac = dfac * odd * odd / 4.0;
    s = __dadd_rn(s, __dmul_rn(__dmul_rn(ratio, dfac), np_powi(zr2, k)));
  }
  return np_div(cb * s, bessel_i0(x));
}

// The JIT-friendly K0 approximation the reference uses inside Vint
// (pulsesuite/PSTD3D/coulomb.py:38-66): 23 below 1e-10, a 19-term series
// with (1/k - gamma) weights below 2, bare asymptote above, 0 past 100.
__device__ inline double bessel_k0_crude(double x) {
  if (x > 100.0) return 0.0;
  if (x < 1e-10) return 23.0;
  if (x < 2.0) {
    double x2 = x * x;
    double result = -log(0.5 * x) - kEuler;
    double term = 1.0;
    for (int k = 1; k < 20; ++k) {
      term = __dmul_rn(__dmul_rn(term, 0.25), x2) / (double)(k * k);
      result = __dadd_rn(result, __dmul_rn(term, 1.0 / (double)k - kEuler));
      if (fabs(term) < 1e-15) break;
    }
    return result;
  }
  return sqrt(kPi / (2.0 * x)) * exp(-x);
}

// eps(q; n1D) of one table block at density n1d (coulomb.py:1185-1190).
__device__ __forceinline__ double eps1d(const double* __restrict__ blk, int nk, int q,
                                        double n1d) {
  double chie = blk[5 * nk + q], chih = blk[6 * nk + q];
  double qe = blk[7 * nk + q], qh = blk[8 * nk + q];
  double le = log(fabs((qe - kPi * n1d) / (qe + n1d)));
  double lh = log(fabs((qh - kPi * n1d) / (qh + n1d)));
  return (1.0 - __dmul_rn(__dmul_rn(chie, 2.0), le)) - __dmul_rn(__dmul_rn(chih, 2.0), lh);
}

// ---------------------------------------------------------------------------
// Block reductions (fixed tree: the result of a wire never depends on what
// other wires share the launch).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace psb
