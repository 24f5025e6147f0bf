// Shared device definitions: storage layout, run constants and the exact
// arithmetic helpers used by the NEMOLite2D kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nemo {

// original/nemolite2d.f90:15-18
constexpr double kPi = 3.1415926535897932;
constexpr double kG = 9.80665;
constexpr double kOmega = 7.292116e-05;

// Storage of every 2-D field: one pitched array over ji in [-2, pitch-3],
// jj in [-1, jpj+1]; element (ji,jj) at base[(jj+1)*pitch + ji+2].  Fortran
// bounds (0:jpi,1:jpj) etc. are windows of it, so the C-grid staggering
// needs no per-field index arithmetic.  pitch is a multiple of 32 doubles,
// so rows start on 256-byte boundaries and every even ji starts a 16-byte
// pair; the pitch leaves room for the pair (jpi+1, jpi+2).
struct Layout {
  int jpi, jpj;
  long pitch;
  long rows;  // jpj + 3
  __host__ __device__ __forceinline__ long idx(int ji, int jj) const {
    return (long)(jj + 1) * pitch + (ji + 2);
  }
  __host__ __device__ long elems() const { return rows * pitch; }
};

inline long layout_pitch(int jpi) { return ((long)(jpi + 6) + 31) / 32 * 32; }

// Per-run constants.  The reference's grid is uniform (original/nemolite2d.f90
// :210-217): every e1* equals dx, every e2* equals dy, every e12* equals
// dx*dy.  Products, sums and sines are formed on the host exactly as the
// Fortran forms them, so device and host agree bit for bit.
struct Consts {
  double e1t, e2t, e1u, e2u, e1v, e2v;
  double e12t, e12u, e12v;
  double two_dx, two_dy;     // e1v(i)+e1v(i+1), e2u(j)+e2u(j+1)
  double rdt, visc, g;
  double fcor;               // 2*omega*SIN(gphi*d2r), :503, :594
  double cfric;              // 1 + cbfr*rdt, :514, :606
  // round-to-nearest reciprocals for the corrected constant divisions
  double r_e1t, r_e2t, r_e12t, r_e12u, r_e12v, r_2dx, r_2dy, r_cfric;
  // RN((1 - cfric*r_cfric)/cfric): with r_cfric, 1/cfric to about 2^-106
  double r_cfric_lo;
  // Products of constants for the default build's folded forms (formed on
  // the host): 0.5*e12t/e12u, 0.5*e12t/e12v, 0.5*e2t, 0.5*e1t, two_dy/8,
  // two_dx/8, rdt/e12t, rdt/e12u, rdt/e12v, visc*e2u/e1t, visc*e1u/2/two_dy,
  // visc*e1v/e2t, visc*e2v/2/two_dx, fcor*e12u/4, -fcor*e12v/4, -g*e2u,
  // -g*e1v.
  double k_su, k_sv, h_e2t, h_e1t, e_2dy, e_2dx, k_ssh, k_u, k_v;
  double vis_u1, vis_u2, vis_v1, vis_v2, cor_u, cor_v, hpg_u, hpg_v;
};

// Mask of original/nemolite2d.f90:184-202: 1 water, 0 land (west, east and
// north walls), -1 open water outside the domain (south row).
__host__ __device__ __forceinline__ int ptmask(int ji, int jj, int jpi, int jpj) {
  if (ji <= 0 || ji >= jpi + 1 || jj >= jpj + 1) return 0;
  if (jj <= 0) return -1;
  return 1;
}

// True for a nonzero |q| < 2^-959 and for an infinite or NaN q: the cases
// where the corrected quotient below is not proven exact.  +-0 is exact.
__device__ __forceinline__ bool quotient_out_of_range(double q) {
  unsigned t = ((unsigned)__double2hiint(q) << 1) | (unsigned)(__double2loint(q) != 0);
  return (t - 1u) < ((64u << 21) - 1u) || t >= (0x7ffu << 21);
}

// Quotient a/b correctly rounded, given rb = RN(1/b) formed on the host.
// Markstein's theorem (IBM J. Res. Dev. 34(1), 1990): with q = RN(a*rb) and
// the exact remainder r = a - b*q (one fma), RN(q + r*rb) = RN(a/b) whenever
// no intermediate underflows or overflows.  Quotients outside the proven
// range take the IEEE division instead.  Writing the last step as
// -fma(-r, rb, -q) keeps the sign of a zero quotient.
__device__ __forceinline__ double div_const(double a, double b, double rb) {
  double q = __dmul_rn(a, rb);
  if (quotient_out_of_range(q)) return a / b;
  double r = fma(-q, b, a);
  return -fma(-r, rb, -q);
}

// 1/b by two Newton-Raphson steps, y <- y + y*(1 - b*y) with fused
// multiply-adds, from a single-precision seed (relative error below 2^-22,
// so the second step leaves an error near 2^-88 before the last rounding).
// The result is RN(1/b) unless 1/b lies that close to a rounding boundary;
// callers that need RN(1/b) verify it against an IEEE division once per
// static divisor (launch_recip) and keep the stored quotient otherwise.
// b must be a normal number within single-precision range.
__device__ __forceinline__ double recip_seed(double b) {
  float yf;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(__double2float_rn(b)));
  return (double)yf;
}
// One Newton step: relative error about 2^-46.
__device__ __forceinline__ double recip_nr1(double b) {
  const double y = recip_seed(b);
  return fma(y, fma(-b, y, 1.0), y);
}
__device__ __forceinline__ double recip_nr(double b) {
  const double y = recip_nr1(b);
  return fma(y, fma(-b, y, 1.0), y);
}

constexpr unsigned long long kSign = 0x8000000000000000ull;

__device__ __forceinline__ bool sign_clear(double w) { return __double2hiint(w) >= 0; }

// First-order upwind value across a face with normal velocity w, lo/hi the
// values on the low/high-index side.  Equals, bit for bit,
//   (0.5 + SIGN(0.5,w))*lo + (0.5 - SIGN(0.5,w))*hi
// (original/nemolite2d.f90:454-471, :542-559) for finite operands: the two
// coefficients are exactly 1 and +0, so the value is main + (+0*other) with
// (main, other) = (lo, hi) when w's sign bit is clear, else (hi, lo); one
// fma forms that sum with a single rounding and the IEEE signed-zero rule.
__device__ __forceinline__ double upwind(double w, double lo, double hi) {
  const bool pos = sign_clear(w);
  return fma(0.0, pos ? hi : lo, pos ? lo : hi);
}
// (0.5 - SIGN(0.5,w))*hi alone (the slip-wall forms at :460, :548)
__device__ __forceinline__ double upwind_hi_only(double w, double hi) {
  unsigned long long hb = (unsigned long long)__double_as_longlong(hi);
  return sign_clear(w) ? __longlong_as_double((long long)(hb & kSign)) : hi;
}
// (0.5 + SIGN(0.5,w))*lo alone (:467, :555)
__device__ __forceinline__ double upwind_lo_only(double w, double lo) {
  unsigned long long lb = (unsigned long long)__double_as_longlong(lo);
  return sign_clear(w) ? lo : __longlong_as_double((long long)(lb & kSign));
}

}  // namespace nemo
