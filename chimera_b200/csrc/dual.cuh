// dual.cuh -- forward-mode dual numbers for the adjoint's local Jacobians.
//
// Dual<N> carries a value and N tangents.  Evaluating one of the templated
// device functions of mhd_device.cuh (get_primitive, the Riemann solvers,
// conserved_floors, limit_slope) with Dual arguments returns the outputs and
// their exact derivatives with respect to the seeded inputs, through the same
// operations and the same branch decisions as the FP64 forward: comparisons
// look at values only, so at a kink the derivative is that of the branch the
// forward took (a one-sided derivative), except at an exact tie of a min / max
// (and |x| at 0), where it is the mean of the two one-sided derivatives.
// sign() / copysign() have zero derivative in their sign argument.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "mhd_device.cuh"

namespace chimera {

template <int N> struct Dual {
  double v;
  double d[N];
  __host__ __device__ constexpr Dual() : v(0.0), d{} {}
  __host__ __device__ constexpr Dual(double x) : v(x), d{} {}
  __host__ __device__ constexpr Dual(int x) : v(double(x)), d{} {}
};

template <int N> __device__ __forceinline__ Dual<N> seed(double v, int k) {
  Dual<N> r(v);
  r.d[k] = 1.0;
  return r;
}

#define DUAL_BIN(OP, VEXPR, DEXPR)                                                   \
  template <int N> __device__ __forceinline__ Dual<N> operator OP(const Dual<N>& a, const Dual<N>& b) { \
    Dual<N> r;                                                                       \
    r.v = VEXPR;                                                                     \
    _Pragma("unroll") for (int k = 0; k < N; ++k) r.d[k] = DEXPR;                    \
    return r;                                                                        \
  }
DUAL_BIN(+, a.v + b.v, a.d[k] + b.d[k])
DUAL_BIN(-, a.v - b.v, a.d[k] - b.d[k])
DUAL_BIN(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef DUAL_BIN

template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}

template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}

// mixed forms with plain doubles
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
  return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) { return a / Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

#define DUAL_CMP(OP)                                                                                     \
  template <int N> __device__ __forceinline__ bool operator OP(const Dual<N>& a, const Dual<N>& b) { return a.v OP b.v; } \
  template <int N> __device__ __forceinline__ bool operator OP(const Dual<N>& a, double b) { return a.v OP b; }            \
  template <int N> __device__ __forceinline__ bool operator OP(double a, const Dual<N>& b) { return a OP b.v; }
DUAL_CMP(<)
DUAL_CMP(>)
DUAL_CMP(<=)
DUAL_CMP(>=)
#undef DUAL_CMP

template <int N> __device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = sqrt(a.v);
  const double h = (r.v > 0.0) ? 0.5 / r.v : 0.0;   // one-sided: zero derivative at sqrt(0)
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * h;
  return r;
}

template <int N> __device__ __forceinline__ Dual<N> dcopysign(const Dual<N>& a, const Dual<N>& b) {
  // |a| with the sign of b; the derivative follows a's magnitude only
  const bool flip = (signbit(a.v) != signbit(b.v));
  return flip ? -a : a;
}

template <int N> __device__ __forceinline__ bool disfinite(const Dual<N>& a) { return isfinite(a.v); }

// min / max of two duals.  At an exact tie -- common here: in a uniform region
// the left and right face states are bit-identical, so e.g. HLLE's
// min(vx_L - cf_L, vx_R - cf_R) ties -- the derivative is the mean of the two
// one-sided ones, which is what a central difference sees; off a tie it is
// the derivative of the larger / smaller argument.
template <int N> __device__ __forceinline__ Dual<N> tie_mean(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = 0.5 * (a.d[k] + b.d[k]);
  return r;
}
template <int N> __device__ __forceinline__ Dual<N> dmax(const Dual<N>& a, const Dual<N>& b) {
  return (a.v > b.v) ? a : ((b.v > a.v) ? b : tie_mean(a, b));
}
template <int N> __device__ __forceinline__ Dual<N> dmin(const Dual<N>& a, const Dual<N>& b) {
  return (a.v < b.v) ? a : ((b.v < a.v) ? b : tie_mean(a, b));
}
// |x| with zero derivative at x = 0 (the central difference there)
template <int N> __device__ __forceinline__ Dual<N> dabs(const Dual<N>& a) {
  return (a.v < 0.0) ? -a : ((a.v > 0.0) ? a : Dual<N>(0.0));
}

// min / max against plain constants (the floors of mhd_device.cuh)
template <int N> __device__ __forceinline__ Dual<N> dmax(const Dual<N>& a, double b) { return (a.v > b) ? a : Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> dmax(double a, const Dual<N>& b) { return (a > b.v) ? Dual<N>(a) : b; }
template <int N> __device__ __forceinline__ Dual<N> dmin(const Dual<N>& a, double b) { return (a.v < b) ? a : Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> dmin(double a, const Dual<N>& b) { return (a < b.v) ? Dual<N>(a) : b; }

template <int N> struct K<Dual<N>> {
  static constexpr double P_floor = 1.0e-12;
  static constexpr double rho_floor = 1.0e-12;
  static constexpr double e_floor_frac = 1.0e-10;
};

}  // namespace chimera
