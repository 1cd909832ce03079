// Shared device helpers for the subface finite-volume kernels (sm_100a).
//
// The plain-FP64 kernels are compiled with --fmad=false and evaluate every
// expression in the same order as the reference Fortran, so a kernel and the CPU
// restatement of the same routine produce the same bits.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

namespace subfv {

constexpr double kGamma = 7.0 / 5.0;

// Error bits a kernel records in the step status word (it never traps).
enum StatusBits : unsigned {
  kErrMeshCheck = 1u << 0,   // check_mesh failed (mesh_geometry_module.F90:403-408)
  kErrNonFinite = 1u << 1,   // a non-finite state, volume or time step
  kErrNegDensity = 1u << 2,  // negative specific volume / density
  kErrBadOmega = 1u << 3,    // positivity limiter gave omega <= 1e-6 (ns_euler_module.F90:595)
  kErrGmres = 1u << 4,       // GMRES did not converge (warning)
  kErrIndex = 1u << 5,       // an index outside its array (checked builds)
};

// x / D for D = 3 or 6, bit-identical to the IEEE quotient (round to nearest), by a
// multiply with the rounded reciprocal R = RN(1/D) and one remainder correction
// (Markstein's correction step for division with a fused multiply-add):
//   q0 = RN(x R),  e = x - D q0 (exact, one FMA),  q = RN(q0 + e R) (one FMA).
// Why it is exact for D = 3 * 2^k: R = (1/D)(1 - 2^-54), so x R is within half an ulp of
// x/D and q0 within one ulp; then x - D q0 is a small multiple of ulp(q0), exactly
// representable. q0 + e R = x/D - (e/D) 2^-54 differs from x/D by less than
// ulp(x/D) 2^-54, while x/D is at least ulp(x/D)/6 away from every rounding midpoint
// (x is a multiple of 2 or 4 ulp(x/D), and 2K - 3(2M + 1) is odd), so both round to the
// same double. Zero (its sign), subnormal or huge x, infinities and NaN take the plain
// division. The kernels that use it stay bit-identical to the CPU restatement, which
// divides; subfv_probe_div_const checks it against CUDA's division.
template <int D>
__host__ __device__ inline double div_const(double x) {
  static_assert(D == 3 || D == 6, "exact only for 3 * 2^k, checked for 3 and 6");
  constexpr double R = 1.0 / D;
  const double ax = fabs(x);
  if (!(ax >= 0x1p-960 && ax <= 0x1p960)) return x / D;
  const double q0 = x * R;
  const double e = fma(-q0, (double)D, x);
  return fma(e, R, q0);
}
__host__ __device__ inline double div3(double x) { return div_const<3>(x); }
__host__ __device__ inline double div6(double x) { return div_const<6>(x); }

// gfortran's inline NORM2 of a 3-vector: scaled sum of squares, scale starting at 1.
__host__ __device__ inline double fnorm2_3(double a0, double a1, double a2) {
  // With every |a_i| <= 1 the scale stays 1, each a_i / scale is a_i exactly and a zero
  // term adds nothing, so the scaled sum below reduces to this one, bit for bit.
  if (fabs(a0) <= 1.0 && fabs(a1) <= 1.0 && fabs(a2) <= 1.0) return sqrt(a0 * a0 + a1 * a1 + a2 * a2);
  double scale = 1.0, res = 0.0;
  const double a[3] = {a0, a1, a2};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (a[i] != 0.0) {
      double ax = fabs(a[i]);
      if (ax > scale) {
        double v = scale / ax;
        res = 1.0 + res * v * v;
        scale = ax;
      } else {
        double v = ax / scale;
        res += v * v;
      }
    }
  }
  return scale * sqrt(res);
}

// Lagrangian pressure (lagrange_module.F90:429-436); u = (tau, u, v, w, e).
__host__ __device__ inline double lag_pressure(double tau, double u1, double u2, double u3, double e) {
  double n = fnorm2_3(u1, u2, u3);
  return (kGamma - 1.0) / tau * (e - 0.5 * (n * n));
}

__host__ __device__ inline double dot3(double a0, double a1, double a2, double b0, double b1, double b2) {
  double s = 0.0;
  s = s + a0 * b0;
  s = s + a1 * b1;
  s = s + a2 * b2;
  return s;
}

// min over non-negative doubles through their bit patterns (order independent, exact)
__device__ inline void atomic_min_pos(double* addr, double v) {
  atomicMin(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

void set_error(const std::string& msg);

#define SUBFV_CUDA(call)                                                          \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      ::subfv::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));     \
      return -1;                                                                  \
    }                                                                             \
  } while (0)

// Device-side scalars of a time loop; one struct per in-flight problem.
struct LagScalars {
  double dtmin;               // running CFL minimum of the current step
  double dt;                  // time step of the current step
  double t, t_max, cfl;
  unsigned long long steps;   // steps taken
  int done;                   // t >= t_max: later steps are no-ops
  int skip;                   // this step was a no-op
};

// Cell record on the device: tau (or rho), the three velocities / momenta, energy, mass,
// pressure, pad. The pressure is recomputed whenever the state changes, with the same
// function the reference calls, so reading it is bit-identical to recomputing it.
constexpr int kRec = 8;
constexpr int kRhs = 6;  // rhs record: five residuals and a pad

inline int grid_for(long long n, int block) { return (int)((n + block - 1) / block); }

}  // namespace subfv
