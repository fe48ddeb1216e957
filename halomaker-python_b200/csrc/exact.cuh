// Explicitly rounded FP64 arithmetic.  The ranking quantities of AdaptaHOP
// (distances, densities, saddle and threshold tests) must round exactly like
// the reference's gfortran build, which uses separate IEEE multiplies and adds
// (no fused multiply-add).  These wrappers make every rounding step explicit
// so the compiler cannot contract them, independently of -fmad.
#pragma once
#include <cuda_runtime.h>

namespace ahop {

__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double xsqrt(double a) { return __dsqrt_rn(a); }

// Periodic component distance of the reference (f90:2931-2932):
//   dx = |a - b| ; dx = max(0, min(dx, L - dx))
__device__ __forceinline__ double pdist(double a, double b, double L) {
  double dx = fabs(xsub(a, b));
  double w = xsub(L, dx);
  dx = fmin(dx, w);
  return fmax(0.0, dx);
}

// Squared periodic distance, summed as ((dx*dx + dy*dy) + dz*dz) (f90:2933-2941).
__device__ __forceinline__ double pdist2(double ax, double ay, double az, double bx, double by, double bz,
                                         double Lx, double Ly, double Lz) {
  double dx = pdist(ax, bx, Lx);
  double dy = pdist(ay, by, Ly);
  double dz = pdist(az, bz, Lz);
  return xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
}

// The same squared distance for a pair known to be less than half a period
// apart on every axis: then |a - b| <= L/2 <= L - |a - b| (also after
// rounding, which is monotone), so the periodic minimum and the clamp at 0
// return |a - b|, and squaring drops the sign.  Same bits as pdist2.
__device__ __forceinline__ double dist2_near(double ax, double ay, double az, double bx, double by, double bz) {
  const double dx = xsub(ax, bx), dy = xsub(ay, by), dz = xsub(az, bz);
  return xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
}

// Cubic-spline kernel of the reference (f90:3270-3287), same evaluation order.
__device__ __forceinline__ double spline(double x) {
  if (x <= 1.0) {
    double x2 = xmul(x, x);
    double x3 = xmul(x2, x);
    return xadd(xsub(1.0, xmul(1.5, x2)), xmul(0.75, x3));
  } else if (x <= 2.0) {
    double y = xsub(2.0, x);
    double y3 = xmul(xmul(y, y), y);
    return xmul(0.25, y3);
  }
  return 0.0;
}

// Order-preserving map of a non-negative double to uint64 (for atomics/sorts).
__device__ __host__ __forceinline__ unsigned long long dbits(double v) {
#ifdef __CUDA_ARCH__
  return (unsigned long long)__double_as_longlong(v);
#else
  unsigned long long u;
  __builtin_memcpy(&u, &v, 8);
  return u;
#endif
}

}  // namespace ahop
