// kernels.cuh -- device-side value arithmetic and the three Green's functions.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace xfmm {

constexpr double INV4PI = 0.079577471545947667884441881686257181;  // 1 / (4 pi)

// ------------------------------------------------------------ values: R, or complex as R2
template <class R> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };

template <class V> struct Base { using type = V; };
template <> struct Base<float2> { using type = float; };
template <> struct Base<double2> { using type = double; };

template <class V> __device__ __forceinline__ V vzero();
template <> __device__ __forceinline__ float vzero<float>() { return 0.f; }
template <> __device__ __forceinline__ double vzero<double>() { return 0.0; }
template <> __device__ __forceinline__ float2 vzero<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double2 vzero<double2>() { return make_double2(0.0, 0.0); }

__device__ __forceinline__ void vfma(float& acc, float a, float b) { acc = fmaf(a, b, acc); }
__device__ __forceinline__ void vfma(double& acc, double a, double b) { acc = fma(a, b, acc); }
__device__ __forceinline__ void vfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
__device__ __forceinline__ void vfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ float vscale(float a, float s) { return a * s; }
__device__ __forceinline__ double vscale(double a, double s) { return a * s; }
__device__ __forceinline__ float2 vscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 vscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ double vadd(double a, double b) { return a + b; }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 vadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// ------------------------------------------------------------ reciprocal square root
// FP32: the hardware approximation.  FP64: an FP32 seed refined by two Newton-Raphson
// steps y <- y (3 - x y^2) / 2 (quadratic convergence: ~2^-22 -> 2^-44 -> full precision),
// the same idea as the reference's rsqrt approximation + Newton steps (vec.h:655-670).
// NS: Newton steps for FP64 (2 for FP64 results; 1, ~2^-44, where the result feeds FP32 work).
template <int NS = 2> __device__ __forceinline__ float rsqrt_any(float x) { return rsqrtf(x); }
template <int NS = 2> __device__ __forceinline__ double rsqrt_any(double x) {
  double y = (double)rsqrtf((float)x);
  const double hx = 0.5 * x;
#pragma unroll
  for (int i = 0; i < NS; i++) y = y * (1.5 - hx * y * y);
  return y;
}
__device__ __forceinline__ float exp_any(float x) { return __expf(x); }
__device__ __forceinline__ double exp_any(double x) { return exp(x); }
__device__ __forceinline__ void sincos_any(float x, float* s, float* c) { __sincosf(x, s, c); }
__device__ __forceinline__ void sincos_any(double x, double* s, double* c) { sincos(x, s, c); }

// ------------------------------------------------------------ kernels
// Potentials/gradients of a unit-free charge q at relative offset (dx,dy,dz) = x_t - x_s, before the
// common 1/(4 pi) factor.  r == 0 contributes nothing (laplace.h:57, modified_helmholtz.h:61, helmholtz.h:64).
enum KernelId { K_LAPLACE = 0, K_YUKAWA = 1, K_HELMHOLTZ = 2 };

template <int KER, class R, int NS = 2> struct Green;

template <class R, int NS> struct Green<K_LAPLACE, R, NS> {
  using Q = R;  // charge / value type
  R k_re, k_im;
  __device__ __forceinline__ void pot(R dx, R dy, R dz, Q q, Q& acc) const {
    const R r2 = dx * dx + dy * dy + dz * dz;
    const R invr = r2 > R(0) ? rsqrt_any<NS>(r2) : R(0);
    acc += q * invr;
  }
  __device__ __forceinline__ void grad(R dx, R dy, R dz, Q q, Q& p, Q& gx, Q& gy, Q& gz) const {
    const R r2 = dx * dx + dy * dy + dz * dz;
    const R invr = r2 > R(0) ? rsqrt_any<NS>(r2) : R(0);
    const R qi = q * invr;
    const R qi3 = qi * invr * invr;
    p += qi;
    gx -= qi3 * dx;
    gy -= qi3 * dy;
    gz -= qi3 * dz;
  }
};

template <class R, int NS> struct Green<K_YUKAWA, R, NS> {
  using Q = R;
  R k_re, k_im;
  __device__ __forceinline__ void pot(R dx, R dy, R dz, Q q, Q& acc) const {
    const R r2 = dx * dx + dy * dy + dz * dz;
    const R invr = r2 > R(0) ? rsqrt_any<NS>(r2) : R(0);
    const R r = r2 * invr;
    acc += q * exp_any(-k_re * r) * invr;
  }
  __device__ __forceinline__ void grad(R dx, R dy, R dz, Q q, Q& p, Q& gx, Q& gy, Q& gz) const {
    const R r2 = dx * dx + dy * dy + dz * dz;
    const R invr = r2 > R(0) ? rsqrt_any<NS>(r2) : R(0);
    const R r = r2 * invr;
    const R kern = q * exp_any(-k_re * r) * invr;  // modified_helmholtz.h:159-164
    const R c = kern * (k_re * r + R(1)) * invr * invr;
    p += kern;
    gx -= c * dx;
    gy -= c * dy;
    gz -= c * dz;
  }
};

template <class R, int NS> struct Green<K_HELMHOLTZ, R, NS> {
  using Q = typename C2<R>::type;
  R k_re, k_im;
  // G = e^{ikr}/r = e^{-Im(k) r} (cos Re(k) r + i sin Re(k) r) / r   (helmholtz.h:241-249)
  __device__ __forceinline__ void pot(R dx, R dy, R dz, Q q, Q& acc) const {
    const R r2 = dx * dx + dy * dy + dz * dz;
    if (!(r2 > R(0))) return;
    const R invr = rsqrt_any<NS>(r2);
    const R r = r2 * invr;
    R sn, cs;
    sincos_any(k_re * r, &sn, &cs);
    const R e = exp_any(-k_im * r) * invr;
    const R gr = e * cs, gi = e * sn;
    acc.x += q.x * gr - q.y * gi;
    acc.y += q.x * gi + q.y * gr;
  }
  // grad = (i k / r - 1/r^2) G q (x_t - x_s)   (helmholtz.h:371-375)
  __device__ __forceinline__ void grad(R dx, R dy, R dz, Q q, Q& p, Q& gx, Q& gy, Q& gz) const {
    const R r2 = dx * dx + dy * dy + dz * dz;
    if (!(r2 > R(0))) return;
    const R invr = rsqrt_any<NS>(r2);
    const R r = r2 * invr;
    R sn, cs;
    sincos_any(k_re * r, &sn, &cs);
    const R e = exp_any(-k_im * r) * invr;
    const R gr = e * cs, gi = e * sn;
    const R pr = q.x * gr - q.y * gi, pi = q.x * gi + q.y * gr;
    p.x += pr;
    p.y += pi;
    // c = i k / r - 1/r^2 = (-k_im/r - 1/r^2) + i (k_re / r)
    const R cr = -k_im * invr - invr * invr, ci = k_re * invr;
    const R fr = cr * pr - ci * pi, fi = cr * pi + ci * pr;
    gx.x += fr * dx;
    gx.y += fi * dx;
    gy.x += fr * dy;
    gy.y += fi * dy;
    gz.x += fr * dz;
    gz.y += fi * dz;
  }
};

// operator+= for complex accumulators used by the generic code above
__device__ __forceinline__ float2& operator+=(float2& a, const float2& b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}
__device__ __forceinline__ double2& operator+=(double2& a, const double2& b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}

}  // namespace xfmm
