// evaluate.cu -- upward and downward passes of the KIFMM on the GPU.
//
// Stage map (reference -> here):
//   P2M   fmm_scale_invariant.h:163-195 / fmm.h:156-185  k_surf_pot (Laplace mixed: k_surf_pot_lap_f2) check
//                                                        potentials + row gather, two FP64 library GEMMs
//                                                        (pinv factors), scaled scatter (0.5^l)
//   M2M   fmm_scale_invariant.h:233-253 / fmm.h:221-241  row gather + library GEMM per level, K = 8 nsurf
//   P2L   fmm_base.h:127-154                             k_p2l
//   M2L   fmm_scale_invariant.h:407-440, 560-646;        real kernels: k_m2l_fwd_r + k_hadamard_dt/_rt (opt-in:
//         fmm.h:395-446, 631-788                         k_hadamard_dc on tcgen05) + k_m2l_bwd_r (FP64:
//                                                        k_hadamard, k_m2l_bwd); complex kernel (p <= 12): k_m2l_fwd_c
//                                                        + Hadamard + k_m2l_bwd_c; real p > 10 or p > 12:
//                                                        k_m2l_grid_up + cuFFT + k_transpose + Hadamard +
//                                                        k_transpose + cuFFT + k_m2l_gather_dn
//   L2L   fmm_scale_invariant.h:256-275 / fmm.h:244-263  row gather + library GEMM per level, N = 8 nsurf
//   L2P   fmm_scale_invariant.h:198-230 / fmm.h:188-218  scaled row gather, two library GEMMs (the mixed
//                                                        path's first factor FP32), scatter; then the far
//                                                        part of the target evaluation
//   M2P   fmm_base.h:97-124                              far part: k_eval (Laplace mixed: k_far_lap)
//   P2P   fmm_base.h:82-94                               near part: k_near (Laplace mixed: k_near_lap_f2)
// Results stay in tree order until get_values scatters them (python/exafmm.cpp:194-207).
#include <cufft.h>

#include <algorithm>
#include <cstdlib>
#include <type_traits>
#include <cmath>

#include "kernels.cuh"
#include "tcgen05.cuh"
#include "xfmm_internal.h"

namespace xfmm {

#define XCUFFT2(call)                                                                                \
  do {                                                                                               \
    cufftResult st_ = (call);                                                                        \
    if (st_ != CUFFT_SUCCESS)                                                                        \
      throw Error(XFMM_ERR_CUDA, std::string("cuFFT ") + #call + " failed: " + std::to_string((int)st_)); \
  } while (0)

namespace {

inline int nblk(int64_t n, int t = 256) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

template <class R> struct R4;
template <> struct R4<float> { using type = float4; };
template <> struct R4<double> { using type = double4; };

template <class Q> __device__ __forceinline__ Q load_charge(const double4& s, const double* qim, int64_t j);
template <> __device__ __forceinline__ float load_charge<float>(const double4& s, const double*, int64_t) {
  return (float)s.w;
}
template <> __device__ __forceinline__ double load_charge<double>(const double4& s, const double*, int64_t) {
  return s.w;
}
template <> __device__ __forceinline__ float2 load_charge<float2>(const double4& s, const double* qim, int64_t j) {
  return make_float2((float)s.w, (float)qim[j]);
}
template <> __device__ __forceinline__ double2 load_charge<double2>(const double4& s, const double* qim, int64_t j) {
  return make_double2(s.w, qim[j]);
}

template <class To> __device__ __forceinline__ To cvt(float v);
template <class To> __device__ __forceinline__ To cvt(double v);
template <class To> __device__ __forceinline__ To cvt(float2 v);
template <class To> __device__ __forceinline__ To cvt(double2 v);
template <> __device__ __forceinline__ float cvt<float>(float v) { return v; }
template <> __device__ __forceinline__ float cvt<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ double cvt<double>(float v) { return (double)v; }
template <> __device__ __forceinline__ double cvt<double>(double v) { return v; }
template <> __device__ __forceinline__ float2 cvt<float2>(float2 v) { return v; }
template <> __device__ __forceinline__ float2 cvt<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ double2 cvt<double2>(float2 v) { return make_double2(v.x, v.y); }
template <> __device__ __forceinline__ double2 cvt<double2>(double2 v) { return v; }

// FP64 accumulation of FP32/FP64 partials
__device__ __forceinline__ void acc64(double& a, float b) { a += (double)b; }
__device__ __forceinline__ void acc64(double& a, double b) { a += b; }
__device__ __forceinline__ void acc64(double2& a, float2 b) {
  a.x += (double)b.x;
  a.y += (double)b.y;
}
__device__ __forceinline__ void acc64(double2& a, double2 b) {
  a.x += b.x;
  a.y += b.y;
}
template <class Q> struct Acc64 { using type = double; };
template <> struct Acc64<float2> { using type = double2; };
template <> struct Acc64<double2> { using type = double2; };

__device__ __forceinline__ double shfl_x(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ double2 shfl_x(double2 v, int o) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}
__device__ __forceinline__ void put_out(double* o, double v, double s, int acc) { *o = acc ? *o + v * s : v * s; }
__device__ __forceinline__ void put_out(double* o, double2 v, double s, int acc) {
  o[0] = acc ? o[0] + v.x * s : v.x * s;
  o[1] = acc ? o[1] + v.y * s : v.y * s;
}

// ================================================================ target evaluation (P2P + M2P + L2P)
struct EvalArgs {
  const int *eval_leafs, *leafs, *nsrcs, *ntrgs, *level;
  int n_eval;
  const int64_t *sbeg, *tbeg;
  const double4 *center, *src4, *trg4;
  const double* src_qim;
  const int64_t *p2p_off, *m2p_off;
  const int *p2p, *m2p;
  const double* surf_base;
  int nsurf;
  const void* up;  // working values [nnodes][nsurf]
  const void* eq;  // working values [nleafs][nsurf]
  double* out;     // tree order, 4 values per target (complex: interleaved)
  double k_re, k_im;
  int do_near, do_far, accumulate, hilo;
};

constexpr int EVAL_WARPS = 4;

// R: arithmetic of the pair interactions; W: value type of the upward equivalent densities (M2P
// sources).  The downward equivalent densities (L2P sources) are FP64 (the pinv output).
#ifndef XFMM_FAR_NS32
#define XFMM_FAR_NS32 1  // Newton steps of the FP64 far field when the working precision is FP32
#endif
template <int KER, class R, class W>
__global__ void __launch_bounds__(32 * EVAL_WARPS) k_eval(EvalArgs a) {
  // with an FP32 working precision (W), one Newton step on the FP64 reciprocal square root (~2^-44)
  using G = Green<KER, R, std::is_same<typename Base<W>::type, float>::value ? XFMM_FAR_NS32 : 2>;
  using Q = typename G::Q;
  using A = typename Acc64<Q>::type;
  using V4 = typename R4<R>::type;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * EVAL_WARPS + wid;
  if (w >= a.n_eval) return;
  __shared__ V4 s_xyz[EVAL_WARPS][32];
  __shared__ V4 s_lo[EVAL_WARPS][32];  // FP32: low parts of the leaf-relative coordinates
  __shared__ Q s_q[EVAL_WARPS][32];
  constexpr bool HILO = sizeof(R) == 4;
  const G g{(R)a.k_re, (R)a.k_im};
  const int pos = a.eval_leafs[w];
  const int node = a.leafs[pos];
  const int T = a.ntrgs[node];
  const int64_t tb = a.tbeg[node];
  const double4 c = a.center[node];
  using Q64 = typename Acc64<Q>::type;
  const W* upv = (const W*)a.up;
  const Q64* eqv = (const Q64*)a.eq;
  for (int t0 = 0, Tc = 0; t0 < T; t0 += Tc) {
    // blocks of 32 targets, the last 17..32 as 16 + the rest, so that the split of the sources over
    // 2..32 lanes per target keeps the lanes busy
    Tc = T - t0 > 32 ? 32 : (T - t0 > 16 ? 16 : T - t0);
    int G2 = 1;  // lanes per target: source stride
    while (G2 * 2 * Tc <= 32) G2 *= 2;
    const int tl = lane / G2, sub = lane % G2;
    const bool active = tl < Tc;
    // leaf-relative target coordinates; in FP32 as hi + lo so that differences keep ~FP32
    // relative accuracy of the separation itself (not of the leaf size)
    R tx = 0, ty = 0, tz = 0, lx = 0, ly = 0, lz = 0;
    if (active) {
      const double4 t = a.trg4[tb + t0 + tl];
      const double dx = t.x - c.x, dy = t.y - c.y, dz = t.z - c.z;
      tx = (R)dx;
      ty = (R)dy;
      tz = (R)dz;
      lx = (R)(dx - (double)tx);
      ly = (R)(dy - (double)ty);
      lz = (R)(dz - (double)tz);
    }
    A P, GX, GY, GZ;
    P = GX = GY = GZ = A();
    // one staged chunk of <= 32 sources: lanes accumulate their share, then FP64 accumulation
    auto consume = [&](int cnt) {
      __syncwarp();
      Q p = vzero<Q>(), gx = vzero<Q>(), gy = vzero<Q>(), gz = vzero<Q>();
      if (active) {
        if (HILO && a.hilo) {
          for (int j = sub; j < cnt; j += G2) {
            const V4 s = s_xyz[wid][j], sl = s_lo[wid][j];
            g.grad((tx - s.x) + (lx - sl.x), (ty - s.y) + (ly - sl.y), (tz - s.z) + (lz - sl.z), s_q[wid][j], p, gx,
                   gy, gz);
          }
        } else {
          for (int j = sub; j < cnt; j += G2) {
            const V4 s = s_xyz[wid][j];
            g.grad(tx - s.x, ty - s.y, tz - s.z, s_q[wid][j], p, gx, gy, gz);
          }
        }
      }
      acc64(P, p);
      acc64(GX, gx);
      acc64(GY, gy);
      acc64(GZ, gz);
      __syncwarp();
    };
    if (a.do_near) {
      for (int64_t e = a.p2p_off[node]; e < a.p2p_off[node + 1]; e++) {
        const int s = a.p2p[e];
        const int ns = a.nsrcs[s];
        const int64_t sb = a.sbeg[s];
        for (int j0 = 0; j0 < ns; j0 += 32) {
          const int cnt = min(32, ns - j0);
          if (lane < cnt) {
            const double4 sv = a.src4[sb + j0 + lane];
            const double dx = sv.x - c.x, dy = sv.y - c.y, dz = sv.z - c.z;
            const R hx = (R)dx, hy = (R)dy, hz = (R)dz;
            s_xyz[wid][lane] = V4{hx, hy, hz, (R)0};
            s_lo[wid][lane] = V4{(R)(dx - (double)hx), (R)(dy - (double)hy), (R)(dz - (double)hz), (R)0};
            s_q[wid][lane] = load_charge<Q>(sv, a.src_qim, sb + j0 + lane);
          }
          consume(cnt);
        }
      }
    }
    if (a.do_far) {
      const int n = a.nsurf;
      // M2P: W-list nodes' upward equivalent surfaces (1.05 box, fmm_base.h:103-121)
      for (int64_t e = a.m2p_off[node]; e < a.m2p_off[node + 1]; e++) {
        const int s = a.m2p[e];
        const double4 cs = a.center[s];
        const double b = 1.05 * cs.w;
        for (int j0 = 0; j0 < n; j0 += 32) {
          const int cnt = min(32, n - j0);
          if (lane < cnt) {
            const int k = j0 + lane;
            s_xyz[wid][lane] = V4{(R)(cs.x + a.surf_base[3 * k] * b - c.x), (R)(cs.y + a.surf_base[3 * k + 1] * b - c.y),
                                  (R)(cs.z + a.surf_base[3 * k + 2] * b - c.z), (R)0};
            s_lo[wid][lane] = V4{(R)0, (R)0, (R)0, (R)0};
            s_q[wid][lane] = cvt<Q>(upv[(int64_t)s * n + k]);
          }
          consume(cnt);
        }
      }
      // L2P: own downward equivalent surface (2.95 box, fmm_scale_invariant.h:221-228)
      const double b = 2.95 * c.w;
      for (int j0 = 0; j0 < n; j0 += 32) {
        const int cnt = min(32, n - j0);
        if (lane < cnt) {
          const int k = j0 + lane;
          s_xyz[wid][lane] = V4{(R)(a.surf_base[3 * k] * b), (R)(a.surf_base[3 * k + 1] * b),
                                (R)(a.surf_base[3 * k + 2] * b), (R)0};
          s_lo[wid][lane] = V4{(R)0, (R)0, (R)0, (R)0};
          s_q[wid][lane] = cvt<Q>(eqv[(int64_t)pos * n + k]);
        }
        consume(cnt);
      }
    }
    for (int o = 1; o < G2; o <<= 1) {
      P = vadd(P, shfl_x(P, o));
      GX = vadd(GX, shfl_x(GX, o));
      GY = vadd(GY, shfl_x(GY, o));
      GZ = vadd(GZ, shfl_x(GZ, o));
    }
    if (active && sub == 0) {
      const int stride = (KER == K_HELMHOLTZ) ? 8 : 4;
      double* o = a.out + (tb + t0 + tl) * stride;
      const int vs = stride / 4;
      put_out(o, P, INV4PI, a.accumulate);
      put_out(o + vs, GX, INV4PI, a.accumulate);
      put_out(o + 2 * vs, GY, INV4PI, a.accumulate);
      put_out(o + 3 * vs, GZ, INV4PI, a.accumulate);
    }
  }
}

// Far field (M2P + L2P) of the Laplace mixed path, in FP64: the sums over equivalent densities cancel
// strongly, so every term needs FP64.  Warp per target leaf, targets mapped to lanes as in k_eval; the
// equivalent surfaces (each W-list node's upward surface, then the leaf's own downward surface) are
// staged 128 points at a time as FP64 (x, y, z, density) relative to the leaf centre, and each lane runs
// four points at once into four partial sums, so the FP64 pipe has independent work between the
// long-latency steps.  1/r: the FP64 reciprocal-square-root approximation instruction (relative error
// below 2^-22.9) and one Newton step (~2^-44).  No pair coincides: a target lies at least 1.95 r from
// its own downward surface, and W-list nodes are not adjacent to the leaf.
__device__ __forceinline__ double rsqrt_approx64(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}
constexpr int FAR_CH = 128;  // surface points staged per chunk
__device__ __forceinline__ void far_pair(double tx, double ty, double tz, const double4& s, double& p, double& gx,
                                         double& gy, double& gz) {
  const double dx = tx - s.x, dy = ty - s.y, dz = tz - s.z;
  const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
  double y = rsqrt_approx64(r2);
  y = y * fma(-0.5 * r2, y * y, 1.5);
  const double qi = s.w * y;
  const double qi3 = qi * (y * y);
  p += qi;
  gx = fma(-qi3, dx, gx);
  gy = fma(-qi3, dy, gy);
  gz = fma(-qi3, dz, gz);
}
// the far field of evaluation leaf w (one warp); spw: the warp's FAR_CH staged surface points
template <class W>
__device__ __forceinline__ void far_leaf_lap(const EvalArgs& a, int w, int lane, double4* spw) {
  const int pos = a.eval_leafs[w];
  const int node = a.leafs[pos];
  const int T = a.ntrgs[node];
  const int64_t tb = a.tbeg[node];
  const double4 c = a.center[node];
  const int n = a.nsurf;
  const W* upv = (const W*)a.up;
  const double* eqv = (const double*)a.eq;
  for (int t0 = 0, Tc = 0; t0 < T; t0 += Tc) {
    // blocks of 32 targets, the last 17..32 as 16 + the rest; 2..32 lanes per target split the points
    Tc = T - t0 > 32 ? 32 : (T - t0 > 16 ? 16 : T - t0);
    int G2 = 1;
    while (G2 * 2 * Tc <= 32) G2 *= 2;
    const int tl = lane / G2, sub = lane % G2;
    const bool active = tl < Tc;
    double tx = 0, ty = 0, tz = 0;
    if (active) {
      const double4 t = a.trg4[tb + t0 + tl];
      tx = t.x - c.x;
      ty = t.y - c.y;
      tz = t.z - c.z;
    }
    double P[4] = {0, 0, 0, 0}, GX[4] = {0, 0, 0, 0}, GY[4] = {0, 0, 0, 0}, GZ[4] = {0, 0, 0, 0};
    auto consume = [&](int cnt) {
      __syncwarp();
      if (active) {
        int j = sub;
        for (; j + 3 * G2 < cnt; j += 4 * G2) {
#pragma unroll
          for (int u = 0; u < 4; u++) far_pair(tx, ty, tz, spw[j + u * G2], P[u], GX[u], GY[u], GZ[u]);
        }
        for (; j < cnt; j += G2) far_pair(tx, ty, tz, spw[j], P[0], GX[0], GY[0], GZ[0]);
      }
      __syncwarp();
    };
    // M2P: W-list nodes' upward equivalent surfaces (1.05 box, fmm_base.h:103-121)
    for (int64_t e = a.m2p_off[node]; e < a.m2p_off[node + 1]; e++) {
      const int s = a.m2p[e];
      const double4 cs = a.center[s];
      const double b = 1.05 * cs.w;
      for (int j0 = 0; j0 < n; j0 += FAR_CH) {
        const int cnt = min(FAR_CH, n - j0);
        for (int i = lane; i < cnt; i += 32) {
          const int k = j0 + i;
          spw[i] = make_double4(cs.x + a.surf_base[3 * k] * b - c.x, cs.y + a.surf_base[3 * k + 1] * b - c.y,
                                    cs.z + a.surf_base[3 * k + 2] * b - c.z, (double)upv[(int64_t)s * n + k]);
        }
        consume(cnt);
      }
    }
    // L2P: own downward equivalent surface (2.95 box, fmm_scale_invariant.h:221-228)
    const double b = 2.95 * c.w;
    for (int j0 = 0; j0 < n; j0 += FAR_CH) {
      const int cnt = min(FAR_CH, n - j0);
      for (int i = lane; i < cnt; i += 32) {
        const int k = j0 + i;
        spw[i] = make_double4(a.surf_base[3 * k] * b, a.surf_base[3 * k + 1] * b, a.surf_base[3 * k + 2] * b,
                                  eqv[(int64_t)pos * n + k]);
      }
      consume(cnt);
    }
    double p = (P[0] + P[1]) + (P[2] + P[3]), gx = (GX[0] + GX[1]) + (GX[2] + GX[3]);
    double gy = (GY[0] + GY[1]) + (GY[2] + GY[3]), gz = (GZ[0] + GZ[1]) + (GZ[2] + GZ[3]);
    for (int o = 1; o < G2; o <<= 1) {
      p += __shfl_xor_sync(0xffffffffu, p, o);
      gx += __shfl_xor_sync(0xffffffffu, gx, o);
      gy += __shfl_xor_sync(0xffffffffu, gy, o);
      gz += __shfl_xor_sync(0xffffffffu, gz, o);
    }
    if (active && sub == 0) {
      double* o = a.out + (tb + t0 + tl) * 4;
      o[0] += p * INV4PI;
      o[1] += gx * INV4PI;
      o[2] += gy * INV4PI;
      o[3] += gz * INV4PI;
    }
  }
}
template <class W>
__global__ void __launch_bounds__(32 * EVAL_WARPS) k_far_lap(EvalArgs a) {
  __shared__ double4 sp[EVAL_WARPS][FAR_CH];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * EVAL_WARPS + wid;
  if (w >= a.n_eval) return;
  far_leaf_lap<W>(a, w, lane, sp[wid]);
}
// The far field of every system of a batch: each warp takes work items (system, evaluation leaf) from one
// queue (a global counter, zeroed before the launch) in the order of `items` until it runs dry.
template <class W>
__global__ void __launch_bounds__(32 * EVAL_WARPS)
    k_far_lap_queue(const EvalArgs* __restrict__ args, const int2* __restrict__ items, int64_t nitems,
                    unsigned int* __restrict__ counter) {
  __shared__ double4 sp[EVAL_WARPS][FAR_CH];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (;;) {
    unsigned int k = 0;
    if (lane == 0) k = atomicAdd(counter, 1u);
    k = __shfl_sync(0xffffffffu, k, 0);
    if ((int64_t)k >= nitems) break;
    const int2 it = items[k];
    far_leaf_lap<W>(args[it.x], it.y, lane, sp[wid]);
    __syncwarp();
  }
}

// ================================================================ near field (P2P)
// Warp per target leaf.  The sources of the leaf's P2P list form one continuous stream that is
// staged 32 at a time in shared memory as leaf-relative coordinates (FP32: hi + lo parts, so the
// separation keeps FP32 relative accuracy); only the stream's last chunk is padded (zero charges,
// far away).  Lanes map to targets in one of two ways:
//   T >= 32 : TPL targets per lane (t = lane + 32 u), every staged source reused TPL times;
//   T <  32 : G lanes per target (G = 32 / 2^ceil(log2 T)), each taking every G-th source of a
//             chunk, partial sums combined with shuffles at the end.
// FP32 chunk sums are accumulated in FP64.
struct NearArgs {
  const int *eval_leafs, *leafs, *nsrcs, *ntrgs;
  int n_eval;
  const int64_t *sbeg, *tbeg, *p2p_off;
  const int* p2p;
  const double4 *center, *src4, *trg4;
  const double* src_qim;
  double* out;
  double k_re, k_im;
};

template <class R> struct Stage4;
template <> struct Stage4<float> { using type = float4; };
template <> struct Stage4<double> { using type = double4; };

constexpr int NEAR_SEG = 64;  // P2P-list entries held per batch

template <class R>
struct NearSmem {
  typename Stage4<R>::type hi[32], lo[32];
  int64_t seg_beg[NEAR_SEG];
  int seg_pre[NEAR_SEG + 1];
};

template <int KER, class R, int TPL>
__device__ __forceinline__ void near_leaf(const NearArgs& a, int node, int lane, NearSmem<R>& sm) {
  using G = Green<KER, R>;
  using Q = typename G::Q;
  using A = typename Acc64<Q>::type;
  constexpr bool CPLX = KER == K_HELMHOLTZ;
  constexpr bool HILO = sizeof(R) == 4;
  const G g{(R)a.k_re, (R)a.k_im};
  const int T = a.ntrgs[node];
  const int64_t tb = a.tbeg[node];
  const double4 c = a.center[node];
  const int64_t e0 = a.p2p_off[node], e1 = a.p2p_off[node + 1];
  // lane -> (target slot, source sub-lane)
  int G2 = 1;
  if (TPL == 1)
    while (G2 * 2 * T <= 32) G2 *= 2;
  const int tl = lane / G2, sub = lane % G2;
  const int nper = 32 / G2;  // sources per lane per chunk
  for (int t0 = 0; t0 < T; t0 += 32 * TPL) {
    R tx[TPL], ty[TPL], tz[TPL], lx[TPL], ly[TPL], lz[TPL];
    A P[TPL], GX[TPL], GY[TPL], GZ[TPL];
#pragma unroll
    for (int u = 0; u < TPL; u++) {
      const int t = t0 + tl + 32 * u;
      double dx = 0, dy = 0, dz = 0;
      if (t < T) {
        const double4 v = a.trg4[tb + t];
        dx = v.x - c.x;
        dy = v.y - c.y;
        dz = v.z - c.z;
      }
      tx[u] = (R)dx;
      ty[u] = (R)dy;
      tz[u] = (R)dz;
      lx[u] = (R)(dx - (double)tx[u]);
      ly[u] = (R)(dy - (double)ty[u]);
      lz[u] = (R)(dz - (double)tz[u]);
      P[u] = GX[u] = GY[u] = GZ[u] = A();
    }
    for (int64_t eb = e0; eb < e1; eb += NEAR_SEG) {
      // segment table of this batch: begin offsets and an inclusive prefix of counts
      const int nseg = (int)(e1 - eb < NEAR_SEG ? e1 - eb : NEAR_SEG);
      __syncwarp();
      int carry = 0;
      for (int k0 = 0; k0 < nseg; k0 += 32) {
        const int k = k0 + lane;
        int cnt = 0;
        if (k < nseg) {
          const int sn = a.p2p[eb + k];
          cnt = a.nsrcs[sn];
          sm.seg_beg[k] = a.sbeg[sn];
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        if (k < nseg) sm.seg_pre[k + 1] = carry + incl;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) sm.seg_pre[0] = 0;
      __syncwarp();
      const int total = carry;
      int seg = 0;  // per-lane cursor into the segment table
      for (int p0 = 0; p0 < total; p0 += 32) {
        const int pos = p0 + lane;
        __syncwarp();
        if (pos < total) {
          while (sm.seg_pre[seg + 1] <= pos) seg++;
          const int64_t si = sm.seg_beg[seg] + (pos - sm.seg_pre[seg]);
          const double4 sv = a.src4[si];
          const double dx = sv.x - c.x, dy = sv.y - c.y, dz = sv.z - c.z;
          const R hx = (R)dx, hy = (R)dy, hz = (R)dz;
          const R qi = CPLX ? (R)a.src_qim[si] : (R)0;
          sm.hi[lane] = {hx, hy, hz, (R)sv.w};
          if constexpr (HILO || CPLX)
            sm.lo[lane] = {(R)(dx - (double)hx), (R)(dy - (double)hy), (R)(dz - (double)hz), qi};
        } else {
          sm.hi[lane] = {(R)1e3, (R)1e3, (R)1e3, (R)0};  // zero-charge padding, far from every target
          if constexpr (HILO || CPLX) sm.lo[lane] = {(R)0, (R)0, (R)0, (R)0};
        }
        __syncwarp();
        Q p[TPL], gx[TPL], gy[TPL], gz[TPL];
#pragma unroll
        for (int u = 0; u < TPL; u++) p[u] = gx[u] = gy[u] = gz[u] = vzero<Q>();
#pragma unroll 4
        for (int jj = 0; jj < nper; jj++) {
          const int j = jj * G2 + sub;
          const auto h = sm.hi[j];
          typename Stage4<R>::type l{};  // low parts (FP32) and imaginary charges (complex); FP64 real: none
          if constexpr (HILO || CPLX) l = sm.lo[j];
          Q q;
          if constexpr (CPLX) q = Q{h.w, l.w};
          else q = h.w;
#pragma unroll
          for (int u = 0; u < TPL; u++) {
            R dx, dy, dz;
            if constexpr (HILO) {
              dx = (tx[u] - h.x) + (lx[u] - l.x);
              dy = (ty[u] - h.y) + (ly[u] - l.y);
              dz = (tz[u] - h.z) + (lz[u] - l.z);
            } else {
              dx = tx[u] - h.x;
              dy = ty[u] - h.y;
              dz = tz[u] - h.z;
            }
            g.grad(dx, dy, dz, q, p[u], gx[u], gy[u], gz[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < TPL; u++) {
          acc64(P[u], p[u]);
          acc64(GX[u], gx[u]);
          acc64(GY[u], gy[u]);
          acc64(GZ[u], gz[u]);
        }
      }
    }
    if (TPL == 1) {
      for (int o = 1; o < G2; o <<= 1) {
        P[0] = vadd(P[0], shfl_x(P[0], o));
        GX[0] = vadd(GX[0], shfl_x(GX[0], o));
        GY[0] = vadd(GY[0], shfl_x(GY[0], o));
        GZ[0] = vadd(GZ[0], shfl_x(GZ[0], o));
      }
    }
#pragma unroll
    for (int u = 0; u < TPL; u++) {
      const int t = t0 + tl + 32 * u;
      if (t < T && sub == 0) {
        const int stride = CPLX ? 8 : 4, vs = stride / 4;
        double* o = a.out + (tb + t) * stride;
        put_out(o, P[u], INV4PI, 0);
        put_out(o + vs, GX[u], INV4PI, 0);
        put_out(o + 2 * vs, GY[u], INV4PI, 0);
        put_out(o + 3 * vs, GZ[u], INV4PI, 0);
      }
    }
  }
}

// ---------------------------------------------------------------- Laplace FP32 near field, paired FP32
// Same mapping and streaming as near_leaf, but two sources are processed per instruction with the
// sm_100 paired FP32 operations (__ffma2_rn / __fadd2_rn / __fmul2_rn): the staged sources are laid
// out structure-of-arrays so that sources (j, j+1) load as one float2, and the target's coordinates
// are duplicated into both halves once per chunk.
// Coordinates are taken relative to the centre of the target leaf: each staged source is moved there in
// FP64 and rounded to FP32 once per chunk (shared by every target of the warp), each target once, so a
// pair's separation is a single FP32 subtraction of two values no larger than the 3 x 3 x 3 leaf
// neighbourhood (a few leaf radii).  Its error is a few FP32 ulps of that neighbourhood's size, not of
// the root's.  That is not enough for the closest pairs (the few pairs a few 1e-5 apart dominate the
// gradient's norm over all targets), so 1/r is taken of max(r^2, d^2), d = NEAR_CLOSE x the leaf
// radius: a pair closer than d (r == 0 among them) contributes a bounded FP32 value.  Those pairs are
// found once per tree with the same FP32 arithmetic (k_close_scan) and, after the near field, k_close_fix
// replaces each one's FP32 contribution with the exact FP64 one (pairs at r == 0 in FP64 contribute
// nothing, laplace.h:57).  The error left in the FP32 pairs, ~2^-24 x (neighbourhood radius /
// separation), is then bounded by separations above d.
constexpr float NEAR_CLOSE = 0.125f;
// the squared close-pair distance of a leaf of radius r (the same FP32 value in every kernel that tests it)
__device__ __forceinline__ float near_close2(double r) {
  const float d = (float)(NEAR_CLOSE * r);
  return d * d;
}
// a source or target relative to the leaf centre, rounded to FP32 (the same in every kernel)
__device__ __forceinline__ float3 leaf_rel(const double4& v, const double4& cn) {
  return make_float3((float)(v.x - cn.x), (float)(v.y - cn.y), (float)(v.z - cn.z));
}
#ifndef XFMM_NEAR_CH
#define XFMM_NEAR_CH 64
#endif
constexpr int NEAR_CH = XFMM_NEAR_CH;  // sources staged per chunk (32 or 64)
static_assert(NEAR_CH == 32 || NEAR_CH == 64, "NEAR_CH");
struct NearSmemF2 {
  // source pair k = sources 2k, 2k+1 relative to the leaf centre: {x, x'}, {y, y'} and {z, z'}, {q, q'}
  float4 pr[NEAR_CH / 2][2];
  int64_t seg_beg[NEAR_SEG];
  int seg_pre[NEAR_SEG + 1];
};

__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

template <int TPL>
__device__ __forceinline__ void near_leaf_lap_f2(const NearArgs& a, int node, int lane, NearSmemF2& sm) {
  const int T = a.ntrgs[node];
  const int64_t tb = a.tbeg[node];
  const int64_t e0 = a.p2p_off[node], e1 = a.p2p_off[node + 1];
  const double4 cn = a.center[node];
  int G2 = 1;  // at most 16 lanes per target
  if (TPL == 1)
    while (G2 * 2 * T <= 32 && G2 < 16) G2 *= 2;
  const int tl = lane / G2, sub = lane % G2;
  const int npl = NEAR_CH / 2 / G2;  // source pairs per lane per chunk
  const float2 M1 = make_float2(-1.f, -1.f);
  const float dc2 = near_close2(cn.w);  // close-pair threshold, squared
  for (int t0 = 0; t0 < T; t0 += 32 * TPL) {
    float2 TX[TPL], TY[TPL], TZ[TPL];
    double P[TPL], GX[TPL], GY[TPL], GZ[TPL];
#pragma unroll
    for (int u = 0; u < TPL; u++) {
      const int t = t0 + tl + 32 * u;
      float3 tr = make_float3(0.f, 0.f, 0.f);
      if (t < T) tr = leaf_rel(a.trg4[tb + t], cn);
      TX[u] = dup2(tr.x);
      TY[u] = dup2(tr.y);
      TZ[u] = dup2(tr.z);
      P[u] = GX[u] = GY[u] = GZ[u] = 0.0;
    }
    for (int64_t eb = e0; eb < e1; eb += NEAR_SEG) {
      const int nseg = (int)(e1 - eb < NEAR_SEG ? e1 - eb : NEAR_SEG);
      __syncwarp();
      int carry = 0;
      for (int k0 = 0; k0 < nseg; k0 += 32) {
        const int k = k0 + lane;
        int cnt = 0, sn = -1;
        if (k < nseg) {
          sn = a.p2p[eb + k];
          cnt = a.nsrcs[sn];
          sm.seg_beg[k] = a.sbeg[sn];
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        if (k < nseg) sm.seg_pre[k + 1] = carry + incl;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) sm.seg_pre[0] = 0;
      __syncwarp();
      const int total = carry;
      int seg = 0;
      for (int p0 = 0; p0 < total; p0 += NEAR_CH) {
        __syncwarp();
#pragma unroll
        for (int h = 0; h < NEAR_CH / 32; h++) {
          const int pos = p0 + 32 * h + lane;
          // zero-charge padding far away: contributes 0 and is never close
          float x = 1e18f, y = 1e18f, z = 1e18f, q = 0.f;
          if (pos < total) {
            while (sm.seg_pre[seg + 1] <= pos) seg++;
            const double4 v = a.src4[sm.seg_beg[seg] + (pos - sm.seg_pre[seg])];
            const float3 sr = leaf_rel(v, cn);
            x = sr.x;
            y = sr.y;
            z = sr.z;
            q = (float)v.w;
          }
          float* r = reinterpret_cast<float*>(sm.pr[16 * h + (lane >> 1)]) + (lane & 1);  // float2 slot
          r[0] = x;
          r[2] = y;
          r[4] = z;
          r[6] = q;
        }
        __syncwarp();
        float2 p2[TPL], gx2[TPL], gy2[TPL], gz2[TPL];
#pragma unroll
        for (int u = 0; u < TPL; u++) p2[u] = gx2[u] = gy2[u] = gz2[u] = make_float2(0.f, 0.f);
        // pairs closer than the threshold (r == 0 among them) give 1/max(r, d): replaced exactly later
#pragma unroll 4
        for (int jj = 0; jj < npl; jj++) {
          const int jp = jj * G2 + sub;  // source pair
          const float4 A0 = sm.pr[jp][0], A1 = sm.pr[jp][1];
          const float2 SX = make_float2(A0.x, A0.y), SY = make_float2(A0.z, A0.w);
          const float2 SZ = make_float2(A1.x, A1.y), Q = make_float2(A1.z, A1.w);
#pragma unroll
          for (int u = 0; u < TPL; u++) {
            const float2 dx = __ffma2_rn(SX, M1, TX[u]);  // t - s
            const float2 dy = __ffma2_rn(SY, M1, TY[u]);
            const float2 dz = __ffma2_rn(SZ, M1, TZ[u]);
            float2 r2 = __fmul2_rn(dx, dx);
            r2 = __ffma2_rn(dy, dy, r2);
            r2 = __ffma2_rn(dz, dz, r2);
            const float2 inv = make_float2(rsqrtf(fmaxf(r2.x, dc2)), rsqrtf(fmaxf(r2.y, dc2)));
            const float2 qi = __fmul2_rn(Q, inv);
            const float2 qi3 = __fmul2_rn(qi, __fmul2_rn(inv, inv));
            p2[u] = __fadd2_rn(p2[u], qi);
            gx2[u] = __ffma2_rn(qi3, dx, gx2[u]);  // sign applied when accumulating
            gy2[u] = __ffma2_rn(qi3, dy, gy2[u]);
            gz2[u] = __ffma2_rn(qi3, dz, gz2[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < TPL; u++) {
          P[u] += (double)(p2[u].x + p2[u].y);
          GX[u] -= (double)(gx2[u].x + gx2[u].y);
          GY[u] -= (double)(gy2[u].x + gy2[u].y);
          GZ[u] -= (double)(gz2[u].x + gz2[u].y);
        }
      }
    }
    if (TPL == 1) {
      for (int o = 1; o < G2; o <<= 1) {
        P[0] += __shfl_xor_sync(0xffffffffu, P[0], o);
        GX[0] += __shfl_xor_sync(0xffffffffu, GX[0], o);
        GY[0] += __shfl_xor_sync(0xffffffffu, GY[0], o);
        GZ[0] += __shfl_xor_sync(0xffffffffu, GZ[0], o);
      }
    }
#pragma unroll
    for (int u = 0; u < TPL; u++) {
      const int t = t0 + tl + 32 * u;
      if (t < T && sub == 0) {
        double* o = a.out + (tb + t) * 4;
        o[0] = P[u] * INV4PI;
        o[1] = GX[u] * INV4PI;
        o[2] = GY[u] * INV4PI;
        o[3] = GZ[u] * INV4PI;
      }
    }
  }
}

#ifndef XFMM_NEARF2_MINB
#define XFMM_NEARF2_MINB 6  // minimum resident blocks per SM asked of the register allocator (measured best of 1..8)
#endif
#ifndef XFMM_NEARF2_TPL
#define XFMM_NEARF2_TPL 2  // largest number of targets per lane (2 or 4)
#endif
__global__ void __launch_bounds__(128, XFMM_NEARF2_MINB) k_near_lap_f2(NearArgs a) {
  __shared__ NearSmemF2 sm[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * 4 + wid;
  if (w >= a.n_eval) return;
  const int node = a.leafs[a.eval_leafs[w]];
  const int T = a.ntrgs[node];
  if (T <= 32) near_leaf_lap_f2<1>(a, node, lane, sm[wid]);
  else if (T <= 64 || XFMM_NEARF2_TPL == 2) near_leaf_lap_f2<2>(a, node, lane, sm[wid]);
  else near_leaf_lap_f2<XFMM_NEARF2_TPL>(a, node, lane, sm[wid]);
}

// The near field's close pairs (k_near_lap_f2): every (target, source) of a leaf's U list whose FP32
// leaf-relative separation, computed exactly as the near-field kernel computes it, is not above the
// leaf's close-pair distance.  Warp per target leaf; the U-list sources pass through shared memory 32 at
// a time.  FILL = false counts them (one global counter), FILL = true writes (target position in tree
// order, source position, leaf node, 0) at positions taken from a second counter.
template <bool FILL>
__global__ void __launch_bounds__(128) k_close_scan(NearArgs a, unsigned long long* __restrict__ counter,
                                                    int4* __restrict__ pairs, int64_t capacity) {
  __shared__ float4 ss[4][32];
  __shared__ int sidx[4][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * 4 + wid;
  if (w >= a.n_eval) return;
  const int node = a.leafs[a.eval_leafs[w]];
  const int T = a.ntrgs[node];
  const int64_t tb = a.tbeg[node];
  const double4 cn = a.center[node];
  const float dc2 = near_close2(cn.w);
  unsigned long long found = 0;
  for (int64_t e = a.p2p_off[node]; e < a.p2p_off[node + 1]; e++) {
    const int sn = a.p2p[e];
    const int ns = a.nsrcs[sn];
    const int64_t sb = a.sbeg[sn];
    for (int j0 = 0; j0 < ns; j0 += 32) {
      __syncwarp();
      if (j0 + lane < ns) {
        const float3 r = leaf_rel(a.src4[sb + j0 + lane], cn);
        ss[wid][lane] = make_float4(r.x, r.y, r.z, 0.f);
        sidx[wid][lane] = (int)(sb + j0 + lane);
      }
      __syncwarp();
      const int cnt = min(32, ns - j0);
      for (int t = lane; t < T; t += 32) {
        const float3 tr = leaf_rel(a.trg4[tb + t], cn);
        for (int j = 0; j < cnt; j++) {
          const float4 sr = ss[wid][j];
          const float dx = __fmaf_rn(sr.x, -1.f, tr.x), dy = __fmaf_rn(sr.y, -1.f, tr.y),
                      dz = __fmaf_rn(sr.z, -1.f, tr.z);
          float r2 = __fmul_rn(dx, dx);
          r2 = __fmaf_rn(dy, dy, r2);
          r2 = __fmaf_rn(dz, dz, r2);
          if (!(r2 > dc2)) {
            if (FILL) {
              const unsigned long long k = atomicAdd(counter, 1ull);
              if ((int64_t)k < capacity) pairs[k] = make_int4((int)(tb + t), sidx[wid][j], node, 0);
            } else {
              found++;
            }
          }
        }
      }
    }
  }
  if (!FILL) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) found += __shfl_xor_sync(0xffffffffu, found, o);
    if (lane == 0 && found) atomicAdd(counter, found);
  }
}

// For each close pair: the exact FP64 contribution (r == 0 skipped, laplace.h:57) in place of the bounded
// FP32 one that k_near_lap_f2 added (recomputed with the same operations; the gradient's FP32 product is
// taken exactly in FP64, as the fused multiply-add took it).
__global__ void k_close_fix(const int4* __restrict__ pairs, int64_t n, NearArgs a1, const NearArgs* __restrict__ args) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int4 pr = pairs[k];
  const NearArgs& a = args ? args[pr.w] : a1;  // one system, or system pr.w of a batch
  const double4 tv = a.trg4[pr.x], sv = a.src4[pr.y], cn = a.center[pr.z];
  const float dc2 = near_close2(cn.w);
  const float3 tr = leaf_rel(tv, cn), sr = leaf_rel(sv, cn);
  const float dx = __fmaf_rn(sr.x, -1.f, tr.x), dy = __fmaf_rn(sr.y, -1.f, tr.y), dz = __fmaf_rn(sr.z, -1.f, tr.z);
  float r2 = __fmul_rn(dx, dx);
  r2 = __fmaf_rn(dy, dy, r2);
  r2 = __fmaf_rn(dz, dz, r2);
  const float inv = rsqrtf(fmaxf(r2, dc2));
  const float qi = __fmul_rn((float)sv.w, inv);
  const float qi3 = __fmul_rn(qi, __fmul_rn(inv, inv));
  double p = -(double)qi, gx = (double)qi3 * dx, gy = (double)qi3 * dy, gz = (double)qi3 * dz;  // remove FP32
  const double ex = tv.x - sv.x, ey = tv.y - sv.y, ez = tv.z - sv.z;
  const double e2 = ex * ex + ey * ey + ez * ez;
  if (e2 > 0.0) {
    const double ir = rsqrt(e2), qe = sv.w * ir, qe3 = qe * ir * ir;
    p += qe;
    gx -= qe3 * ex;
    gy -= qe3 * ey;
    gz -= qe3 * ez;
  }
  double* o = a.out + (int64_t)pr.x * 4;
  atomicAdd(o, p * INV4PI);
  atomicAdd(o + 1, gx * INV4PI);
  atomicAdd(o + 2, gy * INV4PI);
  atomicAdd(o + 3, gz * INV4PI);
}

#ifndef XFMM_NEAR_MAXTPL
#define XFMM_NEAR_MAXTPL 2  // targets per lane of the FP32 near-field kernel (compile-time tunable)
#endif
#ifndef XFMM_NEAR_MINB
#define XFMM_NEAR_MINB 1  // minimum resident blocks per SM requested from the register allocator
#endif

template <int KER, class R>
__global__ void __launch_bounds__(128, XFMM_NEAR_MINB) k_near(NearArgs a) {
  __shared__ NearSmem<R> sm[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * 4 + wid;
  if (w >= a.n_eval) return;
  const int node = a.leafs[a.eval_leafs[w]];
  const int T = a.ntrgs[node];
  if constexpr (sizeof(R) == 4) {
    if (T <= 32 || XFMM_NEAR_MAXTPL == 1) near_leaf<KER, R, 1>(a, node, lane, sm[wid]);
    else if (T <= 64 || XFMM_NEAR_MAXTPL == 2) near_leaf<KER, R, (XFMM_NEAR_MAXTPL >= 2 ? 2 : 1)>(a, node, lane, sm[wid]);
    else if (T <= 96 || XFMM_NEAR_MAXTPL == 3) near_leaf<KER, R, (XFMM_NEAR_MAXTPL >= 3 ? 3 : 1)>(a, node, lane, sm[wid]);
    else near_leaf<KER, R, (XFMM_NEAR_MAXTPL >= 4 ? 4 : 1)>(a, node, lane, sm[wid]);
  } else {
    // FP64: one target per lane keeps occupancy up (two per lane: 134 registers, 27.6 -> 31.3 ms at 4M)
    near_leaf<KER, R, 1>(a, node, lane, sm[wid]);
  }
}

// ================================================================ P2M check potentials and P2L
// Potential at `n` surface points (base * b around centre cn) from body range(s); warp per node.
// The Laplace operators are scale-invariant: computed for root radius pre_r0, they serve a tree of root
// radius r0 = lambda pre_r0 unchanged except for a factor lambda on the check potentials that come straight
// from bodies (P2M, P2L).  With the kernel 1 / (4 pi r), K(lambda x, lambda y) = K(x, y) / lambda: the
// check-to-equivalent pseudo-inverse scales by lambda, M2M and L2L (pseudo-inverse times kernel matrix)
// not at all, and the M2L kernel table by 1 / lambda.  Scaling the P2M check potentials by lambda gives the
// true upward densities; the M2L then yields lambda times the true downward check potentials, which P2L
// must match, and the unscaled pseudo-inverse of L2P maps them to the true downward densities.
inline double op_scale(const Fmm& f, const Tree& t) { return f.kernel == XFMM_LAPLACE ? t.r0 / f.pre_r0 : 1.0; }

struct SurfPotArgs {
  const int* nodes;  // node per warp (P2M: leafs; P2L: p2l_nodes)
  int count;
  const int *nsrcs, *p2l, *level;
  const int64_t *sbeg, *p2l_off;
  const double4 *center, *src4;
  const double* src_qim;
  const double* surf_base;
  int nsurf;
  double alpha;        // 2.95 (P2M check) or 1.05 (P2L dn check)
  void* out;           // working values
  int out_by_node;     // 0: row = warp index (P2M chk[pos]); 1: row = node (P2L into dn, accumulate)
  double k_re, k_im;
  double scale;        // 1 / (4 pi) x op_scale(f, t): the Green's function constant and the operators' r0 scale
};

template <int KER, class R>
__global__ void __launch_bounds__(128) k_surf_pot(SurfPotArgs a) {
  using G = Green<KER, R>;
  using Q = typename G::Q;
  using V4 = typename R4<R>::type;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * 4 + wid;
  if (w >= a.count) return;
  __shared__ V4 s_xyz[4][32];
  __shared__ Q s_q[4][32];
  const G g{(R)a.k_re, (R)a.k_im};
  const int node = a.nodes[w];
  const double4 c = a.center[node];
  const double b = a.alpha * c.w;
  const int n = a.nsurf;
  Q* out = (Q*)a.out + (int64_t)(a.out_by_node ? node : w) * n;
  const bool p2l = a.out_by_node;
  const int64_t e0 = p2l ? a.p2l_off[node] : 0, e1 = p2l ? a.p2l_off[node + 1] : 1;
  bool first = !p2l;
  for (int64_t e = e0; e < e1; e++) {
    const int s = p2l ? a.p2l[e] : node;
    const int ns = a.nsrcs[s];
    const int64_t sb = a.sbeg[s];
    for (int j0 = 0; j0 < ns || (first && j0 == 0); j0 += 32) {
      const int cnt = max(0, min(32, ns - j0));
      if (lane < cnt) {
        const double4 sv = a.src4[sb + j0 + lane];
        s_xyz[wid][lane] = V4{(R)(sv.x - c.x), (R)(sv.y - c.y), (R)(sv.z - c.z), (R)0};
        s_q[wid][lane] = load_charge<Q>(sv, a.src_qim, sb + j0 + lane);
      }
      __syncwarp();
      for (int k = lane; k < n; k += 32) {
        const R px = (R)(a.surf_base[3 * k] * b), py = (R)(a.surf_base[3 * k + 1] * b),
                pz = (R)(a.surf_base[3 * k + 2] * b);
        Q acc = vzero<Q>();
        for (int j = 0; j < cnt; j++) {
          const V4 sx = s_xyz[wid][j];
          g.pot(px - sx.x, py - sx.y, pz - sx.z, s_q[wid][j], acc);
        }
        acc = vscale(acc, (typename Base<Q>::type)a.scale);
        out[k] = first ? acc : vadd(out[k], acc);
      }
      first = false;
      __syncwarp();
    }
  }
}

// P2M check potentials of the Laplace mixed path with paired FP32: two sources per instruction
// (__ffma2_rn etc.), 64 sources staged per chunk as float2 pairs, each lane holding SP_KB check points
// per block.  The check surface (half-width 2.95 r) lies at least 1.95 r from every body of the leaf,
// so no pair coincides (no r == 0 mask) and single FP32 coordinates relative to the leaf centre keep
// the separations accurate to a few ulps.  Padding sources have zero charge.
constexpr int SP_KB = 8;  // check points per lane per block
struct SurfSmemF2 {
  float4 pr[32][2];  // source pair j = sources 2j, 2j + 1: {x, x, y, y}, {z, z, q, q}
};
__global__ void __launch_bounds__(128) k_surf_pot_lap_f2(SurfPotArgs a) {
  __shared__ SurfSmemF2 sm[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * 4 + wid;
  if (w >= a.count) return;
  const int node = a.nodes[w];
  const double4 c = a.center[node];
  const double b = a.alpha * c.w;
  const int n = a.nsurf, ns = a.nsrcs[node];
  const int64_t sb = a.sbeg[node];
  float* out = (float*)a.out + (int64_t)w * n;
  const float2 M1 = make_float2(-1.f, -1.f);
  for (int j0 = 0; j0 < ns || j0 == 0; j0 += 64) {
    const bool first = j0 == 0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int j = j0 + 32 * h + lane;
      float x = 0.f, y = 0.f, z = 0.f, q = 0.f;
      if (j < ns) {
        const double4 sv = a.src4[sb + j];
        x = (float)(sv.x - c.x);
        y = (float)(sv.y - c.y);
        z = (float)(sv.z - c.z);
        q = (float)sv.w;
      }
      float* r = reinterpret_cast<float*>(sm[wid].pr[16 * h + (lane >> 1)]) + (lane & 1);
      r[0] = x;
      r[2] = y;
      r[4] = z;
      r[6] = q;
    }
    __syncwarp();
    const int npair = (min(64, max(ns - j0, 0)) + 1) >> 1;
    for (int k0 = 0; k0 < n; k0 += 32 * SP_KB) {
      const int nk = min(SP_KB, (n - k0 + 31) >> 5);  // slots of this block holding points (warp-uniform)
      float2 px[SP_KB], py[SP_KB], pz[SP_KB], acc[SP_KB];
#pragma unroll
      for (int i = 0; i < SP_KB; i++) {
        const int k = min(k0 + lane + 32 * i, n - 1);  // lanes past the end repeat the last point
        px[i] = dup2((float)(a.surf_base[3 * k] * b));
        py[i] = dup2((float)(a.surf_base[3 * k + 1] * b));
        pz[i] = dup2((float)(a.surf_base[3 * k + 2] * b));
        acc[i] = make_float2(0.f, 0.f);
      }
      for (int jp = 0; jp < npair; jp++) {
        const float4 A = sm[wid].pr[jp][0], B = sm[wid].pr[jp][1];
        const float2 SX = make_float2(A.x, A.y), SY = make_float2(A.z, A.w);
        const float2 SZ = make_float2(B.x, B.y), Q = make_float2(B.z, B.w);
#pragma unroll
        for (int i = 0; i < SP_KB; i++) {
          if (i >= nk) break;
          const float2 dx = __ffma2_rn(SX, M1, px[i]), dy = __ffma2_rn(SY, M1, py[i]), dz = __ffma2_rn(SZ, M1, pz[i]);
          float2 r2 = __fmul2_rn(dx, dx);
          r2 = __ffma2_rn(dy, dy, r2);
          r2 = __ffma2_rn(dz, dz, r2);
          acc[i] = __ffma2_rn(Q, make_float2(rsqrtf(r2.x), rsqrtf(r2.y)), acc[i]);
        }
      }
#pragma unroll
      for (int i = 0; i < SP_KB; i++) {
        const int k = k0 + lane + 32 * i;
        if (k < n) {
          const float o = (acc[i].x + acc[i].y) * (float)a.scale;
          out[k] = first ? o : out[k] + o;
        }
      }
    }
    __syncwarp();
  }
}

// ================================================================ M2L grid fallback (cuFFT, p beyond the DFT kernels)
template <class W>
__global__ void k_m2l_grid_up(const int* __restrict__ src, int nsrc, const int* __restrict__ child0,
                              const W* __restrict__ up, int nsurf, const int* __restrict__ conv2surf, int nconv,
                              W* __restrict__ grid) {
  const int64_t total = (int64_t)nsrc * 8 * nconv;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int g = (int)(e % nconv);
    const int64_t sc = e / nconv;
    const int sidx = (int)(sc >> 3), c = (int)(sc & 7);
    const int k = conv2surf[g];
    grid[e] = k >= 0 ? up[((int64_t)child0[src[sidx]] + c) * nsurf + k] : vzero<W>();
  }
}

// out[col][row] = in[row][col] for an R x C matrix of complex values (32x32 tiles)
template <class CT>
__global__ void k_transpose(const CT* __restrict__ in, CT* __restrict__ out, int64_t R, int64_t C) {
  __shared__ CT tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t r = r0 + i, c = c0 + threadIdx.x;
    if (r < R && c < C) tile[i][threadIdx.x] = in[r * C + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < R && c < C) out[c * R + r] = tile[threadIdx.x][i];
  }
}
// x rounded to TF32 (10 explicit mantissa bits), to nearest with ties away from zero: half of the 13
// dropped bits' range is added to the magnitude and the dropped bits are cleared (a carry moves into
// the exponent when the rounding crosses a binade).  Integer ALU work, where the conversion instruction
// would run on the much narrower transcendental/conversion pipe.
__device__ __forceinline__ uint32_t tf32_head(float x) { return (__float_as_uint(x) + 0x1000u) & 0xffffe000u; }
template <class CT>
void transpose(const CT* in, CT* out, int64_t R, int64_t C, cudaStream_t s) {
  dim3 grid((unsigned)((C + 31) / 32), (unsigned)((R + 31) / 32));
  XREQUIRE(grid.y < 65536, XFMM_ERR_UNSUPPORTED, "transpose too tall");
  k_transpose<CT><<<grid, dim3(32, 8), 0, s>>>(in, out, R, C);
  XLAUNCH();
}

// Hadamard product per frequency (fmm_scale_invariant.h:343-399; intrinsics.h matmult_8x8x2):
//   out[f][t][tc] = sum_ipos sum_sc T[ipos][f][sc*8 + tc] * in[f][src(t, ipos)][sc]
// The FP64 path's form runs on the FP64 tensor cores (k_hadamard_d64), the mixed path's forms on the
// TF32 tensor cores (k_hadamard_dt, k_hadamard_rt below).

// Hadamard product of the FP64 path on the FP64 tensor cores (DMMA, mma.sync m8n8k4 f64), dense form for
// every target: per frequency, D[target][16] = A[target][26 x 16] B[26 x 16][16] as in k_hadamard_dt,
// accumulated in FP64 by the tensor core across the positions.  A warp owns HAD64_TW tiles of 8 targets;
// per (tile, position) eight DMMAs (4 reduction steps x 2 output halves) add the position's products to the
// tile's accumulators.  The reduction index of step c is input real 4 t + c, so that a lane (g, t) supplies
// the reals 4 t .. 4 t + 3 of its target g's source spectrum (32 contiguous bytes) and receives the output
// component 4 h + t (re, im) of target g.  A position none of a tile's 8 targets occupies is skipped (warp
// ballot); sources are loaded one position ahead.
constexpr int HAD64_NT = 256, HAD64_TW = 2;
constexpr int HAD64_TT = (HAD64_NT / 32) * 8 * HAD64_TW;  // targets per CTA
constexpr size_t HAD64_SMEM = (size_t)26 * 4 * 2 * 32 * sizeof(double);

__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// tab: [26][ld] compact source index of target k at each position (-1: empty or padding); rows: [ld]
// output row of target k (-1: padding); ld a multiple of HAD64_TT
__global__ void __launch_bounds__(HAD64_NT, 2)
    k_hadamard_d64(const double2* __restrict__ T, const double2* __restrict__ in, double2* __restrict__ out,
                   const int* __restrict__ tab, int ld, const int* __restrict__ rows, int nsrc, int ntrg, int nfreq) {
  // sB[((ipos * 4 + c) * 2 + h) * 32 + lane] = B[input real 4 t + c][output real 8 h + g] for that lane
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sB = reinterpret_cast<double*>(smem_raw);
  const int f = blockIdx.y, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int e = tid; e < 26 * 4 * 2 * 32; e += HAD64_NT) {
    const int ln = e & 31, h = (e >> 5) & 1, c = (e >> 6) & 3, ipos = e >> 8;
    const int gg = ln >> 2, tt = ln & 3;
    const int sc = 2 * tt + (c >> 1), ri = c & 1;      // input real 4 tt + c: component sc, re / im
    const int o = 8 * h + gg, tc = o >> 1, ro = o & 1;  // output real o: component tc, re / im
    const double2 m = T[((int64_t)ipos * nfreq + f) * 64 + sc * 8 + tc];
    // output re <- (Re m, -Im m) . (in re, in im); output im <- (Im m, Re m)
    sB[e] = ro == 0 ? (ri == 0 ? m.x : -m.y) : (ri == 0 ? m.y : m.x);
  }
  __syncthreads();
  const int g = lane >> 2, t = lane & 3;
  const double2* inf = in + (int64_t)f * nsrc * 8 + 2 * t;  // components 2 t, 2 t + 1: reals 4 t .. 4 t + 3
  auto load4 = [&](int sidx) {
    if (sidx < 0) return make_double4(0.0, 0.0, 0.0, 0.0);
    const double2 u = __ldg(inf + (int64_t)sidx * 8), v = __ldg(inf + (int64_t)sidx * 8 + 1);
    return make_double4(u.x, u.y, v.x, v.y);
  };
  const int base = blockIdx.x * HAD64_TT + wid * 8 * HAD64_TW + g;  // this lane's target in tile j: base + 8 j
  double acc[HAD64_TW][2][2];
  int src[HAD64_TW], srcn[HAD64_TW];
  double4 x[HAD64_TW];
#pragma unroll
  for (int j = 0; j < HAD64_TW; j++) {
#pragma unroll
    for (int h = 0; h < 2; h++) acc[j][h][0] = acc[j][h][1] = 0.0;
    src[j] = tab[base + 8 * j];
    srcn[j] = tab[ld + base + 8 * j];
    x[j] = load4(src[j]);
  }
  for (int ipos = 0; ipos < 26; ipos++) {
    // next position's source pieces, and the position after's source indices
    double4 xn[HAD64_TW];
    int srcnn[HAD64_TW];
#pragma unroll
    for (int j = 0; j < HAD64_TW; j++) {
      xn[j] = ipos + 1 < 26 ? load4(srcn[j]) : make_double4(0.0, 0.0, 0.0, 0.0);
      srcnn[j] = ipos + 2 < 26 ? tab[(ipos + 2) * ld + base + 8 * j] : -1;
    }
    double b[4][2];
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
      for (int h = 0; h < 2; h++) b[c][h] = sB[((ipos * 4 + c) * 2 + h) * 32 + lane];
#pragma unroll
    for (int j = 0; j < HAD64_TW; j++) {
      if (__ballot_sync(0xffffffffu, src[j] >= 0) == 0u) continue;  // no target of the tile here
      const double a[4] = {x[j].x, x[j].y, x[j].z, x[j].w};
#pragma unroll
      for (int c = 0; c < 4; c++)
#pragma unroll
        for (int h = 0; h < 2; h++) dmma_884(acc[j][h], a[c], b[c][h]);
    }
#pragma unroll
    for (int j = 0; j < HAD64_TW; j++) {
      src[j] = srcn[j];
      srcn[j] = srcnn[j];
      x[j] = xn[j];
    }
  }
  double2* of = out + (int64_t)f * ntrg * 8;
#pragma unroll
  for (int j = 0; j < HAD64_TW; j++) {
    const int row = rows[base + 8 * j];
    if (row < 0) continue;
#pragma unroll
    for (int h = 0; h < 2; h++) of[(int64_t)row * 8 + 4 * h + t] = make_double2(acc[j][h][0], acc[j][h][1]);
  }
}

// M2L Hadamard product of the mixed path on the tensor cores (below).  Targets are split by how many of
// the 26 relative positions are occupied: dense targets (at least HAD_DENSE_MIN) keep their sums in
// registers across the positions (k_hadamard_dt); sparse targets -- the deepest nonleaf level, ~7 of 26 --
// are scheduled by position (k_hadamard_rt): a CTA owns HADR_TT sparse targets at one frequency, their
// pairs are grouped by position and packed on the host into rounds of HADR_RW pairs that share one 8x8
// block, and each pair's products are added to its output row with 16-byte vector atomics resolved in
// L2 (the sums are taken in a run-dependent order) on rows the same CTA zeroed first.
// Spectra and products are frequency-major, (frequency f, node, child c) at [(f * nnodes + node) * 8 + c]:
// a CTA (one frequency) reads its sources from one block of the spectra and writes its rows contiguously.
#ifndef XFMM_HAD_DENSE_MIN
#define XFMM_HAD_DENSE_MIN 12
#endif
constexpr int HAD_DENSE_MIN = XFMM_HAD_DENSE_MIN;  // occupied positions that make a target dense
#ifndef XFMM_HAD_DENSE_GROUP_MIN
#define XFMM_HAD_DENSE_GROUP_MIN 256
#endif
constexpr int HAD_DENSE_GROUP_MIN = XFMM_HAD_DENSE_GROUP_MIN;  // dense targets a group needs for the dense form
constexpr int HADR_NT = 256;            // threads per CTA
constexpr int HADR_TT = 512;            // targets per tile
constexpr int HADR_RW = 64;             // pairs per round (4 row tiles of 16)
#ifndef XFMM_HADR_TPC
#define XFMM_HADR_TPC 4
#endif
constexpr int HADR_TPC = XFMM_HADR_TPC;  // default tiles per CTA (one B fill per frequency for all of them)


// Hadamard product, dense form on the tensor cores (FP32 accuracy from three TF32 products).
// Per frequency the dense product is a real GEMM, D[target][16] = A[target][26 x 16] B[26 x 16][16]:
// a target's row of A holds its 26 source spectra (8 complex = 16 reals each, zero where a position is
// empty) and B holds each position's 8x8 complex block as 2x2 real blocks ([re, im] -> [re, im]).
// Warp-level m16n8k8 TF32 MMAs: A and B are split into TF32 heads and tails, and each position's
// Ah Bh + Ah Bt + At Bh (small terms first; the tail-tail product, 2^-22 relative, is dropped) is
// formed in a fresh MMA accumulator and added to FP32 running sums.  The reduction
// index of each 8-wide step is ordered so that a lane's A fragment is one 16-byte piece of a source
// spectrum (lane quad t of a row loads reals 4t..4t+3), and the B fragments of every (position, lane)
// are laid out per frequency in shared memory.  A warp owns 64 targets as 4 tiles of 16 rows.
#ifndef XFMM_HADT_TILES
#define XFMM_HADT_TILES 4  // row tiles of 16 targets per warp
#endif
constexpr int HADT_NT = 256;                                    // threads per CTA
constexpr int HADT_TILES = XFMM_HADT_TILES;
constexpr int HADT_TT = (HADT_NT / 32) * 16 * HADT_TILES;      // targets per CTA tile
#ifndef XFMM_HADT_TPC
#define XFMM_HADT_TPC 1
#endif
constexpr int HADT_TPC = XFMM_HADT_TPC;                         // CTA tiles per CTA (one B fill for all)
constexpr size_t HADT_SMEM = (size_t)26 * 4 * 32 * 16;

__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
// head and tail of x: x = head + tail exactly, head a TF32 value
__device__ __forceinline__ void tf32_split(float x, uint32_t& h, uint32_t& t) {
  h = tf32_head(x);
  t = tf32_head(x - __uint_as_float(h));
}

// The B fragments of frequency f for every (position, reduction step c, output half h, lane):
// sB[(ipos * 4 + c * 2 + h) * 32 + lane] = {b0 head, b1 head, b0 tail, b1 tail}, step c covering the
// source components 2 t + c and half h the target components 4 h .. 4 h + 3 (t = lane % 4).
__device__ __forceinline__ void hadt_fill_b(uint4* sB, const float2* __restrict__ T, int f, int nfreq, int tid,
                                            int nthreads) {
  for (int e = tid; e < 26 * 4 * 32; e += nthreads) {
    const int ln = e & 31, q = (e >> 5) & 3, ipos = e >> 7;
    const int c = q >> 1, h = q & 1, g = ln >> 2, t = ln & 3;
    const int sc = 2 * t + c, tc = 4 * h + (g >> 1);
    const float2 m = T[((int64_t)ipos * nfreq + f) * 64 + sc * 8 + tc];
    // input real (sc, re) -> b0, (sc, im) -> b1; output real (tc, g & 1): re <- (Re m, -Im m), im <- (Im m, Re m)
    const float v0 = (g & 1) ? m.y : m.x, v1 = (g & 1) ? m.x : -m.y;
    uint4 b;
    tf32_split(v0, b.x, b.z);
    tf32_split(v1, b.y, b.w);
    sB[e] = b;
  }
}

// D (16 x 16) += rows (x0: row g, x1: row g + 8) times the position's B, one fresh MMA accumulator:
// d[h][0..1] = row g, target component 4 h + t (re, im); d[h][2..3] = row g + 8
__device__ __forceinline__ void hadt_tile(const float4& x0, const float4& x1, const uint4 (&b)[4], float (&d)[2][4]) {
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int i = 0; i < 4; i++) d[h][i] = 0.f;
#pragma unroll
  for (int c = 0; c < 2; c++) {
    uint32_t a0h, a0t, a1h, a1t, a2h, a2t, a3h, a3t;
    tf32_split(c == 0 ? x0.x : x0.z, a0h, a0t);
    tf32_split(c == 0 ? x1.x : x1.z, a1h, a1t);
    tf32_split(c == 0 ? x0.y : x0.w, a2h, a2t);
    tf32_split(c == 0 ? x1.y : x1.w, a3h, a3t);
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uint4 bb = b[c * 2 + h];
      mma_tf32(d[h], a0t, a1t, a2t, a3t, bb.x, bb.y);
      mma_tf32(d[h], a0h, a1h, a2h, a3h, bb.z, bb.w);
      mma_tf32(d[h], a0h, a1h, a2h, a3h, bb.x, bb.y);
    }
  }
}

// Round form on the tensor cores (sparse targets): each round of 64 same-position pairs as 4 row tiles of
// 16 (pair 16 j + g and 16 j + 8 + g of tile j); lanes t and t ^ 1 trade halves so each adds 16 bytes
// (two target components of one pair) with a vector atomic.  Rounds [r0, r1) at one frequency: warp wid
// takes every (HADR_NT / 32)-th round; inf points at the frequency's spectra (+ lane quad offset t), of at
// its product rows, and the rows were zeroed by the same CTA.
__device__ __forceinline__ void hadr_rounds(const uint4* sB, const float4* __restrict__ inf, float2* of,
                                            const int* __restrict__ rpos, const int2* __restrict__ ent, int r0,
                                            int r1, int wid, int lane) {
  constexpr int NW = HADR_NT / 32;
  static_assert(HADR_RW == 64, "a round is 4 row tiles of 16 pairs");
  const int g = lane >> 2, t = lane & 3;
  // a round's pairs (source, output row) and their spectra, all loads in flight at once
  auto load_round = [&](int r, int2 (&ee)[4][2], float4 (&xx)[4][2]) {
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int rr = 0; rr < 2; rr++) ee[j][rr] = ent[(int64_t)r * HADR_RW + 16 * j + 8 * rr + g];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int rr = 0; rr < 2; rr++)
        xx[j][rr] = ee[j][rr].x >= 0 ? __ldg(inf + (int64_t)ee[j][rr].x * 4) : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  for (int r = r0 + wid; r < r1; r += NW) {
    const int ipos = rpos[r];
    uint4 b[4];
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = sB[(ipos * 4 + q) * 32 + lane];
    int2 ee[4][2];
    float4 xx[4][2];
    load_round(r, ee, xx);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      float d[2][4];
      hadt_tile(xx[j][0], xx[j][1], b, d);
      const bool odd = t & 1;
      const int2 e = odd ? ee[j][1] : ee[j][0];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        // even t keeps row g (components 4h + t, 4h + t + 1); odd t keeps row g + 8 (4h + t - 1, 4h + t)
        const float2 send = odd ? make_float2(d[h][0], d[h][1]) : make_float2(d[h][2], d[h][3]);
        const float rx = __shfl_xor_sync(0xffffffffu, send.x, 1), ry = __shfl_xor_sync(0xffffffffu, send.y, 1);
        const float4 v = odd ? make_float4(rx, ry, d[h][2], d[h][3]) : make_float4(d[h][0], d[h][1], rx, ry);
        if (e.x >= 0) atomicAdd(reinterpret_cast<float4*>(of + (int64_t)e.y * 8 + 4 * h + (t & ~1)), v);
      }
    }
  }
}

__global__ void __launch_bounds__(HADR_NT, 3)  // 3 blocks/SM measured best (80 registers, a 16-byte spill)
    k_hadamard_rt(const float2* __restrict__ T, const float2* __restrict__ in, float2* __restrict__ out,
                  const int* __restrict__ tile_r, const int* __restrict__ rpos, const int2* __restrict__ ent,
                  const int* __restrict__ rows, int ntiles, int tpc, int nsrc, int ntrg, int nfreq) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint4* sB = reinterpret_cast<uint4*>(smem_raw);
  const int f = blockIdx.y, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  // tiles [tb, te) share this CTA's B fragments of frequency f
  const int tb = blockIdx.x * tpc, te = min(ntiles, tb + tpc);
  float2* of = out + (int64_t)f * ntrg * 8;
  // every product of these tiles' targets at frequency f is added by this CTA: their rows start at zero
  for (int e = tid; e < (te - tb) * HADR_TT * 4; e += HADR_NT) {
    const int row = rows[tb * HADR_TT + (e >> 2)];
    if (row >= 0) reinterpret_cast<float4*>(of + (int64_t)row * 8)[e & 3] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  hadt_fill_b(sB, T, f, nfreq, tid, HADR_NT);
  __syncthreads();
  const float4* inf = reinterpret_cast<const float4*>(in + (int64_t)f * nsrc * 8) + (lane & 3);
  hadr_rounds(sB, inf, of, rpos, ent, tile_r[tb], tile_r[te], wid, lane);
}

// The round form over the sparse tiles of many systems that share one operator table (a batch of Laplace
// systems): tiles[k] = (system, its tile), and a CTA covers tiles [tb, te) of the list, possibly of several
// systems, with one B fill per frequency.
struct HadSys {
  const float2* in;     // spectra [f][source][child]
  float2* out;          // products [f][target][child]
  const int* tile_r;    // rounds of each sparse tile (CSR)
  const int* rpos;      // relative position of each round
  const int2* ent;      // pairs of each round
  const int* rows;      // HADR_TT output rows per tile
  int nsrc, ntrg;
};
__global__ void __launch_bounds__(HADR_NT, 3)
    k_hadamard_rt_batch(const float2* __restrict__ T, const HadSys* __restrict__ sys, const int2* __restrict__ tiles,
                        int ntiles, int tpc, int nfreq) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint4* sB = reinterpret_cast<uint4*>(smem_raw);
  const int f = blockIdx.y, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int tb = blockIdx.x * tpc, te = min(ntiles, tb + tpc);
  for (int k = tb; k < te; k++) {
    const int2 tl = tiles[k];
    const HadSys& S = sys[tl.x];
    float2* of = S.out + (int64_t)f * S.ntrg * 8;
    const int* rows = S.rows + (int64_t)tl.y * HADR_TT;
    for (int e = tid; e < HADR_TT * 4; e += HADR_NT) {
      const int row = rows[e >> 2];
      if (row >= 0) reinterpret_cast<float4*>(of + (int64_t)row * 8)[e & 3] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  hadt_fill_b(sB, T, f, nfreq, tid, HADR_NT);
  __syncthreads();
  for (int k = tb; k < te; k++) {
    const int2 tl = tiles[k];
    const HadSys& S = sys[tl.x];
    const float4* inf = reinterpret_cast<const float4*>(S.in + (int64_t)f * S.nsrc * 8) + (lane & 3);
    hadr_rounds(sB, inf, S.out + (int64_t)f * S.ntrg * 8, S.rpos, S.ent, S.tile_r[tl.y], S.tile_r[tl.y + 1], wid,
                lane);
  }
}

// tab: [26][ld] compact source index of dense target k at each position (-1: empty or padding);
// rows: [ld] output row of dense target k (-1: padding).  ld is a multiple of HADT_TT.
__global__ void __launch_bounds__(HADT_NT, 2)
    k_hadamard_dt(const float2* __restrict__ T, const float2* __restrict__ in, float2* __restrict__ out,
                  const int* __restrict__ tab, int ld, const int* __restrict__ rows, int nsrc, int ntrg, int nfreq) {
  // sB[(ipos * 4 + c * 2 + h) * 32 + lane] = {b0 head, b1 head, b0 tail, b1 tail} of reduction step c
  // (source components 2 t + c) and output half h (target components 4 h .. 4 h + 3) for that lane
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint4* sB = reinterpret_cast<uint4*>(smem_raw);  // 26 * 4 * 32 entries
  const int f = blockIdx.y, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  hadt_fill_b(sB, T, f, nfreq, tid, HADT_NT);
  __syncthreads();
  const int g = lane >> 2, t = lane & 3;
  const float4* inf = reinterpret_cast<const float4*>(in + (int64_t)f * nsrc * 8) + t;
  // CTA tiles [blockIdx.x * HADT_TPC, ...) of HADT_TT targets share this CTA's B fragments of frequency f
  for (int ct = blockIdx.x * HADT_TPC; ct < min(ld / HADT_TT, (blockIdx.x + 1) * HADT_TPC); ct++) {
  const int base = ct * HADT_TT + wid * 16 * HADT_TILES + g;  // tile j, rows g / g + 8: base + 16 j (+ 8)
  float acc[HADT_TILES][2][4];
#pragma unroll
  for (int j = 0; j < HADT_TILES; j++)
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int i = 0; i < 4; i++) acc[j][h][i] = 0.f;
  float4 x[HADT_TILES][2];
  int srcn[HADT_TILES][2];  // source indices of the next position, loaded one position ahead
#pragma unroll
  for (int j = 0; j < HADT_TILES; j++)
#pragma unroll
    for (int r = 0; r < 2; r++) srcn[j][r] = tab[base + 16 * j + 8 * r];
  for (int ipos = 0; ipos < 26; ipos++) {
#pragma unroll
    for (int j = 0; j < HADT_TILES; j++)
#pragma unroll
      for (int r = 0; r < 2; r++) {
        const int src = srcn[j][r];
        if (ipos + 1 < 26) srcn[j][r] = tab[(ipos + 1) * ld + base + 16 * j + 8 * r];
        x[j][r] = src >= 0 ? __ldg(inf + (int64_t)src * 4) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    uint4 b[4];
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = sB[(ipos * 4 + q) * 32 + lane];
#pragma unroll
    for (int j = 0; j < HADT_TILES; j++) {
      // this position's products in a fresh MMA accumulator, then added to the running sums with
      // round-to-nearest FP32 adds (the MMA's own accumulation is not rounded to nearest)
      float d[2][4];
      hadt_tile(x[j][0], x[j][1], b, d);
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int i = 0; i < 4; i++) acc[j][h][i] += d[h][i];
    }
  }
  // D fragment: row g (and g + 8), columns 2t, 2t + 1 of half h = target component 4 h + t (re, im)
  float2* of = out + (int64_t)f * ntrg * 8;
#pragma unroll
  for (int j = 0; j < HADT_TILES; j++)
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int row = rows[base + 16 * j + 8 * r];
      if (row < 0) continue;
#pragma unroll
      for (int h = 0; h < 2; h++) of[(int64_t)row * 8 + 4 * h + t] = make_float2(acc[j][h][2 * r], acc[j][h][2 * r + 1]);
    }
  }
}

// Hadamard product, dense form on the sm_100 tensor cores through tcgen05 (FP32 accuracy from three TF32
// products, as in k_hadamard_dt), as a warp-specialised pipeline.  A CTA owns 128 dense targets (target
// slot i = TMEM lane i) and HADC_FPB frequencies, i.e. a stream of 26 HADC_FPB positions.
//   * Warps 0-3 (one per TMEM lane quarter) produce and consume: per position, the 4 lanes of a quad load
//     one source spectrum as 4 contiguous 16-byte pieces (one position ahead), split it into TF32 head
//     and tail and store both into the position's TMEM stage (operand A, `tcgen05.st.16x256b`), then
//     arrive on the stage's `full` barrier.  Before reusing a stage they wait for its `done` barrier,
//     read the products of the position HADC_S earlier back (`tcgen05.ld`) and add them to FP32 running
//     sums in registers (round-to-nearest adds; the tensor core's own accumulation never spans more than
//     one position); after a frequency's last position they store its 128 output rows.
//   * Warp 4 issues: per frequency one bulk copy of the 26 positions' B blocks (built once per operator
//     in the MMA layout by k_hadc_btab) into shared memory, then per position, once the stage is full,
//     six M128 N16 K8 kind::tf32 MMAs (A tail x B head, A head x B tail, A head x B head per 8-wide
//     step) into the stage's fresh TMEM accumulator, committed to `done`.
// No CTA-wide barrier inside the stream.  Every wait is bounded (about a second); a wait that runs out
// ends the waiting role's loop, the others then run out in turn, the CTA releases its TMEM and *status
// is set.
constexpr int HADC_NT = 160;                                // 4 producer/consumer warps + 1 MMA warp
constexpr int HADC_S = 4;                                   // TMEM stages
constexpr int HADC_D = 4;                                   // positions gathered ahead (cp.async ring)
constexpr int HADC_R = HADC_D + 1;                          // ring slots: 128 rows x 64 bytes each
constexpr int HADC_FPB = 8;                                 // frequencies per CTA
constexpr uint32_t HADC_BBYTES = 26 * 2048;                 // B of one frequency: [position][head, tail] 1 KB each
// dynamic shared memory per CTA: B, then the gather ring; at least 96 KB so that at most two CTAs share an
// SM, whose TMEM (512 columns) holds exactly two allocations of HADC_TMEM_COLS
constexpr size_t HADC_RING = (size_t)HADC_R * 128 * 64;
constexpr size_t HADC_SMEM = HADC_BBYTES + HADC_RING > 96 * 1024 ? HADC_BBYTES + HADC_RING : 96 * 1024;
static_assert(3 * HADC_SMEM > 228 * 1024 && 2 * HADC_SMEM <= 227 * 1024, "two CTAs per SM");
constexpr uint32_t HADC_TMEM_COLS = 256;                    // A: HADC_S x 32 columns, then D: HADC_S x 16
constexpr uint32_t HADC_DCOL = 32 * HADC_S;                 // first D column
constexpr long long HADC_WAIT = 2000000000LL;               // SM cycles (about a second) before a wait gives up
static_assert(HADC_DCOL + 16 * HADC_S <= HADC_TMEM_COLS, "TMEM columns");

// The A columns (reduction index) are a permutation of the 16 input reals fixed by the TMEM store shape
// (16x256b): the 4 lanes of a quad load one source spectrum as 4 contiguous 16-byte pieces, lane q the
// reals 4q .. 4q + 3, which land in columns 2q, 2q + 1, 8 + 2q, 9 + 2q.  Column of input real k:
__host__ __device__ __forceinline__ int hadc_col(int k) {
  const int q = k >> 2, r = k & 3;
  return r < 2 ? 2 * q + r : 8 + 2 * q + (r - 2);
}
// byte offset of B element (output real n, A column c) in the 1 KB block of one (position, part):
// core matrix (c / 4, n / 8) at 256 (c / 4) + 128 (n / 8), its row n % 8 at 16 (n % 8), column c % 4
__host__ __device__ __forceinline__ uint32_t hadc_boff(int n, int c) {
  return (uint32_t)((c >> 2) * 256 + (n >> 3) * 128 + (n & 7) * 16 + (c & 3) * 4);
}
// btab[f] (HADC_BBYTES per frequency): factor m(sc, tc) of position ipos -> the real 2 x 2 block
// (outputs 2 tc, 2 tc + 1; inputs 2 sc, 2 sc + 1) = [[Re m, -Im m], [Im m, Re m]], TF32 head then tail
__global__ void k_hadc_btab(const float2* __restrict__ T, int nfreq, unsigned char* __restrict__ btab) {
  const int64_t total = (int64_t)nfreq * 26 * 64;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int f = (int)(e / (26 * 64)), ipos = (int)(e / 64 % 26), sc = (int)(e >> 3 & 7), tc = (int)(e & 7);
    const float2 m = T[((int64_t)ipos * nfreq + f) * 64 + sc * 8 + tc];
    const float v[4] = {m.x, -m.y, m.y, m.x};
    unsigned char* blk = btab + (int64_t)f * HADC_BBYTES + ipos * 2048;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint32_t off = hadc_boff(2 * tc + (j >> 1), hadc_col(2 * sc + (j & 1)));
      uint32_t h, t;
      tf32_split(v[j], h, t);
      *reinterpret_cast<uint32_t*>(blk + off) = h;
      *reinterpret_cast<uint32_t*>(blk + 1024 + off) = t;
    }
  }
}
// a bounded wait whose outcome every lane of the warp shares
__device__ __forceinline__ bool hadc_wait(uint32_t mbar, uint32_t parity) {
  return __all_sync(0xffffffffu, tc5::mbar_wait(mbar, parity, HADC_WAIT));
}

__global__ void __launch_bounds__(HADC_NT, 2)
    k_hadamard_dc(const unsigned char* __restrict__ btab, const float2* __restrict__ in, float2* __restrict__ out,
                  const int* __restrict__ tab, int ld, const int* __restrict__ rows, int nsrc, int ntrg, int nfreq,
                  int* __restrict__ status) {
  using namespace tc5;
  extern __shared__ __align__(16) unsigned char smem_raw[];  // B blocks of the current frequency, gather ring
  __shared__ __align__(8) uint64_t mbar[2 * HADC_S + 2];       // full[S], done[S], B half 0, B half 1
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
  const uint32_t sB = smem_u32(smem_raw);
  const uint32_t full0 = smem_u32(&mbar[0]), done0 = smem_u32(&mbar[HADC_S]), barB0 = smem_u32(&mbar[2 * HADC_S]);
  if (wid == 0) {
    tmem_alloc(smem_u32(&tmem_base), HADC_TMEM_COLS);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int s = 0; s < HADC_S; s++) {
      mbar_init(full0 + 8 * s, 4);
      mbar_init(done0 + 8 * s, 1);
    }
    mbar_init(barB0, 1);
    mbar_init(barB0 + 8, 1);
    fence_mbar_init();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tm = __shfl_sync(0xffffffffu, tmem_base, 0);
  const int fbeg = blockIdx.y * HADC_FPB, nf = min(HADC_FPB, nfreq - fbeg);
  const int G = 26 * nf;  // positions in this CTA's stream
  bool ok = true;
  if (wid == 4) {
    // ---------------- MMA warp
    // B in two halves (positions 0-12, 13-25), each refilled for the next frequency as soon as the MMAs
    // that read it have completed: half 0 once position 12 is done (checked before position 12 + S, which
    // reuses its stage), half 1 once position 25 is done (checked before the next frequency's position
    // S - 1); frequency fi waits for half h on phase fi & 1 of its barrier.
    constexpr uint32_t IDESC = idesc_tf32(128, 16);
    constexpr uint32_t HB = HADC_BBYTES / 2;
    static_assert(HADC_S <= 13 && HB % 16 == 0, "B halves");
    auto load_half = [&](int h, int fi) {
      if (elect_one()) {
        mbar_arrive_expect_tx(barB0 + 8 * h, HB);
        bulk_g2s(sB + h * HB, btab + (int64_t)(fbeg + fi) * HADC_BBYTES + h * HB, HB, barB0 + 8 * h);
      }
      __syncwarp();
    };
    load_half(0, 0);
    load_half(1, 0);
    int issued = 0;
    for (int gi = 0; gi < G && ok; gi++) {
      const int fi = gi / 26, p = gi - 26 * fi, s = gi % HADC_S;
      if (gi >= HADC_S && (p == 12 + HADC_S || p == HADC_S - 1)) {
        // the MMAs of position gi - S (12, or the previous frequency's 25) and all before it are done:
        // the half they read takes the next frequency's blocks
        ok = hadc_wait(done0 + 8 * s, ((gi - HADC_S) / HADC_S) & 1);
        if (!ok) break;
        if (p == 12 + HADC_S && fi + 1 < nf) load_half(0, fi + 1);
        if (p == HADC_S - 1) load_half(1, fi);
      }
      if (p == 0 || p == 13) {
        ok = hadc_wait(barB0 + 8 * (p == 13), fi & 1);
        if (!ok) break;
      }
      ok = hadc_wait(full0 + 8 * s, (gi / HADC_S) & 1);
      if (!ok) break;
      fence_after_sync();
      if (elect_one()) {
        const uint32_t dd = tm + HADC_DCOL + 16 * s, aa = tm + 32 * s, bb = sB + p * 2048;
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
          const uint64_t bh = sdesc_nosw(bb + 512 * kk, 256, 128), bt = sdesc_nosw(bb + 1024 + 512 * kk, 256, 128);
          mma_tf32_ts(dd, aa + 16 + 8 * kk, bh, IDESC, kk);  // fresh sums at the first step
          mma_tf32_ts(dd, aa + 8 * kk, bt, IDESC, 1);
          mma_tf32_ts(dd, aa + 8 * kk, bh, IDESC, 1);
        }
        commit(done0 + 8 * s);
      }
      __syncwarp();
      issued = gi + 1;
    }
    // on an early end, the MMAs in flight get a bounded time to finish before the TMEM is released
    if (!ok && issued > 0) hadc_wait(done0 + 8 * ((issued - 1) % HADC_S), ((issued - 1) / HADC_S) & 1);
  } else {
    // ---------------- producer / consumer warps (lane quarter wid)
    const int g = lane >> 2, q = lane & 3;
    const int k = blockIdx.x * 128 + tid;  // this lane's target slot = TMEM lane tid
    const uint32_t tw = tm + ((uint32_t)(wid * 32) << 16);
    const int row = rows[k];
    float acc[16];
#pragma unroll
    for (int i = 0; i < 16; i++) acc[i] = 0.f;
    auto inf_of = [&](int gi) {
      return reinterpret_cast<const float4*>(in + (int64_t)(fbeg + gi / 26) * nsrc * 8);
    };
    auto take = [&](int gp, int s) {  // products of stream position gp (stage s) into the sums
      fence_after_sync();
      uint32_t d[16];
      ld_32x32b_x16(tw + HADC_DCOL + 16 * s, d);
      wait_ld();
#pragma unroll
      for (int i = 0; i < 16; i++) acc[i] += __uint_as_float(d[i]);
      if (gp % 26 == 25) {  // a frequency's last position: its rows are complete
        if (row >= 0) {
          float4* o = reinterpret_cast<float4*>(out + ((int64_t)(fbeg + gp / 26) * ntrg + row) * 8);
#pragma unroll
          for (int i = 0; i < 4; i++) o[i] = make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);
        }
#pragma unroll
        for (int i = 0; i < 16; i++) acc[i] = 0.f;
      }
    };
    // gather ring: slot r holds, per warp and lane, the lane's 4 spectrum pieces (rows g + 8 i) of one
    // position; each lane reads back only what it copied itself
    const uint32_t ring = sB + HADC_BBYTES + (uint32_t)((wid * 4) * 32 + lane) * 16;
    auto gather = [&](int gi, int idx) {  // cp.async of position gi into its slot (one commit group)
      const float4* inf = inf_of(gi);
      const uint32_t slot = ring + (uint32_t)(gi % HADC_R) * (128 * 64);
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int src = __shfl_sync(0xffffffffu, idx, g + 8 * i);
        cp_async16(slot + i * 32 * 16, src >= 0 ? (const void*)(inf + (int64_t)src * 4 + q) : (const void*)in,
                   src >= 0 ? 16u : 0u);
      }
      cp_async_commit();
    };
    // positions 0 .. D-1 in flight, the index of position D ready
#pragma unroll
    for (int i = 0; i < HADC_D; i++) {
      if (i < G) gather(i, tab[(i % 26) * ld + k]);
      else cp_async_commit();
    }
    int idxn = HADC_D < G ? tab[(HADC_D % 26) * ld + k] : -1;
    for (int gi = 0; gi < G && ok; gi++) {
      const int s = gi % HADC_S;
      if (gi + HADC_D < G) gather(gi + HADC_D, idxn);
      else cp_async_commit();  // keep one group per position
      if (gi + HADC_D + 1 < G) idxn = tab[((gi + HADC_D + 1) % 26) * ld + k];
      cp_async_wait<HADC_D>();  // position gi's group has landed
      float4 x[4];
      {
        const float4* sl = reinterpret_cast<const float4*>(smem_raw + HADC_BBYTES + (size_t)(gi % HADC_R) * (128 * 64)) +
                           (wid * 4) * 32 + lane;
#pragma unroll
        for (int i = 0; i < 4; i++) x[i] = sl[i * 32];
      }
      if (gi >= HADC_S) {  // the stage's previous position is done: take its products, then reuse it
        ok = hadc_wait(done0 + 8 * s, ((gi - HADC_S) / HADC_S) & 1);
        if (!ok) break;
        take(gi - HADC_S, s);
      }
#pragma unroll
      for (int h = 0; h < 2; h++) {  // rows 16 h + g (x[2h]) and 16 h + g + 8 (x[2h + 1]) of the warp
        const float4 a = x[2 * h], b = x[2 * h + 1];
        const float xs[8] = {a.x, a.y, b.x, b.y, a.z, a.w, b.z, b.w};
        uint32_t ah[8], at[8];
#pragma unroll
        for (int i = 0; i < 8; i++) tf32_split(xs[i], ah[i], at[i]);
        const uint32_t ta = tw + ((uint32_t)(16 * h) << 16) + 32 * s;
        st_16x256b_x2(ta, ah);
        st_16x256b_x2(ta + 16, at);
      }
      wait_st();
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(full0 + 8 * s);
    }
    cp_async_wait<0>();
    for (int gp = max(G - HADC_S, 0); gp < G && ok; gp++) {  // the last positions' products
      const int s = gp % HADC_S;
      ok = hadc_wait(done0 + 8 * s, (gp / HADC_S) & 1);
      if (!ok) break;
      take(gp, s);
    }
  }
  fence_before_sync();
  __syncthreads();
  if (wid == 0) {
    fence_after_sync();
    tmem_dealloc(tm, HADC_TMEM_COLS);
  }
  if (!ok && lane == 0) atomicExch(status, 1);
}

// ---------------------------------------------------------------- M2L transforms of the real kernels
// The convolution grid of one child is n1^3 (n1 = 2p), index a + b n1 + c n1^2 (a fastest).  The upward
// equivalent values occupy the corner [0, p)^3 (geometry.h:101-134, up), the downward check values are
// read from the corner [p, 2p)^3 (down).  The forward transform is the real-to-half-complex DFT of the
// grid (factor e^{-2 pi i k n / n1}, unnormalised, frequency f = (kc n1 + kb)(p + 1) + ka), the backward
// one the half-complex-to-real DFT (factor e^{+...}, unnormalised): the transforms of the reference's
// FFTW plans (fmm_scale_invariant.h:560-646).  Because only a p^3 corner of each input is non-zero and
// only a p^3 corner of each output is used, both are computed as three passes of direct sums, one axis
// at a time, in shared memory: no grid is materialised, and each spectrum value is written once by
// the forward transform (k_m2l_fwd_r, below) and read once by the backward one (k_m2l_bwd_r below; FP64:
// k_m2l_bwd here), in the Hadamard product's [frequency][node][child] layout.  A CTA handles FtCpb(R)
// children of one node: their spectrum values of one frequency are contiguous.  The expansion order P
// is a template parameter (2 <= P <= FT_PMAX), so every loop unrolls; k_m2l_bwd keeps each DFT factor
// w^(jk mod n1) in a register chosen at compile time.
constexpr int FT_NT = 256;
constexpr int FT_PMAX = 10;
template <class R> struct FtCpb;
template <> struct FtCpb<float> { static constexpr int v = 8; };   // 64-byte chunks of float2
template <> struct FtCpb<double> { static constexpr int v = 4; };  // 64-byte chunks of double2
template <class R> struct FtMinB;  // k_m2l_bwd (FP64 only)
template <> struct FtMinB<double> { static constexpr int v = 1; };

// calls fn(std::integral_constant<int, p>) for 2 <= p <= FT_PMAX
template <class F>
void ft_dispatch(int p, F&& fn) {
  switch (p) {
    case 2: fn(std::integral_constant<int, 2>()); break;
    case 3: fn(std::integral_constant<int, 3>()); break;
    case 4: fn(std::integral_constant<int, 4>()); break;
    case 5: fn(std::integral_constant<int, 5>()); break;
    case 6: fn(std::integral_constant<int, 6>()); break;
    case 7: fn(std::integral_constant<int, 7>()); break;
    case 8: fn(std::integral_constant<int, 8>()); break;
    case 9: fn(std::integral_constant<int, 9>()); break;
    case 10: fn(std::integral_constant<int, 10>()); break;
    default: throw Error(XFMM_ERR_UNSUPPORTED, "M2L transform kernels cover 2 <= p <= 10");
  }
}

template <class R>
size_t ft_fwd_smem(int p) {  // k_m2l_bwd's shared memory: [CPB][p][n1][H] + [CPB][p][p][H] complex values
  const int n1 = 2 * p, h = p + 1, cpb = FtCpb<R>::v;
  return sizeof(typename C2<R>::type) * ((size_t)cpb * p * p * h + (size_t)cpb * p * n1 * h);
}
template <class R>
size_t ft_bwd_smem(int p) { return ft_fwd_smem<R>(p); }

template <class CT>
__device__ __forceinline__ CT ft_mul(CT a, CT b) {
  return CT{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// w[m] = e^{sign 2 pi i m / n1} from the (cos, sin) table
template <class CT, int N>
__device__ __forceinline__ void ft_load_w(const double* __restrict__ tw, double sign, CT (&w)[N]) {
#pragma unroll
  for (int m = 0; m < N; m++) {
    w[m].x = (decltype(w[m].x))tw[2 * m];
    w[m].y = (decltype(w[m].x))(sign * tw[2 * m + 1]);
  }
}

// dn[child of target trg[t]][k] += scale[t] * backward DFT of spec[.][t][child] at map_dn[k]
template <class R, int P>
__global__ void __launch_bounds__(FT_NT, FtMinB<R>::v)
    k_m2l_bwd(const int* __restrict__ trg, int nt, const int* __restrict__ child0,
              const typename C2<R>::type* __restrict__ spec, int nsurf, const int* __restrict__ map_dn,
              const double* __restrict__ tw, const R* __restrict__ scale, R* __restrict__ dn) {
  using CT = typename C2<R>::type;
  constexpr int CPB = FtCpb<R>::v, N = 2 * P, H = P + 1, NC = N * H;
  const int t = blockIdx.x, ch0 = blockIdx.y * CPB, tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CT* sZ1 = reinterpret_cast<CT*>(smem_raw);  // [CPB][c' < P][kb < N][ka < H]
  CT* sZ2 = sZ1 + CPB * P * NC;               // [CPB][c' < P][b' < P][ka < H]
  __shared__ CT sw[2 * FT_PMAX];
  CT w[N];
  ft_load_w(tw, 1.0, w);
  if (tid < N) sw[tid] = CT{(R)tw[2 * tid], (R)tw[2 * tid + 1]};
  // pass A, along kc, to the outputs c = P + c', one column (ch, kb, ka) per task.  With kc = k + P j
  // (j = 0, 1): w^{(k + P j) m} = (-1)^{j m} w^{k m}, so output m = P + c' is the P-term sum over k of
  // (v[k] + v[k + P]) w^{k m} for even m and (v[k] - v[k + P]) w^{k m} for odd m.
  for (int e = tid; e < NC * CPB; e += FT_NT) {
    const int ch = e % CPB, col = e / CPB;
    const CT* y = spec + ((int64_t)col * nt + t) * 8 + ch0 + ch;
    const int64_t fstride = (int64_t)NC * nt * 8;
    CT up[P], um[P];
#pragma unroll
    for (int k = 0; k < P; k++) {
      const CT a = y[k * fstride], b = y[(k + P) * fstride];
      up[k] = CT{a.x + b.x, a.y + b.y};
      um[k] = CT{a.x - b.x, a.y - b.y};
    }
#pragma unroll
    for (int cc = 0; cc < P; cc++) {
      const bool odd = (P + cc) & 1;
      CT acc = odd ? um[0] : up[0];
#pragma unroll
      for (int k = 1; k < P; k++) vfma(acc, odd ? um[k] : up[k], w[(k * (P + cc)) % N]);
      sZ1[(ch * P + cc) * NC + col] = acc;
    }
  }
  __syncthreads();
  // pass B, along kb, to the outputs b = P + b', one column (ch, c', ka) per task
  for (int e = tid; e < CPB * P * H; e += FT_NT) {  // same pairing of kb and kb + P as pass A
    const int ka = e % H, cc = e / H;
    CT up[P], um[P];
#pragma unroll
    for (int k = 0; k < P; k++) {
      const CT a = sZ1[(cc * N + k) * H + ka], b = sZ1[(cc * N + k + P) * H + ka];
      up[k] = CT{a.x + b.x, a.y + b.y};
      um[k] = CT{a.x - b.x, a.y - b.y};
    }
#pragma unroll
    for (int bb = 0; bb < P; bb++) {
      const bool odd = (P + bb) & 1;
      CT acc = odd ? um[0] : up[0];
#pragma unroll
      for (int k = 1; k < P; k++) vfma(acc, odd ? um[k] : up[k], w[(k * (P + bb)) % N]);
      sZ2[(cc * P + bb) * H + ka] = acc;
    }
  }
  __syncthreads();
  // pass C, along ka (half-complex to real: weight 2 except at ka = 0 and ka = N/2), at the check points;
  // the factor index (ka a mod N) depends on the point, so the factors are read from shared memory
  const int64_t node0 = (int64_t)child0[trg[t]] + ch0;
  const R sc = scale[t];
  for (int e = tid; e < CPB * nsurf; e += FT_NT) {
    const int ch = e / nsurf, k = e - ch * nsurf, g = map_dn[k];
    const int a = g % N, b = g / N % N - P, c = g / (N * N) - P;
    const CT* z = sZ2 + ((ch * P + c) * P + b) * H;
    R y = z[0].x;
    for (int ka = 1, m = a; ka < H; ka++) {
      const R wgt = 2 * ka == N ? (R)1 : (R)2;
      const CT ww = sw[m];
      y += wgt * (z[ka].x * ww.x - z[ka].y * ww.y);
      m += a;
      if (m >= N) m -= N;
    }
    R* d = dn + (node0 + ch) * nsurf + k;
    *d += sc * y;
  }
}

// ---------------------------------------------------------------- M2L transforms of the complex kernel
// The Helmholtz kernel's transforms are full complex DFTs of the n1^3 grid (forward factor
// e^{-2 pi i k n / n1}, backward e^{+...}, both unnormalised; frequency f = (kc n1 + kb) n1 + ka): the
// C2C transforms of the reference's FFTW plans (fmm.h:631-788).  They are pruned as the real ones are
// (input corner [0, p)^3, output corner [p, 2p)^3; three passes of direct sums in shared memory, outputs
// k and k + p of a length-p input from even and odd partial sums).
constexpr int FTC_PMAX = 12;
template <class F>
void ftc_dispatch(int p, F&& fn) {
  switch (p) {
    case 2: fn(std::integral_constant<int, 2>()); break;
    case 3: fn(std::integral_constant<int, 3>()); break;
    case 4: fn(std::integral_constant<int, 4>()); break;
    case 5: fn(std::integral_constant<int, 5>()); break;
    case 6: fn(std::integral_constant<int, 6>()); break;
    case 7: fn(std::integral_constant<int, 7>()); break;
    case 8: fn(std::integral_constant<int, 8>()); break;
    case 9: fn(std::integral_constant<int, 9>()); break;
    case 10: fn(std::integral_constant<int, 10>()); break;
    case 11: fn(std::integral_constant<int, 11>()); break;
    case 12: fn(std::integral_constant<int, 12>()); break;
    default: throw Error(XFMM_ERR_UNSUPPORTED, "complex M2L transform kernels cover 2 <= p <= 12");
  }
}
// y[k] for k < 2P from x[0..P): y[k] = sum_m x[m] w^{k m}, w[j] = e^{sign 2 pi i j / 2P}; outputs k and
// k + P are even + odd and even - odd (w^{(k + P) m} = (-1)^m w^{k m}); out(k, value) stores one output
template <int P, class CT, class WT, class Out>
__device__ __forceinline__ void ftc_dft_p(const CT (&x)[P], const WT& w, Out&& out) {
  constexpr int N = 2 * P;
#pragma unroll
  for (int k = 0; k < P; k++) {
    CT ev = x[0], od = ft_mul(x[1], w[k % N]);
#pragma unroll
    for (int m = 2; m < P; m += 2) vfma(ev, x[m], w[(k * m) % N]);
#pragma unroll
    for (int m = 3; m < P; m += 2) vfma(od, x[m], w[(k * m) % N]);
    out(k, CT{ev.x + od.x, ev.y + od.y});
    out(k + P, CT{ev.x - od.x, ev.y - od.y});
  }
}
// y[P + j] for j < P from X[0..2P): y[P + j] = sum_k X[k] w^{k (P + j)}; with k = k' + P i,
// w^{(k' + P i)(P + j)} = (-1)^{i (P + j)} w^{k' (P + j)}: a P-term sum of X[k'] +- X[k' + P]
template <int P, class CT, class WT, class Out>
__device__ __forceinline__ void ftc_idft_upper(const CT (&up)[P], const CT (&um)[P], const WT& w, Out&& out) {
  constexpr int N = 2 * P;
#pragma unroll
  for (int j = 0; j < P; j++) {
    const bool odd = (P + j) & 1;
    CT acc = odd ? um[0] : up[0];
#pragma unroll
    for (int k = 1; k < P; k++) vfma(acc, odd ? um[k] : up[k], w[(k * (P + j)) % N]);
    out(j, acc);
  }
}

// Children per CTA of the complex forward transform: the spectrum values of one frequency of all 8
// children of a node are one 64-byte (float2) or 128-byte (double2) row, written by consecutive lanes.
template <class R> struct FtcCpb;
template <> struct FtcCpb<float> { static constexpr int v = 8; };
template <> struct FtcCpb<double> { static constexpr int v = 4; };
#ifndef XFMM_FTC_JS
#define XFMM_FTC_JS 3
#endif
constexpr int FTC_JS = XFMM_FTC_JS;  // first-axis base frequencies j per slab: outputs ka = j and j + p
#ifndef XFMM_FTC_FWD_MINB
#define XFMM_FTC_FWD_MINB 1  // FP32: resident CTAs per SM the forward transform's registers are set for
#endif
template <class R> struct FtcFwdMinB { static constexpr int v = sizeof(R) == 4 ? XFMM_FTC_FWD_MINB : 1; };
template <class R>
size_t ftc_fwd_smem(int p) {  // per child and slab: [p][p][2 JS] + [p][n1][2 JS] complex values
  return sizeof(typename C2<R>::type) * FtcCpb<R>::v * (size_t)p * (p + 2 * p) * 2 * FTC_JS;
}
#ifndef XFMM_FTC_JSB
#define XFMM_FTC_JSB 2
#endif
constexpr int FTC_JSB = XFMM_FTC_JSB;  // base frequencies per slab of the backward transform
// per CTA: [p][n1][CPB][2 JSB] + [p][p] rows of CPB 2 JSB + 1 (odd: the point-indexed reads of pass C
// fall on different banks) complex values
template <class R>
size_t ftc_bwd_smem(int p) {
  constexpr int ZS = FtcCpb<R>::v * 2 * FTC_JSB;
  return sizeof(typename C2<R>::type) * ((size_t)p * 2 * p * ZS + (size_t)p * p * (ZS + 1));
}

// spec[(f*ns + s)*8 + child] = forward complex DFT of the children ch0 .. ch0 + CPB - 1 of source node
// src[s].  The first-axis frequencies ka are taken in slabs (base frequencies j0 .. j0 + JS - 1 and their
// partners j + p); per slab the three passes run on the slab's columns only, and the grid input is read
// through the grid -> surface map (values outside the surface are zero) from the L1-resident rows of up.
template <class R, int P>
__global__ void __launch_bounds__(FT_NT, FtcFwdMinB<R>::v)
    k_m2l_fwd_c(const int* __restrict__ src, int ns, const int* __restrict__ child0,
                const typename C2<R>::type* __restrict__ up, int nsurf, const int* __restrict__ conv2surf,
                const double* __restrict__ tw, typename C2<R>::type* __restrict__ spec) {
  using CT = typename C2<R>::type;
  constexpr int N = 2 * P, CPB = FtcCpb<R>::v, KS = 2 * FTC_JS;
  const int s = blockIdx.x, ch0 = blockIdx.y * CPB, tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CT* sA = reinterpret_cast<CT*>(smem_raw);  // [c < P][b < P][ch][slot < KS]
  CT* sB = sA + P * P * CPB * KS;            // [c < P][kb < N][ch][slot]
  __shared__ int sidx[P * P * P];            // grid corner [c][b][a] -> surface index or -1
  __shared__ CT sw[N];                       // w[m] = e^{-2 pi i m / N}: the same factor in every lane
  if (tid < N) sw[tid] = CT{(R)tw[2 * tid], (R)(-tw[2 * tid + 1])};
  for (int e = tid; e < P * P * P; e += FT_NT) {
    const int a = e % P, b = (e / P) % P, c = e / (P * P);
    sidx[e] = conv2surf[(c * N + b) * N + a];
  }
  const int64_t node0 = (int64_t)child0[src[s]] + ch0;
  const int64_t fstride = (int64_t)N * N * ns * 8;
  for (int j0 = 0; j0 < P; j0 += FTC_JS) {
    __syncthreads();  // sidx and sw ready; the previous slab's sA / sB reads done
    // pass 1, along a: task (c, b, ch); slots 2 q and 2 q + 1 hold ka = j0 + q and j0 + q + P
    for (int e = tid; e < P * P * CPB; e += FT_NT) {
      const int ch = e % CPB, cb = e / CPB;
      const CT* u = up + (node0 + ch) * nsurf;
      CT x[P];
#pragma unroll
      for (int a = 0; a < P; a++) {
        const int k = sidx[cb * P + a];
        x[a] = k >= 0 ? __ldg(u + k) : CT{(R)0, (R)0};
      }
#pragma unroll
      for (int q = 0; q < FTC_JS; q++) {
        const int j = j0 + q;
        if (j >= P) break;
        CT ev = x[0], od{(R)0, (R)0};
#pragma unroll
        for (int a = 1; a < P; a++) vfma(a & 1 ? od : ev, x[a], sw[(j * a) % N]);  // j known at run time only
        sA[(cb * CPB + ch) * KS + 2 * q] = CT{ev.x + od.x, ev.y + od.y};
        sA[(cb * CPB + ch) * KS + 2 * q + 1] = CT{ev.x - od.x, ev.y - od.y};
      }
    }
    __syncthreads();
    // pass 2, along b: task (c, ch, slot)
    for (int e = tid; e < P * CPB * KS; e += FT_NT) {
      const int sl = e % KS, ch = (e / KS) % CPB, c = e / (KS * CPB);
      CT x[P];
#pragma unroll
      for (int b = 0; b < P; b++) x[b] = sA[((c * P + b) * CPB + ch) * KS + sl];
      ftc_dft_p<P>(x, sw, [&](int kb, CT v) { sB[((c * N + kb) * CPB + ch) * KS + sl] = v; });
    }
    __syncthreads();
    // pass 3, along c: task (kb, slot, ch), children fastest: the CPB children of one frequency are
    // written by consecutive lanes
    for (int e = tid; e < N * KS * CPB; e += FT_NT) {
      const int ch = e % CPB, sl = (e / CPB) % KS, kb = e / (CPB * KS);
      const int j = j0 + sl / 2;
      if (j >= P) continue;
      const int ka = j + (sl & 1) * P;
      CT x[P];
#pragma unroll
      for (int c = 0; c < P; c++) x[c] = sB[((c * N + kb) * CPB + ch) * KS + sl];
      CT* o = spec + ((int64_t)(kb * N + ka) * ns + s) * 8 + ch0 + ch;
      ftc_dft_p<P>(x, sw, [&](int kc, CT v) { o[kc * fstride] = v; });
    }
  }
}

// dn[child ch0 + ch of target trg[t]][k] += scale[t] * backward complex DFT of spec[.][t][child] at map_dn[k],
// for the CPB children ch0 .. of the CTA.  The first-axis frequencies ka are taken in slabs as in the
// forward transform: per slab, pass A (along kc, rows of CPB children read by consecutive lanes) and
// pass B (along kb) run on the slab's columns, and pass C adds the slab's terms of the last sum (along
// ka) to per-point sums kept in registers (point i of the thread: k = tid + i FT_NT over CPB nsurf).
template <class R> struct FtcMinB;  // resident CTAs per SM of the backward transform (registers)
template <> struct FtcMinB<float> { static constexpr int v = 2; };
template <> struct FtcMinB<double> { static constexpr int v = 1; };
template <class R, int P>
__global__ void __launch_bounds__(FT_NT, FtcMinB<R>::v)
    k_m2l_bwd_c(const int* __restrict__ trg, int nt, const int* __restrict__ child0,
                const typename C2<R>::type* __restrict__ spec, int nsurf, const int* __restrict__ map_dn,
                const double* __restrict__ tw, const R* __restrict__ scale, typename C2<R>::type* __restrict__ dn) {
  using CT = typename C2<R>::type;
  constexpr int N = 2 * P, CPB = FtcCpb<R>::v, JS = FTC_JSB, KS = 2 * JS, ZS = CPB * KS + 1;
  constexpr int NPT = (CPB * (6 * (P - 1) * (P - 1) + 2) + FT_NT - 1) / FT_NT;  // points per thread
  const int t = blockIdx.x, ch0 = blockIdx.y * CPB, tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CT* sZ1 = reinterpret_cast<CT*>(smem_raw);  // [c' < P][kb < N][ch][slot < KS]
  CT* sZ2 = sZ1 + P * N * CPB * KS;           // [c' < P][b' < P] rows of ZS: [ch][slot], one pad
  __shared__ CT sw[N];                        // w[m] = e^{+2 pi i m / N}, read by broadcast (passes A, B)
  if (tid < N) sw[tid] = CT{(R)tw[2 * tid], (R)tw[2 * tid + 1]};
  CT acc[NPT];
#pragma unroll
  for (int i = 0; i < NPT; i++) acc[i] = CT{(R)0, (R)0};
  const int64_t fstride = (int64_t)N * N * nt * 8;
  for (int j0 = 0; j0 < P; j0 += JS) {
    __syncthreads();  // sw ready; the previous slab's sZ2 reads done
    // pass A, along kc, to c = P + c': task (kb, slot, ch), children fastest (one row per frequency)
    for (int e = tid; e < N * KS * CPB; e += FT_NT) {
      const int ch = e % CPB, sl = (e / CPB) % KS, kb = e / (CPB * KS);
      const int j = j0 + sl / 2;
      if (j >= P) continue;
      const int ka = j + (sl & 1) * P;
      const CT* y = spec + ((int64_t)(kb * N + ka) * nt + t) * 8 + ch0 + ch;
      CT up[P], um[P];
#pragma unroll
      for (int k = 0; k < P; k++) {
        const CT a = y[k * fstride], b = y[(k + P) * fstride];
        up[k] = CT{a.x + b.x, a.y + b.y};
        um[k] = CT{a.x - b.x, a.y - b.y};
      }
      ftc_idft_upper<P>(up, um, sw, [&](int cc, CT v) { sZ1[((cc * N + kb) * CPB + ch) * KS + sl] = v; });
    }
    __syncthreads();
    // pass B, along kb, to b = P + b': task (c', ch, slot)
    for (int e = tid; e < P * CPB * KS; e += FT_NT) {
      const int sl = e % KS, ch = (e / KS) % CPB, cc = e / (KS * CPB);
      if (j0 + sl / 2 >= P) continue;
      CT up[P], um[P];
#pragma unroll
      for (int k = 0; k < P; k++) {
        const CT a = sZ1[((cc * N + k) * CPB + ch) * KS + sl], b = sZ1[((cc * N + k + P) * CPB + ch) * KS + sl];
        up[k] = CT{a.x + b.x, a.y + b.y};
        um[k] = CT{a.x - b.x, a.y - b.y};
      }
      ftc_idft_upper<P>(up, um, sw, [&](int bb, CT v) { sZ2[(cc * P + bb) * ZS + ch * KS + sl] = v; });
    }
    __syncthreads();
    // pass C, this slab's terms of the sum along ka at each point: (Z[j] + (-1)^a Z[j + P]) w^{j a}
#pragma unroll
    for (int i = 0; i < NPT; i++) {
      const int e = tid + i * FT_NT;
      if (e < CPB * nsurf) {
        const int ch = e / nsurf, k = e - ch * nsurf, g = map_dn[k];
        const int a = g % N, b = g / N % N - P, c = g / (N * N) - P;
        const CT* z = sZ2 + (c * P + b) * ZS + ch * KS;
        const R sgn = (a & 1) ? (R)-1 : (R)1;
#pragma unroll
        for (int q = 0; q < JS; q++) {
          const int jj = j0 + q;
          if (jj >= P) break;
          const CT v{z[2 * q].x + sgn * z[2 * q + 1].x, z[2 * q].y + sgn * z[2 * q + 1].y};
          vfma(acc[i], v, sw[(jj * a) % N]);
        }
      }
    }
  }
  const int64_t node0 = (int64_t)child0[trg[t]] + ch0;
  const R sc = scale[t];
#pragma unroll
  for (int i = 0; i < NPT; i++) {
    const int e = tid + i * FT_NT;
    if (e < CPB * nsurf) {
      CT* d = dn + node0 * nsurf + e;  // child ch0 + e / nsurf, point e % nsurf
      *d = CT{d->x + sc * acc[i].x, d->y + sc * acc[i].y};
    }
  }
}

// ---------------------------------------------------------------- slabbed M2L transforms of the real kernels
// The real transforms (half spectrum along the first axis, H = p + 1 frequencies ka) computed as the
// complex ones are: CPB children per CTA (one spectrum row of a frequency read or written by consecutive
// lanes), the first-axis frequencies in slabs of FTR_KS, so that a CTA needs ~37 KB of shared memory
// (p = 8) instead of 110 KB and three or more CTAs share an SM; DFT factors are read from shared memory
// (the same factor in every lane: broadcast).  The backward transform keeps each check point's running
// sum along the last axis in registers across the slabs.
#ifndef XFMM_FTR_KS
#define XFMM_FTR_KS 3
#endif
#ifndef XFMM_FTR_MINB_F
#define XFMM_FTR_MINB_F 4
#endif
constexpr int FTR_KS = XFMM_FTR_KS;
#ifndef XFMM_FTR_BWD_MINB_HI
#define XFMM_FTR_BWD_MINB_HI 3  // backward transform, p >= 9 (more per-point sums per thread; measured at p = 10)
#endif
template <class R> struct FtrMinB;
template <> struct FtrMinB<float> { static constexpr int v = XFMM_FTR_MINB_F; };
template <> struct FtrMinB<double> { static constexpr int v = 1; };
template <class R, int P> struct FtrBwdMinB {
  static constexpr int v = (sizeof(R) == 4 && P >= 9) ? XFMM_FTR_BWD_MINB_HI : FtrMinB<R>::v;
};
template <class R>
size_t ftr_fwd_smem(int p) {  // [p][p][CPB][KS] + [p][n1][CPB][KS] complex values
  return sizeof(typename C2<R>::type) * (size_t)p * 3 * p * FtCpb<R>::v * FTR_KS;
}
template <class R>
size_t ftr_bwd_smem(int p) {  // [p][n1][CPB][KS] + [p][p] rows of CPB KS + 1 complex values
  const size_t zs = (size_t)FtCpb<R>::v * FTR_KS;
  return sizeof(typename C2<R>::type) * ((size_t)p * 2 * p * zs + (size_t)p * p * (zs + 1));
}

// spec[(f*ns + s)*8 + ch0 + ch] = forward real-to-half-complex DFT of the children ch0 .. ch0 + CPB - 1 of
// source node src[s], f = (kc n1 + kb) H + ka
template <class R, int P>
__global__ void __launch_bounds__(FT_NT, FtrMinB<R>::v)
    k_m2l_fwd_r(const int* __restrict__ src, int ns, const int* __restrict__ child0, const R* __restrict__ up,
                int nsurf, const int* __restrict__ conv2surf, const double* __restrict__ tw,
                typename C2<R>::type* __restrict__ spec) {
  using CT = typename C2<R>::type;
  constexpr int N = 2 * P, H = P + 1, CPB = FtCpb<R>::v, KS = FTR_KS;
  const int s = blockIdx.x, ch0 = blockIdx.y * CPB, tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CT* sA = reinterpret_cast<CT*>(smem_raw);  // [c < P][b < P][ch][slot < KS]
  CT* sB = sA + P * P * CPB * KS;            // [c < P][kb < N][ch][slot]
  __shared__ int sidx[P * P * P];            // grid corner [c][b][a] -> surface index or -1
  __shared__ CT sw[N];                       // w[m] = e^{-2 pi i m / N}
  if (tid < N) sw[tid] = CT{(R)tw[2 * tid], (R)(-tw[2 * tid + 1])};
  for (int e = tid; e < P * P * P; e += FT_NT) {
    const int a = e % P, b = (e / P) % P, c = e / (P * P);
    sidx[e] = conv2surf[(c * N + b) * N + a];
  }
  const int64_t node0 = (int64_t)child0[src[s]] + ch0;
  const int64_t fstride = (int64_t)N * H * ns * 8;  // kc -> kc + 1
  for (int k0 = 0; k0 < H; k0 += KS) {
    __syncthreads();  // sidx and sw ready; the previous slab's reads done
    // pass 1, along a (real input): task (c, b, ch), slot sl = ka - k0
    for (int e = tid; e < P * P * CPB; e += FT_NT) {
      const int ch = e % CPB, cb = e / CPB;
      const R* u = up + (node0 + ch) * nsurf;
      R x[P];
#pragma unroll
      for (int a = 0; a < P; a++) {
        const int k = sidx[cb * P + a];
        x[a] = k >= 0 ? __ldg(u + k) : (R)0;
      }
#pragma unroll
      for (int sl = 0; sl < KS; sl++) {
        const int ka = k0 + sl;
        if (ka >= H) break;
        R re = x[0], im = 0;
#pragma unroll
        for (int a = 1; a < P; a++) {
          const CT ww = sw[(ka * a) % N];
          re += x[a] * ww.x;
          im += x[a] * ww.y;
        }
        sA[(cb * CPB + ch) * KS + sl] = CT{re, im};
      }
    }
    __syncthreads();
    // pass 2, along b: task (c, ch, slot)
    for (int e = tid; e < P * CPB * KS; e += FT_NT) {
      const int sl = e % KS, ch = (e / KS) % CPB, c = e / (KS * CPB);
      if (k0 + sl >= H) continue;
      CT x[P];
#pragma unroll
      for (int b = 0; b < P; b++) x[b] = sA[((c * P + b) * CPB + ch) * KS + sl];
      ftc_dft_p<P>(x, sw, [&](int kb, CT v) { sB[((c * N + kb) * CPB + ch) * KS + sl] = v; });
    }
    __syncthreads();
    // pass 3, along c: task (kb, slot, ch), children fastest
    for (int e = tid; e < N * KS * CPB; e += FT_NT) {
      const int ch = e % CPB, sl = (e / CPB) % KS, kb = e / (CPB * KS);
      const int ka = k0 + sl;
      if (ka >= H) continue;
      CT x[P];
#pragma unroll
      for (int c = 0; c < P; c++) x[c] = sB[((c * N + kb) * CPB + ch) * KS + sl];
      CT* o = spec + ((int64_t)(kb * H + ka) * ns + s) * 8 + ch0 + ch;
      ftc_dft_p<P>(x, sw, [&](int kc, CT v) { o[kc * fstride] = v; });
    }
  }
}

// dn[child ch0 + ch of target trg[t]][k] += scale[t] * backward half-complex-to-real DFT of spec[.][t][child]
// at map_dn[k] (weight 2 on the half spectrum's interior frequencies 0 < ka < N / 2)
template <class R, int P>
__global__ void __launch_bounds__(FT_NT, (FtrBwdMinB<R, P>::v))
    k_m2l_bwd_r(const int* __restrict__ trg, int nt, const int* __restrict__ child0,
                const typename C2<R>::type* __restrict__ spec, int nsurf, const int* __restrict__ map_dn,
                const double* __restrict__ tw, const R* __restrict__ scale, R* __restrict__ dn) {
  using CT = typename C2<R>::type;
  constexpr int N = 2 * P, H = P + 1, CPB = FtCpb<R>::v, KS = FTR_KS, ZS = CPB * KS + 1;
  constexpr int NPT = (CPB * (6 * (P - 1) * (P - 1) + 2) + FT_NT - 1) / FT_NT;  // points per thread
  const int t = blockIdx.x, ch0 = blockIdx.y * CPB, tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CT* sZ1 = reinterpret_cast<CT*>(smem_raw);  // [c' < P][kb < N][ch][slot < KS]
  CT* sZ2 = sZ1 + P * N * CPB * KS;           // [c' < P][b' < P] rows of ZS: [ch][slot], one pad
  __shared__ CT sw[N];                        // w[m] = e^{+2 pi i m / N}
  if (tid < N) sw[tid] = CT{(R)tw[2 * tid], (R)tw[2 * tid + 1]};
  R acc[NPT];
#pragma unroll
  for (int i = 0; i < NPT; i++) acc[i] = 0;
  const int64_t fstride = (int64_t)N * H * nt * 8;
  for (int k0 = 0; k0 < H; k0 += KS) {
    __syncthreads();  // sw ready; the previous slab's sZ2 reads done
    // pass A, along kc, to c = P + c': task (kb, slot, ch), children fastest
    for (int e = tid; e < N * KS * CPB; e += FT_NT) {
      const int ch = e % CPB, sl = (e / CPB) % KS, kb = e / (CPB * KS);
      const int ka = k0 + sl;
      if (ka >= H) continue;
      const CT* y = spec + ((int64_t)(kb * H + ka) * nt + t) * 8 + ch0 + ch;
      CT up[P], um[P];
#pragma unroll
      for (int k = 0; k < P; k++) {
        const CT a = y[k * fstride], b = y[(k + P) * fstride];
        up[k] = CT{a.x + b.x, a.y + b.y};
        um[k] = CT{a.x - b.x, a.y - b.y};
      }
      ftc_idft_upper<P>(up, um, sw, [&](int cc, CT v) { sZ1[((cc * N + kb) * CPB + ch) * KS + sl] = v; });
    }
    __syncthreads();
    // pass B, along kb, to b = P + b': task (c', ch, slot)
    for (int e = tid; e < P * CPB * KS; e += FT_NT) {
      const int sl = e % KS, ch = (e / KS) % CPB, cc = e / (KS * CPB);
      if (k0 + sl >= H) continue;
      CT up[P], um[P];
#pragma unroll
      for (int k = 0; k < P; k++) {
        const CT a = sZ1[((cc * N + k) * CPB + ch) * KS + sl], b = sZ1[((cc * N + k + P) * CPB + ch) * KS + sl];
        up[k] = CT{a.x + b.x, a.y + b.y};
        um[k] = CT{a.x - b.x, a.y - b.y};
      }
      ftc_idft_upper<P>(up, um, sw, [&](int bb, CT v) { sZ2[(cc * P + bb) * ZS + ch * KS + sl] = v; });
    }
    __syncthreads();
    // pass C, this slab's terms along ka at each point: wgt Re(Z[ka] w^{ka a})
#pragma unroll
    for (int i = 0; i < NPT; i++) {
      const int e = tid + i * FT_NT;
      if (e < CPB * nsurf) {
        const int ch = e / nsurf, k = e - ch * nsurf, g = map_dn[k];
        const int a = g % N, b = g / N % N - P, c = g / (N * N) - P;
        const CT* z = sZ2 + (c * P + b) * ZS + ch * KS;
#pragma unroll
        for (int sl = 0; sl < KS; sl++) {
          const int ka = k0 + sl;
          if (ka >= H) break;
          const CT ww = sw[(ka * a) % N];
          const R wgt = (ka == 0 || 2 * ka == N) ? (R)1 : (R)2;
          acc[i] += wgt * (z[sl].x * ww.x - z[sl].y * ww.y);
        }
      }
    }
  }
  const int64_t node0 = (int64_t)child0[trg[t]] + ch0;
  const R sc = scale[t];
#pragma unroll
  for (int i = 0; i < NPT; i++) {
    const int e = tid + i * FT_NT;
    if (e < CPB * nsurf) dn[node0 * nsurf + e] += sc * acc[i];  // child ch0 + e / nsurf, point e % nsurf
  }
}

// dn[child c of target t][k] += scale[t] * grid[(t*8 + c)*nconv + map_dn[k]]   (fmm_scale_invariant.h:639-643)
template <class W, class RB>
__global__ void k_m2l_gather_dn(const int* __restrict__ trg, int ntrg, const int* __restrict__ child0,
                                const W* __restrict__ grid, int nconv, const int* __restrict__ map_dn, int nsurf,
                                const RB* __restrict__ scale, W* __restrict__ dn) {
  const int64_t total = (int64_t)ntrg * 8 * nsurf;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % nsurf);
    const int64_t tc = e / nsurf;
    const int t = (int)(tc >> 3), c = (int)(tc & 7);
    W* d = dn + ((int64_t)child0[trg[t]] + c) * nsurf + k;
    *d = vadd(*d, vscale(grid[tc * nconv + map_dn[k]], scale[t]));
  }
}

// ================================================================ misc
// Sources of the Laplace paired-FP32 near field: hi/lo FP32 parts of (x - o), FP32 charge.
// *bad becomes nonzero if any of v[0, n) is NaN or infinite
__global__ void k_count_nonfinite(const double* __restrict__ v, int64_t n, int* __restrict__ bad) {
  int found = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    found |= !isfinite(v[i]);
  if (__syncthreads_or(found) && threadIdx.x == 0) atomicOr(bad, 1);
}
__global__ void k_set_charges(const double* __restrict__ q, const int* __restrict__ perm, int64_t n, int cplx,
                              double4* __restrict__ src4, double* __restrict__ qim) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t j = perm[i];
  if (cplx) {
    src4[i].w = q[2 * j];
    qim[i] = q[2 * j + 1];
  } else {
    src4[i].w = q[j];
  }
}
__global__ void k_scatter_out(const double* __restrict__ in, const int* __restrict__ perm, int64_t n, int width,
                              double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t j = perm[i];
  for (int c = 0; c < width; c++) out[j * width + c] = in[i * width + c];
}

}  // namespace

// ================================================================ workspace
// Rows of one batch of translation GEMMs (translate.cu): per row its A and C offsets in real elements of
// the buffers (complex values count twice) and its scale.
struct GemmRows {
  int M = 0;
  DBuf<int64_t> a, c;
  DBuf<double> al64;
};

struct Workspace {
  int precision = -1, kernel = -1, p = 0;
  size_t vsz = 0;
  DBuf<char> up, dn, chk;  // working precision
  DBuf<double> tc_scratch;  // FP64 sums of the split-K tensor-core translations (zero between uses)
  DBuf<int4> close_pairs;   // Laplace mixed near field: the close pairs (k_close_scan), found once per tree
  int64_t n_close = -1;     // -1: not searched yet
  DBuf<char> ybuf, eq;     // FP64: pinv intermediate (rows of the kept singular directions), downward
                           // equivalent densities of the leaves
  DBuf<double> out;
  DBuf<int> status;   // set by a kernel whose bounded wait ran out (0: none)
  // leaves grouped by level (P2M / L2P operators are per level except for Laplace)
  std::vector<int> leaf_level_off;
  GemmRows p2m1, p2m2, l2p1, l2p2;  // two factors each (rows grouped by leaf level)
  std::vector<GemmRows> m2m, l2l;  // per level of the parent
  // M2L
  DBuf<char> grid, specA, specB;
  std::vector<cufftHandle> fwd, bwd;
  // Hadamard tiling: per group, tiles of TT targets; CSR over (tile, ipos) of (local target, source)
  std::vector<int> had_tile0;  // first tile of each group (ngroups + 1)
  // FP32: sparse targets in the round form (per tile the range of rounds and HADR_TT output rows; per
  // round its relative position and HADR_RW pairs), dense targets in the dense form (per group a
  // [26][ld] source table and ld output rows)
  DBuf<int> hadr_tile, hadr_pos, hadr_row;
  DBuf<int2> hadr_ent;
  DBuf<int> hadd_tab, hadd_row;
  std::vector<int64_t> hadd_tab0, hadd_row0;
  std::vector<int> hadd_ld;
  bool hadt_attr = false, hadrt_attr = false, hadc_attr = false, had64_attr = false;
  // dense Hadamard targets on tcgen05 (k_hadamard_dc) instead of mma.sync (k_hadamard_dt): chosen when the
  // workspace is created, by XFMM_HADAMARD_TCGEN05=1 in the environment
  bool had_tc5 = false;
  DBuf<unsigned char> hadc_btab;      // its B blocks per frequency (k_hadc_btab), built for one operator table
  const void* hadc_btab_T = nullptr;
  int hadc_btab_nf = 0;
  // M2L transforms: own pruned DFT kernels (real p <= 10, complex p <= 12, shared memory permitting) or
  // cuFFT on the grid
  bool fused = false;
  size_t ft_fwd_smem = 0, ft_bwd_smem = 0;
  int64_t launches = 0;  // kernels of this library launched by the last evaluate
  cudaEvent_t ev[9] = {};
  std::vector<cudaEvent_t> m2l_ev;  // 4 per M2L group
  bool ev_ok = false;
  ~Workspace() {
    for (auto h : fwd) cufftDestroy(h);
    for (auto h : bwd) cufftDestroy(h);
    if (ev_ok) {
      for (auto& e : ev) cudaEventDestroy(e);
      for (auto& e : m2l_ev) cudaEventDestroy(e);
    }
  }
};

void release_workspace(Tree& t) {
  for (auto& w : t.ws) {
    delete w;
    w = nullptr;
  }
}

namespace {

template <class RB>
void upload_rows(GemmRows& g, const std::vector<int64_t>& a, const std::vector<int64_t>& c,
                 const std::vector<double>& al, cudaStream_t s) {
  g.M = (int)a.size();
  g.a.upload(a, s);
  g.c.upload(c, s);
  g.al64.upload(al, s);
}

Workspace& workspace(Fmm& f, Tree& t, cudaStream_t s) {
  Workspace*& w = t.ws[f.precision];
  if (w && w->kernel == f.kernel && w->p == f.p) return *w;
  delete w;
  w = new Workspace();
  Workspace& W = *w;
  W.precision = f.precision;
  W.kernel = f.kernel;
  W.p = f.p;
  const bool cplx = f.is_complex();
  W.vsz = (f.mixed() ? 4 : 8) * (cplx ? 2 : 1);
  const int n = f.nsurf;
  W.up.alloc((size_t)t.nnodes * n * W.vsz);
  W.dn.alloc((size_t)t.nnodes * n * W.vsz);
  W.chk.alloc((size_t)std::max(t.nleafs, 1) * n * W.vsz);
  W.ybuf.alloc((size_t)std::max(t.nleafs, 1) * n * 8 * (cplx ? 2 : 1));
  W.eq.alloc((size_t)std::max(t.nleafs, 1) * n * 8 * (cplx ? 2 : 1));
  W.out.alloc((size_t)t.ntrg * 4 * (cplx ? 2 : 1));
  W.status.alloc(1);
  {
    const char* e = std::getenv("XFMM_HADAMARD_TCGEN05");
    W.had_tc5 = e && e[0] == '1';
  }
  XCUDA(cudaMemsetAsync(W.status.p, 0, sizeof(int), s));
  // leaf rows grouped by level: P2M (chk[pos] -> up[node]) and L2P (dn[node] -> eq[pos])
  const bool lap = f.kernel == XFMM_LAPLACE;
  std::vector<int> order(t.nleafs);
  for (int i = 0; i < t.nleafs; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return t.h_level[t.h_leafs[x]] < t.h_level[t.h_leafs[y]]; });
  W.leaf_level_off.assign(t.depth + 2, 0);
  {
    std::vector<int64_t> idn, nodes;
    std::vector<double> al, one;
    int cur = 0;
    for (int l = 0; l <= t.depth; l++) {
      W.leaf_level_off[l] = cur;
      while (cur < t.nleafs && t.h_level[t.h_leafs[order[cur]]] == l) cur++;
    }
    W.leaf_level_off[t.depth + 1] = cur;
    const int64_t rn = (int64_t)n * (cplx ? 2 : 1);  // row length in real elements
    for (int i : order) {
      const int node = t.h_leafs[i];
      idn.push_back((int64_t)i * rn);
      nodes.push_back((int64_t)node * rn);
      al.push_back(lap ? std::pow(0.5, t.h_level[node]) : 1.0);
      one.push_back(1.0);
    }
    // P2M: chk[i] -U^H-> eq[i] (scratch) -V S+, 0.5^l-> up[node];  L2P: dn[node] -> chk[i] (scratch) -> eq[i]
    upload_rows<double>(W.p2m1, idn, idn, one, s);
    upload_rows<double>(W.p2m2, idn, nodes, al, s);
    upload_rows<double>(W.l2p1, nodes, idn, one, s);
    upload_rows<double>(W.l2p2, idn, idn, al, s);
  }
  W.m2m.clear();
  W.l2l.clear();
  W.m2m.resize(t.depth + 1);
  W.l2l.resize(t.depth + 1);
  for (int l = 0; l <= t.depth; l++) {
    std::vector<int64_t> ma, mc, la, lc;
    std::vector<double> one;
    for (int k : t.h_nonleafs)
      if (t.h_level[k] == l) {
        const int64_t rn = (int64_t)n * (cplx ? 2 : 1);
        ma.push_back((int64_t)t.h_child0[k] * rn);
        mc.push_back((int64_t)k * rn);
        la.push_back((int64_t)k * rn);
        lc.push_back((int64_t)t.h_child0[k] * rn);
        one.push_back(1.0);
      }
    upload_rows<double>(W.m2m[l], ma, mc, one, s);
    upload_rows<double>(W.l2l[l], la, lc, one, s);
  }
  if (f.mixed()) {
    // FP64 scratch of the split-K tensor-core M2M / L2L of the small levels, zeroed once
    const int cw = cplx ? 2 : 1;
    int64_t need = 0;
    for (int l = 0; l <= t.depth; l++) {
      need = std::max(need, tgemm_tc_scratch(W.m2m[l].M, cw * n, cw * 8 * n, 1));
      need = std::max(need, tgemm_tc_scratch(W.l2l[l].M, cw * 8 * n, cw * n, 1));
    }
    if (need > 0) {
      W.tc_scratch.alloc((size_t)need);
      XCUDA(cudaMemsetAsync(W.tc_scratch.p, 0, W.tc_scratch.bytes(), s));
    }
  }
  // M2L buffers and FFT plans
  const int ng = (int)t.m2l_src_off.size() - 1;
  int maxn = 1;
  for (int g = 0; g < ng; g++) {
    maxn = std::max(maxn, t.m2l_src_off[g + 1] - t.m2l_src_off[g]);
    maxn = std::max(maxn, t.m2l_trg_off[g + 1] - t.m2l_trg_off[g]);
  }
  const size_t rsz = f.mixed() ? 4 : 8;  // real scalar size
  {
    constexpr size_t kMaxSmem = 227 * 1024;
    const size_t fw = f.mixed() ? ftr_fwd_smem<float>(f.p) : ftr_fwd_smem<double>(f.p);
    const size_t bw = f.mixed() ? ft_bwd_smem<float>(f.p) : ft_bwd_smem<double>(f.p);
    const size_t cw = std::max(f.mixed() ? ftc_fwd_smem<float>(f.p) : ftc_fwd_smem<double>(f.p),
                               f.mixed() ? ftc_bwd_smem<float>(f.p) : ftc_bwd_smem<double>(f.p));
    W.fused = cplx ? (f.p <= FTC_PMAX && cw <= kMaxSmem) : (f.p <= FT_PMAX && fw <= kMaxSmem && bw <= kMaxSmem);
  }
  W.specA.alloc((size_t)maxn * 8 * f.nfreq * 2 * rsz);
  W.specB.alloc((size_t)maxn * 8 * f.nfreq * 2 * rsz);
  int dims[3] = {f.n1, f.n1, f.n1};
  cufftType tf = cplx ? (f.mixed() ? CUFFT_C2C : CUFFT_Z2Z) : (f.mixed() ? CUFFT_R2C : CUFFT_D2Z);
  cufftType tb = cplx ? (f.mixed() ? CUFFT_C2C : CUFFT_Z2Z) : (f.mixed() ? CUFFT_C2R : CUFFT_Z2D);
  if (!W.fused) W.grid.alloc((size_t)maxn * 8 * f.nconv * rsz * (cplx ? 2 : 1));
  for (int g = 0; g < ng && !W.fused; g++) {
    const int ns = t.m2l_src_off[g + 1] - t.m2l_src_off[g], nt = t.m2l_trg_off[g + 1] - t.m2l_trg_off[g];
    cufftHandle hf = 0, hb = 0;
    if (ns > 0) {
      XCUFFT2(cufftPlanMany(&hf, 3, dims, nullptr, 1, f.nconv, nullptr, 1, f.nfreq, tf, 8 * ns));
      XCUFFT2(cufftSetStream(hf, s));
    }
    if (nt > 0) {
      XCUFFT2(cufftPlanMany(&hb, 3, dims, nullptr, 1, f.nfreq, nullptr, 1, f.nconv, tb, 8 * nt));
      XCUFFT2(cufftSetStream(hb, s));
    }
    W.fwd.push_back(hf);
    W.bwd.push_back(hb);
  }
  if (f.mixed()) {
    // Targets with at least HAD_DENSE_MIN occupied positions go to the dense form, in tiles of HADT_TT
    // (table [26][ld], padded with -1).  The others go to the round form: tiles of HADR_TT targets;
    // per tile and relative position the pairs (source index, output row) in rounds
    // of HADR_RW, padded with source -1.  Both write disjoint rows of the group's output.
    std::vector<int> tile_r, pos, srow, dtab, drow;
    std::vector<int2> ent;
    W.had_tile0.assign(ng + 1, 0);
    W.hadd_tab0.assign(ng, 0);
    W.hadd_row0.assign(ng, 0);
    W.hadd_ld.assign(ng, 0);
    int ntiles = 0;
    for (int g = 0; g < ng; g++) {
      W.had_tile0[g] = ntiles;
      const int tb = t.m2l_trg_off[g], te = t.m2l_trg_off[g + 1];
      std::vector<int> dense, sparse;
      for (int tt = tb; tt < te; tt++) {
        int cnt = 0;
        for (int ipos = 0; ipos < 26; ipos++) cnt += t.h_m2l_tab[26 * (size_t)tt + ipos] >= 0;
        (cnt >= HAD_DENSE_MIN ? dense : sparse).push_back(tt);
      }
      // a group with few dense targets would leave most rows of the dense form's tiles (HADT_TT targets,
      // one tile per frequency) empty; the round form packs its pairs into full rounds instead
      if ((int)dense.size() < HAD_DENSE_GROUP_MIN) {
        sparse.insert(sparse.end(), dense.begin(), dense.end());
        std::sort(sparse.begin(), sparse.end());
        dense.clear();
      }
      // dense targets level by level (node order within a level is Morton order): the targets of one
      // tile are then spatially compact and share most of their sources in L2
      std::stable_sort(dense.begin(), dense.end(),
                       [&](int a, int b) { return t.h_level[t.h_m2l_trg[a]] < t.h_level[t.h_m2l_trg[b]]; });
      const int ld = (int)((dense.size() + HADT_TT - 1) / HADT_TT) * HADT_TT;
      W.hadd_ld[g] = ld;
      W.hadd_tab0[g] = (int64_t)dtab.size();
      W.hadd_row0[g] = (int64_t)drow.size();
      dtab.resize(dtab.size() + (size_t)26 * ld, -1);
      drow.resize(drow.size() + ld, -1);
      for (size_t k = 0; k < dense.size(); k++) {
        const int tt = dense[k];
        drow[W.hadd_row0[g] + k] = tt - tb;
        for (int ipos = 0; ipos < 26; ipos++)
          dtab[W.hadd_tab0[g] + (size_t)ipos * ld + k] = t.h_m2l_tab[26 * (size_t)tt + ipos];
      }
      for (size_t k0 = 0; k0 < sparse.size(); k0 += HADR_TT, ntiles++) {
        tile_r.push_back((int)pos.size());
        const size_t k1 = std::min(sparse.size(), k0 + HADR_TT);
        for (size_t k = k0; k < k0 + HADR_TT; k++) srow.push_back(k < k1 ? sparse[k] - tb : -1);
        for (int ipos = 0; ipos < 26; ipos++) {
          int n = 0;
          for (size_t k = k0; k < k1; k++) {
            const int sidx = t.h_m2l_tab[26 * (size_t)sparse[k] + ipos];
            if (sidx < 0) continue;
            if (n == 0) {
              pos.push_back(ipos);
              ent.resize(ent.size() + HADR_RW, make_int2(-1, 0));
            }
            ent[ent.size() - HADR_RW + n] = make_int2(sidx, sparse[k] - tb);  // source, output row
            if (++n == HADR_RW) n = 0;
          }
        }
      }
    }
    W.had_tile0[ng] = ntiles;
    tile_r.push_back((int)pos.size());
    if (ent.empty()) {
      pos.push_back(0);
      ent.resize(HADR_RW, make_int2(-1, 0));
    }
    if (srow.empty()) srow.push_back(-1);
    if (dtab.empty()) dtab.push_back(-1);
    if (drow.empty()) drow.push_back(-1);
    W.hadr_tile.upload(tile_r, s);
    W.hadr_pos.upload(pos, s);
    W.hadr_ent.upload(ent, s);
    W.hadr_row.upload(srow, s);
    W.hadd_tab.upload(dtab, s);
    W.hadd_row.upload(drow, s);
  } else {
    // FP64: every target in the dense form on the FP64 tensor cores (k_hadamard_d64): per group a [26][ld]
    // source table and ld output rows, targets level by level (Morton order inside a level), padded to
    // whole CTA tiles
    std::vector<int> dtab, drow;
    W.had_tile0.assign(ng + 1, 0);
    W.hadd_tab0.assign(ng, 0);
    W.hadd_row0.assign(ng, 0);
    W.hadd_ld.assign(ng, 0);
    for (int g = 0; g < ng; g++) {
      const int tb = t.m2l_trg_off[g], te = t.m2l_trg_off[g + 1];
      std::vector<int> all;
      for (int tt = tb; tt < te; tt++) all.push_back(tt);
      std::stable_sort(all.begin(), all.end(),
                       [&](int a, int b) { return t.h_level[t.h_m2l_trg[a]] < t.h_level[t.h_m2l_trg[b]]; });
      const int ld = (int)((all.size() + HAD64_TT - 1) / HAD64_TT) * HAD64_TT;
      W.hadd_ld[g] = ld;
      W.hadd_tab0[g] = (int64_t)dtab.size();
      W.hadd_row0[g] = (int64_t)drow.size();
      dtab.resize(dtab.size() + (size_t)26 * ld, -1);
      drow.resize(drow.size() + ld, -1);
      for (size_t k = 0; k < all.size(); k++) {
        const int tt = all[k];
        drow[W.hadd_row0[g] + k] = tt - tb;
        for (int ipos = 0; ipos < 26; ipos++)
          dtab[W.hadd_tab0[g] + (size_t)ipos * ld + k] = t.h_m2l_tab[26 * (size_t)tt + ipos];
      }
    }
    if (dtab.empty()) dtab.push_back(-1);
    if (drow.empty()) drow.push_back(-1);
    W.hadd_tab.upload(dtab, s);
    W.hadd_row.upload(drow, s);
  }
  for (auto& e : W.ev) XCUDA(cudaEventCreate(&e));
  W.m2l_ev.resize(4 * (size_t)ng);
  for (auto& e : W.m2l_ev) XCUDA(cudaEventCreate(&e));
  W.ev_ok = true;
  XCUDA(cudaStreamSynchronize(s));
  return W;
}

inline const LevelOps& level_ops(const Fmm& f, int level) { return f.ops[f.kernel == XFMM_LAPLACE ? 0 : level]; }

template <class RB> const RB* m2l_scale_of(const Tree& t);
template <> const float* m2l_scale_of<float>(const Tree& t) { return t.m2l_scale.p; }
template <> const double* m2l_scale_of<double>(const Tree& t) { return t.m2l_scale64.p; }

// The near field's close pairs of this tree (count, then fill), once per workspace; no allocation while
// evaluating afterwards.
void find_close_pairs(Workspace& ws, const NearArgs& na, int n_eval, cudaStream_t s) {
  DBuf<unsigned long long> cnt(2);
  XCUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes(), s));
  if (n_eval > 0) {
    k_close_scan<false><<<nblk(n_eval, 4), 128, 0, s>>>(na, cnt.p, nullptr, 0);
    XLAUNCH();
  }
  unsigned long long n = 0;
  XCUDA(cudaMemcpyAsync(&n, cnt.p, sizeof(n), cudaMemcpyDeviceToHost, s));
  XCUDA(cudaStreamSynchronize(s));
  ws.close_pairs.alloc(std::max<unsigned long long>(n, 1));
  if (n > 0) {
    k_close_scan<true><<<nblk(n_eval, 4), 128, 0, s>>>(na, cnt.p + 1, ws.close_pairs.p, (int64_t)n);
    XLAUNCH();
    XCUDA(cudaStreamSynchronize(s));  // cnt is released on return
  }
  ws.n_close = (int64_t)n;
}

constexpr int DOWN_PRE = 1, DOWN_NEAR = 2, DOWN_FAR = 4, DOWN_ALL = 7;
constexpr int M2L_FWD = 1, M2L_HAD_SPARSE = 2, M2L_HAD_DENSE = 4, M2L_BWD = 8, M2L_ALL = 15;
// parts of the downward pass before the near field: the M2L parts above (P2L with the forward transforms),
// then L2L, then L2P's check-to-equivalent step
constexpr int PRE_L2L = 16, PRE_DC2E = 32, PRE_ALL = M2L_ALL | PRE_L2L | PRE_DC2E;
// parts of the upward pass: P2M's check potentials, its two pseudo-inverse GEMMs, M2M
constexpr int UP_CHK = 1, UP_M2M = 2, UP_PINV = 4, UP_P2M = UP_CHK | UP_PINV, UP_ALL = 7;

// ------------------------------------------------------------------ engine, per kernel and precision
template <int KER, class R>
struct Engine {
  using W = typename Green<KER, R>::Q;          // working value: R or complex
  using V64 = typename Green<KER, double>::Q;   // FP64 value (pinv GEMMs, downward equivalent densities)
  using CT = typename C2<R>::type;              // spectrum value
  static constexpr int CW = KER == K_HELMHOLTZ ? 2 : 1;  // reals per value

  static void upward(Fmm& f, Tree& t, Workspace& ws, cudaStream_t s, int parts = UP_ALL) {
    const int n = f.nsurf;
    if (parts & UP_P2M) {
      if (parts & UP_CHK) {
        ws.launches = 0;
        XCUDA(cudaEventRecord(ws.ev[0], s));
      }
      // P2M: check potentials of every leaf, then the pinv (UC2E) GEMM per leaf level
      if (t.nleafs && (parts & UP_CHK)) {
        SurfPotArgs a{t.leafs.p,  t.nleafs, t.nsrcs.p,     nullptr,  t.level.p, t.sbeg.p,   nullptr, t.center.p,
                      t.src4.p,   t.src_qim.p, f.surf_base.p, n,      2.95,      ws.chk.p, 0,         f.k_re, f.k_im,
                      INV4PI * op_scale(f, t)};
        if constexpr (KER == K_LAPLACE && sizeof(R) == 4)
          k_surf_pot_lap_f2<<<nblk(t.nleafs, 4), 128, 0, s>>>(a);
        else
          k_surf_pot<KER, R><<<nblk(t.nleafs, 4), 128, 0, s>>>(a);
        XLAUNCH();
        ws.launches++;
      }
      if (t.nleafs && (parts & UP_PINV)) {
        // e = 0.5^l (V S+) (U^H c) per leaf level, two FP64 GEMMs on the tensor cores: y over the kept
        // singular directions only, then e scattered to the leaves' up rows with the level's scale.
        // (An FP32 first factor, as in L2P below, measured 1.4e-7 more potential error at p = 8 and 3e-7
        // at p = 10: the upward densities feed every later translation.)
        for (int l = 0; l <= t.depth; l++) {
          if (KER == K_LAPLACE && l > 0) break;
          const int r0 = ws.leaf_level_off[l], r1 = ws.leaf_level_off[l + 1];
          const int m = KER == K_LAPLACE ? ws.p2m1.M : r1 - r0;
          const int off = KER == K_LAPLACE ? 0 : r0;
          if (m <= 0) continue;
          const LevelOps& op = level_ops(f, l);
          const int rk = op.rank;
          TGemm g1{m, CW * rk, CW * n, ws.p2m1.a.p + off, ws.p2m1.c.p + off, nullptr, (int64_t)CW * n, 0, (int64_t)CW * n};
          tgemm_f64<R, double>(g1, (const R*)ws.chk.p, op.tg_p2m1.p, (double*)ws.ybuf.p, s);
          TGemm g2{m, CW * n, CW * rk, ws.p2m2.a.p + off, ws.p2m2.c.p + off, ws.p2m2.al64.p + off, (int64_t)CW * n, 0,
                   (int64_t)CW * n};
          tgemm_f64<double, R>(g2, (const double*)ws.ybuf.p, op.tg_p2m2.p, (R*)ws.up.p, s);
          ws.launches += 2;
        }
      }
      if (parts & UP_PINV) XCUDA(cudaEventRecord(ws.ev[1], s));
    }
    if (!(parts & UP_M2M)) return;
    // M2M: deepest parents first (post-order); per level one GEMM of the parents' 8 children rows
    // (contiguous per parent) with the [8n][n] operator, written to the parents' rows
    for (int l = t.depth - 1; l >= 0; l--) {
      const GemmRows& g = ws.m2m[l];
      if (g.M <= 0) continue;
      const LevelOps& op = level_ops(f, l);
      // the parents' rows start at zero (clear_values): the products are added to them, as the reference
      // adds each child's contribution (fmm_scale_invariant.h:243-251)
      TGemm gm{g.M, CW * n, CW * 8 * n, g.a.p, g.c.p, nullptr, (int64_t)CW * n, 1, (int64_t)CW * n};
      gm.status = ws.status.p;
      gm.scratch = ws.tc_scratch.p;
      gm.scratch_len = (int64_t)ws.tc_scratch.n;
      if constexpr (sizeof(R) == 4)
        tgemm_tc<float>(gm, (const float*)ws.up.p, op.tg_m2m_h.p, op.tg_m2m_l.p, op.ld_m2m, (float*)ws.up.p, s);
      else
        tgemm_f64<double, double>(gm, (const double*)ws.up.p, op.tg_m2m.p, (double*)ws.up.p, s);
      ws.launches++;
    }
    XCUDA(cudaEventRecord(ws.ev[2], s));
  }

  // phase: which parts of every group's M2L to run (M2L_FWD, M2L_HAD_SPARSE, M2L_HAD_DENSE, M2L_BWD)
  static void m2l(Fmm& f, Tree& t, Workspace& ws, cudaStream_t s, int phase = M2L_ALL) {
    const int n = f.nsurf, nconv = f.nconv, nfreq = f.nfreq;
    const int ng = (int)t.m2l_src_off.size() - 1;
    for (int g = 0; g < ng; g++) {
      cudaEvent_t* ev = ws.m2l_ev.data() + 4 * g;
      const int ns = t.m2l_src_off[g + 1] - t.m2l_src_off[g], nt = t.m2l_trg_off[g + 1] - t.m2l_trg_off[g];
      if (ns == 0 || nt == 0) continue;
      const int* src = t.m2l_src.p + t.m2l_src_off[g];
      const int* trg = t.m2l_trg.p + t.m2l_trg_off[g];
      const int tab_level = KER == K_LAPLACE ? 0 : g + 1;
      const CT* T = (const CT*)f.ops[tab_level].m2l_T.p;
      if (phase & M2L_FWD) {
        XCUDA(cudaEventRecord(ev[0], s));
        // upward equivalent DFT (fmm_scale_invariant.h:560-604) -> specB [f][s][c]
        if constexpr (KER != K_HELMHOLTZ) {
          if (ws.fused) {
            ft_dispatch(f.p, [&](auto pc) {
              constexpr int PP = decltype(pc)::value;
              const size_t smem = ftr_fwd_smem<R>(PP);
              if (ws.ft_fwd_smem < smem) {
                XCUDA(cudaFuncSetAttribute(k_m2l_fwd_r<R, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                ws.ft_fwd_smem = smem;
              }
              k_m2l_fwd_r<R, PP><<<dim3(ns, 8 / FtCpb<R>::v), FT_NT, smem, s>>>(
                  src, ns, t.child0.p, (const R*)ws.up.p, n, f.conv_to_surf_up.p, f.dft_tw.p, (CT*)ws.specB.p);
            });
            XLAUNCH();
            ws.launches++;
          }
        } else if (ws.fused) {
          ftc_dispatch(f.p, [&](auto pc) {
            constexpr int PP = decltype(pc)::value;
            const size_t smem = ftc_fwd_smem<R>(PP);
            if (ws.ft_fwd_smem < smem) {
              XCUDA(cudaFuncSetAttribute(k_m2l_fwd_c<R, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
              ws.ft_fwd_smem = smem;
            }
            k_m2l_fwd_c<R, PP><<<dim3(ns, 8 / FtcCpb<R>::v), FT_NT, smem, s>>>(
                src, ns, t.child0.p, (const CT*)ws.up.p, n, f.conv_to_surf_up.p, f.dft_tw.p, (CT*)ws.specB.p);
          });
          XLAUNCH();
          ws.launches++;
        }
        if (!ws.fused) {
          k_m2l_grid_up<W><<<std::min<int64_t>(nblk((int64_t)ns * 8 * nconv), 148 * 32), 256, 0, s>>>(
              src, ns, t.child0.p, (const W*)ws.up.p, n, f.conv_to_surf_up.p, nconv, (W*)ws.grid.p);
          XLAUNCH();
          ws.launches++;
          XCUFFT2(cufftSetStream(ws.fwd[g], s));
          exec_fwd(ws.fwd[g], ws.grid.p, ws.specA.p);
          ws.launches++;
          transpose<CT>((const CT*)ws.specA.p, (CT*)ws.specB.p, (int64_t)ns * 8, nfreq, s);  // -> [f][s][c]
        }
        XCUDA(cudaEventRecord(ev[1], s));
      }
      if (phase & (M2L_HAD_SPARSE | M2L_HAD_DENSE)) {
        // Hadamard product
        const int ntiles = ws.had_tile0[g + 1] - ws.had_tile0[g];
        if constexpr (sizeof(CT) == 8) {
          XREQUIRE(nfreq < 65536, XFMM_ERR_UNSUPPORTED, "too many frequencies for the Hadamard grid");
          if (ntiles > 0 && (phase & M2L_HAD_SPARSE)) {
            const int* rows = ws.hadr_row.p + (int64_t)ws.had_tile0[g] * HADR_TT;
            if (!ws.hadrt_attr) {
              XCUDA(cudaFuncSetAttribute(k_hadamard_rt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HADT_SMEM));
              ws.hadrt_attr = true;
            }
            const int tpc = t.hadr_tpc > 0 ? t.hadr_tpc : HADR_TPC;
            k_hadamard_rt<<<dim3((ntiles + tpc - 1) / tpc, nfreq), HADR_NT, HADT_SMEM, s>>>(
                T, (const CT*)ws.specB.p, (CT*)ws.specA.p, ws.hadr_tile.p + ws.had_tile0[g], ws.hadr_pos.p,
                ws.hadr_ent.p, rows, ntiles, tpc, ns, nt, nfreq);
            XLAUNCH();
            ws.launches++;
          }
          if (ws.hadd_ld[g] > 0 && ws.had_tc5 && (phase & M2L_HAD_DENSE)) {
            if (!ws.hadc_attr) {
              XCUDA(cudaFuncSetAttribute(k_hadamard_dc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HADC_SMEM));
              ws.hadc_attr = true;
            }
            if (ws.hadc_btab_T != (const void*)T || ws.hadc_btab_nf != nfreq) {  // B blocks in the MMA layout
              ws.hadc_btab.reserve((size_t)nfreq * HADC_BBYTES);
              k_hadc_btab<<<std::min<int64_t>(nblk((int64_t)nfreq * 26 * 64), 148 * 16), 256, 0, s>>>(T, nfreq,
                                                                                                    ws.hadc_btab.p);
              XLAUNCH();
              ws.launches++;
              ws.hadc_btab_T = T;
              ws.hadc_btab_nf = nfreq;
            }
            k_hadamard_dc<<<dim3(ws.hadd_ld[g] / 128, (nfreq + HADC_FPB - 1) / HADC_FPB), HADC_NT, HADC_SMEM, s>>>(
                ws.hadc_btab.p, (const CT*)ws.specB.p, (CT*)ws.specA.p, ws.hadd_tab.p + ws.hadd_tab0[g], ws.hadd_ld[g],
                ws.hadd_row.p + ws.hadd_row0[g], ns, nt, nfreq, ws.status.p);
            XLAUNCH();
            ws.launches++;
          } else if (ws.hadd_ld[g] > 0 && (phase & M2L_HAD_DENSE)) {
            if (!ws.hadt_attr) {
              XCUDA(cudaFuncSetAttribute(k_hadamard_dt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HADT_SMEM));
              ws.hadt_attr = true;
            }
            k_hadamard_dt<<<dim3((ws.hadd_ld[g] / HADT_TT + HADT_TPC - 1) / HADT_TPC, nfreq), HADT_NT, HADT_SMEM, s>>>(
                T, (const CT*)ws.specB.p, (CT*)ws.specA.p, ws.hadd_tab.p + ws.hadd_tab0[g], ws.hadd_ld[g],
                ws.hadd_row.p + ws.hadd_row0[g], ns, nt, nfreq);
            XLAUNCH();
            ws.launches++;
          }
        } else {
          XREQUIRE(nfreq < 65536, XFMM_ERR_UNSUPPORTED, "too many frequencies for the Hadamard grid");
          if (ws.hadd_ld[g] > 0 && (phase & M2L_HAD_DENSE)) {
            if (!ws.had64_attr) {
              XCUDA(cudaFuncSetAttribute(k_hadamard_d64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HAD64_SMEM));
              ws.had64_attr = true;
            }
            k_hadamard_d64<<<dim3(ws.hadd_ld[g] / HAD64_TT, nfreq), HAD64_NT, HAD64_SMEM, s>>>(
                T, (const CT*)ws.specB.p, (CT*)ws.specA.p, ws.hadd_tab.p + ws.hadd_tab0[g], ws.hadd_ld[g],
                ws.hadd_row.p + ws.hadd_row0[g], ns, nt, nfreq);
            XLAUNCH();
            ws.launches++;
          }
        }
        XCUDA(cudaEventRecord(ev[2], s));
      }
      if (phase & M2L_BWD) {
        // inverse DFT of specA [f][t][c] to the downward check potentials (fmm_scale_invariant.h:606-646)
        if constexpr (KER != K_HELMHOLTZ) {
          if (ws.fused) {
            ft_dispatch(f.p, [&](auto pc) {
              constexpr int PP = decltype(pc)::value;
            if constexpr (sizeof(R) == 4) {  // FP64: the unslabbed form (measured faster at 1 CTA per SM)
              const size_t smem = ftr_bwd_smem<R>(PP);
              if (ws.ft_bwd_smem < smem) {
                XCUDA(cudaFuncSetAttribute(k_m2l_bwd_r<R, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                ws.ft_bwd_smem = smem;
              }
              k_m2l_bwd_r<R, PP><<<dim3(nt, 8 / FtCpb<R>::v), FT_NT, smem, s>>>(
                  trg, nt, t.child0.p, (const CT*)ws.specA.p, n, f.map_dn.p, f.dft_tw.p,
                  m2l_scale_of<R>(t) + t.m2l_trg_off[g], (R*)ws.dn.p);
            } else {
              const size_t smem = ft_bwd_smem<R>(PP);
              if (ws.ft_bwd_smem < smem) {
                XCUDA(cudaFuncSetAttribute(k_m2l_bwd<R, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                ws.ft_bwd_smem = smem;
              }
              k_m2l_bwd<R, PP><<<dim3(nt, 8 / FtCpb<R>::v), FT_NT, smem, s>>>(
                  trg, nt, t.child0.p, (const CT*)ws.specA.p, n, f.map_dn.p, f.dft_tw.p,
                  m2l_scale_of<R>(t) + t.m2l_trg_off[g], (R*)ws.dn.p);
            }
            });
            XLAUNCH();
            ws.launches++;
          }
        } else if (ws.fused) {
          ftc_dispatch(f.p, [&](auto pc) {
            constexpr int PP = decltype(pc)::value;
            const size_t smem = ftc_bwd_smem<R>(PP);
            if (ws.ft_bwd_smem < smem) {
              XCUDA(cudaFuncSetAttribute(k_m2l_bwd_c<R, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
              ws.ft_bwd_smem = smem;
            }
            k_m2l_bwd_c<R, PP><<<dim3(nt, 8 / FtcCpb<R>::v), FT_NT, smem, s>>>(trg, nt, t.child0.p, (const CT*)ws.specA.p, n,
                                                               f.map_dn.p, f.dft_tw.p,
                                                               m2l_scale_of<R>(t) + t.m2l_trg_off[g], (CT*)ws.dn.p);
          });
          XLAUNCH();
          ws.launches++;
        }
        if (!ws.fused) {
          ws.launches++;
          transpose<CT>((const CT*)ws.specA.p, (CT*)ws.specB.p, nfreq, (int64_t)nt * 8, s);  // -> [t][c][f]
          XCUFFT2(cufftSetStream(ws.bwd[g], s));
          exec_bwd(ws.bwd[g], ws.specB.p, ws.grid.p);
          k_m2l_gather_dn<W, R><<<std::min<int64_t>(nblk((int64_t)nt * 8 * n), 148 * 32), 256, 0, s>>>(
              trg, nt, t.child0.p, (const W*)ws.grid.p, nconv, f.map_dn.p, n,
              m2l_scale_of<R>(t) + t.m2l_trg_off[g], (W*)ws.dn.p);
          XLAUNCH();
          ws.launches += 2;
        }
        XCUDA(cudaEventRecord(ev[3], s));
      }
    }
  }

  static void exec_fwd(cufftHandle h, void* in, void* out) {
    if (KER == K_HELMHOLTZ) {
      if (sizeof(R) == 4) XCUFFT2(cufftExecC2C(h, (cufftComplex*)in, (cufftComplex*)out, CUFFT_FORWARD));
      else XCUFFT2(cufftExecZ2Z(h, (cufftDoubleComplex*)in, (cufftDoubleComplex*)out, CUFFT_FORWARD));
    } else {
      if (sizeof(R) == 4) XCUFFT2(cufftExecR2C(h, (cufftReal*)in, (cufftComplex*)out));
      else XCUFFT2(cufftExecD2Z(h, (cufftDoubleReal*)in, (cufftDoubleComplex*)out));
    }
  }
  static void exec_bwd(cufftHandle h, void* in, void* out) {
    if (KER == K_HELMHOLTZ) {
      if (sizeof(R) == 4) XCUFFT2(cufftExecC2C(h, (cufftComplex*)in, (cufftComplex*)out, CUFFT_INVERSE));
      else XCUFFT2(cufftExecZ2Z(h, (cufftDoubleComplex*)in, (cufftDoubleComplex*)out, CUFFT_INVERSE));
    } else {
      if (sizeof(R) == 4) XCUFFT2(cufftExecC2R(h, (cufftComplex*)in, (cufftReal*)out));
      else XCUFFT2(cufftExecZ2D(h, (cufftDoubleComplex*)in, (cufftDoubleReal*)out));
    }
  }

  // the far field (M2P + L2P evaluation), added to the near field's values
  static EvalArgs far_args(Fmm& f, Tree& t, Workspace& ws) {
    EvalArgs a{t.eval_leafs.p, t.leafs.p, t.nsrcs.p,   t.ntrgs.p, t.level.p, t.n_eval_leafs, t.sbeg.p,
               t.tbeg.p,       t.center.p, t.src4.p,   t.trg4.p,  t.src_qim.p, t.p2p_off.p,  t.m2p_off.p,
               t.p2p.p,        t.m2p.p,   f.surf_base.p, f.nsurf, ws.up.p,   ws.eq.p,        ws.out.p,
               f.k_re,         f.k_im,    1,           1,         0,         1};
    a.do_near = 0;
    a.accumulate = 1;
    return a;
  }

  static NearArgs near_args(Fmm& f, Tree& t, Workspace& ws) {
    return NearArgs{t.eval_leafs.p, t.leafs.p, t.nsrcs.p,   t.ntrgs.p, t.n_eval_leafs, t.sbeg.p, t.tbeg.p,
                    t.p2p_off.p,    t.p2p.p,   t.center.p,  t.src4.p,  t.trg4.p,       t.src_qim.p, ws.out.p,
                    f.k_re,         f.k_im};
  }

  // phases: DOWN_PRE (P2L, M2L, L2L, L2P check-to-equivalent), DOWN_NEAR (P2P), DOWN_FAR (M2P + L2P
  // evaluation, added to the near field's values); an evaluate runs all three in this order
  static void downward(Fmm& f, Tree& t, Workspace& ws, cudaStream_t s, int phases = DOWN_ALL, int m2l_phase = PRE_ALL) {
    const int n = f.nsurf;
    if (phases & DOWN_PRE) downward_pre(f, t, ws, s, m2l_phase);
    if (t.n_eval_leafs && (phases & DOWN_NEAR)) {
      NearArgs na = near_args(f, t, ws);
      if constexpr (KER == K_LAPLACE && sizeof(R) == 4) {
        if (ws.n_close < 0) find_close_pairs(ws, na, t.n_eval_leafs, s);
        k_near_lap_f2<<<nblk(t.n_eval_leafs, 4), 128, 0, s>>>(na);
        XLAUNCH();
        ws.launches++;
        if (ws.n_close > 0) {
          k_close_fix<<<nblk(ws.n_close, 256), 256, 0, s>>>(ws.close_pairs.p, ws.n_close, na, nullptr);
          XLAUNCH();
          ws.launches++;
        }
      } else {
        k_near<KER, R><<<nblk(t.n_eval_leafs, 4), 128, 0, s>>>(na);
        XLAUNCH();
        ws.launches++;
      }
    }
    if (phases & DOWN_NEAR) XCUDA(cudaEventRecord(ws.ev[8], s));
    if (t.n_eval_leafs && (phases & DOWN_FAR)) {
      const EvalArgs a = far_args(f, t, ws);
      const int blocks = nblk(t.n_eval_leafs, EVAL_WARPS);
      if constexpr (KER == K_LAPLACE && sizeof(R) == 4)
        k_far_lap<W><<<blocks, 32 * EVAL_WARPS, 0, s>>>(a);
      else
        k_eval<KER, double, W><<<blocks, 32 * EVAL_WARPS, 0, s>>>(a);
      XLAUNCH();
      ws.launches++;
    }
    if (phases & DOWN_FAR) XCUDA(cudaEventRecord(ws.ev[7], s));
  }

  // m2l_phase: the parts to run (PRE_ALL for an evaluate): the M2L parts (P2L with the forward transforms),
  // L2L (PRE_L2L) and L2P's check-to-equivalent step (PRE_DC2E)
  static void downward_pre(Fmm& f, Tree& t, Workspace& ws, cudaStream_t s, int m2l_phase = PRE_ALL) {
    const int n = f.nsurf;
    // P2L (X list) into downward check potentials
    if (t.n_p2l_nodes && (m2l_phase & M2L_FWD)) {
      SurfPotArgs a{t.p2l_nodes.p, t.n_p2l_nodes, t.nsrcs.p,     t.p2l.p, t.level.p, t.sbeg.p, t.p2l_off.p, t.center.p,
                    t.src4.p,      t.src_qim.p,   f.surf_base.p, n,       1.05,      ws.dn.p,  1,           f.k_re,
                    f.k_im,        INV4PI * op_scale(f, t)};
      k_surf_pot<KER, R><<<nblk(t.n_p2l_nodes, 4), 128, 0, s>>>(a);
      XLAUNCH();
      ws.launches++;
    }
    if (m2l_phase & M2L_FWD) XCUDA(cudaEventRecord(ws.ev[3], s));
    // M2L
    if (t.n_m2l_trg) m2l(f, t, ws, s, m2l_phase);
    if (m2l_phase & M2L_BWD) XCUDA(cudaEventRecord(ws.ev[4], s));
    if (m2l_phase & PRE_L2L) {
      // L2L: shallowest parents first (pre-order); per level one GEMM of the parents' rows with the
      // [n][8n] operator, added to the 8 children rows (contiguous per parent)
      for (int l = 0; l < t.depth; l++) {
        const GemmRows& g = ws.l2l[l];
        if (g.M <= 0) continue;
        const LevelOps& op = level_ops(f, l);
        TGemm gl{g.M, CW * 8 * n, CW * n, g.a.p, g.c.p, nullptr, (int64_t)CW * 8 * n, 1, (int64_t)CW * n};
        gl.status = ws.status.p;
        gl.scratch = ws.tc_scratch.p;
        gl.scratch_len = (int64_t)ws.tc_scratch.n;
        if constexpr (sizeof(R) == 4)
          tgemm_tc<float>(gl, (const float*)ws.dn.p, op.tg_l2l_h.p, op.tg_l2l_l.p, op.ld_l2l, (float*)ws.dn.p, s);
        else
          tgemm_f64<double, double>(gl, (const double*)ws.dn.p, op.tg_l2l.p, (double*)ws.dn.p, s);
        ws.launches++;
      }
      XCUDA(cudaEventRecord(ws.ev[5], s));
    }
    if (!(m2l_phase & PRE_DC2E)) return;
    // L2P part 1: downward check -> equivalent (DC2E) per leaf level, e = conj(U) S+ (conj(VH) 0.5^l c):
    // y over the kept singular directions, then e to the leaf positions (FP64).
    if (t.nleafs) {
      for (int l = 0; l <= t.depth; l++) {
        if (KER == K_LAPLACE && l > 0) break;
        const int r0 = ws.leaf_level_off[l], r1 = ws.leaf_level_off[l + 1];
        const int m = KER == K_LAPLACE ? ws.l2p1.M : r1 - r0;
        const int off = KER == K_LAPLACE ? 0 : r0;
        if (m <= 0) continue;
        const LevelOps& op = level_ops(f, l);
        const int rk = op.rank;
        TGemm g1{m, CW * rk, CW * n, ws.l2p1.a.p + off, ws.l2p1.c.p + off, ws.l2p2.al64.p + off, (int64_t)CW * n, 0,
                 (int64_t)CW * n};
        // The mixed path's downward check values are FP32 and conj(VH) is orthogonal: y = conj(VH) c runs
        // at FP32 accuracy (TF32 x 3), then e = conj(U) S+ y, whose 1/s amplification needs FP64.  These
        // densities feed only the leaf's own targets (measured: +0.5e-7 potential error at p = 8, +1e-7
        // at p = 10).
        g1.status = ws.status.p;
        if constexpr (sizeof(R) == 4 && KER != K_HELMHOLTZ)
          tgemm_tc<double>(g1, (const float*)ws.dn.p, op.tg_l2p1_h.p, op.tg_l2p1_l.p, op.ld_l2p1, (double*)ws.ybuf.p, s);
        else
          tgemm_f64<R, double>(g1, (const R*)ws.dn.p, op.tg_l2p1.p, (double*)ws.ybuf.p, s);
        TGemm g2{m, CW * n, CW * rk, ws.l2p2.a.p + off, ws.l2p2.c.p + off, nullptr, (int64_t)CW * n, 0, (int64_t)CW * n};
        tgemm_f64<double, double>(g2, (const double*)ws.ybuf.p, op.tg_l2p2.p, (double*)ws.eq.p, s);
        ws.launches += 2;
      }
    }
    XCUDA(cudaEventRecord(ws.ev[6], s));
  }
};

template <class F>
void dispatch(const Fmm& f, F&& fn) {
  if (f.kernel == XFMM_LAPLACE) {
    if (f.mixed()) fn(Engine<K_LAPLACE, float>());
    else fn(Engine<K_LAPLACE, double>());
  } else if (f.kernel == XFMM_MODIFIED_HELMHOLTZ) {
    if (f.mixed()) fn(Engine<K_YUKAWA, float>());
    else fn(Engine<K_YUKAWA, double>());
  } else {
    if (f.mixed()) fn(Engine<K_HELMHOLTZ, float>());
    else fn(Engine<K_HELMHOLTZ, double>());
  }
}

void check_ready(const Fmm& f, const Tree& t) {
  XREQUIRE(t.lists_built, XFMM_ERR_STATE, "evaluate before build_list");
  XREQUIRE(t.m2l_ready, XFMM_ERR_STATE, "evaluate before M2L_setup");
  XREQUIRE(f.precomputed, XFMM_ERR_STATE, "evaluate before precompute");
  XREQUIRE(f.pre_r0 == t.r0 || f.kernel == XFMM_LAPLACE, XFMM_ERR_STATE,
           "operators were precomputed for another root radius");
  XREQUIRE(f.kernel == XFMM_LAPLACE || f.pre_depth >= t.depth, XFMM_ERR_STATE,
           "operators were precomputed for a shallower tree");
  XREQUIRE(t.nsurf_lists == f.nsurf, XFMM_ERR_STATE, "lists were built for another expansion order");
  XREQUIRE((t.m2l_grouped_by_level != 0) == (f.kernel != XFMM_LAPLACE), XFMM_ERR_STATE,
           "M2L_setup was done for another kernel family");
}

}  // namespace

// ================================================================ public (internal API)
void set_charges(Fmm& f, Tree& t, const double* q, bool on_device, cudaStream_t s) {
  const int64_t n = t.nsrc;
  const int vs = f.is_complex() ? 2 : 1;
  const double* dq = q;
  if (!on_device) {
    // host charges: copied to a grow-only staging buffer owned by the tree and checked there for
    // non-finite values before any of them replaces the current charges; the call returns once the
    // caller's buffer has been read
    t.stage_q.upload(q, n * vs, s);
    dq = t.stage_q.p;
    t.stage_flag.reserve(1);
    XCUDA(cudaMemsetAsync(t.stage_flag.p, 0, sizeof(int), s));
    k_count_nonfinite<<<std::max<int64_t>(1, std::min<int64_t>(nblk(n * vs), 4 * 148)), 256, 0, s>>>(
        dq, n * vs, t.stage_flag.p);
    XLAUNCH();
    int bad = 0;
    XCUDA(cudaMemcpyAsync(&bad, t.stage_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    XCUDA(cudaStreamSynchronize(s));
    if (bad) throw Error(XFMM_ERR_NUMERIC, "non-finite value in charges");
  }
  k_set_charges<<<nblk(n), 256, 0, s>>>(dq, t.src_perm.p, n, f.is_complex(), t.src4.p, t.src_qim.p);
  XLAUNCH();
}

void clear_values(Fmm& f, Tree& t, cudaStream_t s) {
  check_ready(f, t);
  Workspace& ws = workspace(f, t, s);
  XCUDA(cudaMemsetAsync(ws.up.p, 0, ws.up.bytes(), s));
  XCUDA(cudaMemsetAsync(ws.dn.p, 0, ws.dn.bytes(), s));
}

void upward_pass(Fmm& f, Tree& t, cudaStream_t s) {
  check_ready(f, t);
  Workspace& ws = workspace(f, t, s);
  dispatch(f, [&](auto e) { decltype(e)::upward(f, t, ws, s); });
}

void downward_pass(Fmm& f, Tree& t, cudaStream_t s) {
  check_ready(f, t);
  Workspace& ws = workspace(f, t, s);
  dispatch(f, [&](auto e) { decltype(e)::downward(f, t, ws, s); });
}

// ================================================================ many systems in one evaluate
// Persistent near field over the target leaves of every system of a batch: each warp takes work items
// (system, target leaf) from one queue (a global counter, zeroed before the launch) in the order of
// `items` (largest pair count first) until it runs dry.  tpl: the largest number of targets a lane holds
// (1 or 2), the height of the warp's target tile.
__global__ void __launch_bounds__(128, XFMM_NEARF2_MINB)
    k_near_lap_f2_queue(const NearArgs* __restrict__ args, const int2* __restrict__ items, int64_t nitems,
                        unsigned int* __restrict__ counter, int tpl) {
  __shared__ NearSmemF2 sm[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (;;) {
    unsigned int k = 0;
    if (lane == 0) k = atomicAdd(counter, 1u);
    k = __shfl_sync(0xffffffffu, k, 0);
    if ((int64_t)k >= nitems) break;
    const int2 it = items[k];
    const NearArgs& a = args[it.x];
    const int node = a.leafs[a.eval_leafs[it.y]];
    const int T = a.ntrgs[node];
    if (T <= 32 || tpl == 1) near_leaf_lap_f2<1>(a, node, lane, sm[wid]);
    else near_leaf_lap_f2<2>(a, node, lane, sm[wid]);
    __syncwarp();
  }
}
template <int KER, class R>
__global__ void __launch_bounds__(128, XFMM_NEAR_MINB)
    k_near_queue(const NearArgs* __restrict__ args, const int2* __restrict__ items, int64_t nitems,
                 unsigned int* __restrict__ counter, int tpl) {
  __shared__ NearSmem<R> sm[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (;;) {
    unsigned int k = 0;
    if (lane == 0) k = atomicAdd(counter, 1u);
    k = __shfl_sync(0xffffffffu, k, 0);
    if ((int64_t)k >= nitems) break;
    const int2 it = items[k];
    const NearArgs& a = args[it.x];
    const int node = a.leafs[a.eval_leafs[it.y]];
    const int T = a.ntrgs[node];
    if (sizeof(R) == 4 && T > 32 && tpl >= 2) near_leaf<KER, R, 2>(a, node, lane, sm[wid]);
    else near_leaf<KER, R, 1>(a, node, lane, sm[wid]);
    __syncwarp();
  }
}
// pairs of one system, tagged with its index in .w, appended to a batch list
__global__ void k_tag_pairs(const int4* __restrict__ src, int64_t n, int sys, int4* __restrict__ dst) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < n) {
    int4 v = src[k];
    v.w = sys;
    dst[k] = v;
  }
}

struct Batch {
  std::vector<Fmm*> fmm;
  std::vector<Tree*> tree;
  int kernel = 0, precision = 0;
  DBuf<NearArgs> args;
  DBuf<int2> items;
  int64_t nitems = 0;
  DBuf<unsigned int> counter;
  DBuf<int4> close;
  int64_t nclose = 0;
  std::vector<int> order;  // systems, most bodies first (dealt to the streams in this order)
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  int near_ctas_per_sm = 0, near_tpl = 2;  // tuning (0: the kernel's resident limit)
  // mixed Laplace systems sharing one operator table: the sparse M2L Hadamard of every system in one launch
  bool had_batched = false;
  const float2* had_T = nullptr;
  int had_nfreq = 0, had_tpc = HADR_TPC, nhtiles = 0;
  DBuf<HadSys> hsys;
  DBuf<int2> htiles;
  // with the shared table also the M2M and L2L of every system, per level one GEMM over all systems' rows
  std::vector<GemmRows> bm2m, bl2l;  // row offsets rebased onto system 0's up / dn arrays
  DBuf<double> bscratch;             // FP64 scratch of their split K (zero between uses)
  GemmRows bp2m1, bp2m2, bl2p1, bl2p2;  // P2M and L2P pseudo-inverse factors of every system's leaves
  int* bstatus = nullptr;            // system 0's device status flag (bounded waits)
  // mixed Laplace: the far field of every system as one persistent launch over (system, leaf) items
  DBuf<EvalArgs> fargs;
  DBuf<int2> fitems;
  int64_t nfitems = 0;
  DBuf<unsigned int> fcounter;
  ~Batch() {
    for (auto e : events) cudaEventDestroy(e);
    for (auto st : streams) cudaStreamDestroy(st);
  }
};

Batch* batch_create(Fmm** fmms, Tree** trees, int n, cudaStream_t s) {
  XREQUIRE(n > 0, XFMM_ERR_ARG, "a batch needs at least one system");
  auto* b = new Batch();
  try {
    b->kernel = fmms[0]->kernel;
    b->precision = fmms[0]->precision;
    std::vector<NearArgs> hargs(n);
    std::vector<std::pair<int64_t, int2>> work;
    std::vector<int64_t> bodies(n);
    for (int k = 0; k < n; k++) {
      Fmm& f = *fmms[k];
      Tree& t = *trees[k];
      XREQUIRE(f.kernel == b->kernel && f.precision == b->precision, XFMM_ERR_ARG,
               "the systems of a batch share one kernel and one precision");
      check_ready(f, t);
      Workspace& ws = workspace(f, t, s);
      b->fmm.push_back(&f);
      b->tree.push_back(&t);
      dispatch(f, [&](auto e) { hargs[k] = decltype(e)::near_args(f, t, ws); });
      bodies[k] = t.ntrg;
      // work items: target leaves, costed by their pair counts
      std::vector<int64_t> poff = t.p2p_off.download(s);
      std::vector<int> pl = t.p2p.download(s, (size_t)t.np2p);
      std::vector<int> el = t.eval_leafs.download(s, (size_t)t.n_eval_leafs);
      for (int i = 0; i < t.n_eval_leafs; i++) {
        const int node = t.h_leafs[el[i]];
        int64_t ns = 0;
        for (int64_t e = poff[node]; e < poff[node + 1]; e++) ns += t.h_nsrcs[pl[e]];
        work.push_back({(int64_t)t.h_ntrgs[node] * ns, make_int2(k, i)});
      }
      if (f.kernel == XFMM_LAPLACE && f.mixed() && ws.n_close < 0 && t.n_eval_leafs > 0)
        find_close_pairs(ws, hargs[k], t.n_eval_leafs, s);
      if (f.kernel == XFMM_LAPLACE && f.mixed()) b->nclose += std::max<int64_t>(ws.n_close, 0);
    }
    if (b->kernel == XFMM_LAPLACE && b->precision == XFMM_MIXED) {
      // far-field items: evaluation leaves costed by targets x surface points evaluated (own + W list)
      std::vector<EvalArgs> fa(n);
      std::vector<std::pair<int64_t, int2>> fw;
      for (int k = 0; k < n; k++) {
        Fmm& f = *fmms[k];
        Tree& t = *trees[k];
        Workspace& ws = workspace(f, t, s);
        fa[k] = Engine<K_LAPLACE, float>::far_args(f, t, ws);
        std::vector<int64_t> moff = t.m2p_off.download(s);
        std::vector<int> el = t.eval_leafs.download(s, (size_t)t.n_eval_leafs);
        for (int i = 0; i < t.n_eval_leafs; i++) {
          const int node = t.h_leafs[el[i]];
          fw.push_back({(int64_t)t.h_ntrgs[node] * f.nsurf * (1 + moff[node + 1] - moff[node]), make_int2(k, i)});
        }
      }
      std::stable_sort(fw.begin(), fw.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
      std::vector<int2> fi(fw.size());
      for (size_t i = 0; i < fw.size(); i++) fi[i] = fw[i].second;
      b->nfitems = (int64_t)fi.size();
      if (!fi.empty()) b->fitems.upload(fi, s);
      b->fargs.upload(fa, s);
      b->fcounter.alloc(1);
    }
    std::stable_sort(work.begin(), work.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    std::vector<int2> items(work.size());
    for (size_t i = 0; i < work.size(); i++) items[i] = work[i].second;
    b->nitems = (int64_t)items.size();
    b->items.upload(items, s);
    b->args.upload(hargs, s);
    b->counter.alloc(1);
    if (b->nclose > 0) {
      b->close.alloc((size_t)b->nclose);
      int64_t off = 0;
      for (int k = 0; k < n; k++) {
        Workspace& ws = *trees[k]->ws[fmms[k]->precision];
        if (ws.n_close <= 0) continue;
        k_tag_pairs<<<nblk(ws.n_close, 256), 256, 0, s>>>(ws.close_pairs.p, ws.n_close, k, b->close.p + off);
        XLAUNCH();
        off += ws.n_close;
      }
    }
    // one operator table for every system (one Fmm), mixed Laplace (one M2L group): the sparse Hadamard
    // tiles of all systems as one list
    bool shared = b->kernel == XFMM_LAPLACE && b->precision == XFMM_MIXED;
    for (int k = 1; k < n && shared; k++) shared = fmms[k] == fmms[0];
    if (shared) {
      std::vector<HadSys> hs(n);
      std::vector<int2> tl;
      for (int k = 0; k < n; k++) {
        Tree& t = *trees[k];
        Workspace& ws = *t.ws[fmms[k]->precision];
        HadSys& h = hs[k];
        h = HadSys{};
        if (t.n_m2l_trg == 0 || t.m2l_src_off.size() != 2) continue;
        h.in = (const float2*)ws.specB.p;
        h.out = (float2*)ws.specA.p;
        h.tile_r = ws.hadr_tile.p + ws.had_tile0[0];
        h.rpos = ws.hadr_pos.p;
        h.ent = ws.hadr_ent.p;
        h.rows = ws.hadr_row.p + (int64_t)ws.had_tile0[0] * HADR_TT;
        h.nsrc = t.m2l_src_off[1] - t.m2l_src_off[0];
        h.ntrg = t.m2l_trg_off[1] - t.m2l_trg_off[0];
        for (int j = 0; j < ws.had_tile0[1] - ws.had_tile0[0]; j++) tl.push_back(make_int2(k, j));
      }
      // per-level translations over all systems' rows: offsets rebased onto system 0's up / dn arrays (every
      // system's arrays are separate allocations, 256-byte aligned: the rebased offsets keep 16-byte rows).
      // A rebased offset reaches from system 0's array into another system's allocation: this relies on the
      // device's single flat address space (every allocation of the context is addressed from one base),
      // not on C++ pointer rules, and the offsets are only ever applied on the device.
      int maxd = 0;
      for (int k = 0; k < n; k++) maxd = std::max(maxd, trees[k]->depth);
      const int prec = fmms[0]->precision, ns = fmms[0]->nsurf;
      Workspace& w0 = *trees[0]->ws[prec];
      const float* up0 = (const float*)w0.up.p;
      const float* dn0 = (const float*)w0.dn.p;
      b->bm2m.resize(maxd);
      b->bl2l.resize(maxd);
      int64_t need = 0;
      for (int l = 0; l < maxd; l++) {
        std::vector<int64_t> ma, mc, la, lc;
        for (int k = 0; k < n; k++) {
          Tree& t = *trees[k];
          Workspace& ws = *t.ws[prec];
          if (l >= t.depth) continue;
          const int64_t du = (const float*)ws.up.p - up0, dd = (const float*)ws.dn.p - dn0;
          const GemmRows& gm = ws.m2m[l];
          const GemmRows& gl = ws.l2l[l];
          if (gm.M > 0) {
            const std::vector<int64_t> a = gm.a.download(s, (size_t)gm.M), c = gm.c.download(s, (size_t)gm.M);
            for (int i = 0; i < gm.M; i++) {
              ma.push_back(a[i] + du);
              mc.push_back(c[i] + du);
            }
          }
          if (gl.M > 0) {
            const std::vector<int64_t> a = gl.a.download(s, (size_t)gl.M), c = gl.c.download(s, (size_t)gl.M);
            for (int i = 0; i < gl.M; i++) {
              la.push_back(a[i] + dd);
              lc.push_back(c[i] + dd);
            }
          }
        }
        upload_rows<double>(b->bm2m[l], ma, mc, std::vector<double>(ma.size(), 1.0), s);
        upload_rows<double>(b->bl2l[l], la, lc, std::vector<double>(la.size(), 1.0), s);
        need = std::max(need, tgemm_tc_scratch((int)ma.size(), ns, 8 * ns, 1));
        need = std::max(need, tgemm_tc_scratch((int)la.size(), 8 * ns, ns, 1));
      }
      // the pseudo-inverse factors of P2M and L2P over every system's leaves (one leaf group for Laplace):
      // A and C offsets rebased onto system 0's arrays, each in its own element unit
      {
        auto rel = [](const DBuf<char>& x, const DBuf<char>& x0, size_t es) {
          return (int64_t)((x.p - x0.p) / (int64_t)es);
        };
        std::vector<int64_t> a1, c1, a2, c2, la1, lc1, la2, lc2;
        std::vector<double> al2, lal1;
        for (int k = 0; k < n; k++) {
          Workspace& ws = *trees[k]->ws[prec];
          const int64_t dchk = rel(ws.chk, w0.chk, sizeof(float)), dy = rel(ws.ybuf, w0.ybuf, sizeof(double)),
                        dup = rel(ws.up, w0.up, sizeof(float)), ddn = rel(ws.dn, w0.dn, sizeof(float)),
                        deq = rel(ws.eq, w0.eq, sizeof(double));
          auto take = [&](const GemmRows& g, int64_t da, int64_t dc, std::vector<int64_t>& va,
                          std::vector<int64_t>& vc, std::vector<double>* val) {
            if (g.M <= 0) return;
            const std::vector<int64_t> a = g.a.download(s, (size_t)g.M), c = g.c.download(s, (size_t)g.M);
            std::vector<double> al;
            if (val) al = g.al64.download(s, (size_t)g.M);
            for (int i = 0; i < g.M; i++) {
              va.push_back(a[i] + da);
              vc.push_back(c[i] + dc);
              if (val) val->push_back(al[i]);
            }
          };
          XREQUIRE(ws.p2m1.M == ws.p2m2.M && ws.l2p1.M == ws.l2p2.M, XFMM_ERR_STATE,
                   "pseudo-inverse factor rows differ");
          take(ws.p2m1, dchk, dy, a1, c1, nullptr);
          take(ws.p2m2, dy, dup, a2, c2, &al2);
          take(ws.l2p1, ddn, dy, la1, lc1, nullptr);
          // L2P's first factor takes its per-row scale from the second factor's rows (as in the evaluate)
          take(ws.l2p2, dy, deq, la2, lc2, &lal1);
        }
        upload_rows<double>(b->bp2m1, a1, c1, std::vector<double>(a1.size(), 1.0), s);
        upload_rows<double>(b->bp2m2, a2, c2, al2, s);
        upload_rows<double>(b->bl2p1, la1, lc1, lal1, s);
        upload_rows<double>(b->bl2p2, la2, lc2, std::vector<double>(la2.size(), 1.0), s);
        need = std::max(need, tgemm_tc_scratch((int)la1.size(), fmms[0]->ops[0].rank, ns, 0));
      }
      if (need > 0) {
        b->bscratch.alloc((size_t)need);
        XCUDA(cudaMemsetAsync(b->bscratch.p, 0, b->bscratch.bytes(), s));
      }
      b->bstatus = w0.status.p;
      b->had_batched = true;
      b->had_T = (const float2*)fmms[0]->ops[0].m2l_T.p;
      b->had_nfreq = fmms[0]->nfreq;
      b->nhtiles = (int)tl.size();
      b->hsys.upload(hs, s);
      if (!tl.empty()) b->htiles.upload(tl, s);
      XREQUIRE(b->had_nfreq < 65536, XFMM_ERR_UNSUPPORTED, "too many frequencies for the Hadamard grid");
      XCUDA(cudaFuncSetAttribute(k_hadamard_rt_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HADT_SMEM));
    }
    b->order.resize(n);
    for (int k = 0; k < n; k++) b->order[k] = k;
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return bodies[x] > bodies[y]; });
    XCUDA(cudaStreamSynchronize(s));
  } catch (...) {
    delete b;
    throw;
  }
  return b;
}

void batch_free(Batch* b) { delete b; }

void batch_schedule(const int64_t* sizes, int n, int nstreams, int* stream_of) {
  XREQUIRE(n >= 0 && nstreams >= 1, XFMM_ERR_ARG, "batch schedule needs n >= 0 and nstreams >= 1");
  std::vector<int> order(n);
  for (int k = 0; k < n; k++) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return sizes[x] > sizes[y]; });
  std::vector<int64_t> load(std::max(1, std::min(nstreams, std::max(n, 1))), 0);
  for (int k : order) {
    const int j = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    stream_of[k] = j;
    load[j] += sizes[k];
  }
}

void batch_set_tuning(Batch* b, int option, int value) {
  if (option == XFMM_BATCH_NEAR_CTAS_PER_SM) {
    XREQUIRE(value >= 0 && value <= 32, XFMM_ERR_ARG, "CTAs per SM out of range (0..32)");
    b->near_ctas_per_sm = value;
  } else if (option == XFMM_BATCH_NEAR_TARGETS_PER_LANE) {
    XREQUIRE(value == 1 || value == 2, XFMM_ERR_ARG, "targets per lane must be 1 or 2");
    b->near_tpl = value;
  } else if (option == XFMM_BATCH_HADAMARD_TILES_PER_CTA) {
    XREQUIRE(value >= 0 && value <= 64, XFMM_ERR_ARG, "Hadamard tiles per CTA must be 0..64");
    b->had_tpc = value > 0 ? value : HADR_TPC;
  } else {
    XREQUIRE(false, XFMM_ERR_ARG, "unknown batch tuning option");
  }
}

// One evaluate of every system: charges (device, caller's order; null: keep the current ones) in,
// potentials and gradients out (device, caller's order).  The per-system stages before and after the
// near field run on `nstreams` streams forked from s (systems dealt largest first, each to the stream
// with the fewest bodies so far); the near field of all systems is one persistent launch on s.
void batch_evaluate(Batch* b, const double* const* charges, double* const* outs, int nstreams, cudaStream_t s) {
  const int n = (int)b->fmm.size();
  nstreams = std::max(1, std::min(nstreams, n));
  while ((int)b->streams.size() < nstreams) {
    cudaStream_t st;
    XCUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->streams.push_back(st);
  }
  while (b->events.size() < (size_t)5 * (nstreams + 1)) {
    cudaEvent_t e;
    XCUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->events.push_back(e);
  }
  std::vector<int64_t> sizes(n);
  for (int k = 0; k < n; k++) sizes[k] = b->tree[k]->ntrg;
  std::vector<int> stream_of(n);
  batch_schedule(sizes.data(), n, nstreams, stream_of.data());
  std::vector<std::vector<int>> lists(nstreams);
  for (int k : b->order) lists[stream_of[k]].push_back(k);
  auto fork_join = [&](int evbase, auto&& body) {
    if (nstreams == 1) {
      for (int k : lists[0]) body(k, s);
      return;
    }
    XCUDA(cudaEventRecord(b->events[evbase], s));
    for (int j = 0; j < nstreams; j++) {
      XCUDA(cudaStreamWaitEvent(b->streams[j], b->events[evbase], 0));
      for (int k : lists[j]) body(k, b->streams[j]);
      XCUDA(cudaEventRecord(b->events[evbase + 1 + j], b->streams[j]));
      XCUDA(cudaStreamWaitEvent(s, b->events[evbase + 1 + j], 0));
    }
  };
  // before the near field: upward pass, P2L, M2L and L2L per system.  With one shared operator table (mixed
  // Laplace) the parts that share it run as one launch over all systems: the M2M and L2L of each level, and
  // the sparse M2L Hadamard between the systems' forward and backward transforms.
  const int E = nstreams + 1;
  Fmm& f0 = *b->fmm[0];
  auto per_system = [&](int evbase, int up_parts, int pre_parts, bool first) {
    fork_join(evbase, [&](int k, cudaStream_t st) {
      Fmm& f = *b->fmm[k];
      Tree& t = *b->tree[k];
      if (first) {
        if (charges && charges[k]) set_charges(f, t, charges[k], true, st);
        clear_values(f, t, st);
      }
      Workspace& ws = workspace(f, t, st);
      dispatch(f, [&](auto e) {
        if (up_parts) decltype(e)::upward(f, t, ws, st, up_parts);
        if (pre_parts) decltype(e)::downward(f, t, ws, st, DOWN_PRE, pre_parts);
      });
    });
  };
  auto batched_tr = [&](const GemmRows& g, bool m2m) {
    if (g.M <= 0) return;
    const int nn = f0.nsurf;
    const LevelOps& op = f0.ops[0];
    float* up0 = (float*)b->tree[0]->ws[f0.precision]->up.p;
    float* dn0 = (float*)b->tree[0]->ws[f0.precision]->dn.p;
    TGemm gg = m2m ? TGemm{g.M, nn, 8 * nn, g.a.p, g.c.p, nullptr, (int64_t)nn, 1, (int64_t)nn}
                   : TGemm{g.M, 8 * nn, nn, g.a.p, g.c.p, nullptr, (int64_t)8 * nn, 1, (int64_t)nn};
    gg.status = b->bstatus;
    gg.scratch = b->bscratch.p;
    gg.scratch_len = (int64_t)b->bscratch.n;
    if (m2m) tgemm_tc<float>(gg, up0, op.tg_m2m_h.p, op.tg_m2m_l.p, op.ld_m2m, up0, s);
    else tgemm_tc<float>(gg, dn0, op.tg_l2l_h.p, op.tg_l2l_l.p, op.ld_l2l, dn0, s);
  };
  if (!b->had_batched) {
    per_system(0, UP_ALL, PRE_ALL, true);
  } else {
    Workspace& w0 = *b->tree[0]->ws[f0.precision];
    const int nn = f0.nsurf, rk = f0.ops[0].rank;
    const LevelOps& op = f0.ops[0];
    per_system(0, UP_CHK, 0, true);
    if (b->bp2m1.M > 0) {  // P2M's pseudo-inverse factors of every system's leaves
      TGemm g1{b->bp2m1.M, rk, nn, b->bp2m1.a.p, b->bp2m1.c.p, nullptr, (int64_t)nn, 0, (int64_t)nn};
      tgemm_f64<float, double>(g1, (const float*)w0.chk.p, op.tg_p2m1.p, (double*)w0.ybuf.p, s);
      TGemm g2{b->bp2m2.M, nn, rk, b->bp2m2.a.p, b->bp2m2.c.p, b->bp2m2.al64.p, (int64_t)nn, 0, (int64_t)nn};
      tgemm_f64<double, float>(g2, (const double*)w0.ybuf.p, op.tg_p2m2.p, (float*)w0.up.p, s);
    }
    for (int l = (int)b->bm2m.size() - 1; l >= 0; l--) batched_tr(b->bm2m[l], true);
    per_system(E, 0, M2L_FWD | M2L_HAD_DENSE, false);
    if (b->nhtiles > 0) {
      const int tpc = std::max(1, b->had_tpc);
      k_hadamard_rt_batch<<<dim3((b->nhtiles + tpc - 1) / tpc, b->had_nfreq), HADR_NT, HADT_SMEM, s>>>(
          b->had_T, b->hsys.p, b->htiles.p, b->nhtiles, tpc, b->had_nfreq);
      XLAUNCH();
    }
    per_system(2 * E, 0, M2L_BWD, false);
    for (int l = 0; l < (int)b->bl2l.size(); l++) batched_tr(b->bl2l[l], false);
    if (b->bl2p1.M > 0) {  // L2P's check-to-equivalent factors of every system's leaves
      TGemm g1{b->bl2p1.M, rk, nn, b->bl2p1.a.p, b->bl2p1.c.p, b->bl2p1.al64.p, (int64_t)nn, 0, (int64_t)nn};
      g1.status = b->bstatus;
      g1.scratch = b->bscratch.p;
      g1.scratch_len = (int64_t)b->bscratch.n;
      tgemm_tc<double>(g1, (const float*)w0.dn.p, op.tg_l2p1_h.p, op.tg_l2p1_l.p, op.ld_l2p1, (double*)w0.ybuf.p, s);
      TGemm g2{b->bl2p2.M, nn, rk, b->bl2p2.a.p, b->bl2p2.c.p, nullptr, (int64_t)nn, 0, (int64_t)nn};
      tgemm_f64<double, double>(g2, (const double*)w0.ybuf.p, op.tg_l2p2.p, (double*)w0.eq.p, s);
    }
  }
  // the near field of every system: one persistent launch draining the work queue
  if (b->nitems > 0) {
    int dev = 0, nsm = 148;
    XCUDA(cudaGetDevice(&dev));
    XCUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    XCUDA(cudaMemsetAsync(b->counter.p, 0, sizeof(unsigned int), s));
    const bool lapf2 = b->kernel == XFMM_LAPLACE && b->precision == XFMM_MIXED;
    auto launch = [&](auto kern) {
      int per_sm = 0;
      XCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0));
      if (b->near_ctas_per_sm > 0) per_sm = std::min(per_sm, b->near_ctas_per_sm);
      const int64_t need = (b->nitems + 3) / 4;
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)std::max(per_sm, 1) * nsm, need));
      kern<<<grid, 128, 0, s>>>(b->args.p, b->items.p, b->nitems, b->counter.p, b->near_tpl);
      XLAUNCH();
    };
    if (lapf2) launch(k_near_lap_f2_queue);
    else if (b->kernel == XFMM_LAPLACE) launch(k_near_queue<K_LAPLACE, double>);
    else if (b->kernel == XFMM_MODIFIED_HELMHOLTZ)
      b->precision == XFMM_MIXED ? launch(k_near_queue<K_YUKAWA, float>) : launch(k_near_queue<K_YUKAWA, double>);
    else
      b->precision == XFMM_MIXED ? launch(k_near_queue<K_HELMHOLTZ, float>) : launch(k_near_queue<K_HELMHOLTZ, double>);
    if (lapf2 && b->nclose > 0) {
      NearArgs none{};
      k_close_fix<<<nblk(b->nclose, 256), 256, 0, s>>>(b->close.p, b->nclose, none, b->args.p);
      XLAUNCH();
    }
  }
  // the far field (one persistent launch over every system's leaves for mixed Laplace), then the results
  const bool far_queue = b->nfitems > 0;
  if (far_queue) {
    int dev = 0, nsm = 148, per_sm = 0;
    XCUDA(cudaGetDevice(&dev));
    XCUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    XCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_far_lap_queue<float>, 32 * EVAL_WARPS, 0));
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((int64_t)std::max(per_sm, 1) * nsm, (b->nfitems + EVAL_WARPS - 1) / EVAL_WARPS));
    XCUDA(cudaMemsetAsync(b->fcounter.p, 0, sizeof(unsigned int), s));
    k_far_lap_queue<float><<<grid, 32 * EVAL_WARPS, 0, s>>>(b->fargs.p, b->fitems.p, b->nfitems, b->fcounter.p);
    XLAUNCH();
  }
  fork_join(4 * E, [&](int k, cudaStream_t st) {
    Fmm& f = *b->fmm[k];
    Tree& t = *b->tree[k];
    Workspace& ws = workspace(f, t, st);
    if (!far_queue) dispatch(f, [&](auto e) { decltype(e)::downward(f, t, ws, st, DOWN_FAR); });
    get_values(f, t, outs[k], st);
  });
}

// Device times of the last upward + downward pass (ms): 0 P2M, 1 M2M, 2 P2L, 3 M2L, 4 L2L,
// 5 L2P check->equivalent, 6 target evaluation (P2P + M2P + L2P), 7 total, 8-10 M2L FFT / Hadamard / iFFT.
namespace {
// An mbarrier (expecting one arrival) whose phase nothing completes; the wait runs out after `limit`
// cycles and the kernel reports it through *status, as the pipelined kernels do.
__global__ void k_selftest_wait(long long limit, int* status) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = tc5::smem_u32(&bar);
  if (threadIdx.x == 0) {
    tc5::mbar_init(b, 1);
    tc5::fence_mbar_init();
  }
  __syncthreads();
  const bool ok = __all_sync(0xffffffffu, tc5::mbar_wait(b, 0, limit));
  if (!ok && threadIdx.x == 0) atomicExch(status, 1);
}
}  // namespace

void selftest_bounded_wait(int64_t limit_cycles) {
  XREQUIRE(limit_cycles >= 1 && limit_cycles <= 1000000000LL, XFMM_ERR_ARG, "limit_cycles outside 1..1e9");
  DBuf<int> status(1);
  XCUDA(cudaMemset(status.p, 0, sizeof(int)));
  k_selftest_wait<<<1, 32>>>(limit_cycles, status.p);
  XLAUNCH();
  XCUDA(cudaDeviceSynchronize());
  int h = 0;
  XCUDA(cudaMemcpy(&h, status.p, sizeof(int), cudaMemcpyDeviceToHost));
  XREQUIRE(!h, XFMM_ERR_TIMEOUT, "bounded device-side wait ran out (self-test)");
}

// After the caller's stream has been synchronised: XFMM_ERR_TIMEOUT when a bounded device-side wait of the
// last pass ran out (the flag is cleared for the next pass).
void check_device_status(Fmm& f, Tree& t) {
  Workspace* ws = t.ws[f.precision];
  if (!ws) return;
  int dev_status = 0;
  XCUDA(cudaMemcpy(&dev_status, ws->status.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (dev_status) {
    XCUDA(cudaMemset(ws->status.p, 0, sizeof(int)));
    XREQUIRE(false, XFMM_ERR_TIMEOUT, "a bounded device-side wait ran out in the last pass (results incomplete)");
  }
}

void stage_times(Fmm& f, Tree& t, double* ms14) {
  Workspace* ws = t.ws[f.precision];
  XREQUIRE(ws, XFMM_ERR_STATE, "no evaluate has run");
  XCUDA(cudaEventSynchronize(ws->ev[7]));
  int dev_status = 0;
  XCUDA(cudaMemcpy(&dev_status, ws->status.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (dev_status) {
    XCUDA(cudaMemset(ws->status.p, 0, sizeof(int)));
    XREQUIRE(false, XFMM_ERR_TIMEOUT, "a bounded device-side wait ran out in the last pass (results incomplete)");
  }
  auto el = [](cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? (double)ms : 0.0;
  };
  const int pairs[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}, {0, 7}};
  for (int i = 0; i < 8; i++) ms14[i] = el(ws->ev[pairs[i][0]], ws->ev[pairs[i][1]]);
  ms14[8] = ms14[9] = ms14[10] = 0;
  const int ng = (int)ws->m2l_ev.size() / 4;
  for (int g = 0; g < ng; g++) {
    const int ns = t.m2l_src_off[g + 1] - t.m2l_src_off[g], nt = t.m2l_trg_off[g + 1] - t.m2l_trg_off[g];
    if (ns == 0 || nt == 0) continue;
    cudaEvent_t* e = ws->m2l_ev.data() + 4 * g;
    ms14[8] += el(e[0], e[1]);
    ms14[9] += el(e[1], e[2]);
    ms14[10] += el(e[2], e[3]);
  }
  for (int i = 0; i < 11; i++) f.stage_ms[i] = ms14[i];
  ms14[11] = (double)ws->launches;
  ms14[12] = el(ws->ev[6], ws->ev[8]);  // near field (P2P)
  ms14[13] = el(ws->ev[8], ws->ev[7]);  // far field (M2P + L2P)
}

void get_values(Fmm& f, Tree& t, double* out_dev, cudaStream_t s) {
  Workspace& ws = workspace(f, t, s);
  const int width = 4 * (f.is_complex() ? 2 : 1);
  k_scatter_out<<<nblk(t.ntrg), 256, 0, s>>>(ws.out.p, t.trg_perm.p, t.ntrg, width, out_dev);
  XLAUNCH();
  ws.launches++;
}

// xfmm_gradient_p2p: one "leaf" of all targets against one "leaf" of all sources
namespace {
struct RawP2P {
  DBuf<double4> s4, t4;
  DBuf<double> qim;
};
__global__ void k_pack_raw(const double* xyz, const double* q, int64_t n, int cplx, double4* out, double* qim) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_double4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], q ? (cplx ? q[2 * i] : q[i]) : 0.0);
  if (q && cplx) qim[i] = q[2 * i + 1];
}
template <int KER, class R>
__global__ void __launch_bounds__(128) k_raw_p2p(const double4* __restrict__ s4, const double* __restrict__ qim,
                                                  int64_t ns, const double4* __restrict__ t4, int64_t nt,
                                                  double k_re, double k_im, double* __restrict__ out) {
  using G = Green<KER, R>;
  using Q = typename G::Q;
  using A = typename Acc64<Q>::type;
  using V4 = typename R4<R>::type;
  __shared__ double4 sx[128];
  __shared__ Q sq[128];
  const G g{(R)k_re, (R)k_im};
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const double4 tv = t < nt ? t4[t] : make_double4(0, 0, 0, 0);
  A P, GX, GY, GZ;
  P = GX = GY = GZ = A();
  for (int64_t j0 = 0; j0 < ns; j0 += 128) {
    const int cnt = (int)(ns - j0 < 128 ? ns - j0 : 128);
    __syncthreads();
    if (threadIdx.x < cnt) {
      const double4 sv = s4[j0 + threadIdx.x];
      sx[threadIdx.x] = sv;
      sq[threadIdx.x] = load_charge<Q>(sv, qim, j0 + threadIdx.x);
    }
    __syncthreads();
    Q p = vzero<Q>(), gx = vzero<Q>(), gy = vzero<Q>(), gz = vzero<Q>();
    for (int j = 0; j < cnt; j++) {
      const double4 s = sx[j];  // differences in FP64, the kernel in R
      g.grad((R)(tv.x - s.x), (R)(tv.y - s.y), (R)(tv.z - s.z), sq[j], p, gx, gy, gz);
    }
    acc64(P, p);
    acc64(GX, gx);
    acc64(GY, gy);
    acc64(GZ, gz);
  }
  if (t < nt) {
    const int stride = (KER == K_HELMHOLTZ) ? 8 : 4, vs = stride / 4;
    double* o = out + t * stride;
    put_out(o, P, INV4PI, 1);
    put_out(o + vs, GX, INV4PI, 1);
    put_out(o + 2 * vs, GY, INV4PI, 1);
    put_out(o + 3 * vs, GZ, INV4PI, 1);
  }
}
}  // namespace

void gradient_p2p_raw(int kernel, double k_re, double k_im, int precision, const double* src, int64_t ns,
                      const double* q, const double* trg, int64_t nt, double* out, cudaStream_t s) {
  const int cplx = kernel == XFMM_HELMHOLTZ;
  RawP2P r;
  r.s4.alloc(std::max<int64_t>(ns, 1));
  r.t4.alloc(std::max<int64_t>(nt, 1));
  r.qim.alloc(std::max<int64_t>(ns, 1));
  k_pack_raw<<<nblk(ns), 256, 0, s>>>(src, q, ns, cplx, r.s4.p, r.qim.p);
  k_pack_raw<<<nblk(nt), 256, 0, s>>>(trg, nullptr, nt, 0, r.t4.p, nullptr);
  XLAUNCH();
  const int blocks = nblk(nt, 128);
  const bool m = precision == XFMM_MIXED;
  if (kernel == XFMM_LAPLACE) {
    if (m) k_raw_p2p<K_LAPLACE, float><<<blocks, 128, 0, s>>>(r.s4.p, r.qim.p, ns, r.t4.p, nt, k_re, k_im, out);
    else k_raw_p2p<K_LAPLACE, double><<<blocks, 128, 0, s>>>(r.s4.p, r.qim.p, ns, r.t4.p, nt, k_re, k_im, out);
  } else if (kernel == XFMM_MODIFIED_HELMHOLTZ) {
    if (m) k_raw_p2p<K_YUKAWA, float><<<blocks, 128, 0, s>>>(r.s4.p, r.qim.p, ns, r.t4.p, nt, k_re, k_im, out);
    else k_raw_p2p<K_YUKAWA, double><<<blocks, 128, 0, s>>>(r.s4.p, r.qim.p, ns, r.t4.p, nt, k_re, k_im, out);
  } else {
    if (m) k_raw_p2p<K_HELMHOLTZ, float><<<blocks, 128, 0, s>>>(r.s4.p, r.qim.p, ns, r.t4.p, nt, k_re, k_im, out);
    else k_raw_p2p<K_HELMHOLTZ, double><<<blocks, 128, 0, s>>>(r.s4.p, r.qim.p, ns, r.t4.p, nt, k_re, k_im, out);
  }
  XLAUNCH();
  XCUDA(cudaStreamSynchronize(s));
}

// The evaluation of gradient_p2p_raw with the packed bodies in device scratch that the caller owns
// (s4: ns double4, qim: ns doubles, t4: nt double4, each 32-byte aligned).  Asynchronous on s; no
// allocation and no synchronisation.  The packing kernels write every scratch entry the P2P kernel
// reads, so the scratch needs no initial contents.
void gradient_p2p_scratch(int kernel, double k_re, double k_im, int precision, const double* src, int64_t ns,
                          const double* q, const double* trg, int64_t nt, double* out, double4* s4, double* qim,
                          double4* t4, cudaStream_t s) {
  const int cplx = kernel == XFMM_HELMHOLTZ;
  if (ns > 0) k_pack_raw<<<nblk(ns), 256, 0, s>>>(src, q, ns, cplx, s4, qim);
  k_pack_raw<<<nblk(nt), 256, 0, s>>>(trg, nullptr, nt, 0, t4, nullptr);
  XLAUNCH();
  const int blocks = nblk(nt, 128);
  const bool m = precision == XFMM_MIXED;
  if (kernel == XFMM_LAPLACE) {
    if (m) k_raw_p2p<K_LAPLACE, float><<<blocks, 128, 0, s>>>(s4, qim, ns, t4, nt, k_re, k_im, out);
    else k_raw_p2p<K_LAPLACE, double><<<blocks, 128, 0, s>>>(s4, qim, ns, t4, nt, k_re, k_im, out);
  } else if (kernel == XFMM_MODIFIED_HELMHOLTZ) {
    if (m) k_raw_p2p<K_YUKAWA, float><<<blocks, 128, 0, s>>>(s4, qim, ns, t4, nt, k_re, k_im, out);
    else k_raw_p2p<K_YUKAWA, double><<<blocks, 128, 0, s>>>(s4, qim, ns, t4, nt, k_re, k_im, out);
  } else {
    if (m) k_raw_p2p<K_HELMHOLTZ, float><<<blocks, 128, 0, s>>>(s4, qim, ns, t4, nt, k_re, k_im, out);
    else k_raw_p2p<K_HELMHOLTZ, double><<<blocks, 128, 0, s>>>(s4, qim, ns, t4, nt, k_re, k_im, out);
  }
  XLAUNCH();
}

// FmmBase::verify (fmm_base.h:208-267) on the device: FP64 direct sum over all sources
void verify(Fmm& f, Tree& t, int sample, double* err2, cudaStream_t s) {
  Workspace& ws = workspace(f, t, s);
  std::vector<int> trg_leaves;
  if (sample) {
    const int stride = t.nleafs / 10;
    for (int i = 0; i < 10 && i * stride < t.nleafs; i++) trg_leaves.push_back(t.h_leafs[i * stride]);
  } else {
    trg_leaves = t.h_leafs;
  }
  std::vector<int64_t> tb = t.tbeg.download(s);
  std::vector<int64_t> rows;
  for (int node : trg_leaves)
    for (int k = 0; k < t.h_ntrgs[node]; k++) rows.push_back(tb[node] + k);
  const int cplx = f.is_complex();
  const int width = 4 * (cplx ? 2 : 1);
  std::vector<double4> htrg = t.trg4.download(s);
  std::vector<double> hout = ws.out.download(s);
  std::vector<double> txyz(3 * rows.size());
  for (size_t i = 0; i < rows.size(); i++) {
    txyz[3 * i] = htrg[rows[i]].x;
    txyz[3 * i + 1] = htrg[rows[i]].y;
    txyz[3 * i + 2] = htrg[rows[i]].z;
  }
  std::vector<double4> hsrc = t.src4.download(s);
  std::vector<double> hqim = t.src_qim.download(s);
  std::vector<double> sxyz(3 * t.nsrc), q(t.nsrc * (cplx ? 2 : 1));
  for (int64_t i = 0; i < t.nsrc; i++) {
    sxyz[3 * i] = hsrc[i].x;
    sxyz[3 * i + 1] = hsrc[i].y;
    sxyz[3 * i + 2] = hsrc[i].z;
    if (cplx) {
      q[2 * i] = hsrc[i].w;
      q[2 * i + 1] = hqim[i];
    } else {
      q[i] = hsrc[i].w;
    }
  }
  DBuf<double> ds, dq, dt, dout;
  ds.upload(sxyz, s);
  dq.upload(q, s);
  dt.upload(txyz, s);
  dout.alloc(std::max<size_t>(rows.size(), 1) * width);
  XCUDA(cudaMemsetAsync(dout.p, 0, dout.bytes(), s));
  gradient_p2p_raw(f.kernel, f.k_re, f.k_im, XFMM_FP64, ds.p, t.nsrc, dq.p, dt.p, (int64_t)rows.size(), dout.p, s);
  std::vector<double> ex = dout.download(s);
  double pd = 0, pn = 0, gd = 0, gn = 0;
  const int vs = cplx ? 2 : 1;
  for (size_t i = 0; i < rows.size(); i++)
    for (int c = 0; c < 4; c++)
      for (int v = 0; v < vs; v++) {
        const double e = ex[i * width + c * vs + v], a = hout[rows[i] * width + c * vs + v];
        (c == 0 ? pd : gd) += (e - a) * (e - a);
        (c == 0 ? pn : gn) += e * e;
      }
  err2[0] = std::sqrt(pd / pn);
  err2[1] = std::sqrt(gd / gn);
}

}  // namespace xfmm
