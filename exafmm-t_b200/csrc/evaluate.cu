// evaluate.cu -- upward and downward passes of the KIFMM on the GPU.
//
// Stage map (reference -> here):
//   P2M   fmm_scale_invariant.h:163-195 / fmm.h:156-185  k_p2m (check potentials) + gemm_rows (pinv, 0.5^l)
//   M2M   fmm_scale_invariant.h:233-253 / fmm.h:221-241  gemm_rows per level, K = 8 nsurf (children contiguous)
//   P2L   fmm_base.h:127-154                             k_p2l
//   M2L   fmm_scale_invariant.h:407-440, 560-646;        k_m2l_grid_up + cuFFT + k_transpose + k_hadamard
//         fmm.h:395-446, 631-788                         + k_transpose + cuFFT + k_m2l_gather_dn
//   L2L   fmm_scale_invariant.h:256-275 / fmm.h:244-263  gemm_rows per level, N = 8 nsurf
//   L2P   fmm_scale_invariant.h:198-230 / fmm.h:188-218  gemm_rows (pinv^T, 0.5^l) + k_eval (far part)
//   M2P   fmm_base.h:97-124                              k_eval (far part)
//   P2P   fmm_base.h:82-94                               k_eval (near part)
// The near and far target evaluations share one warp-per-leaf kernel; results stay in
// tree order until get_values scatters them (python/exafmm.cpp:194-207).
#include <cufft.h>

#include <algorithm>
#include <cmath>

#include "kernels.cuh"
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

template <int KER, class R>
__global__ void __launch_bounds__(32 * EVAL_WARPS) k_eval(EvalArgs a) {
  using G = Green<KER, R>;
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
  const Q* upv = (const Q*)a.up;
  const Q* eqv = (const Q*)a.eq;
  for (int t0 = 0; t0 < T; t0 += 32) {
    const int Tc = min(32, T - t0);
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
            s_q[wid][lane] = upv[(int64_t)s * n + k];
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
          s_q[wid][lane] = eqv[(int64_t)pos * n + k];
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

// ================================================================ P2M check potentials and P2L
// Potential at `n` surface points (base * b around centre cn) from body range(s); warp per node.
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
        acc = vscale(acc, (typename Base<Q>::type)INV4PI);
        out[k] = first ? acc : vadd(out[k], acc);
      }
      first = false;
      __syncwarp();
    }
  }
}

// ================================================================ translation GEMMs
// C[coff[i] + j] (+)= alpha[i] * sum_k A[aoff[i] + k] * B[k*N + j]   (rows gathered/scattered)
template <class V, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_gemm_rows(int M, int N, int K, const V* __restrict__ A,
                                                                      const int64_t* __restrict__ aoff,
                                                                      const V* __restrict__ B, V* __restrict__ C,
                                                                      const int64_t* __restrict__ coff,
                                                                      const typename Base<V>::type* __restrict__ alpha,
                                                                      int accumulate) {
  using RB = typename Base<V>::type;
  constexpr int NT = (BM / TM) * (BN / TN);
  __shared__ V As[BK][BM];
  __shared__ V Bs[BK][BN];
  const int tid = threadIdx.x;
  const int tx = tid % (BN / TN), ty = tid / (BN / TN);
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  V acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) acc[i][j] = vzero<V>();
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int e = tid; e < BM * BK; e += NT) {
      const int r = e / BK, kk = e % BK;
      const int row = m0 + r, k = k0 + kk;
      As[kk][r] = (row < M && k < K) ? A[aoff[row] + k] : vzero<V>();
    }
    for (int e = tid; e < BK * BN; e += NT) {
      const int kk = e / BN, cc = e % BN;
      const int k = k0 + kk, col = n0 + cc;
      Bs[kk][cc] = (k < K && col < N) ? B[(int64_t)k * N + col] : vzero<V>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      V av[TM], bv[TN];
#pragma unroll
      for (int i = 0; i < TM; i++) av[i] = As[kk][ty * TM + i];
#pragma unroll
      for (int j = 0; j < TN; j++) bv[j] = Bs[kk][tx * TN + j];
#pragma unroll
      for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) vfma(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < TM; i++) {
    const int row = m0 + ty * TM + i;
    if (row >= M) continue;
    const RB al = alpha ? alpha[row] : RB(1);
    V* crow = C + coff[row];
#pragma unroll
    for (int j = 0; j < TN; j++) {
      const int col = n0 + tx * TN + j;
      if (col < N) {
        const V v = vscale(acc[i][j], al);
        crow[col] = accumulate ? vadd(crow[col], v) : v;
      }
    }
  }
}

template <class V>
void gemm_rows(int M, int N, int K, const V* A, const int64_t* aoff, const V* B, V* C, const int64_t* coff,
               const typename Base<V>::type* alpha, int accumulate, cudaStream_t s) {
  if (M <= 0) return;
  constexpr bool cplx = sizeof(V) == 2 * sizeof(typename Base<V>::type);
  if (cplx) {
    dim3 grid((N + 63) / 64, (M + 31) / 32);
    k_gemm_rows<V, 32, 64, 8, 2, 4><<<grid, 256, 0, s>>>(M, N, K, A, aoff, B, C, coff, alpha, accumulate);
  } else {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    k_gemm_rows<V, 64, 64, 16, 4, 4><<<grid, 256, 0, s>>>(M, N, K, A, aoff, B, C, coff, alpha, accumulate);
  }
  XLAUNCH();
}

// ================================================================ M2L
// grid[(s*8 + c)*nconv + g] = up[child c of source s][surface point mapped to g] (0 elsewhere)
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
template <class CT>
void transpose(const CT* in, CT* out, int64_t R, int64_t C, cudaStream_t s) {
  dim3 grid((unsigned)((C + 31) / 32), (unsigned)((R + 31) / 32));
  XREQUIRE(grid.y < 65536, XFMM_ERR_UNSUPPORTED, "transpose too tall");
  k_transpose<CT><<<grid, dim3(32, 8), 0, s>>>(in, out, R, C);
  XLAUNCH();
}

// Hadamard product per frequency (fmm_scale_invariant.h:343-399; intrinsics.h matmult_8x8x2):
//   out[f][t][tc] = sum_ipos sum_sc T[ipos][f][sc*8 + tc] * in[f][src(t, ipos)][sc]
template <class CT, int KC>
__global__ void __launch_bounds__(256) k_hadamard(const CT* __restrict__ T, const CT* __restrict__ in,
                                                   CT* __restrict__ out, const int* __restrict__ tab, int nsrc,
                                                   int ntrg, int nfreq) {
  extern __shared__ unsigned char smem_raw[];
  CT* sT = (CT*)smem_raw;  // [26][KC][64]
  const int f0 = blockIdx.x * KC;
  for (int e = threadIdx.x; e < 26 * KC * 64; e += blockDim.x) {
    const int j = e % 64, kk = (e / 64) % KC, ipos = e / (64 * KC);
    const int f = f0 + kk;
    sT[e] = f < nfreq ? T[((int64_t)ipos * nfreq + f) * 64 + j] : vzero<CT>();
  }
  __syncthreads();
  for (int kk = 0; kk < KC; kk++) {
    const int f = f0 + kk;
    if (f >= nfreq) break;
    const CT* inf = in + (int64_t)f * nsrc * 8;
    for (int t = threadIdx.x; t < ntrg; t += blockDim.x) {
      CT acc[8];
#pragma unroll
      for (int i = 0; i < 8; i++) acc[i] = vzero<CT>();
      for (int ipos = 0; ipos < 26; ipos++) {
        const int s = tab[t * 26 + ipos];
        if (s < 0) continue;
        CT v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = inf[(int64_t)s * 8 + i];
        const CT* M = sT + (ipos * KC + kk) * 64;
#pragma unroll
        for (int sc = 0; sc < 8; sc++)
#pragma unroll
          for (int tc = 0; tc < 8; tc++) vfma(acc[tc], M[sc * 8 + tc], v[sc]);
      }
      CT* o = out + ((int64_t)f * ntrg + t) * 8;
#pragma unroll
      for (int i = 0; i < 8; i++) o[i] = acc[i];
    }
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
struct GemmRows {
  int M = 0;
  DBuf<int64_t> a, c;
  DBuf<float> al32;
  DBuf<double> al64;
};

struct Workspace {
  int precision = -1, kernel = -1, p = 0;
  size_t vsz = 0;
  DBuf<char> up, dn, chk, eq;
  DBuf<double> out;
  // leaves grouped by level (P2M / L2P operators are per level except for Laplace)
  std::vector<int> leaf_level_off;
  GemmRows p2m1, p2m2, l2p1, l2p2;  // two factors each (rows grouped by leaf level)
  std::vector<GemmRows> m2m, l2l;  // per level of the parent
  // M2L
  DBuf<char> grid, specA, specB;
  std::vector<cufftHandle> fwd, bwd;
  size_t hadamard_smem = 0;
  int64_t launches = 0;  // kernels of this library launched by the last evaluate
  cudaEvent_t ev[8] = {};
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
  std::vector<float> f(al.begin(), al.end());
  g.al32.upload(f, s);
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
  W.eq.alloc((size_t)std::max(t.nleafs, 1) * n * W.vsz);
  W.out.alloc((size_t)t.ntrg * 4 * (cplx ? 2 : 1));
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
    for (int i : order) {
      const int node = t.h_leafs[i];
      idn.push_back((int64_t)i * n);
      nodes.push_back((int64_t)node * n);
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
        ma.push_back((int64_t)t.h_child0[k] * n);
        mc.push_back((int64_t)k * n);
        la.push_back((int64_t)k * n);
        lc.push_back((int64_t)t.h_child0[k] * n);
        one.push_back(1.0);
      }
    upload_rows<double>(W.m2m[l], ma, mc, one, s);
    upload_rows<double>(W.l2l[l], la, lc, one, s);
  }
  // M2L buffers and FFT plans
  const int ng = (int)t.m2l_src_off.size() - 1;
  int maxn = 1;
  for (int g = 0; g < ng; g++) {
    maxn = std::max(maxn, t.m2l_src_off[g + 1] - t.m2l_src_off[g]);
    maxn = std::max(maxn, t.m2l_trg_off[g + 1] - t.m2l_trg_off[g]);
  }
  const size_t rsz = f.mixed() ? 4 : 8;  // real scalar size
  const size_t grid_vals = (size_t)maxn * 8 * f.nconv;
  W.grid.alloc(grid_vals * rsz * (cplx ? 2 : 1));
  W.specA.alloc((size_t)maxn * 8 * f.nfreq * 2 * rsz);
  W.specB.alloc((size_t)maxn * 8 * f.nfreq * 2 * rsz);
  int dims[3] = {f.n1, f.n1, f.n1};
  cufftType tf = cplx ? (f.mixed() ? CUFFT_C2C : CUFFT_Z2Z) : (f.mixed() ? CUFFT_R2C : CUFFT_D2Z);
  cufftType tb = cplx ? (f.mixed() ? CUFFT_C2C : CUFFT_Z2Z) : (f.mixed() ? CUFFT_C2R : CUFFT_Z2D);
  for (int g = 0; g < ng; g++) {
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
  for (auto& e : W.ev) XCUDA(cudaEventCreate(&e));
  W.m2l_ev.resize(4 * (size_t)ng);
  for (auto& e : W.m2l_ev) XCUDA(cudaEventCreate(&e));
  W.ev_ok = true;
  XCUDA(cudaStreamSynchronize(s));
  return W;
}

template <class W>
struct Ops {
  const W *p2m1, *p2m2, *l2p1, *l2p2, *m2m, *l2l;
};
template <class W>
Ops<W> ops_of(const Fmm& f, int level) {
  const LevelOps& o = f.ops[f.kernel == XFMM_LAPLACE ? 0 : level];
  return Ops<W>{(const W*)o.p2m_B1.p, (const W*)o.p2m_B2.p, (const W*)o.l2p_B1.p, (const W*)o.l2p_B2.p,
                (const W*)o.m2m_B.p,  (const W*)o.l2l_B.p};
}

template <class RB> const RB* alpha_of(const GemmRows& g);
template <> const float* alpha_of<float>(const GemmRows& g) { return g.al32.p; }
template <> const double* alpha_of<double>(const GemmRows& g) { return g.al64.p; }

template <class RB> const RB* m2l_scale_of(const Tree& t);
template <> const float* m2l_scale_of<float>(const Tree& t) { return t.m2l_scale.p; }
template <> const double* m2l_scale_of<double>(const Tree& t) { return t.m2l_scale64.p; }

// ------------------------------------------------------------------ engine, per kernel and precision
template <int KER, class R>
struct Engine {
  using W = typename Green<KER, R>::Q;  // working value: R or complex
  using CT = typename C2<R>::type;      // spectrum value

  static void upward(Fmm& f, Tree& t, Workspace& ws, cudaStream_t s) {
    const int n = f.nsurf;
    ws.launches = 0;
    XCUDA(cudaEventRecord(ws.ev[0], s));
    // P2M: check potentials of every leaf, then the pinv (UC2E) GEMM per leaf level
    if (t.nleafs) {
      SurfPotArgs a{t.leafs.p,  t.nleafs, t.nsrcs.p,     nullptr,  t.level.p, t.sbeg.p,   nullptr, t.center.p,
                    t.src4.p,   t.src_qim.p, f.surf_base.p, n,      2.95,      ws.chk.p, 0,         f.k_re, f.k_im};
      k_surf_pot<KER, R><<<nblk(t.nleafs, 4), 128, 0, s>>>(a);
      XLAUNCH();
      ws.launches++;
      W* up = (W*)ws.up.p;
      for (int l = 0; l <= t.depth; l++) {
        if (KER == K_LAPLACE && l > 0) break;
        const int r0 = ws.leaf_level_off[l], r1 = ws.leaf_level_off[l + 1];
        const int m = KER == K_LAPLACE ? ws.p2m1.M : r1 - r0;
        const int off = KER == K_LAPLACE ? 0 : r0;
        if (m <= 0) continue;
        const Ops<W> o = ops_of<W>(f, l);
        ws.launches++;
        gemm_rows<W>(m, n, n, (const W*)ws.chk.p, ws.p2m1.a.p + off, o.p2m1, (W*)ws.eq.p, ws.p2m1.c.p + off,
                     nullptr, 0, s);
        ws.launches++;
        gemm_rows<W>(m, n, n, (const W*)ws.eq.p, ws.p2m2.a.p + off, o.p2m2, up, ws.p2m2.c.p + off,
                     alpha_of<R>(ws.p2m2) + off, 0, s);
      }
    }
    XCUDA(cudaEventRecord(ws.ev[1], s));
    // M2M: deepest parents first (post-order)
    for (int l = t.depth - 1; l >= 0; l--) {
      const GemmRows& g = ws.m2m[l];
      ws.launches++;
        gemm_rows<W>(g.M, n, 8 * n, (const W*)ws.up.p, g.a.p, ops_of<W>(f, l).m2m, (W*)ws.up.p, g.c.p, nullptr, 0, s);
    }
    XCUDA(cudaEventRecord(ws.ev[2], s));
  }

  static void m2l(Fmm& f, Tree& t, Workspace& ws, cudaStream_t s) {
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
      XCUDA(cudaEventRecord(ev[0], s));
      // upward equivalent FFT (fmm_scale_invariant.h:560-604)
      k_m2l_grid_up<W><<<std::min<int64_t>(nblk((int64_t)ns * 8 * nconv), 148 * 32), 256, 0, s>>>(
          src, ns, t.child0.p, (const W*)ws.up.p, n, f.conv_to_surf_up.p, nconv, (W*)ws.grid.p);
      XLAUNCH();
      ws.launches++;
      exec_fwd(ws.fwd[g], ws.grid.p, ws.specA.p);
      ws.launches++;
      transpose<CT>((const CT*)ws.specA.p, (CT*)ws.specB.p, (int64_t)ns * 8, nfreq, s);  // -> [f][s][c]
      XCUDA(cudaEventRecord(ev[1], s));
      // Hadamard product
      constexpr int KC = sizeof(R) == 4 ? 4 : 2;
      const size_t smem = (size_t)26 * KC * 64 * sizeof(CT);
      if (ws.hadamard_smem < smem) {
        XCUDA(cudaFuncSetAttribute(k_hadamard<CT, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ws.hadamard_smem = smem;
      }
      k_hadamard<CT, KC><<<(nfreq + KC - 1) / KC, 256, smem, s>>>(T, (const CT*)ws.specB.p, (CT*)ws.specA.p,
                                                                    t.m2l_tab.p + (int64_t)t.m2l_trg_off[g] * 26, ns,
                                                                    nt, nfreq);
      XLAUNCH();
      ws.launches++;
      XCUDA(cudaEventRecord(ev[2], s));
      // inverse FFT to downward check potentials (fmm_scale_invariant.h:606-646)
      ws.launches++;
      transpose<CT>((const CT*)ws.specA.p, (CT*)ws.specB.p, nfreq, (int64_t)nt * 8, s);  // -> [t][c][f]
      exec_bwd(ws.bwd[g], ws.specB.p, ws.grid.p);
      k_m2l_gather_dn<W, R><<<std::min<int64_t>(nblk((int64_t)nt * 8 * n), 148 * 32), 256, 0, s>>>(
          trg, nt, t.child0.p, (const W*)ws.grid.p, nconv, f.map_dn.p, n,
          m2l_scale_of<R>(t) + t.m2l_trg_off[g], (W*)ws.dn.p);
      XLAUNCH();
      ws.launches++;
      XCUDA(cudaEventRecord(ev[3], s));
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

  static void downward(Fmm& f, Tree& t, Workspace& ws, cudaStream_t s) {
    const int n = f.nsurf;
    // P2L (X list) into downward check potentials
    if (t.n_p2l_nodes) {
      SurfPotArgs a{t.p2l_nodes.p, t.n_p2l_nodes, t.nsrcs.p,     t.p2l.p, t.level.p, t.sbeg.p, t.p2l_off.p, t.center.p,
                    t.src4.p,      t.src_qim.p,   f.surf_base.p, n,       1.05,      ws.dn.p,  1,           f.k_re,
                    f.k_im};
      k_surf_pot<KER, R><<<nblk(t.n_p2l_nodes, 4), 128, 0, s>>>(a);
      XLAUNCH();
      ws.launches++;
    }
    XCUDA(cudaEventRecord(ws.ev[3], s));
    // M2L
    if (t.n_m2l_trg) m2l(f, t, ws, s);
    XCUDA(cudaEventRecord(ws.ev[4], s));
    // L2L: shallowest parents first (pre-order)
    for (int l = 0; l < t.depth; l++) {
      const GemmRows& g = ws.l2l[l];
      ws.launches++;
        gemm_rows<W>(g.M, 8 * n, n, (const W*)ws.dn.p, g.a.p, ops_of<W>(f, l).l2l, (W*)ws.dn.p, g.c.p, nullptr, 1, s);
    }
    XCUDA(cudaEventRecord(ws.ev[5], s));
    // L2P part 1: downward check -> equivalent (DC2E) per leaf level
    if (t.nleafs) {
      for (int l = 0; l <= t.depth; l++) {
        if (KER == K_LAPLACE && l > 0) break;
        const int r0 = ws.leaf_level_off[l], r1 = ws.leaf_level_off[l + 1];
        const int m = KER == K_LAPLACE ? ws.l2p1.M : r1 - r0;
        const int off = KER == K_LAPLACE ? 0 : r0;
        if (m <= 0) continue;
        const Ops<W> o = ops_of<W>(f, l);
        ws.launches++;
        gemm_rows<W>(m, n, n, (const W*)ws.dn.p, ws.l2p1.a.p + off, o.l2p1, (W*)ws.chk.p, ws.l2p1.c.p + off,
                     nullptr, 0, s);
        ws.launches++;
        gemm_rows<W>(m, n, n, (const W*)ws.chk.p, ws.l2p2.a.p + off, o.l2p2, (W*)ws.eq.p, ws.l2p2.c.p + off,
                     alpha_of<R>(ws.l2p2) + off, 0, s);
      }
    }
    XCUDA(cudaEventRecord(ws.ev[6], s));
    // P2P + M2P + L2P target evaluation
    if (t.n_eval_leafs) {
      EvalArgs a{t.eval_leafs.p, t.leafs.p, t.nsrcs.p,   t.ntrgs.p, t.level.p,     t.n_eval_leafs, t.sbeg.p,
                 t.tbeg.p,       t.center.p, t.src4.p,   t.trg4.p,  t.src_qim.p,   t.p2p_off.p,    t.m2p_off.p,
                 t.p2p.p,        t.m2p.p,   f.surf_base.p, n,        ws.up.p,       ws.eq.p,        ws.out.p,
                 f.k_re,         f.k_im,    1,           1,         0,             1};
      k_eval<KER, R><<<nblk(t.n_eval_leafs, EVAL_WARPS), 32 * EVAL_WARPS, 0, s>>>(a);
      XLAUNCH();
      ws.launches++;
    }
    XCUDA(cudaEventRecord(ws.ev[7], s));
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
  XREQUIRE(f.pre_r0 == t.r0, XFMM_ERR_STATE, "operators were precomputed for another root radius");
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
    t.stage_q.upload(q, n * vs, s);  // grow-only staging buffer owned by the tree
    dq = t.stage_q.p;
  }
  k_set_charges<<<nblk(n), 256, 0, s>>>(dq, t.src_perm.p, n, f.is_complex(), t.src4.p, t.src_qim.p);
  XLAUNCH();
  if (!on_device) XCUDA(cudaStreamSynchronize(s));
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

// Device times of the last upward + downward pass (ms): 0 P2M, 1 M2M, 2 P2L, 3 M2L, 4 L2L,
// 5 L2P check->equivalent, 6 target evaluation (P2P + M2P + L2P), 7 total, 8-10 M2L FFT / Hadamard / iFFT.
void stage_times(Fmm& f, Tree& t, double* ms11) {
  Workspace* ws = t.ws[f.precision];
  XREQUIRE(ws, XFMM_ERR_STATE, "no evaluate has run");
  XCUDA(cudaEventSynchronize(ws->ev[7]));
  auto el = [](cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? (double)ms : 0.0;
  };
  const int pairs[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}, {0, 7}};
  for (int i = 0; i < 8; i++) ms11[i] = el(ws->ev[pairs[i][0]], ws->ev[pairs[i][1]]);
  ms11[8] = ms11[9] = ms11[10] = 0;
  const int ng = (int)ws->m2l_ev.size() / 4;
  for (int g = 0; g < ng; g++) {
    const int ns = t.m2l_src_off[g + 1] - t.m2l_src_off[g], nt = t.m2l_trg_off[g + 1] - t.m2l_trg_off[g];
    if (ns == 0 || nt == 0) continue;
    cudaEvent_t* e = ws->m2l_ev.data() + 4 * g;
    ms11[8] += el(e[0], e[1]);
    ms11[9] += el(e[1], e[2]);
    ms11[10] += el(e[2], e[3]);
  }
  for (int i = 0; i < 11; i++) f.stage_ms[i] = ms11[i];
  ms11[11] = (double)ws->launches;
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
