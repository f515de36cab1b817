// translate.cu -- the check-to-equivalent and parent/child translations (P2M and L2P pseudo-inverse
// factors, M2M, L2L) as level-batched GEMMs on the tensor cores, with the row gather, the per-row scale
// and the scatter (or scatter-add) fused into the GEMM.
//
// Every translation of one level is C_r (=|+=) alpha_r * A_r * B over the rows r of that level:
//   P2M  (fmm_scale_invariant.h:163-195)  A_r = check potentials of leaf r, B = UC2E_U^T, then UC2E_V^T,
//                                          alpha_r = 0.5^level on the second factor, C_r = up[leaf]
//   M2M  (fmm_scale_invariant.h:233-253)  A_r = the 8 children's up rows of parent r (contiguous),
//                                          B = [8n][n] stack of M2M[c]^T, C_r = up[parent]
//   L2L  (fmm_scale_invariant.h:256-275)  A_r = dn[parent], B = [n][8n] of L2L[c]^T, C_r += dn[children]
//   L2P  (fmm_scale_invariant.h:198-230)  A_r = 0.5^level dn[leaf], B = DC2E_U^T, then DC2E_V^T
// A complex translation is a real one of twice the size: interleaved complex rows are real rows, and
// the operator is expanded to [2K][2N] with the 2x2 blocks (re, im; -im, re) (expand_operator).
//
// Two kernels:
//   k_tgemm_f64   FP64 on the FP64 tensor path (mma.sync m8n8k4 f64), 64 x 64 output tiles per CTA of 4
//                 warps, K in steps of 16 staged through shared memory: pseudo-inverse factors (their
//                 1/s amplification needs FP64) and every translation of the FP64 path.
//   k_tgemm_tc    FP32 accuracy from three TF32 tensor-core products of head/tail splits
//                 (Ah Bh + Ah Bt + At Bh, the tail-tail term 2^-22 relative dropped) on tcgen05 with
//                 TMEM accumulators, for the mixed path's M2M, L2L and L2P's first factor.  B is split
//                 once per operator (hi/lo arrays).  Each 16-wide K step is formed in a fresh MMA
//                 accumulator and added to FP32 running sums with round-to-nearest adds: the tensor
//                 core's own FP32 accumulation truncates, and over the 2368-term M2M rows it would cost
//                 accuracy.
#include <cuda_runtime.h>

#include <cstdint>

#include "tcgen05.cuh"
#include "xfmm_internal.h"

namespace xfmm {
namespace {

constexpr int TG_BM = 64, TG_BN = 64, TG_NT = 128;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// asynchronous global -> shared copy of VB bytes (16 or 8), of which `valid` are read, the rest zeroed
template <int VB>
__device__ __forceinline__ void cp_async_zfill(uint32_t dst, const void* src, uint32_t valid) {
  if constexpr (VB == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(valid) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Copies a tile of `rows` x `cols` elements (ES bytes each) into shared memory rows of `lds` elements:
// tile row i is global row `row_ptr(i)` (null: zeros) from element `c0`, elements up to `ncols` of the
// row read, the rest zeroed.  Every thread of the CTA takes its share of VB-byte chunks.
template <int VB, int ES, class RowPtr>
__device__ __forceinline__ void tile_async(char* smem, int rows, int cols, int lds, RowPtr row_ptr, int c0, int ncols,
                                           const void* any) {
  constexpr int EPC = VB / ES;  // elements per chunk
  const int cpr = cols / EPC, total = rows * cpr;
  for (int q = threadIdx.x; q < total; q += TG_NT) {
    const int i = q / cpr, cc = (q % cpr) * EPC;
    const char* src = row_ptr(i);
    const int left = ncols - (c0 + cc);
    const uint32_t valid = (src && left > 0) ? (uint32_t)(left >= EPC ? VB : left * ES) : 0u;
    // a chunk that reads nothing still names a global address of the matrix (its first element)
    const char* s = valid ? src + (int64_t)(c0 + cc) * ES : static_cast<const char*>(any);
    cp_async_zfill<VB>(saddr(smem + ((int64_t)i * lds + cc) * ES), s, valid);
  }
}

__device__ __forceinline__ void store_out(float* p, double v, int acc) { *p = acc ? *p + (float)v : (float)v; }
__device__ __forceinline__ void store_out(double* p, double v, int acc) { *p = acc ? *p + v : v; }

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// ---------------------------------------------------------------- FP64 (DMMA)
// C[coff[r] + j] (=|+=) alpha[r] * sum_k A[aoff[r] + k] * B[k * ldb + j], r < M, j < N, k < K.
// A row-major in shared memory ([BM][BK + 4], as TA), B k-major ([BK][BN + 4]), both filled by cp.async
// in a ring of TGD_ST stages.  Warp (wm, wn) owns rows 32 wm .. +31 and columns 32 wn .. +31 as 4 x 4
// m8n8 fragments; lane (g = lane / 4, t = lane % 4) holds A[g][t], B[t][g] and C[g][2t .. 2t + 1].
constexpr int TGD_BK = 16, TGD_ST = 4, TGD_LDA = TGD_BK + 4, TGD_LDB = TG_BN + 4;
template <class TA>
constexpr size_t tgd_smem() {
  return (size_t)TGD_ST * ((size_t)TG_BM * TGD_LDA * sizeof(TA) + (size_t)TGD_BK * TGD_LDB * sizeof(double));
}

template <class TA, class TC, int VA>
__global__ void __launch_bounds__(TG_NT) k_tgemm_f64(int M, int N, int K, const TA* __restrict__ A,
                                                      const int64_t* __restrict__ aoff, const double* __restrict__ B,
                                                      int64_t ldb, const double* __restrict__ alpha, TC* __restrict__ C,
                                                      const int64_t* __restrict__ coff, int acc) {
  extern __shared__ __align__(16) char tgd_sm[];
  TA* As = reinterpret_cast<TA*>(tgd_sm);
  double* Bs = reinterpret_cast<double*>(tgd_sm + (size_t)TGD_ST * TG_BM * TGD_LDA * sizeof(TA));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wm = w >> 1, wn = w & 1;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.x * TG_BM, n0 = blockIdx.y * TG_BN;
  const int nk = (K + TGD_BK - 1) / TGD_BK;
  auto load = [&](int slot, int kt) {
    const int k0 = kt * TGD_BK;
    tile_async<VA, sizeof(TA)>(
        reinterpret_cast<char*>(As + (size_t)slot * TG_BM * TGD_LDA), TG_BM, TGD_BK, TGD_LDA,
        [&](int i) -> const char* {
          const int r = m0 + i;
          return r < M ? reinterpret_cast<const char*>(A + aoff[r]) : nullptr;
        },
        k0, K, A);
    tile_async<16, 8>(
        reinterpret_cast<char*>(Bs + (size_t)slot * TGD_BK * TGD_LDB), TGD_BK, TG_BN, TGD_LDB,
        [&](int i) -> const char* {
          const int k = k0 + i;
          return k < K ? reinterpret_cast<const char*>(B + (int64_t)k * ldb) : nullptr;
        },
        n0, N, B);
  };
  double c[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) c[i][j][0] = c[i][j][1] = 0.0;
#pragma unroll
  for (int st = 0; st < TGD_ST - 1; st++) {
    if (st < nk) load(st, st);
    cp_commit();
  }
  for (int kt = 0; kt < nk; kt++) {
    cp_wait<TGD_ST - 2>();
    __syncthreads();
    const int nx = kt + TGD_ST - 1;
    if (nx < nk) load(nx % TGD_ST, nx);
    cp_commit();
    const TA* a_s = As + (size_t)(kt % TGD_ST) * TG_BM * TGD_LDA;
    const double* b_s = Bs + (size_t)(kt % TGD_ST) * TGD_BK * TGD_LDB;
#pragma unroll
    for (int ks = 0; ks < TGD_BK; ks += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = (double)a_s[(32 * wm + 8 * i + g) * TGD_LDA + ks + t];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = b_s[(ks + t) * TGD_LDB + 32 * wn + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dmma(c[i][j], a[i], b[j]);
    }
  }
  cp_wait<0>();
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = m0 + 32 * wm + 8 * i + g;
    if (r >= M) continue;
    const double al = alpha ? alpha[r] : 1.0;
    TC* crow = C + coff[r];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int col = n0 + 32 * wn + 8 * j + 2 * t + h;
        if (col < N) store_out(crow + col, al * c[i][j][h], acc);
      }
  }
}

// ---------------------------------------------------------------- FP32 accuracy from TF32 (x3)
__device__ __forceinline__ uint32_t tf32_round(float x) {
  // nearest TF32 value (10-bit mantissa) by integer rounding of the 13 dropped bits
  uint32_t u = __float_as_uint(x);
  u += 0x1000u;
  return u & 0xFFFFE000u;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t& h, uint32_t& l) {
  h = tf32_round(x);
  l = tf32_round(x - __uint_as_float(h));
}
// ---------------------------------------------------------------- FP32 accuracy on tcgen05 (TF32 x 3)
// C = alpha A B on the sm_100 tensor cores (tcgen05).  A CTA owns 128 rows (one per TMEM
// lane), 64 columns and a range of 16-wide K steps (K split over blockIdx.z when a level has few rows;
// the parts are then added into C with atomics, C already holding the rows' starting values).
// Per step: the rows' A pieces arrive raw by cp.async two steps ahead (16 bytes per lane, coalesced), in
// place into the stage's A-tail tile or into a raw buffer, and are split into TF32 head and tail one step
// ahead as K-major core matrices (8 rows x 16 bytes, 128 contiguous bytes each); the operator's head and
// tail (pre-split, transposed to [N][K], zero-padded to whole tiles) arrive by cp.async in the same
// layout, two steps ahead.  The proxy
// fence that hands a split step to the tensor core is issued before the next step's copies, so that it
// has none of this thread's copies in flight to wait for (measured: 5% faster M2M and L2L).  One
// elected lane of warp 0 issues the step's six MMAs (M128 N64 K8; Ah Bt + At Bh + Ah Bh per half step,
// the first into a fresh accumulator) into one of two TMEM accumulators and commits them to that
// accumulator's mbarrier.  While they run, every warp reads the previous step's accumulator back (its 32
// lanes x 64 columns) and adds it to FP32 running sums with round-to-nearest adds.  Waits are bounded
// (about a second); one that runs out sets the status flag and ends the loop.
constexpr int TC_BM = 128, TC_BN = 64, TC_BK = 16, TC_NT = 128, TC_D = 2, TC_ST = TC_D + 1;
#ifndef XFMM_TC_KSPLIT_MAX
#define XFMM_TC_KSPLIT_MAX 64  // largest K split of a tensor-core translation GEMM
#endif
#ifndef XFMM_TC_KSPLIT_CTAS
#define XFMM_TC_KSPLIT_CTAS (2 * 2 * 148)  // CTAs a split aims at (two per SM, two waves)
#endif
constexpr uint32_t TC_CORE = 128;                                         // bytes per core matrix
constexpr uint32_t TC_A_BYTES = TC_BM * TC_BK * 4, TC_B_BYTES = TC_BN * TC_BK * 4;
constexpr uint32_t TC_STAGE = 2 * TC_A_BYTES + 2 * TC_B_BYTES;            // A head, A tail, B head, B tail
// shared memory: the stages (+ alignment), and for the raw-buffer form two raw A buffers
constexpr size_t TC_SMEM_IP = TC_ST * (size_t)TC_STAGE + 1024;                    // in place: 3 CTAs per SM
constexpr size_t TC_SMEM_RAW = TC_SMEM_IP + 2 * (size_t)TC_A_BYTES;             // raw buffers: 2 CTAs per SM
template <bool IP> constexpr size_t tc_smem() { return IP ? TC_SMEM_IP : TC_SMEM_RAW; }
constexpr long long TC_WAIT = 2000000000LL;

// byte offset of element (row, k) (k < 16) in a K-major tile of 16-wide rows: core (row / 8, k / 4)
__device__ __forceinline__ uint32_t tc_off(int row, int k) {
  return (uint32_t)(((row >> 3) * 4 + (k >> 2)) * TC_CORE + (row & 7) * 16 + (k & 3) * 4);
}
__device__ __forceinline__ void tc_mma_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// register <- TMEM, shape 32x32b repeated 64 times: lane i of the warp gets 64 consecutive 32-bit columns
// of TMEM lane (lane field of taddr) + i
__device__ __forceinline__ void ld_32x32b_x64(uint32_t taddr, uint32_t (&v)[64]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
               : "r"(taddr)
               : "memory");
}
// cp.async.wait_group with a run-time count (0..3 groups left in flight)
__device__ __forceinline__ void cp_wait_dyn(int n) {
  if (n <= 0) asm volatile("cp.async.wait_group 0;" ::: "memory");
  else if (n == 1) asm volatile("cp.async.wait_group 1;" ::: "memory");
  else if (n == 2) asm volatile("cp.async.wait_group 2;" ::: "memory");
  else asm volatile("cp.async.wait_group 3;" ::: "memory");
}
// Waits (spinning) for the phase of the given parity; false after `limit` SM clock cycles
__device__ __forceinline__ bool mbar_spin(uint32_t mbar, uint32_t parity, long long limit) {
  if (tc5::mbar_try_wait(mbar, parity)) return true;
  const long long t0 = clock64();
  while (!tc5::mbar_try_wait(mbar, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}

template <class TC, int VA, bool IP>
__global__ void __launch_bounds__(TC_NT, IP ? 3 : 2)
    k_tgemm_tc(int M, int N, int K, const float* __restrict__ A, const int64_t* __restrict__ aoff,
               const float* __restrict__ Bth, const float* __restrict__ Btl, int64_t ldbt,
               const double* __restrict__ alpha, TC* __restrict__ C, const int64_t* __restrict__ coff, int acc,
               int* __restrict__ status, double* __restrict__ scratch) {
  using namespace tc5;
  extern __shared__ __align__(16) unsigned char tc_raw[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  unsigned char* sm = tc_raw + ((1024 - (smem_u32(tc_raw) & 1023)) & 1023);  // stages on a 1 KB boundary
  const uint32_t sm_u = smem_u32(sm);
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * TC_BN;
  // this CTA's K steps
  const int nsteps = (K + TC_BK - 1) / TC_BK, per = (nsteps + gridDim.z - 1) / gridDim.z;
  const int c0 = blockIdx.z * per, nc = max(0, min(nsteps, c0 + per) - c0);
  if (w == 0) {
    tmem_alloc(smem_u32(&tmem_base), 128);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    fence_mbar_init();
    abort_flag = 0;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tm = tmem_base;
  // this thread's A pieces: piece q = tid + 128 i -> row (q % 8) + 8 (q / 32), K elements 4 kc .. 4 kc + 3
  // of the step, kc = (q / 8) % 4.  A warp reads 8 rows x 64 bytes (coalesced) and every 8-lane phase of
  // a 16-byte shared-memory access covers one 128-byte core matrix (no bank conflicts).
  auto prow = [](int q) { return (q & 7) + 8 * (q >> 5); };
  int64_t arow[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = m0 + prow(tid + TC_NT * i);
    arow[i] = r < M ? aoff[r] : -1;
  }
  const int kq = ((tid >> 3) & 3) * 4;
  // raw A pieces (zero-filled outside the rows and K) and the operator rows of step c (absolute index),
  // one cp.async group.  In place (IP), a raw piece lands where its TF32 tail will be (the stage's
  // A-tail tile, same core-matrix offset) and the thread that splits it writes the tail over it;
  // otherwise it lands in the raw buffer of its step's parity.
  unsigned char* rawA = sm + TC_ST * (size_t)TC_STAGE;
  auto raw_piece = [&](unsigned char* st, int c, int q) -> unsigned char* {
    if constexpr (IP) return st + TC_A_BYTES + tc_off(prow(q), kq);
    else return rawA + (size_t)(c & 1) * TC_A_BYTES + (size_t)q * 16;
  };
  auto fetch = [&](int c) {
    unsigned char* st = sm + (size_t)(c % TC_ST) * TC_STAGE;
    const int k0 = c * TC_BK;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int q = tid + TC_NT * i, row = prow(q), kk = ((q >> 3) & 3) * 4;
      const int64_t o = (int64_t)(n0 + row) * ldbt + k0 + kk;  // padded operator: always in bounds
      const uint32_t d = tc_off(row, kk);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(st + 2 * TC_A_BYTES + d)), "l"(Bth + o)
                   : "memory");
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(st + 2 * TC_A_BYTES + TC_B_BYTES + d)),
                   "l"(Btl + o)
                   : "memory");
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int k = k0 + kq;
      const int left = K - k;
      const uint32_t dst = smem_u32(raw_piece(st, c, tid + TC_NT * i));
      const bool any = arow[i] >= 0 && left > 0;
      const float* src = any ? A + arow[i] + k : A;  // a chunk that reads nothing still names A
      if constexpr (VA == 16) {
        const uint32_t valid = any ? (uint32_t)(left >= 4 ? 16 : 4 * left) : 0u;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid) : "memory");
      } else {
        const uint32_t v0 = any ? (uint32_t)(left >= 2 ? 8 : 4 * left) : 0u;
        const uint32_t v1 = (any && left > 2) ? (uint32_t)(left >= 4 ? 8 : 4 * (left - 2)) : 0u;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(v0) : "memory");
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst + 8), "l"(v1 ? src + 2 : A), "r"(v1)
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // this thread's raw pieces of step c (its own copies) split into the head and tail tiles of its stage
  auto split = [&](int c) {
    unsigned char* st = sm + (size_t)(c % TC_ST) * TC_STAGE;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int q = tid + TC_NT * i;
      const float4 v = *reinterpret_cast<const float4*>(raw_piece(st, c, q));
      uint32_t h[4], l[4];
      split_tf32(v.x, h[0], l[0]);
      split_tf32(v.y, h[1], l[1]);
      split_tf32(v.z, h[2], l[2]);
      split_tf32(v.w, h[3], l[3]);
      const uint32_t d = tc_off(prow(q), kq);
      *reinterpret_cast<uint4*>(st + d) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(st + TC_A_BYTES + d) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  };
  auto barrier = [&]() {  // shared-memory writes visible to the tensor core, then a CTA barrier
    fence_proxy_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
  };
  float run[TC_BN];
#pragma unroll
  for (int j = 0; j < TC_BN; j++) run[j] = 0.f;
  auto readout = [&](int buf) {  // the warp's 32 lanes x 64 columns in one load, one wait
    uint32_t v[TC_BN];
    ld_32x32b_x64(tm + ((uint32_t)(32 * w) << 16) + (uint32_t)(64 * buf), v);
    wait_ld();
#pragma unroll
    for (int j = 0; j < TC_BN; j++) run[j] = __fadd_rn(run[j], __uint_as_float(v[j]));
  };
  constexpr uint32_t IDESC = idesc_tf32(TC_BM, TC_BN);
  // prologue: steps 0 .. TC_D - 1 fetched, step 0 split
  for (int j = 0; j < TC_D; j++)
    if (j < nc) fetch(c0 + j);
  if (nc > 0) {
    cp_wait_dyn(min(TC_D, nc) - 1);
    split(c0);
  }
  barrier();
  bool ok = true;
  for (int i = 0; i < nc && ok; i++) {
    const int c = c0 + i, s = i & 1;
    if (w == 0) {
      if (elect_one()) {
        const uint32_t st = sm_u + (uint32_t)(c % TC_ST) * TC_STAGE;
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {  // half steps K 8 ks .. 8 ks + 7: core columns 2 ks, 2 ks + 1
          const uint32_t o = 2 * ks * TC_CORE;
          const uint64_t ah = sdesc_nosw(st + o, TC_CORE, 4 * TC_CORE),
                         al = sdesc_nosw(st + TC_A_BYTES + o, TC_CORE, 4 * TC_CORE);
          const uint64_t bh = sdesc_nosw(st + 2 * TC_A_BYTES + o, TC_CORE, 4 * TC_CORE),
                         bl = sdesc_nosw(st + 2 * TC_A_BYTES + TC_B_BYTES + o, TC_CORE, 4 * TC_CORE);
          const uint32_t d = tm + 64 * s;
          tc_mma_ss(d, al, bh, IDESC, ks);  // fresh accumulator at the first MMA of the step
          tc_mma_ss(d, ah, bl, IDESC, 1);
          tc_mma_ss(d, ah, bh, IDESC, 1);
        }
        commit(smem_u32(&mbar[s]));
      }
      __syncwarp();
    }
    if (i >= 1) {
      // the previous step's MMAs are complete: its accumulator is read back, its stage is free
      if (__all_sync(0xffffffffu, mbar_spin(smem_u32(&mbar[s ^ 1]), ((i - 1) >> 1) & 1, TC_WAIT))) {
        fence_after_sync();
        readout(s ^ 1);
      } else {
        ok = false;
        if (lane == 0) abort_flag = 1;
      }
    }
    // step c + 1 is split and made visible to the tensor core (proxy fence) before step c + TC_D's copies
    // are issued (copies of steps c + 1 .. c + TC_D - 1 are in flight; step c + 1's must have landed)
    if (ok && i + 1 < nc) {
      cp_wait_dyn(min(TC_D - 2, nc - 2 - i));
      split(c + 1);
    }
    fence_proxy_async_smem();
    if (ok && i + TC_D < nc) fetch(c + TC_D);  // into the stage of step c - 1
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    ok = abort_flag == 0;
  }
  if (ok && nc > 0) {
    const int i = nc - 1;
    if (__all_sync(0xffffffffu, mbar_spin(smem_u32(&mbar[i & 1]), (i >> 1) & 1, TC_WAIT))) {
      fence_after_sync();
      readout(i & 1);
    } else if (lane == 0) {
      abort_flag = 1;
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  ok = abort_flag == 0;
  if (!ok) {
    if (tid == 0) atomicExch(status, 1);
  } else if (nc > 0) {
    const int r = m0 + 32 * w + lane;
    if (r < M) {
      const double al = alpha ? alpha[r] : 1.0;
      TC* crow = C + coff[r] + n0;
      if (gridDim.z > 1) {
        // a part of a split K: added in FP64 into the scratch row r (k_tc_finish moves it into C)
        double* srow = scratch + (int64_t)r * N + n0;
#pragma unroll
        for (int j = 0; j < TC_BN; j++)
          if (n0 + j < N) atomicAdd(srow + j, al * (double)run[j]);
      } else {
#pragma unroll
        for (int j = 0; j < TC_BN; j++)
          if (n0 + j < N) store_out(crow + j, al * (double)run[j], acc);
      }
    }
  }
  if (w == 0) tmem_dealloc(tm, 128);
}

// C[coff[r] + j] (=|+=) scratch[r][j] for the rows of a split-K tensor-core GEMM, scratch cleared for its
// next use
template <class TC>
__global__ void k_tc_finish(int M, int N, double* __restrict__ scratch, TC* __restrict__ C,
                            const int64_t* __restrict__ coff, int acc) {
  const int64_t total = (int64_t)M * N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / N), j = (int)(e % N);
    store_out(C + coff[r] + j, scratch[e], acc);
    scratch[e] = 0.0;
  }
}

// out[j][k] = E[k][j] for the real form E ([KR][NR]) of B, TF32 head and tail, zero outside E, for
// j < npad, k < ldbt: the transposed operator of k_tgemm_tc
template <class TS>
__global__ void k_expand_operator_t(const TS* __restrict__ B, int K, int N, int64_t ldb, int cplx, int npad,
                                    int64_t ldbt, float* __restrict__ ohi, float* __restrict__ olo) {
  const int KR = cplx ? 2 * K : K, NR = cplx ? 2 * N : N;
  const int64_t total = (int64_t)npad * ldbt;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / ldbt), k = (int)(e % ldbt);
    double v = 0.0;
    if (j < NR && k < KR) {
      if (!cplx) {
        v = (double)B[(int64_t)k * ldb + j];
      } else {
        const int kk = k >> 1, jj = j >> 1;
        const double re = (double)B[2 * ((int64_t)kk * ldb + jj)], im = (double)B[2 * ((int64_t)kk * ldb + jj) + 1];
        v = (k & 1) == 0 ? ((j & 1) == 0 ? re : im) : ((j & 1) == 0 ? -im : re);
      }
    }
    const float f = (float)v;
    const float h = __uint_as_float(tf32_round(f));
    ohi[e] = h;
    olo[e] = __uint_as_float(tf32_round(f - h));
  }
}

// ---------------------------------------------------------------- operator preparation
// out[k][j] of the real form of B ([K][N] real, or [K][N] complex expanded to [2K][2N] with the blocks
// (re, im; -im, re), so that an interleaved complex row times it is the complex product), as FP64 and/or
// as a TF32 head + tail split of its FP32 value.
template <class TS>
__global__ void k_expand_operator(const TS* __restrict__ B, int K, int N, int64_t ldb, int cplx,
                                  double* __restrict__ o64, float* __restrict__ ohi, float* __restrict__ olo) {
  const int KR = cplx ? 2 * K : K, NR = cplx ? 2 * N : N;
  const int64_t total = (int64_t)KR * NR;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / NR), j = (int)(e % NR);
    double v;
    if (!cplx) {
      v = (double)B[(int64_t)k * ldb + j];
    } else {
      const int kk = k >> 1, jj = j >> 1;
      const double re = (double)B[2 * ((int64_t)kk * ldb + jj)], im = (double)B[2 * ((int64_t)kk * ldb + jj) + 1];
      // rows 2kk (real part of a_k) and 2kk + 1 (imaginary part) against columns 2jj (real) and 2jj + 1
      v = (k & 1) == 0 ? ((j & 1) == 0 ? re : im) : ((j & 1) == 0 ? -im : re);
    }
    if (o64) o64[e] = v;
    if (ohi) {
      const float f = (float)v;
      const float h = __uint_as_float(tf32_round(f));
      ohi[e] = h;
      olo[e] = __uint_as_float(tf32_round(f - h));
    }
  }
}

inline int tg_blocks(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

}  // namespace

void expand_operator(const void* B, bool b_single, int K, int N, int64_t ldb, bool cplx, double* o64, float* ohi,
                     float* olo, cudaStream_t s) {
  const int64_t total = (int64_t)(cplx ? 2 * K : K) * (cplx ? 2 * N : N);
  if (b_single)
    k_expand_operator<float><<<tg_blocks(total), 256, 0, s>>>((const float*)B, K, N, ldb, cplx, o64, ohi, olo);
  else
    k_expand_operator<double><<<tg_blocks(total), 256, 0, s>>>((const double*)B, K, N, ldb, cplx, o64, ohi, olo);
  XLAUNCH();
}

template <class TA, class TC>
void tgemm_f64(const TGemm& g, const TA* A, const double* B, TC* C, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0) return;
  // B rows (ldb doubles) and A rows must start 8-byte aligned; 16-byte copies where they start 16-byte
  // aligned (A offsets multiples of astep elements)
  XREQUIRE(g.ldb % 2 == 0 && g.astep % 2 == 0, XFMM_ERR_UNSUPPORTED, "translation rows must be 16-byte aligned");
  const dim3 grid((g.M + TG_BM - 1) / TG_BM, (g.N + TG_BN - 1) / TG_BN);
  constexpr size_t smem = tgd_smem<TA>();
  const bool a16 = (g.astep * (int64_t)sizeof(TA)) % 16 == 0;
  auto go = [&](auto kern) {
    XCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, TG_NT, smem, s>>>(g.M, g.N, g.K, A, g.aoff, B, g.ldb, g.alpha, C, g.coff, g.accumulate);
  };
  if (a16) go(k_tgemm_f64<TA, TC, 16>);
  else go(k_tgemm_f64<TA, TC, 8>);
  XLAUNCH();
}
template <class TC>
void tgemm_tc(const TGemm& g, const float* A, const float* Bth, const float* Btl, int64_t ldbt, TC* C,
              cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0) return;
  XREQUIRE(g.status && g.astep % 2 == 0 && ldbt % TC_BK == 0, XFMM_ERR_UNSUPPORTED,
           "tensor-core translation: status flag and aligned rows required");
  // K split over blockIdx.z for levels with few row tiles (two CTAs per SM, about two waves), in parts
  // of at least 8 steps; only where C is accumulated into (the parts are added with atomics)
  const int mt = (g.M + TC_BM - 1) / TC_BM, nt = (g.N + TC_BN - 1) / TC_BN, nsteps = (g.K + TC_BK - 1) / TC_BK;
  int kz = 1;
  if (g.accumulate) {
    const int want = (XFMM_TC_KSPLIT_CTAS + mt * nt - 1) / (mt * nt);
    kz = std::max(1, std::min(std::min(want, nsteps / 8), XFMM_TC_KSPLIT_MAX));
  }
  if (kz > 1) {
    // the parts meet in an FP64 scratch ([M][N], zero between uses), then one pass adds it into C
    XREQUIRE(g.scratch && g.scratch_len >= (int64_t)g.M * g.N, XFMM_ERR_UNSUPPORTED,
             "split tensor-core translation: scratch too small");
  }
  const dim3 grid(mt, nt, kz);
  // In place, three CTAs share an SM; measured faster except for short K (fewer than 32 steps) with many
  // column tiles (the Laplace L2L: 0.86 ms with the raw buffers, 1.06 ms in place), which keeps the raw
  // buffers and two CTAs per SM.
  const bool ip = !(nsteps < 32 && nt >= 16);
  auto go = [&](auto kern, size_t smem) {
    XCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, TC_NT, smem, s>>>(g.M, g.N, g.K, A, g.aoff, Bth, Btl, ldbt, g.alpha, C, g.coff, g.accumulate,
                                   g.status, g.scratch);
  };
  if (g.astep % 4 == 0) ip ? go(k_tgemm_tc<TC, 16, true>, TC_SMEM_IP) : go(k_tgemm_tc<TC, 16, false>, TC_SMEM_RAW);
  else ip ? go(k_tgemm_tc<TC, 8, true>, TC_SMEM_IP) : go(k_tgemm_tc<TC, 8, false>, TC_SMEM_RAW);
  XLAUNCH();
  if (kz > 1) {
    k_tc_finish<TC><<<tg_blocks((int64_t)g.M * g.N), 256, 0, s>>>(g.M, g.N, g.scratch, C, g.coff, g.accumulate);
    XLAUNCH();
  }
}
// the FP64 scratch (doubles) a split tgemm_tc of M x N needs, 0 when it does not split
int64_t tgemm_tc_scratch(int M, int N, int K, int accumulate) {
  const int mt = (M + TC_BM - 1) / TC_BM, nt = (N + TC_BN - 1) / TC_BN, nsteps = (K + TC_BK - 1) / TC_BK;
  if (!accumulate || M <= 0 || N <= 0) return 0;
  const int want = (XFMM_TC_KSPLIT_CTAS + mt * nt - 1) / (mt * nt);
  const int kz = std::max(1, std::min(std::min(want, nsteps / 8), XFMM_TC_KSPLIT_MAX));
  return kz > 1 ? (int64_t)M * N : 0;
}
template void tgemm_tc<float>(const TGemm&, const float*, const float*, const float*, int64_t, float*, cudaStream_t);
template void tgemm_tc<double>(const TGemm&, const float*, const float*, const float*, int64_t, double*, cudaStream_t);

void expand_operator_t(const void* B, bool b_single, int K, int N, int64_t ldb, bool cplx, int npad, int64_t ldbt,
                       float* ohi, float* olo, cudaStream_t s) {
  const int64_t total = (int64_t)npad * ldbt;
  if (b_single)
    k_expand_operator_t<float><<<tg_blocks(total), 256, 0, s>>>((const float*)B, K, N, ldb, cplx, npad, ldbt, ohi, olo);
  else
    k_expand_operator_t<double><<<tg_blocks(total), 256, 0, s>>>((const double*)B, K, N, ldb, cplx, npad, ldbt, ohi,
                                                                 olo);
  XLAUNCH();
}

template void tgemm_f64<float, float>(const TGemm&, const float*, const double*, float*, cudaStream_t);
template void tgemm_f64<float, double>(const TGemm&, const float*, const double*, double*, cudaStream_t);
template void tgemm_f64<double, float>(const TGemm&, const double*, const double*, float*, cudaStream_t);
template void tgemm_f64<double, double>(const TGemm&, const double*, const double*, double*, cudaStream_t);

}  // namespace xfmm

namespace xfmm {

// The GEMM forms of one level's translation operators (kept beside the precompute's own copies).
void prepare_translation_operands(const Fmm& f, LevelOps& op, cudaStream_t s) {
  const int n = f.nsurf, cw = f.is_complex() ? 2 : 1;
  const bool cplx = f.is_complex();
  const size_t nn = (size_t)cw * n * cw * n;
  op.tg_p2m1.alloc(nn);
  op.tg_p2m2.alloc(nn);
  op.tg_l2p1.alloc(nn);
  op.tg_l2p2.alloc(nn);
  expand_operator(op.p2m_B1.p, false, n, n, n, cplx, op.tg_p2m1.p, nullptr, nullptr, s);
  expand_operator(op.p2m_B2.p, false, n, n, n, cplx, op.tg_p2m2.p, nullptr, nullptr, s);
  expand_operator(op.l2p_B1.p, false, n, n, n, cplx, op.tg_l2p1.p, nullptr, nullptr, s);
  expand_operator(op.l2p_B2.p, false, n, n, n, cplx, op.tg_l2p2.p, nullptr, nullptr, s);
  if (f.mixed()) {
    // transposed ([N][K]), rows padded to whole 64-column tiles and to a multiple of 16 K elements, TF32
    // head and tail: the operands of the tensor-core GEMM (tgemm_tc)
    auto tr = [&](const void* B, int K, int N, int64_t ldb, bool c, DBuf<float>& hi, DBuf<float>& lo, int64_t& ldbt) {
      const int KR = c ? 2 * K : K, NR = c ? 2 * N : N;
      const int npad = (NR + 63) / 64 * 64;
      ldbt = (KR + 15) / 16 * 16;
      hi.alloc((size_t)npad * ldbt);
      lo.alloc((size_t)npad * ldbt);
      expand_operator_t(B, true, K, N, ldb, c, npad, ldbt, hi.p, lo.p, s);
    };
    tr(op.m2m_B.p, 8 * n, n, n, cplx, op.tg_m2m_h, op.tg_m2m_l, op.ld_m2m);
    tr(op.l2l_B.p, n, 8 * n, 8 * n, cplx, op.tg_l2l_h, op.tg_l2l_l, op.ld_l2l);
    if (!cplx) tr(op.l2p_B1f.p, n, n, n, false, op.tg_l2p1_h, op.tg_l2p1_l, op.ld_l2p1);
  } else {
    op.tg_m2m.alloc(8 * nn);
    op.tg_l2l.alloc(8 * nn);
    expand_operator(op.m2m_B.p, false, 8 * n, n, n, cplx, op.tg_m2m.p, nullptr, nullptr, s);
    expand_operator(op.l2l_B.p, false, n, 8 * n, 8 * n, cplx, op.tg_l2l.p, nullptr, nullptr, s);
  }
}

}  // namespace xfmm
