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
// Two kernels, both 64 x 64 output tiles per CTA of 4 warps (2 x 2 warps of 32 x 32), K in steps of 16
// staged through shared memory (k-major, padded rows), next step prefetched into registers:
//   k_tgemm_f64   FP64 on the FP64 tensor path (mma.sync m8n8k4 f64): pseudo-inverse factors (their
//                 1/s amplification needs FP64) and every translation of the FP64 path.
//   k_tgemm_tf32  FP32 accuracy from three TF32 tensor-core products of head/tail splits
//                 (Ah Bh + Ah Bt + At Bh, the tail-tail term 2^-22 relative dropped) for the mixed path's
//                 M2M, L2L and L2P's first factor.  B is split once per operator (hi/lo arrays).  Each
//                 16-wide K step is formed in a fresh MMA accumulator and added to FP32 running sums
//                 with round-to-nearest adds: the tensor core's own FP32 accumulation truncates, and over
//                 the 2368-term M2M rows it would cost accuracy.
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
__device__ __forceinline__ void mma_tf32_16x8x8(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// C[coff[r] + j] (=|+=) alpha[r] * sum_k A[aoff[r] + k] * (Bh + Bl)[k * ldb + j] with FP32 A.
// A row-major in shared memory ([BM][BK + 4]), Bh and Bl k-major ([BK][BN + 8]), cp.async ring of TGT_ST
// stages.  Warp (wm, wn) owns rows 32 wm .. +31 (2 m16 fragments) and columns 32 wn .. +31 (4 n8
// fragments); lane (g, t) holds A[g | g+8][t | t+4], B[t | t+4][g] and C[g | g+8][2t .. 2t + 1].
constexpr int TGT_BK = 16, TGT_ST = 3, TGT_LDA = TGT_BK + 4, TGT_LDB = TG_BN + 8;  // 43 KB: 4 CTAs per SM
constexpr size_t TGT_SMEM = (size_t)TGT_ST * ((size_t)TG_BM * TGT_LDA + 2 * (size_t)TGT_BK * TGT_LDB) * sizeof(float);

template <class TC, int VB>
__global__ void __launch_bounds__(TG_NT, 4) k_tgemm_tf32(int M, int N, int K, const float* __restrict__ A,
                                                       const int64_t* __restrict__ aoff, const float* __restrict__ Bh,
                                                       const float* __restrict__ Bl, int64_t ldb,
                                                       const double* __restrict__ alpha, TC* __restrict__ C,
                                                       const int64_t* __restrict__ coff, int acc) {
  extern __shared__ __align__(16) float tgt_sm[];
  float* As = tgt_sm;
  float* Hs = As + (size_t)TGT_ST * TG_BM * TGT_LDA;
  float* Ls = Hs + (size_t)TGT_ST * TGT_BK * TGT_LDB;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wm = w >> 1, wn = w & 1;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.x * TG_BM, n0 = blockIdx.y * TG_BN;
  const int nk = (K + TGT_BK - 1) / TGT_BK;
  auto load = [&](int slot, int kt) {
    const int k0 = kt * TGT_BK;
    tile_async<VB, 4>(
        reinterpret_cast<char*>(As + (size_t)slot * TG_BM * TGT_LDA), TG_BM, TGT_BK, TGT_LDA,
        [&](int i) -> const char* {
          const int r = m0 + i;
          return r < M ? reinterpret_cast<const char*>(A + aoff[r]) : nullptr;
        },
        k0, K, A);
    auto brow = [&](const float* Bx) {
      return [=](int i) -> const char* {
        const int k = k0 + i;
        return k < K ? reinterpret_cast<const char*>(Bx + (int64_t)k * ldb) : nullptr;
      };
    };
    tile_async<VB, 4>(reinterpret_cast<char*>(Hs + (size_t)slot * TGT_BK * TGT_LDB), TGT_BK, TG_BN, TGT_LDB, brow(Bh),
                      n0, N, Bh);
    tile_async<VB, 4>(reinterpret_cast<char*>(Ls + (size_t)slot * TGT_BK * TGT_LDB), TGT_BK, TG_BN, TGT_LDB, brow(Bl),
                      n0, N, Bl);
  };
  float run[2][4][4];  // round-to-nearest running sums
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) run[i][j][e] = 0.f;
#pragma unroll
  for (int st = 0; st < TGT_ST - 1; st++) {
    if (st < nk) load(st, st);
    cp_commit();
  }
  for (int kt = 0; kt < nk; kt++) {
    cp_wait<TGT_ST - 2>();
    __syncthreads();
    const int nx = kt + TGT_ST - 1;
    if (nx < nk) load(nx % TGT_ST, nx);
    cp_commit();
    const float* a_s = As + (size_t)(kt % TGT_ST) * TG_BM * TGT_LDA;
    const float* h_s = Hs + (size_t)(kt % TGT_ST) * TGT_BK * TGT_LDB;
    const float* l_s = Ls + (size_t)(kt % TGT_ST) * TGT_BK * TGT_LDB;
    // the stage's 16-wide K step in a fresh accumulator; the three products of each step go out
    // fragment by fragment (8 independent accumulators between dependent MMAs)
    float d[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int e = 0; e < 4; e++) d[i][j][e] = 0.f;
#pragma unroll
    for (int ks = 0; ks < TGT_BK; ks += 8) {
      uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const float* ar = a_s + (32 * wm + 16 * i + g) * TGT_LDA + ks + t;
        split_tf32(ar[0], ah[i][0], al[i][0]);
        split_tf32(ar[8 * TGT_LDA], ah[i][1], al[i][1]);
        split_tf32(ar[4], ah[i][2], al[i][2]);
        split_tf32(ar[8 * TGT_LDA + 4], ah[i][3], al[i][3]);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int o = (ks + t) * TGT_LDB + 32 * wn + 8 * j + g;
        bh[j][0] = __float_as_uint(h_s[o]);
        bh[j][1] = __float_as_uint(h_s[o + 4 * TGT_LDB]);
        bl[j][0] = __float_as_uint(l_s[o]);
        bl[j][1] = __float_as_uint(l_s[o + 4 * TGT_LDB]);
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_tf32_16x8x8(d[i][j], al[i], bh[j][0], bh[j][1]);
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_tf32_16x8x8(d[i][j], ah[i], bl[j][0], bl[j][1]);
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_tf32_16x8x8(d[i][j], ah[i], bh[j][0], bh[j][1]);
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int e = 0; e < 4; e++) run[i][j][e] = __fadd_rn(run[i][j][e], d[i][j][e]);
  }
  cp_wait<0>();
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int hr = 0; hr < 2; hr++) {
      const int r = m0 + 32 * wm + 16 * i + g + 8 * hr;
      if (r >= M) continue;
      const double al = alpha ? alpha[r] : 1.0;
      TC* crow = C + coff[r];
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int col = n0 + 32 * wn + 8 * j + 2 * t + h;
          if (col < N) store_out(crow + col, al * (double)run[i][j][2 * hr + h], acc);
        }
    }
}

// ---------------------------------------------------------------- FP32 accuracy on tcgen05 (TF32 x 3)
// The same C = alpha A B as k_tgemm_tf32 on the sm_100 tensor cores: a CTA owns 128 rows (one per TMEM
// lane) and 64 columns.  Per 16-wide K step the 4 warps load the rows' A pieces (coalesced, 16 bytes per
// lane), split them into TF32 head and tail and store both into shared memory as K-major core matrices
// (8 rows x 16 bytes, 128 contiguous bytes each); the operator's head and tail, pre-split and stored
// transposed ([N][K], zero-padded to whole tiles), arrive by cp.async in the same layout.  One elected
// lane of warp 0 issues the step's six MMAs (M128 N64 K8, Ah Bt + At Bh + Ah Bh per half step, the first
// into a fresh accumulator) into one of two TMEM accumulators and commits them to that accumulator's
// mbarrier.  While they run, every warp reads the previous step's accumulator back (its 32 lanes x 64
// columns) and adds it to FP32 running sums with round-to-nearest adds, then stages the next step.
// Waits are bounded (about a second); one that runs out sets the status flag and ends the loop.
constexpr int TC_BM = 128, TC_BN = 64, TC_BK = 16, TC_NT = 128;
constexpr uint32_t TC_CORE = 128;                                         // bytes per core matrix
constexpr uint32_t TC_A_BYTES = TC_BM * TC_BK * 4, TC_B_BYTES = TC_BN * TC_BK * 4;
constexpr uint32_t TC_STAGE = 2 * TC_A_BYTES + 2 * TC_B_BYTES;            // A head, A tail, B head, B tail
constexpr size_t TC_SMEM = 2 * (size_t)TC_STAGE + 1024;                  // two stages (+ alignment slack)
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

template <class TC, int VA>
__global__ void __launch_bounds__(TC_NT, 4)
    k_tgemm_tc(int M, int N, int K, const float* __restrict__ A, const int64_t* __restrict__ aoff,
               const float* __restrict__ Bth, const float* __restrict__ Btl, int64_t ldbt,
               const double* __restrict__ alpha, TC* __restrict__ C, const int64_t* __restrict__ coff, int acc,
               int* __restrict__ status) {
  using namespace tc5;
  extern __shared__ __align__(16) unsigned char tc_raw[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  // stage buffers on a 1 KB boundary
  unsigned char* sm = tc_raw + ((1024 - (smem_u32(tc_raw) & 1023)) & 1023);
  const uint32_t sm_u = smem_u32(sm);
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * TC_BN;
  const int nc = (K + TC_BK - 1) / TC_BK;
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
  // A rows of this thread's pieces: piece q = tid + 128 i -> row q / 4, core column q % 4
  int64_t arow[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = m0 + ((tid + TC_NT * i) >> 2);
    arow[i] = r < M ? aoff[r] : -1;
  }
  const int kq = (tid & 3) * 4;  // first K element of this thread's pieces
  auto stage = [&](int c) {
    unsigned char* st = sm + (size_t)(c & 1) * TC_STAGE;
    const int k0 = c * TC_BK;
    // operator head / tail rows n0 .. n0 + 63 (transposed, padded: always in bounds)
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int q = tid + TC_NT * i, row = q >> 2, kk = (q & 3) * 4;
      const int64_t o = (int64_t)(n0 + row) * ldbt + k0 + kk;
      const uint32_t d = tc_off(row, kk);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(st + 2 * TC_A_BYTES + d)), "l"(Bth + o)
                   : "memory");
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(st + 2 * TC_A_BYTES + TC_B_BYTES + d)),
                   "l"(Btl + o)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    // A pieces, split into TF32 head and tail
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int row = (tid + TC_NT * i) >> 2;
      float v[4] = {0.f, 0.f, 0.f, 0.f};
      if (arow[i] >= 0) {
        const float* src = A + arow[i] + k0 + kq;
        if (k0 + kq + 3 < K) {
          if constexpr (VA == 16) {
            const float4 x = *reinterpret_cast<const float4*>(src);
            v[0] = x.x, v[1] = x.y, v[2] = x.z, v[3] = x.w;
          } else {
            const float2 x = *reinterpret_cast<const float2*>(src), y = *reinterpret_cast<const float2*>(src + 2);
            v[0] = x.x, v[1] = x.y, v[2] = y.x, v[3] = y.y;
          }
        } else {
#pragma unroll
          for (int e = 0; e < 4; e++)
            if (k0 + kq + e < K) v[e] = src[e];
        }
      }
      uint32_t h[4], l[4];
#pragma unroll
      for (int e = 0; e < 4; e++) split_tf32(v[e], h[e], l[e]);
      const uint32_t d = tc_off(row, kq);
      *reinterpret_cast<uint4*>(st + d) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(st + TC_A_BYTES + d) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  };
  auto publish = [&]() {  // this thread's staged data visible to the tensor core, then a CTA barrier
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    fence_proxy_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
  };
  float run[TC_BN];
#pragma unroll
  for (int j = 0; j < TC_BN; j++) run[j] = 0.f;
  auto readout = [&](int buf) {
    const uint32_t base = tm + ((uint32_t)(32 * w) << 16) + (uint32_t)(64 * buf);
#pragma unroll
    for (int j = 0; j < TC_BN; j += 16) {
      uint32_t v[16];
      ld_32x32b_x16(base + j, v);
      wait_ld();
#pragma unroll
      for (int e = 0; e < 16; e++) run[j + e] = __fadd_rn(run[j + e], __uint_as_float(v[e]));
    }
  };
  constexpr uint32_t IDESC = idesc_tf32(TC_BM, TC_BN);
  bool ok = true;
  if (nc > 0) stage(0);
  publish();
  for (int c = 0; c < nc && ok; c++) {
    const int s = c & 1;
    if (w == 0) {
      if (elect_one()) {
        const uint32_t st = sm_u + (uint32_t)s * TC_STAGE;
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {  // half steps K 8 ks .. 8 ks + 7: core columns 2 ks, 2 ks + 1
          const uint32_t o = 2 * ks * TC_CORE;
          const uint64_t ah = sdesc_nosw(st + o, TC_CORE, 4 * TC_CORE), al = sdesc_nosw(st + TC_A_BYTES + o, TC_CORE, 4 * TC_CORE);
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
    if (c >= 1) {
      // the previous step's MMAs (accumulator and stage s ^ 1) are complete: read it back, then restage
      ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&mbar[s ^ 1]), ((c - 1) >> 1) & 1, TC_WAIT));
      if (ok) {
        fence_after_sync();
        readout(s ^ 1);
      } else if (lane == 0) {
        abort_flag = 1;
      }
    }
    if (ok && c + 1 < nc) stage(c + 1);
    publish();
    ok = abort_flag == 0;
  }
  if (ok && nc > 0) {
    const int c = nc - 1;
    if (__all_sync(0xffffffffu, mbar_wait(smem_u32(&mbar[c & 1]), (c >> 1) & 1, TC_WAIT))) {
      fence_after_sync();
      readout(c & 1);
    } else if (lane == 0) {
      abort_flag = 1;
    }
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  ok = abort_flag == 0;
  if (!ok) {
    if (tid == 0) atomicExch(status, 1);
  } else {
    const int r = m0 + 32 * w + lane;
    if (r < M) {
      const double al = alpha ? alpha[r] : 1.0;
      TC* crow = C + coff[r] + n0;
#pragma unroll
      for (int j = 0; j < TC_BN; j++)
        if (n0 + j < N) store_out(crow + j, al * (double)run[j], acc);
    }
  }
  if (w == 0) tmem_dealloc(tm, 128);
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
void tgemm_tf32(const TGemm& g, const float* A, const float* Bh, const float* Bl, TC* C, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0) return;
  const dim3 grid((g.M + TG_BM - 1) / TG_BM, (g.N + TG_BN - 1) / TG_BN);
  // A rows (offsets multiples of astep floats) and B rows (ldb floats) 16-byte aligned when those are
  // multiples of 4, else 8-byte copies (both at least 8-byte aligned)
  XREQUIRE(g.ldb % 2 == 0 && g.astep % 2 == 0, XFMM_ERR_UNSUPPORTED, "translation rows must be 8-byte aligned");
  const bool v16 = g.astep % 4 == 0 && g.ldb % 4 == 0;
  auto go = [&](auto kern) {
    XCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TGT_SMEM));
    kern<<<grid, TG_NT, TGT_SMEM, s>>>(g.M, g.N, g.K, A, g.aoff, Bh, Bl, g.ldb, g.alpha, C, g.coff, g.accumulate);
  };
  if (v16) go(k_tgemm_tf32<TC, 16>);
  else go(k_tgemm_tf32<TC, 8>);
  XLAUNCH();
}

template <class TC>
void tgemm_tc(const TGemm& g, const float* A, const float* Bth, const float* Btl, int64_t ldbt, TC* C,
              cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0) return;
  XREQUIRE(g.status && g.astep % 2 == 0 && ldbt % TC_BK == 0, XFMM_ERR_UNSUPPORTED,
           "tensor-core translation: status flag and aligned rows required");
  const dim3 grid((g.M + TC_BM - 1) / TC_BM, (g.N + TC_BN - 1) / TC_BN);
  auto go = [&](auto kern) {
    XCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
    kern<<<grid, TC_NT, TC_SMEM, s>>>(g.M, g.N, g.K, A, g.aoff, Bth, Btl, ldbt, g.alpha, C, g.coff, g.accumulate,
                                      g.status);
  };
  if (g.astep % 4 == 0) go(k_tgemm_tc<TC, 16>);
  else go(k_tgemm_tc<TC, 8>);
  XLAUNCH();
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
template void tgemm_tf32<float>(const TGemm&, const float*, const float*, const float*, float*, cudaStream_t);
template void tgemm_tf32<double>(const TGemm&, const float*, const float*, const float*, double*, cudaStream_t);

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
