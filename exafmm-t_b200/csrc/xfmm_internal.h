// xfmm_internal.h -- shared internals of libexafmm_b200.so (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "xfmm.h"

namespace xfmm {

struct Error : std::exception {
  int code;
  std::string msg;
  Error(int c, std::string m) : code(c), msg(std::move(m)) {}
  const char* what() const noexcept override { return msg.c_str(); }
};

#define XFMM_STR2(x) #x
#define XFMM_STR(x) XFMM_STR2(x)
#define XCUDA(call)                                                                                         \
  do {                                                                                                      \
    cudaError_t e_ = (call);                                                                                \
    if (e_ != cudaSuccess)                                                                                  \
      throw ::xfmm::Error(e_ == cudaErrorMemoryAllocation ? XFMM_ERR_OOM : XFMM_ERR_CUDA,                   \
                          std::string(__FILE__ ":" XFMM_STR(__LINE__) " ") + #call + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define XREQUIRE(cond, code, msg)                     \
  do {                                                \
    if (!(cond)) throw ::xfmm::Error((code), (msg));  \
  } while (0)
#define XLAUNCH() XCUDA(cudaGetLastError())

// Owning device buffer (move-only).
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) XCUDA(cudaMalloc(&p, count * sizeof(T)));
  }
  // grow-only reallocation (contents not preserved)
  void reserve(size_t count) {
    if (count > n) alloc(count);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
  void upload(const T* h, size_t count, cudaStream_t s) {
    reserve(count);
    if (count) XCUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
  std::vector<T> download(cudaStream_t s, size_t count = (size_t)-1) const {
    if (count == (size_t)-1) count = n;
    std::vector<T> h(count);
    if (count) {
      XCUDA(cudaMemcpyAsync(h.data(), p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
      XCUDA(cudaStreamSynchronize(s));
    }
    return h;
  }
};

constexpr int LMAX = 21;  // path keys hold 21 octant digits (63 bits): deepest supported level

inline int nsurf_of(int p) { return 6 * (p - 1) * (p - 1) + 2; }

struct Workspace;  // evaluate buffers, one per precision (evaluate.cu)
struct Tree;
void release_workspace(Tree& t);

// Tree + interaction lists on the device, node arrays in the reference's idx order.
struct Tree {
  Workspace* ws[2] = {nullptr, nullptr};  // evaluate workspace per precision
  Tree() = default;
  Tree(const Tree&) = delete;
  Tree& operator=(const Tree&) = delete;
  ~Tree() { release_workspace(*this); }
  int64_t nsrc = 0, ntrg = 0;
  int nnodes = 0, nleafs = 0, nnonleafs = 0, depth = 0, nonadaptive = 0, ncrit = 0, nsurf_lists = 0;
  double x0[3] = {0, 0, 0}, r0 = 0;
  // bodies in tree order: (x, y, z, Re q) and Im q for complex charges
  DBuf<double4> src4, trg4;
  DBuf<double> src_qim;
  DBuf<int> src_perm, trg_perm;
  // nodes
  DBuf<int> level, is_leaf, nsrcs, ntrgs, parent, octant, child0;
  DBuf<int64_t> sbeg, tbeg;
  DBuf<double4> center;  // x, y, z, r
  DBuf<uint64_t> key;    // the reference's Morton key with level offset (hilbert.h:79-107)
  DBuf<int> leafs, nonleafs;
  std::vector<int> h_level, h_is_leaf, h_child0, h_leafs, h_nonleafs, h_ntrgs, h_nsrcs;
  // lists
  bool lists_built = false;
  DBuf<int> colleagues, m2l;
  DBuf<int64_t> p2p_off, m2p_off, p2l_off;
  DBuf<int> p2p, m2p, p2l;
  int64_t np2p = 0, nm2p = 0, np2l = 0;
  // derived schedules
  DBuf<int> nl_by_level;              // nonleafs grouped by level (ascending), pre-order within a level
  std::vector<int> nl_level_off;      // depth+2 offsets into nl_by_level
  DBuf<int> eval_leafs;               // leaf positions (index into leafs) with ntrgs > 0
  int n_eval_leafs = 0;
  DBuf<int> p2l_nodes;                // nodes with a non-empty P2L list
  int n_p2l_nodes = 0;
  DBuf<float> leaf_scale;             // 0.5^level per leaf position (Laplace P2M/L2P scaling)
  DBuf<double> leaf_scale64;
  int64_t p2p_pairs = 0, m2p_pairs = 0, l2p_pairs = 0, m2l_pairs = 0;
  // M2L setup (fmm_scale_invariant.h:277-341 / fmm.h:265-333)
  bool m2l_ready = false;
  int m2l_grouped_by_level = 0;
  DBuf<int> m2l_src;                  // compact source list (node idx), grouped by level if per-level
  std::vector<int> m2l_src_off;       // group offsets
  DBuf<int> m2l_trg;                  // targets (nonleaf node idx), same grouping
  std::vector<int> h_m2l_trg;         // host copy
  std::vector<int> m2l_trg_off;
  DBuf<int> m2l_tab;                  // [n_trg][26] compact source index within its group, -1 if none
  std::vector<int> h_m2l_tab;
  DBuf<float> m2l_scale;              // per target 2^(level+1) (Laplace) else 1
  DBuf<double> m2l_scale64;
  int n_m2l_src = 0, n_m2l_trg = 0;
  // persistent staging for host-side charges and results (no allocation per call)
  DBuf<double> stage_q, stage_out;
  DBuf<int> stage_flag;               // non-finite charges found by the device-side check
  int hadr_tpc = 0;                   // sparse M2L Hadamard: tiles per CTA (0: the built-in default)
};

// Precomputed operators of one level (or the single scale-invariant level).
struct LevelOps {
  // working precision copies (float for mixed, double for fp64); complex types stored as interleaved pairs
  // K(check, equiv) = U S V^H; the pseudo-inverse is applied in FP64 (both precisions), in two factors as the
  // reference does (UC2E_U then UC2E_V, DC2E_U then DC2E_V), never as one product: P = V S+ U^H
  // has entries up to ~1/s_min and a single dot product with it cancels catastrophically.
  DBuf<char> p2m_B1;   // [n][n]      y = U^H c        : B1[k][j] = conj(U[k][j])
  DBuf<char> p2m_B2;   // [n][n]      e = V S+ y       : B2[k][j] = conj(VH[k][j]) / s_k
  DBuf<char> l2p_B1;   // [n][n]      y = conj(VH) c   : B1[k][j] = conj(VH[j][k])
  DBuf<char> l2p_B2;   // [n][n]      e = conj(U) S+ y : B2[k][j] = conj(U[j][k]) / s_k
  DBuf<char> l2p_B1f;  // FP32 copy of l2p_B1 (mixed path, real kernels: the L2P first factor runs in FP32)
  DBuf<char> m2m_B;    // [8n][n]     B[c*n+k][j] = M2M[c][j][k], M2M[c] = (V S+)(U^H K_c)
  DBuf<char> l2l_B;    // [n][8n]     B[k][c*n+j] = M2M[c][k][j] (L2L = M2M^T)
  DBuf<char> m2l_T;    // [26][nfreq][64] complex: entry [s*8+t] (fmm_scale_invariant.h:549-551)
  int rank = 0;        // singular values kept by the pinv threshold: B1 columns / B2 rows beyond are zero
  // the same operators in the form the translation GEMMs (translate.cu) read: real [K][N] row-major, a
  // complex operator expanded to [2K][2N] (expand_operator); FP64 for the pinv factors and the FP64
  // path, TF32 head / tail arrays for the mixed path's M2M, L2L and (real kernels) L2P first factor
  DBuf<double> tg_p2m1, tg_p2m2, tg_l2p1, tg_l2p2, tg_m2m, tg_l2l;
  DBuf<float> tg_m2m_h, tg_m2m_l, tg_l2l_h, tg_l2l_l, tg_l2p1_h, tg_l2p1_l;  // mixed: transposed [N][ld]
  int64_t ld_m2m = 0, ld_l2l = 0, ld_l2p1 = 0;
};

struct Fmm {
  int kernel = 0, p = 0, ncrit = 0, precision = 0;
  double k_re = 0, k_im = 0;
  int nsurf = 0, nconv = 0, nfreq = 0, n1 = 0;
  int depth = 0;
  double x0[3] = {0, 0, 0}, r0 = 0;
  std::string filename;               // operator file in the reference's .dat layout ("" : none)
  bool precomputed = false;
  double pre_r0 = -1;
  int pre_depth = -1;
  std::vector<LevelOps> ops;          // 1 (Laplace) or depth+1 (per-level kernels)
  DBuf<double> surf_base;             // [nsurf][3] unit surface (geometry.h:21-54 before scaling)
  DBuf<int> map_up, map_dn;           // surface index -> conv-grid index (geometry.h:101-134)
  DBuf<int> conv_to_surf_up;          // conv-grid index -> surface index or -1
  DBuf<double> dft_tw;                // [n1] (cos, sin)(2 pi m / n1): factors of the M2L transforms
  std::vector<double> h_surf_base;
  double stage_ms[11] = {0};
  bool is_complex() const { return kernel == XFMM_HELMHOLTZ; }
  bool mixed() const { return precision == XFMM_MIXED; }
};

// tree.cu
void build_tree(Fmm& fmm, Tree& t, const double* src_xyz, const double* trg_xyz, int nonadaptive_depth,
                cudaStream_t s);
void build_lists(Fmm& fmm, Tree& t, cudaStream_t s);
void m2l_setup(Fmm& fmm, Tree& t, cudaStream_t s);
// precompute.cu
void precompute(Fmm& fmm, int depth, cudaStream_t s);
void host_surface_base(int p, std::vector<double>& out);
// evaluate.cu
void set_charges(Fmm& fmm, Tree& t, const double* q, bool on_device, cudaStream_t s);
void clear_values(Fmm& fmm, Tree& t, cudaStream_t s);
void upward_pass(Fmm& fmm, Tree& t, cudaStream_t s);
void downward_pass(Fmm& fmm, Tree& t, cudaStream_t s);
void get_values(Fmm& fmm, Tree& t, double* out_dev, cudaStream_t s);
void stage_times(Fmm& fmm, Tree& t, double* ms14);
void check_device_status(Fmm& f, Tree& t);
void selftest_bounded_wait(int64_t limit_cycles);
void gradient_p2p_raw(int kernel, double k_re, double k_im, int precision, const double* src, int64_t ns,
                      const double* q, const double* trg, int64_t nt, double* out, cudaStream_t s);
void verify(Fmm& fmm, Tree& t, int sample, double* err2, cudaStream_t s);
void gradient_p2p_scratch(int kernel, double k_re, double k_im, int precision, const double* src, int64_t ns,
                          const double* q, const double* trg, int64_t nt, double* out, double4* s4, double* qim,
                          double4* t4, cudaStream_t s);
// translate.cu: level-batched translation GEMMs with fused row gather / scale / scatter.
// C[coff[r] + j] (=|+=) alpha[r] * sum_k A[aoff[r] + k] * B[k * ldb + j] for r < M, j < N, k < K, on
// real views of the rows (complex rows as interleaved reals, operators expanded).
struct TGemm {
  int M = 0, N = 0, K = 0;
  const int64_t* aoff = nullptr;
  const int64_t* coff = nullptr;
  const double* alpha = nullptr;  // null: 1
  int64_t ldb = 0;
  int accumulate = 0;
  int64_t astep = 0;  // every A offset is a multiple of astep elements (alignment of the A rows)
  int* status = nullptr;  // device flag set by a tensor-core GEMM whose bounded wait ran out
  double* scratch = nullptr;  // FP64 [M][N] for a split tensor-core GEMM, zero between uses
  int64_t scratch_len = 0;
};
template <class TA, class TC>
void tgemm_f64(const TGemm& g, const TA* A, const double* B, TC* C, cudaStream_t s);
template <class TC>
void tgemm_tc(const TGemm& g, const float* A, const float* Bth, const float* Btl, int64_t ldbt, TC* C,
              cudaStream_t s);
int64_t tgemm_tc_scratch(int M, int N, int K, int accumulate);
void expand_operator_t(const void* B, bool b_single, int K, int N, int64_t ldb, bool cplx, int npad, int64_t ldbt,
                       float* ohi, float* olo, cudaStream_t s);
void expand_operator(const void* B, bool b_single, int K, int N, int64_t ldb, bool cplx, double* o64, float* ohi,
                     float* olo, cudaStream_t s);
void prepare_translation_operands(const Fmm& f, LevelOps& op, cudaStream_t s);
// evaluate.cu: many systems in one evaluate (xfmm_batch_*)
struct Batch;
Batch* batch_create(Fmm** fmms, Tree** trees, int n, cudaStream_t s);
void batch_free(Batch* b);
void batch_schedule(const int64_t* sizes, int n, int nstreams, int* stream_of);
void batch_set_tuning(Batch* b, int option, int value);
void batch_evaluate(Batch* b, const double* const* charges, double* const* outs, int nstreams, cudaStream_t s);
// capi.cpp: record the message returned by xfmm_last_error() on this thread
void set_last_error(const char* msg);

}  // namespace xfmm
