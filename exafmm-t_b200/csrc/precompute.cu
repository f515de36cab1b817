// precompute.cu -- FP64 precomputation of the translation operators (Fmm::precompute).
//
//   check-to-equivalent pinv  fmm_scale_invariant.h:446-514, fmm.h:451-521 (LAPACK gesvd there,
//                             cuSOLVER gesvd here); P = pinv(K(check 2.95, equiv 1.05)) with the
//                             reference's truncation s_i > 4*eps*s_max (eps = 1e-16 for FP64,
//                             1e-10 for the mixed path so FP32 equivalent densities stay exact
//                             enough); applied in the reference's two factors (see LevelOps)
//   M2M / L2L                 fmm_scale_invariant.h:51-77, fmm.h:47-74: M2M[c] = (V S+)(U^H K(parent check,
//                             child equiv)); L2L[c] == M2M[c]^T (pinv(K^T) = pinv(K)^T)
//   M2L kernel FFT tables     fmm_scale_invariant.h:517-558, fmm.h:524-629: 316 convolution grids ->
//                             3-D FFT (cuFFT, FP64) -> 26 tables [nfreq][8 src x 8 trg] / nconv
// Laplace is scale invariant: one set of level-0 operators.  The other kernels get
// operators for every level 0..depth and M2L tables for child levels 1..depth.
#include <cublas_v2.h>
#include <cufft.h>
#include <cusolverDn.h>

#include <array>
#include <cmath>
#include <cstdio>
#include <map>
#include <tuple>

#include "xfmm_internal.h"

namespace xfmm {

#define XCUBLAS(call)                                                                               \
  do {                                                                                              \
    cublasStatus_t st_ = (call);                                                                    \
    if (st_ != CUBLAS_STATUS_SUCCESS)                                                               \
      throw Error(XFMM_ERR_CUDA, std::string("cuBLAS ") + #call + " failed: " + std::to_string((int)st_)); \
  } while (0)
#define XCUSOLVER(call)                                                                                 \
  do {                                                                                                  \
    cusolverStatus_t st_ = (call);                                                                      \
    if (st_ != CUSOLVER_STATUS_SUCCESS)                                                                 \
      throw Error(XFMM_ERR_CUDA, std::string("cuSOLVER ") + #call + " failed: " + std::to_string((int)st_)); \
  } while (0)
#define XCUFFT(call)                                                                                 \
  do {                                                                                               \
    cufftResult st_ = (call);                                                                        \
    if (st_ != CUFFT_SUCCESS)                                                                        \
      throw Error(XFMM_ERR_CUDA, std::string("cuFFT ") + #call + " failed: " + std::to_string((int)st_)); \
  } while (0)

// geometry.h:21-54: unit surface points before the alpha*r scaling
void host_surface_base(int p, std::vector<double>& c) {
  const int n = nsurf_of(p);
  c.assign(3 * n, 0.0);
  c[0] = c[1] = c[2] = -1.0;
  int cnt = 1;
  for (int i = 0; i < p - 1; i++)
    for (int j = 0; j < p - 1; j++, cnt++) {
      c[3 * cnt] = -1.0;
      c[3 * cnt + 1] = (2.0 * (i + 1) - p + 1) / (p - 1);
      c[3 * cnt + 2] = (2.0 * j - p + 1) / (p - 1);
    }
  for (int i = 0; i < p - 1; i++)
    for (int j = 0; j < p - 1; j++, cnt++) {
      c[3 * cnt] = (2.0 * i - p + 1) / (p - 1);
      c[3 * cnt + 1] = -1.0;
      c[3 * cnt + 2] = (2.0 * (j + 1) - p + 1) / (p - 1);
    }
  for (int i = 0; i < p - 1; i++)
    for (int j = 0; j < p - 1; j++, cnt++) {
      c[3 * cnt] = (2.0 * (i + 1) - p + 1) / (p - 1);
      c[3 * cnt + 1] = (2.0 * j - p + 1) / (p - 1);
      c[3 * cnt + 2] = -1.0;
    }
  for (int i = 0; i < (n / 2) * 3; i++) c[3 * cnt + i] = -c[i];
}

namespace {

// geometry.h:55-62
std::vector<double> host_surface(int p, double r0, int level, const double* ctr, double alpha) {
  std::vector<double> c;
  host_surface_base(p, c);
  const double r = r0 * std::pow(0.5, level);
  const double b = alpha * r;
  for (size_t i = 0; i < c.size() / 3; i++)
    for (int d = 0; d < 3; d++) c[3 * i + d] = c[3 * i + d] * b + ctr[d];
  return c;
}

// geometry.h:101-134 (rounded; identical to the reference's truncation for p <= 20)
std::vector<int> host_surf2conv(int p, bool up) {
  const int n1 = 2 * p;
  const double ctr[3] = {0.5 * (p - 1), 0.5 * (p - 1), 0.5 * (p - 1)};
  std::vector<double> s = host_surface(p, 0.5, 0, ctr, double(p - 1));
  const double off = up ? (p - 1) : (2 * p - 1);
  std::vector<int> m(s.size() / 3);
  for (size_t i = 0; i < m.size(); i++) {
    const int a = (int)std::lround(off - s[3 * i]), b = (int)std::lround(off - s[3 * i + 1]),
              c = (int)std::lround(off - s[3 * i + 2]);
    m[i] = a + b * n1 + c * n1 * n1;
  }
  return m;
}

// geometry.h:156-195
std::vector<std::array<int, 3>> rel_coords(int max_r, int min_r, int step) {
  std::vector<std::array<int, 3>> out;
  for (int k = -max_r; k <= max_r; k += step)
    for (int j = -max_r; j <= max_r; j += step)
      for (int i = -max_r; i <= max_r; i += step)
        if (std::abs(i) >= min_r || std::abs(j) >= min_r || std::abs(k) >= min_r) out.push_back({i, j, k});
  return out;
}
std::vector<int> m2l_index_map() {
  auto m2l = rel_coords(1, 1, 1), helper = rel_coords(3, 2, 1);
  std::map<std::tuple<int, int, int>, int> lut;
  for (size_t i = 0; i < helper.size(); i++) lut[{helper[i][0], helper[i][1], helper[i][2]}] = (int)i;
  std::vector<int> m(26 * 64, -1);
  for (int i = 0; i < 26; i++)
    for (int j1 = 0; j1 < 8; j1++)
      for (int j2 = 0; j2 < 8; j2++) {
        const int a = m2l[i][0] * 2 - (j1 & 1) + (j2 & 1), b = m2l[i][1] * 2 - ((j1 >> 1) & 1) + ((j2 >> 1) & 1),
                  c = m2l[i][2] * 2 - ((j1 >> 2) & 1) + ((j2 >> 2) & 1);
        auto it = lut.find({a, b, c});
        m[i * 64 + j2 * 8 + j1] = it == lut.end() ? -1 : it->second;
      }
  return m;
}

constexpr double FOURPI = 4.0 * 3.14159265358979323846;

// potential of a unit charge (the kernels' scalar formulas, laplace.h:269-274 etc.), complex form
__device__ __forceinline__ double2 green64(int kernel, double k_re, double k_im, double r2) {
  if (r2 == 0) return make_double2(0, 0);
  const double r = sqrt(r2);
  if (kernel == XFMM_LAPLACE) return make_double2(1.0 / r / FOURPI, 0);
  if (kernel == XFMM_MODIFIED_HELMHOLTZ) return make_double2(exp(-k_re * r) / r / FOURPI, 0);
  const double e = exp(-k_im * r) / r / FOURPI;
  double sn, cs;
  sincos(k_re * r, &sn, &cs);
  return make_double2(e * cs, e * sn);
}

// M[i*nt + j] = G(trg_j - src_i)   (fmm_base.h:65-76), real or interleaved complex output
__global__ void k_kernel_matrix(int kernel, double k_re, double k_im, const double* src, int ns, const double* trg,
                                int nt, double* out, int cplx) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)ns * nt) return;
  const int i = (int)(e / nt), j = (int)(e % nt);
  const double dx = trg[3 * j] - src[3 * i], dy = trg[3 * j + 1] - src[3 * i + 1], dz = trg[3 * j + 2] - src[3 * i + 2];
  const double2 g = green64(kernel, k_re, k_im, dx * dx + dy * dy + dz * dz);
  if (cplx) {
    out[2 * e] = g.x;
    out[2 * e + 1] = g.y;
  } else {
    out[e] = g.x;
  }
}

// conv grids of all 316 helper offsets: value at g = potential at origin of a unit charge at grid point g
__global__ void k_conv_values(int kernel, double k_re, double k_im, int p, double a, const double* offs, int nh,
                              double* out, int cplx) {
  const int n1 = 2 * p, nconv = n1 * n1 * n1;
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)nh * nconv) return;
  const int h = (int)(e / nconv), g = (int)(e % nconv);
  const int i = g % n1, j = (g / n1) % n1, k = g / (n1 * n1);
  // geometry.h:85-87
  const double x = (i - p) * a / (p - 1) + offs[3 * h], y = (j - p) * a / (p - 1) + offs[3 * h + 1],
               z = (k - p) * a / (p - 1) + offs[3 * h + 2];
  const double2 gv = green64(kernel, k_re, k_im, x * x + y * y + z * z);
  if (cplx) {
    out[2 * e] = gv.x;
    out[2 * e + 1] = gv.y;
  } else {
    out[e] = gv.x;
  }
}

__global__ void k_sinv(const double* s, int n, double thr, double* sinv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sinv[i] = s[i] > thr ? 1.0 / s[i] : 0.0;
}

// The reference's four check-to-equivalent factors, row-major n x n (fmm_scale_invariant.h:474-479 real,
// 505-512 complex) from cuSOLVER's column-major SVD of A = M^T, M = U_M S VH_M the row-major kernel
// matrix: M = conj(V_c) S U_c^T, so read as row-major arrays the memory of cuSOLVER's U is U_c^T = VH_M and
// the memory of its VT (= V_c^H, column-major) is conj(V_c) = U_M.  UC2E_U = U^H,
// UC2E_V = V S+, DC2E_U = conj(VH), DC2E_V = conj(U) S+ (real kernels: no conjugates).
__global__ void k_ref_factors(const double* Uc, const double* Vc, const double* sinv, int n, int cplx, double* uc2e_u,
                              double* uc2e_v, double* dc2e_u, double* dc2e_v) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n) return;
  const int k = (int)(e / n), j = (int)(e % n);
  const int64_t kj = (int64_t)k * n + j, jk = (int64_t)j * n + k;
  // U_M[k][j] = Vc[k][j], VH_M[k][j] = Uc[k][j]
  if (cplx) {
    const double2* U2 = (const double2*)Uc;
    const double2* V2 = (const double2*)Vc;
    const double2 vjk = V2[jk], ukj = U2[kj], vkj = V2[kj], ujk = U2[jk];
    ((double2*)uc2e_u)[kj] = make_double2(vjk.x, -vjk.y);                    // conj(U_M[j][k])
    ((double2*)uc2e_v)[kj] = make_double2(ujk.x * sinv[j], -ujk.y * sinv[j]);  // conj(VH_M[j][k]) / s_j
    ((double2*)dc2e_u)[kj] = make_double2(ukj.x, -ukj.y);                    // conj(VH_M[k][j])
    ((double2*)dc2e_v)[kj] = make_double2(vkj.x * sinv[j], -vkj.y * sinv[j]);  // conj(U_M[k][j]) / s_j
  } else {
    uc2e_u[kj] = Vc[jk];
    uc2e_v[kj] = Uc[jk] * sinv[j];
    dc2e_u[kj] = Uc[kj];
    dc2e_v[kj] = Vc[kj] * sinv[j];
  }
}

// out[k][j] = keep(k) ? in[j][k] : 0 (n x n, complex as pairs): the GEMM form of a reference factor, with
// the columns of dropped singular directions zeroed (keep: the first `rank` columns; rank = n keeps all)
__global__ void k_factor_T(const double* in, int n, int cplx, int rank, double* out) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n) return;
  const int k = (int)(e / n), j = (int)(e % n);
  const int64_t src = (int64_t)j * n + k;
  const bool keep = k < rank;
  if (cplx) ((double2*)out)[e] = keep ? ((const double2*)in)[src] : make_double2(0, 0);
  else out[e] = keep ? in[src] : 0.0;
}
// columns >= rank of a row-major n x n reference factor set to zero (in place)
__global__ void k_zero_cols(double* a, int n, int cplx, int rank) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n || (int)(e % n) < rank) return;
  if (cplx) ((double2*)a)[e] = make_double2(0, 0);
  else a[e] = 0.0;
}

// T[ipos][f][j] = helper[imap[ipos][j]][f] / nconv
__global__ void k_m2l_tables(const double2* helper, int nfreq, const int* imap, double nconv, double2* T) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= 26ll * nfreq * 64) return;
  const int j = (int)(e % 64), f = (int)((e / 64) % nfreq), ipos = (int)(e / (64ll * nfreq));
  const int h = imap[ipos * 64 + j];
  double2 v = make_double2(0, 0);
  if (h >= 0) {
    const double2 x = helper[(int64_t)h * nfreq + f];
    v = make_double2(x.x / nconv, x.y / nconv);
  }
  T[e] = v;
}

// out[k][j] = (transpose ? A[j][k] : A[k][j]) for an n x n block, written into a wider row layout
__global__ void k_place(const double* A, int n, int transpose, int cplx, int out_ld, int out_row0, int out_col0,
                        void* out, int out_single) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n) return;
  const int k = (int)(e / n), j = (int)(e % n);
  const int64_t src = transpose ? (int64_t)j * n + k : (int64_t)k * n + j;
  const int64_t dst = (int64_t)(out_row0 + k) * out_ld + out_col0 + j;
  if (cplx) {
    const double re = A[2 * src], im = A[2 * src + 1];
    if (out_single) ((float2*)out)[dst] = make_float2((float)re, (float)im);
    else ((double2*)out)[dst] = make_double2(re, im);
  } else {
    if (out_single) ((float*)out)[dst] = (float)A[src];
    else ((double*)out)[dst] = A[src];
  }
}
__global__ void k_to_single(const double* in, float* out, int64_t n) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < n) out[e] = (float)in[e];
}

inline int nb(int64_t n) { return (int)std::max<int64_t>(1, (n + 255) / 256); }

// ---- the reference's operator file (.dat; fmm_scale_invariant.h:86-148, fmm.h:83-138), FP64 build:
//   r0 (8 bytes), then per level (Laplace: level 0 only; the other kernels: levels 0..depth)
//   UC2E_U, UC2E_V, DC2E_U, DC2E_V, M2M[8], L2L[8] (n x n row-major, real or complex values),
//   then the M2L tables of the table levels (Laplace: one; the others: levels 1..depth), 26 per level,
//   each [nfreq][8 x 8][re, im] in doubles.  A file is used only when its size and r0 match, as the
//   reference's load_matrix decides (else the operators are computed and the file rewritten).
struct DatOps {
  std::vector<std::array<std::vector<double>, 4>> fac;
  std::vector<std::vector<double>> m2m, l2l, m2l;
  void alloc(const Fmm& f, int depth) {
    const int nlev = f.kernel == XFMM_LAPLACE ? 1 : depth + 1;
    const int ntab = f.kernel == XFMM_LAPLACE ? 1 : depth;
    fac.assign(nlev, {});
    m2m.assign(nlev, {});
    l2l.assign(nlev, {});
    m2l.assign(ntab, {});
  }
};

size_t dat_bytes(const Fmm& f, int depth) {
  const size_t vs = f.is_complex() ? 2 : 1, n = f.nsurf;
  const size_t nlev = f.kernel == XFMM_LAPLACE ? 1 : depth + 1, ntab = f.kernel == XFMM_LAPLACE ? 1 : depth;
  return sizeof(double) + nlev * 20 * n * n * vs * sizeof(double) + ntab * 26 * (size_t)f.nfreq * 128 * sizeof(double);
}

bool dat_load(const Fmm& f, int depth, DatOps& d) {
  FILE* fp = std::fopen(f.filename.c_str(), "rb");
  if (!fp) return false;
  std::fseek(fp, 0, SEEK_END);
  const long size = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  double r0 = 0;
  bool ok = size >= 0 && (size_t)size == dat_bytes(f, depth) && std::fread(&r0, sizeof(double), 1, fp) == 1 &&
            r0 == f.r0;
  if (ok) {
    d.alloc(f, depth);
    const size_t vs = f.is_complex() ? 2 : 1, nn = (size_t)f.nsurf * f.nsurf * vs;
    auto rd = [&](std::vector<double>& v, size_t cnt) {
      v.resize(cnt);
      return std::fread(v.data(), sizeof(double), cnt, fp) == cnt;
    };
    for (size_t l = 0; ok && l < d.fac.size(); l++) {
      for (int i = 0; i < 4; i++) ok = ok && rd(d.fac[l][i], nn);
      ok = ok && rd(d.m2m[l], 8 * nn) && rd(d.l2l[l], 8 * nn);
    }
    for (size_t t = 0; ok && t < d.m2l.size(); t++) ok = rd(d.m2l[t], 26 * (size_t)f.nfreq * 128);
  }
  std::fclose(fp);
  return ok;
}

void dat_save(const Fmm& f, int depth, const DatOps& d) {
  (void)depth;
  std::remove(f.filename.c_str());
  FILE* fp = std::fopen(f.filename.c_str(), "wb");
  XREQUIRE(fp, XFMM_ERR_ARG, "cannot write the operator file " + f.filename);
  bool ok = std::fwrite(&f.r0, sizeof(double), 1, fp) == 1;
  auto wr = [&](const std::vector<double>& v) { return std::fwrite(v.data(), sizeof(double), v.size(), fp) == v.size(); };
  for (size_t l = 0; ok && l < d.fac.size(); l++) {
    for (int i = 0; i < 4; i++) ok = ok && wr(d.fac[l][i]);
    ok = ok && wr(d.m2m[l]) && wr(d.l2l[l]);
  }
  for (size_t t = 0; ok && t < d.m2l.size(); t++) ok = wr(d.m2l[t]);
  ok = (std::fclose(fp) == 0) && ok;
  XREQUIRE(ok, XFMM_ERR_ARG, "writing the operator file " + f.filename + " failed");
}

struct Handles {
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t sol = nullptr;
  ~Handles() {
    if (blas) cublasDestroy(blas);
    if (sol) cusolverDnDestroy(sol);
  }
};

// Row-major complex or real GEMM C = op(P) Q for n x n matrices (op: identity or transpose, never
// conjugate), on cuBLAS's column-major convention: row-major X is column-major X^T.
void gemm_rm(cublasHandle_t h, int n, bool cplx, const double* P, bool transP, const double* Q, double* C) {
  const cublasOperation_t tp = transP ? CUBLAS_OP_T : CUBLAS_OP_N;
  if (cplx) {
    const cuDoubleComplex one = make_cuDoubleComplex(1, 0), z = make_cuDoubleComplex(0, 0);
    XCUBLAS(cublasZgemm(h, CUBLAS_OP_N, tp, n, n, n, &one, (const cuDoubleComplex*)Q, n, (const cuDoubleComplex*)P, n,
                        &z, (cuDoubleComplex*)C, n));
  } else {
    const double one = 1, z = 0;
    XCUBLAS(cublasDgemm(h, CUBLAS_OP_N, tp, n, n, n, &one, Q, n, P, n, &z, C, n));
  }
}

// M2M[c] = UC2E_V (UC2E_U K_c) and, when l2l is given, L2L[c] = (K_c^T DC2E_V) DC2E_U for the 8 children
// (fmm_scale_invariant.h:51-77, fmm.h:47-74), K_c = K(parent check surface, child c's equivalent surface),
// each n x n row-major at c n^2 of the outputs.
void m2m_products(const Fmm& f, cublasHandle_t blas, int lev, const DBuf<double>& d_chk, DBuf<double>& d_eqv,
                  const DBuf<double>& uc2e_u, const DBuf<double>& uc2e_v, const DBuf<double>& dc2e_u,
                  const DBuf<double>& dc2e_v, DBuf<double>& K, DBuf<double>& Tmp, double* m2m, double* l2l,
                  cudaStream_t s) {
  const int p = f.p, n = f.nsurf;
  const bool cplx = f.is_complex();
  const size_t nn = (size_t)n * n * (cplx ? 2 : 1);
  const auto rel = rel_coords(1, 1, 2);
  const double sc = f.r0 * std::pow(0.5, lev + 1);
  for (int c = 0; c < 8; c++) {
    const double cc[3] = {rel[c][0] * sc, rel[c][1] * sc, rel[c][2] * sc};
    std::vector<double> ceq = host_surface(p, f.r0, lev + 1, cc, 1.05);
    d_eqv.upload(ceq, s);
    k_kernel_matrix<<<nb((int64_t)n * n), 256, 0, s>>>(f.kernel, f.k_re, f.k_im, d_chk.p, n, d_eqv.p, n, K.p, cplx);
    XLAUNCH();
    gemm_rm(blas, n, cplx, uc2e_u.p, false, K.p, Tmp.p);
    gemm_rm(blas, n, cplx, uc2e_v.p, false, Tmp.p, m2m + (size_t)c * nn);
    if (l2l) {
      gemm_rm(blas, n, cplx, K.p, true, dc2e_v.p, Tmp.p);
      gemm_rm(blas, n, cplx, Tmp.p, false, dc2e_u.p, l2l + (size_t)c * nn);
    }
  }
}

}  // namespace

void precompute(Fmm& f, int depth, cudaStream_t s) {
  const int p = f.p, n = f.nsurf, n1 = f.n1, nconv = f.nconv, nfreq = f.nfreq;
  const bool cplx = f.is_complex();
  const int vs = cplx ? 2 : 1;        // doubles per value
  const bool single = f.mixed();
  const size_t wsz = (single ? sizeof(float) : sizeof(double)) * vs;  // bytes per working value
#ifndef XFMM_PINV_EPS_MIXED
#define XFMM_PINV_EPS_MIXED 1e-10
#endif
  const double eps = single ? XFMM_PINV_EPS_MIXED : 1e-16;
  const double r0 = f.r0;
  Handles H;
  XCUBLAS(cublasCreate(&H.blas));
  XCUBLAS(cublasSetStream(H.blas, s));
  XCUSOLVER(cusolverDnCreate(&H.sol));
  XCUSOLVER(cusolverDnSetStream(H.sol, s));

  // geometry tables shared by all levels
  host_surface_base(p, f.h_surf_base);
  f.surf_base.upload(f.h_surf_base, s);
  std::vector<int> mup = host_surf2conv(p, true), mdn = host_surf2conv(p, false);
  f.map_up.upload(mup, s);
  f.map_dn.upload(mdn, s);
  std::vector<int> inv(nconv, -1);
  for (int k = 0; k < n; k++) inv[mup[k]] = k;
  f.conv_to_surf_up.upload(inv, s);
  {
    // e^{2 pi i m / n1} for m < n1, as (cos, sin) pairs: the DFT factors of the M2L transforms
    const int n1 = 2 * p;
    std::vector<double> tw(2 * n1);
    for (int m = 0; m < n1; m++) {
      const double a = 2.0 * 3.14159265358979323846 * m / n1;
      tw[2 * m] = std::cos(a);
      tw[2 * m + 1] = std::sin(a);
    }
    f.dft_tw.upload(tw, s);
  }
  std::vector<int> imap = m2l_index_map();
  DBuf<int> d_imap;
  d_imap.upload(imap, s);
  auto helper_rel = rel_coords(3, 2, 1);

  const int nlev = f.kernel == XFMM_LAPLACE ? 1 : depth + 1;
  const std::vector<int> tab_levels = f.kernel == XFMM_LAPLACE ? std::vector<int>{0} : [&] {
    std::vector<int> v;
    for (int l = 1; l <= depth; l++) v.push_back(l);
    return v;
  }();
  // The reference's FP64 operators (its threshold, its row-major layouts): read from the operator file
  // when it holds this configuration, else computed here and, when a file is named, written to it.
  // The working operators of this precision are derived from them below.
  DatOps dat;
  const bool named = !f.filename.empty();
  const bool loaded = named && dat_load(f, depth, dat);
  if (!loaded) dat.alloc(f, depth);
  f.ops.clear();
  f.ops.resize(nlev);
  const double zero[3] = {0, 0, 0};
  const size_t nn = (size_t)n * n * vs;
  DBuf<double> d_chk, d_eqv, M(nn), S(n), U(nn), VT(nn), K(nn), Tmp(nn), sinv(n);
  DBuf<double> R[4], F[4], M2Mref(8 * nn), L2Lref(8 * nn), M2M(8 * nn);
  for (auto& b : R) b.alloc(nn);
  for (auto& b : F) b.alloc(nn);
  DBuf<int> info(1);
  for (int lev = 0; lev < nlev; lev++) {
    LevelOps& op = f.ops[lev];
    std::vector<double> chk = host_surface(p, r0, lev, zero, 2.95);
    d_chk.upload(chk, s);
    if (loaded) {
      for (int i = 0; i < 4; i++) R[i].upload(dat.fac[lev][i], s);
      M2Mref.upload(dat.m2m[lev], s);
      L2Lref.upload(dat.l2l[lev], s);
    } else {
      // ---- K(check, equiv), its SVD and the reference's factors at its threshold 4e-16 s_max
      std::vector<double> eqv = host_surface(p, r0, lev, zero, 1.05);
      d_eqv.upload(eqv, s);
      k_kernel_matrix<<<nb((int64_t)n * n), 256, 0, s>>>(f.kernel, f.k_re, f.k_im, d_chk.p, n, d_eqv.p, n, M.p, cplx);
      XLAUNCH();
      int lwork = 0;
      if (cplx) XCUSOLVER(cusolverDnZgesvd_bufferSize(H.sol, n, n, &lwork));
      else XCUSOLVER(cusolverDnDgesvd_bufferSize(H.sol, n, n, &lwork));
      DBuf<double> work((size_t)std::max(lwork, 1) * vs), rwork(5 * (size_t)n);
      if (cplx)
        XCUSOLVER(cusolverDnZgesvd(H.sol, 'A', 'A', n, n, (cuDoubleComplex*)M.p, n, S.p, (cuDoubleComplex*)U.p, n,
                                   (cuDoubleComplex*)VT.p, n, (cuDoubleComplex*)work.p, lwork, rwork.p, info.p));
      else
        XCUSOLVER(cusolverDnDgesvd(H.sol, 'A', 'A', n, n, M.p, n, S.p, U.p, n, VT.p, n, work.p, lwork, rwork.p,
                                   info.p));
      int hinfo = 0;
      XCUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      std::vector<double> hs = S.download(s);
      XREQUIRE(hinfo == 0, XFMM_ERR_NUMERIC, "check-to-equivalent SVD did not converge");
      double smax = 0;
      for (double v : hs) smax = std::max(smax, std::fabs(v));
      k_sinv<<<nb(n), 256, 0, s>>>(S.p, n, 1e-16 * smax * 4, sinv.p);
      k_ref_factors<<<nb((int64_t)n * n), 256, 0, s>>>(U.p, VT.p, sinv.p, n, cplx, R[0].p, R[1].p, R[2].p, R[3].p);
      XLAUNCH();
      // M2M[c] = UC2E_V (UC2E_U K(parent check, child equiv)) (fmm_scale_invariant.h:67-71), L2L[c] =
      // K^T DC2E_V DC2E_U (72-74), each n x n row-major
      m2m_products(f, H.blas, lev, d_chk, d_eqv, R[0], R[1], R[2], R[3], K, Tmp, M2Mref.p, L2Lref.p, s);
      if (named) {
        for (int i = 0; i < 4; i++) dat.fac[lev][i] = R[i].download(s);
        dat.m2m[lev] = M2Mref.download(s);
        dat.l2l[lev] = L2Lref.download(s);
      }
    }
    // ---- the working operators of this precision.  Singular directions kept: those with s_k above
    // 4 eps s_max, s_k = 1 / |column k of UC2E_V| (V has unit columns; dropped columns are zero).
    std::vector<double> hv = R[1].download(s);
    std::vector<double> sk(n, 0.0);
    double smax = 0;
    for (int k = 0; k < n; k++) {
      double c2 = 0;
      for (int j = 0; j < n; j++)
        for (int q = 0; q < vs; q++) c2 += hv[((size_t)j * n + k) * vs + q] * hv[((size_t)j * n + k) * vs + q];
      sk[k] = c2 > 0 ? 1.0 / std::sqrt(c2) : 0.0;
      smax = std::max(smax, sk[k]);
    }
    int rank = 0;  // singular values come in descending order: the kept directions are a prefix
    while (rank < n && sk[rank] > 0 && (!single || sk[rank] > 4 * eps * smax)) rank++;
    op.rank = std::max(rank, 1);
    for (int i = 0; i < 4; i++) {
      k_factor_T<<<nb((int64_t)n * n), 256, 0, s>>>(R[i].p, n, cplx, (i == 1 || i == 3) ? op.rank : n, F[i].p);
      XLAUNCH();
    }
    const double* m2m_w = M2Mref.p;  // FP64: the reference's M2M, L2L
    const double* l2l_w = L2Lref.p;
    if (single) {
      // mixed: M2M from the factors truncated at the mixed threshold (L2L = its transpose)
      k_zero_cols<<<nb((int64_t)n * n), 256, 0, s>>>(R[1].p, n, cplx, op.rank);
      k_zero_cols<<<nb((int64_t)n * n), 256, 0, s>>>(R[3].p, n, cplx, op.rank);
      XLAUNCH();
      m2m_products(f, H.blas, lev, d_chk, d_eqv, R[0], R[1], R[2], R[3], K, Tmp, M2M.p, nullptr, s);
      m2m_w = M2M.p;
      l2l_w = nullptr;
    }
    // ---- GEMM operands: the check-to-equivalent factors stay FP64 in both precisions
    DBuf<char>* dst[4] = {&op.p2m_B1, &op.p2m_B2, &op.l2p_B1, &op.l2p_B2};
    for (int i = 0; i < 4; i++) {
      dst[i]->alloc(nn * sizeof(double));
      XCUDA(cudaMemcpyAsync(dst[i]->p, F[i].p, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    // the mixed path's L2P first factor (an orthogonal rotation of FP32 check values) runs in FP32
    if (single && !cplx) {
      op.l2p_B1f.alloc((size_t)n * n * sizeof(float));
      k_to_single<<<nb((int64_t)n * n), 256, 0, s>>>(F[2].p, (float*)op.l2p_B1f.p, (int64_t)n * n);
      XLAUNCH();
    }
    // m2m_B[c n + k][j] = M2M[c][j][k];  l2l_B[k][c n + j] = L2L[c][j][k] (= M2M[c][k][j])
    op.m2m_B.alloc((size_t)8 * n * n * wsz);
    op.l2l_B.alloc((size_t)8 * n * n * wsz);
    for (int c = 0; c < 8; c++) {
      const double* Mc = m2m_w + (size_t)c * nn;
      k_place<<<nb((int64_t)n * n), 256, 0, s>>>(Mc, n, 1, cplx, n, c * n, 0, op.m2m_B.p, single);
      if (l2l_w)
        k_place<<<nb((int64_t)n * n), 256, 0, s>>>(l2l_w + (size_t)c * nn, n, 1, cplx, 8 * n, 0, c * n, op.l2l_B.p,
                                                   single);
      else
        k_place<<<nb((int64_t)n * n), 256, 0, s>>>(Mc, n, 0, cplx, 8 * n, 0, c * n, op.l2l_B.p, single);
    }
    XLAUNCH();
    prepare_translation_operands(f, op, s);
  }

  // ---- M2L tables [26][nfreq][64] complex (the reference's matrix_M2L layout), FP64 then working precision
  const int nh = (int)helper_rel.size();
  if (!tab_levels.empty()) {
    DBuf<double> grid, spec, T64((size_t)26 * nfreq * 64 * 2);
    DBuf<double> offs(3 * (size_t)nh);
    cufftHandle plan = 0;
    if (!loaded) {
      grid.alloc((size_t)nh * nconv * vs);
      spec.alloc((size_t)nh * nfreq * 2);
      int dims[3] = {n1, n1, n1};
      XCUFFT(cufftPlanMany(&plan, 3, dims, nullptr, 1, nconv, nullptr, 1, nfreq, cplx ? CUFFT_Z2Z : CUFFT_D2Z, nh));
      XCUFFT(cufftSetStream(plan, s));
    }
    for (size_t ti = 0; ti < tab_levels.size(); ti++) {
      const int l = tab_levels[ti];
      if (loaded) {
        T64.upload(dat.m2l[ti], s);
      } else {
        std::vector<double> ho(3 * nh);
        for (int h = 0; h < nh; h++)
          for (int d = 0; d < 3; d++)
            ho[3 * h + d] = l == 0 ? helper_rel[h][d] * (r0 / 0.5) : helper_rel[h][d] * r0 * std::pow(0.5, l - 1);
        offs.upload(ho, s);
        const double a = 2 * r0 * std::pow(0.5, l) * 1.05;
        k_conv_values<<<nb((int64_t)nh * nconv), 256, 0, s>>>(f.kernel, f.k_re, f.k_im, p, a, offs.p, nh, grid.p,
                                                               cplx);
        XLAUNCH();
        if (cplx)
          XCUFFT(cufftExecZ2Z(plan, (cufftDoubleComplex*)grid.p, (cufftDoubleComplex*)spec.p, CUFFT_FORWARD));
        else
          XCUFFT(cufftExecD2Z(plan, grid.p, (cufftDoubleComplex*)spec.p));
        k_m2l_tables<<<nb(26ll * nfreq * 64), 256, 0, s>>>((double2*)spec.p, nfreq, d_imap.p, (double)nconv,
                                                            (double2*)T64.p);
        XLAUNCH();
        if (named) dat.m2l[ti] = T64.download(s);
      }
      LevelOps& op = f.ops[l];
      const int64_t cnt = 26ll * nfreq * 64 * 2;
      if (single) {
        op.m2l_T.alloc(cnt * sizeof(float));
        k_to_single<<<nb(cnt), 256, 0, s>>>(T64.p, (float*)op.m2l_T.p, cnt);
        XLAUNCH();
      } else {
        op.m2l_T.alloc(cnt * sizeof(double));
        XCUDA(cudaMemcpyAsync(op.m2l_T.p, T64.p, cnt * sizeof(double), cudaMemcpyDeviceToDevice, s));
      }
    }
    XCUDA(cudaStreamSynchronize(s));
    if (plan) cufftDestroy(plan);
  }
  if (named && !loaded) dat_save(f, depth, dat);
  XCUDA(cudaStreamSynchronize(s));
  f.precomputed = true;
  f.pre_r0 = r0;
  f.pre_depth = depth;
}

}  // namespace xfmm
